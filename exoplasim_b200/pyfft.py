"""Drop-in replacement for ExoPlaSim's f2py module ``exoplasim.pyfft``.

Same function names, argument order and array conventions as the calls
pyburn makes (pyburn.py:606, 711, 810, 840, 867, 1067, 1172):

  inigau(nlat)                              -> (sid, gwd)
  sp2gp(sp, nlat, nlon, ntru, nfs)          sp (NRSP, nlev)      -> gp (nlon, nlat, nlev)
  gp2sp(gp, nlat, nlon, ntru, nfs)          gp (nlon, nlat, nlev)-> sp (NRSP, nlev)
  sp3fc(sp, nlat, nlon, ntru, nfs)          sp (NRSP, nlev)      -> fc (2, nlon/2, nlat, nlev)
  gp3fc(gp)                                 gp (n, lot, nlev)    -> fc (n, lot, nlev)
  fc3gp(fc)                                 fc (n, lot, nlev)    -> gp (n, lot, nlev)
  spvgp(sd, sz, rdcostheta, nlon, ntru, nfs)   -> (gu, gv) each (nlon, nlat, nlev)
  gpvsp(gu, gv, costhetadr, ntru, nfs)         -> (sd, sz) each (NRSP, nlev)
  dv2uv(sd, sz, nlat, nlon, ntru, nlev, nfs)   -> (pu, pv) each (2, nlon/2, nlat, nlev)
  uv2dv(pu, pv, nlat, nlon, ntru, nlev, nfs)   -> (pd, pz) each (2, NCSP, nlev)
  sp2fc / sp2fcdmu / fc2sp / gp2fc / fc2gp / legini  (single-field forms)

Shapes are Fortran-ordered like f2py's results (pyburn transposes them).
The pyfft scalings are kept: fc2gp multiplies by sqrt(2) (pyfft.f90:895),
gp2sp divides by sqrt(2) before the forward FFT (:1160), spvgp/gpvsp take
the radius/cos(lat) factors (:1063, :1106).  Unlike the f2py module, tables
are built once per resolution (not on every call) and the FFT twiddles are
FP64 (pyfft.f90 computes them in 4-byte reals).  Arrays go to the GPU and
back; torch CUDA tensors are accepted too and stay on the device.
exoplasim_b200.pyfft991 is the same module under the name pyburn imports for
NLAT 192 and 320 (pyburn.py:594-602): one GPU FFT serves every even length
from 4 to 4096 whose half has no prime factor above 5, which covers both
modules' lists (pyfft.f90:791-792, pyfft991.f90:793).
"""
import functools

import numpy as np
import torch

from .transforms import Plan

SQRT2 = 1.4142135623730951


@functools.lru_cache(maxsize=16)
def _plan(nlat, nfs):
    return Plan(nlat, pyfft_nfs=int(nfs), plavor=0.0)


def _dev(a):
    """(tensor on cuda float64, is_numpy)"""
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=torch.float64), False
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda"), True


def _out(t, numpy):
    return t.cpu().numpy() if numpy else t


def _spec_levels(sp, ntru):
    """(NRSP, nlev) Fortran-style -> contiguous (nlev, NRSP)."""
    nrsp = (ntru + 1) * (ntru + 2)
    if sp.dim() == 1:
        sp = sp.reshape(nrsp, 1)
    if sp.shape[0] != nrsp:
        raise ValueError(f"spectral array must have {nrsp} rows, got {tuple(sp.shape)}")
    return sp.t().contiguous()


def _check_trunc(p, nlon, ntru):
    """The reference sizes its arrays from (NLON, NTRU); this library derives
    both from NLAT, so a caller's pair must be the triangular one for NLAT."""
    if int(nlon) != p.nlon or int(ntru) != p.ntru:
        raise ValueError(f"NLAT={p.nlat} needs NLON={p.nlon} and NTRU={p.ntru}, got {nlon} and {ntru}")


def _grid_levels(gp):
    """(nlon, nlat, nlev) -> contiguous (nlev, nlat, nlon)."""
    if gp.dim() == 2:
        gp = gp.unsqueeze(-1)
    return gp.permute(2, 1, 0).contiguous()


def inigau(nlat):
    """Gaussian abscissas (sin lat, north first) and weights (gaussmod.f90:5-40)."""
    return _plan(int(nlat), 0).gauss()


def legini(nlat, nlon, ntru, nlev=1, nfs=0):
    """The eight legini tables as (NCSP, NLAT) Fortran-ordered arrays plus the filter."""
    p = _plan(int(nlat), int(nfs))
    tabs = [p.table(n).T for n in ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv")]
    n = np.arange(1, ntru + 2, dtype=np.float32)
    filt = (1 - nfs) + nfs * np.exp(-8.0 * (n / np.float32(ntru)) ** 8).astype(np.float64)
    return (*tabs, filt)


def sp2fc(sp, nlat, nlon, ntru, nlev=1, nfs=0):
    """One field sp(2,NCSP) -> fc(2,NLON/2,NLAT) (pyfft.f90:264)."""
    t, isnp = _dev(sp)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    fc = p.sp2fc(t.reshape(1, p.nrsp))
    return _out(fc[0].reshape(nlat, nlon // 2, 2).permute(2, 1, 0), isnp)


def sp2fcdmu(sp, nlat, nlon, ntru, nlev=1, nfs=0):
    t, isnp = _dev(sp)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    fc = p.sp2fcdmu(t.reshape(1, p.nrsp))
    return _out(fc[0].reshape(nlat, nlon // 2, 2).permute(2, 1, 0), isnp)


def fc2sp(fc, nlat, nlon, ntru, nlev=1, nfs=0):
    """fc(2,NLON/2,NLAT) -> sp(2,NCSP) (pyfft.f90:160)."""
    t, isnp = _dev(fc)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    rows = t.permute(2, 1, 0).contiguous().reshape(1, nlat, nlon)
    sp = p.fc2sp(rows)[0]
    return _out(sp.reshape(p.ncsp, 2).t(), isnp)


def gp2fc(a, n=None, lot=None):
    """(n, lot) grid rows -> Fourier coefficients, not scaled by sqrt(2) (pyfft.f90:814)."""
    t, isnp = _dev(a)
    n = t.shape[0]
    rows = t.t().contiguous()
    Plan.gp2fc(rows)
    return _out(rows.t(), isnp)


def fc2gp(a, n=None, lot=None):
    """(n, lot) Fourier rows -> grid, times sqrt(2) (pyfft.f90:855-898)."""
    t, isnp = _dev(a)
    rows = t.t().contiguous()
    Plan.fc2gp(rows)
    return _out(rows.t() * SQRT2, isnp)


def gp3fc(a):
    """gp2fc level by level: (n, lot, nlev) -> (n, lot, nlev) (pyfft.f90:938)."""
    t, isnp = _dev(a)
    if t.dim() == 2:
        t = t.unsqueeze(-1)
    rows = t.permute(2, 1, 0).contiguous()
    Plan.gp2fc(rows)
    return _out(rows.permute(2, 1, 0), isnp)


def fc3gp(a):
    """fc2gp level by level (with the sqrt(2) of pyfft's fc2gp) (pyfft.f90:905)."""
    t, isnp = _dev(a)
    if t.dim() == 2:
        t = t.unsqueeze(-1)
    rows = t.permute(2, 1, 0).contiguous()
    Plan.fc2gp(rows)
    return _out(rows.permute(2, 1, 0) * SQRT2, isnp)


def sp3fc(sp, nlat, nlon, ntru, nfs=0):
    """sp (NRSP, nlev) -> fc (2, NLON/2, NLAT, nlev) (pyfft.f90:344)."""
    t, isnp = _dev(sp)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    lev = _spec_levels(t, p.ntru)
    fc = p.sp2fc(lev)  # (nlev, nlat, nlon)
    out = fc.reshape(-1, nlat, nlon // 2, 2).permute(3, 2, 1, 0)
    return _out(out, isnp)


def sp2gp(sp, nlat, nlon, ntru, nfs=0):
    """sp (NRSP, nlev) -> gp (NLON, NLAT, nlev): sp2fc + fc2gp * sqrt(2) (pyfft.f90:971)."""
    t, isnp = _dev(sp)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    lev = _spec_levels(t, p.ntru)
    g = p.sp2fc(lev)
    Plan.fc2gp(g)
    g.mul_(SQRT2)
    return _out(g.permute(2, 1, 0), isnp)


def gp2sp(gp, nlat, nlon, ntru, nfs=0):
    """gp (NLON, NLAT, nlev) -> sp (NRSP, nlev): gp2fc(gp/sqrt(2)) + fc2sp (pyfft.f90:1141)."""
    t, isnp = _dev(gp)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    rows = _grid_levels(t) / SQRT2
    Plan.gp2fc(rows)
    sp = p.fc2sp(rows)
    return _out(sp.t(), isnp)


def dv2uv(sd, sz, nlat, nlon, ntru, nlev=None, nfs=0):
    """(div, vort) (NRSP, nlev) -> Fourier (u, v) cos(lat), each (2, NLON/2, NLAT, nlev),
    without the planetary-vorticity offset (pyfft.f90:454-553)."""
    td, isnp = _dev(sd)
    tz, _ = _dev(sz)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    u, v = p.dv2uv(_spec_levels(td, p.ntru), _spec_levels(tz, p.ntru))
    f = lambda t: t.reshape(-1, nlat, nlon // 2, 2).permute(3, 2, 1, 0)  # noqa: E731
    return _out(f(u), isnp), _out(f(v), isnp)


def uv2dv(pu, pv, nlat, nlon, ntru, nlev=None, nfs=0):
    """Fourier (u, v) cos(lat) (2, NLON/2, NLAT, nlev) -> (div, vort) each (2, NCSP, nlev)
    (pyfft.f90:560-690, the folded branch)."""
    tu, isnp = _dev(pu)
    tv, _ = _dev(pv)
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    if tu.dim() == 3:
        tu, tv = tu.unsqueeze(-1), tv.unsqueeze(-1)
    rows = lambda t: t.permute(3, 2, 1, 0).contiguous().reshape(-1, nlat, nlon)  # noqa: E731
    sd, sz = p.uv2dv(rows(tu), rows(tv))
    f = lambda t: t.reshape(-1, p.ncsp, 2).permute(2, 1, 0)  # noqa: E731
    return _out(f(sd), isnp), _out(f(sz), isnp)


def spvgp(sd, sz, rdcostheta, nlon, ntru, nfs=0):
    """(div, vort) spectral -> (u, v) grid times radius/cos(lat) (pyfft.f90:1012-1069)."""
    td, isnp = _dev(sd)
    tz, _ = _dev(sz)
    rc, _ = _dev(rdcostheta)
    nlat = rc.shape[0]
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, nlon, ntru)
    u, v = p.dv2uv(_spec_levels(td, p.ntru), _spec_levels(tz, p.ntru))
    Plan.fc2gp(u)
    Plan.fc2gp(v)
    scale = (rc * SQRT2).view(1, nlat, 1)
    u.mul_(scale)
    v.mul_(scale)
    return _out(u.permute(2, 1, 0), isnp), _out(v.permute(2, 1, 0), isnp)


def gpvsp(gu, gv, costhetadr, ntru, nfs=0):
    """(u, v) grid times cos(lat)/radius -> (div, vort) spectral (pyfft.f90:1076-1133)."""
    tu, isnp = _dev(gu)
    tv, _ = _dev(gv)
    cr, _ = _dev(costhetadr)
    nlat = cr.shape[0]
    p = _plan(int(nlat), int(nfs))
    _check_trunc(p, tu.shape[0], ntru)
    scale = (cr / SQRT2).view(1, nlat, 1)
    u = _grid_levels(tu) * scale
    v = _grid_levels(tv) * scale
    Plan.gp2fc(u)
    Plan.gp2fc(v)
    sd, sz = p.uv2dv(u, v)
    return _out(sd.t(), isnp), _out(sz.t(), isnp)

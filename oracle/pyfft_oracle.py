"""FP64 restatement of the f2py module exoplasim.pyfft (test infrastructure only).

TEST INFRASTRUCTURE ONLY: the checker for exoplasim_b200.pyfft.  Each
function composes the C oracle's legmod/fftmod/fft991mod restatement in the
order exoplasim/pyfft.f90 does, with pyfft's own scalings and layouts:

  sp2gp   pyfft.f90:971-1005   per level: sp2fc (filter sfilt) -> fc2gp, times sqrt(2) (:895)
  gp2sp   pyfft.f90:1141-1174  per level: gp2fc(gp / sqrt(2)) -> fc2sp (folded)
  spvgp   pyfft.f90:1012-1069  dv2uv (no plavor: :531-532 are commented out)
                               -> fc2gp * sqrt(2) -> * rdcostheta(lat)
  gpvsp   pyfft.f90:1076-1133  * costhetadr(lat) / sqrt(2) -> gp2fc -> uv2dv (folded)
  sp3fc   pyfft.f90:344-369    per level sp2fc -> fc(2, NLON/2, NLAT, NLEV)
  gp3fc   pyfft.f90:938-964    gp2fc per level, no sqrt(2)
  fc3gp   pyfft.f90:905-931    fc2gp per level, times sqrt(2)
  dv2uv   pyfft.f90:454-553    -> pu, pv (2, NLON/2, NLAT, NLEV)
  uv2dv   pyfft.f90:560-690    -> pd, pz (2, NCSP, NLEV)

pyburn.py:594-602 picks exoplasim.pyfft991 (the FFT991 transform,
pyfft991.f90:813-883) for NLAT 192 and 320 and exoplasim.pyfft otherwise;
``use991`` selects between the two here.  Arrays follow f2py's Fortran-ordered
shapes.  The FFT twiddles are FP64: the f2py build computes pyfft's twiddle
angles in 4-byte reals (pyfft.f90:1201-1206, no -fdefault-real-8 in
__init__.py:84-85), which perturbs its grids at the 1e-7 level; this
restatement follows the FP64 transform of the model's own fftmod.
"""
import functools

import numpy as np

from oracle import oracle as O

SQRT2 = 1.4142135623730951


@functools.lru_cache(maxsize=8)
def _leg(nlat, nfs):
    return O.Leg(int(nlat), pyfft_nfs=int(nfs))


def _fft(rows, inverse, use991):
    f = O.fc2gp if inverse else O.gp2fc
    return f(rows, use991=use991)


def _fc_fortran(fc_rows):
    """(nlat, nlon) Fourier rows -> (2, nlon/2, nlat)."""
    nlat, nlon = fc_rows.shape
    return fc_rows.reshape(nlat, nlon // 2, 2).transpose(2, 1, 0)


def _fc_rows(fc):
    """(2, nlon/2, nlat) -> (nlat, nlon) Fourier rows."""
    return np.ascontiguousarray(fc.transpose(2, 1, 0)).reshape(fc.shape[2], 2 * fc.shape[1])


def inigau(nlat):
    return O.inigau(int(nlat))


def sp2gp(sp, nlat, nlon, ntru, nfs=0, use991=False):
    L = _leg(nlat, nfs)
    sp = np.asarray(sp, np.float64).reshape(L.nrsp, -1)
    gp = np.zeros((nlon, nlat, sp.shape[1]))
    for v in range(sp.shape[1]):
        g = _fft(L.sp2fc(sp[:, v]), True, use991) * SQRT2
        gp[:, :, v] = g.T
    return gp


def gp2sp(gp, nlat, nlon, ntru, nfs=0, use991=False):
    L = _leg(nlat, nfs)
    gp = np.asarray(gp, np.float64).reshape(nlon, nlat, -1)
    sp = np.zeros((L.nrsp, gp.shape[2]))
    for v in range(gp.shape[2]):
        fc = _fft(gp[:, :, v].T / SQRT2, False, use991)
        sp[:, v] = L.fc2sp(fc, folded=True)
    return sp


def sp3fc(sp, nlat, nlon, ntru, nfs=0):
    L = _leg(nlat, nfs)
    sp = np.asarray(sp, np.float64).reshape(L.nrsp, -1)
    return np.stack([_fc_fortran(L.sp2fc(sp[:, v])) for v in range(sp.shape[1])], axis=-1)


def gp3fc(a, use991=False):
    a = np.asarray(a, np.float64)
    return np.stack([_fft(a[:, :, v].T, False, use991).T for v in range(a.shape[2])], axis=-1)


def fc3gp(a, use991=False):
    a = np.asarray(a, np.float64)
    return np.stack([_fft(a[:, :, v].T, True, use991).T * SQRT2 for v in range(a.shape[2])], axis=-1)


def dv2uv(sd, sz, nlat, nlon, ntru, nfs=0):
    L = _leg(nlat, nfs)
    pu, pv = L.dv2uv(np.ascontiguousarray(np.asarray(sd, np.float64).T),
                     np.ascontiguousarray(np.asarray(sz, np.float64).T), plavor=0.0)
    return (np.stack([_fc_fortran(r) for r in pu], axis=-1),
            np.stack([_fc_fortran(r) for r in pv], axis=-1))


def uv2dv(pu, pv, nlat, nlon, ntru, nfs=0):
    L = _leg(nlat, nfs)
    ru = np.stack([_fc_rows(pu[..., v]) for v in range(pu.shape[3])])
    rv = np.stack([_fc_rows(pv[..., v]) for v in range(pv.shape[3])])
    pd, pz = L.uv2dv(ru, rv, folded=True)
    return (pd.reshape(-1, L.ncsp, 2).transpose(2, 1, 0), pz.reshape(-1, L.ncsp, 2).transpose(2, 1, 0))


def spvgp(sd, sz, rdcostheta, nlon, ntru, nfs=0, use991=False):
    nlat = len(rdcostheta)
    L = _leg(nlat, nfs)
    pu, pv = L.dv2uv(np.ascontiguousarray(np.asarray(sd, np.float64).T),
                     np.ascontiguousarray(np.asarray(sz, np.float64).T), plavor=0.0)
    rc = np.asarray(rdcostheta, np.float64)
    gu = np.stack([(_fft(r, True, use991) * SQRT2 * rc[:, None]).T for r in pu], axis=-1)
    gv = np.stack([(_fft(r, True, use991) * SQRT2 * rc[:, None]).T for r in pv], axis=-1)
    return gu, gv


def gpvsp(gu, gv, costhetadr, ntru, nfs=0, use991=False):
    nlat = len(costhetadr)
    L = _leg(nlat, nfs)
    cr = np.asarray(costhetadr, np.float64)
    gu = np.asarray(gu, np.float64)
    gv = np.asarray(gv, np.float64)
    ru = np.stack([_fft(gu[:, :, v].T * cr[:, None] / SQRT2, False, use991) for v in range(gu.shape[2])])
    rv = np.stack([_fft(gv[:, :, v].T * cr[:, None] / SQRT2, False, use991) for v in range(gv.shape[2])])
    pd, pz = L.uv2dv(ru, rv, folded=True)
    return pd.T.copy(), pz.T.copy()

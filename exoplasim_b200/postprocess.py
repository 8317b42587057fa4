"""pyburn's horizontal transforms of an output dataset on the GPU.

pyburn.py:623-1348 (_transformvar, _transformvectorvar) brings every
variable of a raw output file into the requested horizontal mode by calling
the f2py pyfft module on all output times and levels of the variable at once,
and pyfft rebuilds its Legendre tables on every such call.  These functions
take the same arrays, make the same calls on exoplasim_b200.pyfft (one
batched GPU transform over times x levels, tables built once per resolution)
and return arrays of the same shapes, layouts and roll of the longitudes.

Modes: "grid" (spectral -> Gaussian grid with sp2gp and the half-turn roll
of the longitudes, pyburn.py:684-707; spvgp for a divergence/vorticity pair,
:1039-1069), "spectral" (grid -> modes with gp2sp, :778-816) and "fourier"
(spectral -> Fourier with sp3fc, grid -> Fourier with gp3fc after the
1/sqrt(2), :818-850).  Arrays may be numpy or torch; torch CUDA tensors stay
on the device.  Two cases differ from the reference where it fails: mode
"spectral" of a single-level grid field (times, lat, lon) gives (times,
modes, 2) here, where pyburn.py:798 raises NameError on a misspelt name; and
of a multi-level grid field it gives (times, levels, modes, 2), the shape its
own dims label says, where pyburn returns (times*levels, modes, 2).
"""
import numpy as np
import torch

from . import pyfft

SQRT2 = 1.4142135623730951


def _t(a):
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=torch.float64), False
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda"), True


def _out(t, numpy):
    return t.cpu().numpy() if numpy else t


def transformvar(variable, nlat, nlon, nlev, ntru, mode="grid", physfilter=False):
    """One variable of a dataset, (ntimes[, nlev], NRSP) spectral or
    (ntimes[, nlev], nlat, nlon) grid, brought into `mode` (pyburn.py:623-958)."""
    v, isnp = _t(variable)
    nrsp = (ntru + 1) * (ntru + 2)
    spectral = v.shape[-1] == nrsp
    nfs = int(physfilter)
    if mode == "grid":
        if not spectral:
            return _out(v, isnp)
        ntimes = v.shape[0]
        nlevs = v.shape[1] if v.dim() == 3 else 1
        sp = v.reshape(ntimes * nlevs, nrsp).t()                       # Fortran (NRSP, times*levels)
        gp = pyfft.sp2gp(sp, nlat, nlon, ntru, nfs)                    # (nlon, nlat, times*levels)
        shape = (ntimes, nlevs, nlat, nlon) if v.dim() == 3 else (ntimes, nlat, nlon)
        gp = gp.permute(2, 1, 0).reshape(shape)
        return _out(torch.roll(gp, nlon // 2, dims=-1), isnp)
    if mode == "spectral":
        if spectral:
            out = v
        elif v.dim() in (3, 4):
            lead = v.shape[:-2]
            gp = v.reshape(-1, nlat, nlon).permute(2, 1, 0)           # (nlon, nlat, times*levels)
            out = pyfft.gp2sp(gp, nlat, nlon, ntru, nfs).t().reshape(*lead, nrsp)
        else:
            return _out(v, isnp)                                       # columns and scalars pass through
        return _out(out.reshape(*out.shape[:-1], nrsp // 2, 2), isnp)
    if mode == "fourier":
        if spectral:
            ntimes = v.shape[0]
            nlevs = v.shape[1] if v.dim() == 3 else 1
            sp = v.reshape(ntimes * nlevs, nrsp).t()
            fc = pyfft.sp3fc(sp, nlat, nlon, ntru, nfs)                # (2, nlon/2, nlat, times*levels)
            shape = (ntimes, nlevs, nlat, nlon // 2, 2) if v.dim() == 3 else (ntimes, nlat, nlon // 2, 2)
            return _out(fc.permute(3, 2, 1, 0).reshape(shape), isnp)
        if v.dim() in (3, 4):
            lead = v.shape[:-2]
            gp = (v / SQRT2).reshape(-1, nlat, nlon).permute(2, 1, 0)  # (nlon, nlat, times*levels)
            fc = pyfft.gp3fc(gp)
            return _out(fc.permute(2, 1, 0).reshape(*lead, nlat, nlon // 2, 2), isnp)
        return _out(v, isnp)
    raise ValueError(f"mode {mode!r}: grid, spectral and fourier are the transform modes")


def transformvectorvar(uvar, vvar, lats, nlon, nlev, ntru, mode="grid", physfilter=False, radius=6371220.0):
    """A divergence/vorticity pair (ntimes[, nlev], NRSP) to the grid winds
    u and v (pyburn.py:960-1348, mode "grid"): spvgp with radius / cos(lat),
    then the half-turn roll of the longitudes."""
    if mode != "grid":
        raise ValueError("the vector transform is built for mode 'grid'")
    lats = np.asarray(lats, dtype=np.float64)
    rlats = lats * np.pi / 180.0 if np.nanmax(lats) > 10 else lats
    nlat = len(rlats)
    u, isnp = _t(uvar)
    v, _ = _t(vvar)
    nrsp = (ntru + 1) * (ntru + 2)
    if u.shape[-1] != nrsp:
        return _out(u, isnp), _out(v, isnp)
    ntimes = u.shape[0]
    nlevs = u.shape[1] if u.dim() == 3 else 1
    rdcostheta = radius / np.cos(rlats)
    su = u.reshape(ntimes * nlevs, nrsp).t()
    sv = v.reshape(ntimes * nlevs, nrsp).t()
    gu, gv = pyfft.spvgp(su, sv, torch.as_tensor(rdcostheta, device="cuda"), nlon, ntru, int(physfilter))
    shape = (ntimes, nlevs, nlat, nlon) if u.dim() == 3 else (ntimes, nlat, nlon)
    f = lambda g: torch.roll(g.permute(2, 1, 0).reshape(shape), nlon // 2, dims=-1)  # noqa: E731
    return _out(f(gu), isnp), _out(f(gv), isnp)


def refactor(variable, header, ntimes=None, nlev=10):
    """A code's concatenated values shaped (times[, levels], dim2, dim1) from its
    header, as pyburn.refactorvariable (pyburn.py:497-551)."""
    variable = np.asarray(variable)
    dim1 = max(header[4], header[5])
    dim2 = min(header[4], header[5])
    if header[1] == 1:
        nlevs = nlev
        if ntimes is not None:
            if ntimes * nlevs * dim1 * dim2 < len(variable):
                nlevs = int(len(variable) / (ntimes * dim1 * dim2))
        elif len(variable) % (float(len(variable)) / (dim1 * dim2 * nlevs)) != 0:
            nlevs += 1
    else:
        nlevs = 1
        if ntimes is not None and ntimes * dim1 * dim2 > len(variable):
            ntimes = int(len(variable) // (dim1 * dim2))
    if ntimes is None:
        ntimes = int(len(variable) // (dim1 * dim2 * nlevs))
    if nlevs == 1:
        if dim2 == 1:
            return np.reshape(variable, (ntimes,) if dim1 == 1 else (ntimes, dim1))
        return np.reshape(variable, (ntimes, dim2, dim1))
    if dim2 == 1:
        return np.reshape(variable, (ntimes, nlevs) if dim1 == 1 else (ntimes, nlevs, dim1))
    return np.reshape(variable, (ntimes, nlevs, dim2, dim1))

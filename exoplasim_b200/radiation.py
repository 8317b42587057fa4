"""PyTorch-facing radiation column pass (radmod.f90 radstep) over libexotx.

Column arrays use the reference layout x(NHOR, NLEV) stored as torch tensors
of shape (nlev or nlep, nhor) -- level-major, columns fastest.  dsalb is
(nhor, 2) (Fortran dsalb(2,NHOR)).  sid and cola are per latitude row.
"""
import ctypes as C

import torch

from . import _lib
from ._lib import FP32, FP64, RAD_IO_FIELDS, call

RAD_INPUTS = ("dt", "dq", "dcc", "dql", "dqco2", "dp", "dls", "dicec")
RAD_INOUT = ("dqo3", "gmu0", "dalb", "dsalb", "dtdt")
RAD_OUTPUTS = ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux", "dtdtswr", "dtdtlwr", "dconv")


def default_params(nlev, nhor, nlon, **over):
    """Reference namelist defaults (radmod.f90:27-100) with overrides."""
    p = _lib.RadParams()
    call("exotx_rad_params_default", nlev, nhor, nlon, C.byref(p))
    for k, v in over.items():
        if k in ("rcl1", "rcl2", "acl2", "sigma", "sigmah", "dsigma"):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = float(x)
        elif not hasattr(p, k):
            raise AttributeError(f"unknown radiation parameter {k}")
        else:
            setattr(p, k, v)
    return p


def solarini(starbbtemp, minwavel_nm=316.036116751):
    """Blackbody band split (zsolar1, zsolar2, rcoeff) (radmod.f90:166-376)."""
    z1, z2, rc = C.c_double(), C.c_double(), C.c_double()
    call("exotx_solarini", float(starbbtemp), minwavel_nm * 1e-9, C.byref(z1), C.byref(z2), C.byref(rc))
    return z1.value, z2.value, rc.value


def alloc_outputs(params, dtype=torch.float64, device="cuda"):
    nlev, nhor = params.nlev, params.nhor
    out = {}
    for k in ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux"):
        out[k] = torch.zeros((nlev + 1, nhor), dtype=dtype, device=device)
    for k in ("dtdtswr", "dtdtlwr", "dconv"):
        out[k] = torch.zeros((nlev, nhor), dtype=dtype, device=device)
    return out


def radstep(params, cols, out=None, precision="fp64"):
    """Run radstep on device tensors.

    cols: dict with sid, cola (nlat rows), dt, dq, dcc, dql (nlep, nhor), dqco2 (nlev, nhor),
    dp, dls, dicec (nhor) and the in/out arrays dqo3 (nlev, nhor), gmu0 (nhor), dalb (nhor),
    dsalb (nhor, 2), dtdt (nlev, nhor) -- updated in place.  Returns the output dict.
    """
    prec = FP64 if precision in ("fp64", FP64) else FP32
    dtype = torch.float64 if prec == FP64 else torch.float32
    if out is None:
        out = alloc_outputs(params, dtype)
    io = make_io(cols, out, prec)
    call("exotx_radstep", C.byref(params), prec, C.byref(io),
         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out


def make_io(cols, out, prec):
    """exotx_rad_io over the column and output tensors (zsol optional)."""
    dtype = torch.float64 if prec == FP64 else torch.float32
    io = _lib.RadIO()
    allv = dict(cols)
    allv.update(out)
    for name in RAD_IO_FIELDS:
        t = allv.get(name)
        if t is None:
            if name == "zsol":
                continue
            raise KeyError(f"radstep needs '{name}'")
        if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
            raise TypeError(f"{name} must be a contiguous CUDA {dtype} tensor")
        setattr(io, name, t.data_ptr())
    return io

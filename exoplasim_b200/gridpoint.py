"""The grid-point step of gridpointa on the GPU (plasim.f90:2441-2455).

Between the inverse and the forward transform sets: gp = exp(gp), calcgp
(:2587-2755) and the flux products.  Takes the inverse set's grid output
(6L+3 fields: gu gv gt gd gz gq gpj gpmt gp) and gives the forward set's
input (9L+1 fields: gtn gqn gut gvt guz gvz gke gvpp guq gvq), so that
inverse_set -> gridpoint -> forward_set is gridpointa's transform path with
no host round trip.
"""
import ctypes as C

import torch

from . import _lib
from ._lib import FP32, FP64, call


class GpParams(C.Structure):
    _fields_ = ([("nlev", C.c_int), ("nqspec", C.c_int)] +
                [(n, C.c_double) for n in ("akap", "rdbrv", "adv", "psurf", "ww")] +
                [(n, C.c_double * 64) for n in ("dsigma", "sigmah", "rdsig", "t0", "t01s2", "tkp")] +
                [("g", C.c_double * 4096), ("c", C.c_double * 4096)])


def default_params(nlev, **over):
    """Earth defaults (exotx_gp_params_default); t0, sigmah, dsigma or akap
    overrides re-derive the semi-implicit arrays (initsi)."""
    p = GpParams()
    call("exotx_gp_params_default", nlev, C.byref(p))
    for k, v in over.items():
        if k in ("dsigma", "sigmah", "t0"):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = float(x)
        else:
            setattr(p, k, v)
    if over:
        call("exotx_gp_params_derive", C.byref(p))
    return p


class GpConst:
    """The constants on the device (exotx_gpconst)."""

    def __init__(self, params):
        self.params = params
        self._lib = _lib.load()
        h = C.c_void_p()
        call("exotx_gpconst_create", C.byref(params), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.exotx_gpconst_destroy(h)
            except Exception:
                pass
            self._h = None


def gridpoint(plan, const, gin, gout=None, dw=None, dq=None, precision=None):
    """gin (ninst, 6L+3, NLAT, NLON) -> gout (ninst, 9L+1, NLAT, NLON); float64
    or float32 CUDA tensors.  dw (ninst, L, NLAT, NLON) receives the vertical
    velocity diagnostic when given; dq (ninst, L, NLAT, NLON) is read when
    nqspec = 0."""
    L = const.params.nlev
    squeeze = gin.dim() == 3
    if squeeze:
        gin = gin.unsqueeze(0)
    ninst = gin.shape[0]
    if tuple(gin.shape[1:]) != (6 * L + 3, plan.nlat, plan.nlon) or not gin.is_cuda or not gin.is_contiguous():
        raise ValueError(f"gin must be a contiguous CUDA tensor (ninst, {6 * L + 3}, {plan.nlat}, {plan.nlon})")
    prec = FP64 if gin.dtype == torch.float64 else FP32
    if gout is None:
        gout = torch.empty((ninst, 9 * L + 1, plan.nlat, plan.nlon), dtype=gin.dtype, device=gin.device)
    gout_v = gout.unsqueeze(0) if gout.dim() == 3 else gout
    if tuple(gout_v.shape) != (ninst, 9 * L + 1, plan.nlat, plan.nlon) or gout_v.dtype != gin.dtype:
        raise ValueError("gout has the wrong shape or dtype")
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    call("exotx_gridpoint", plan.handle, const._h, prec, ptr(gin), ptr(gout_v), ptr(dw), ptr(dq), ninst,
         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return gout_v[0] if squeeze else gout_v

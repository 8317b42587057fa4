"""exotx_forward_set_noalloc -- the forward transform set with its scratch
(Fourier intermediate and FFT twiddles) in a fixed array inside the library
instead of allocated device memory -- against exotx_forward_set, through the
C ABI.  The file name makes pytest collect it last; it passes alone in a
fresh process and after the other tests.

Tolerance: the transform tests' bars, max|x-ref|/max|ref| per field below
1e-12 (FP64) and 2e-5 (FP32).  Both entry points launch the same kernels on
the same twiddle values, so in practice they agree exactly.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from exoplasim_b200 import _lib
from exoplasim_b200 import synthetic as S
from exoplasim_b200.transforms import Plan
from tests._util import relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 2e-5}
PREC = {"fp64": 0, "fp32": 1, "mixed": 2}
DT = {"fp64": torch.float64, "fp32": torch.float32}
BAD_DIM, BAD_ARG = 1, 3


def _noalloc(P, prec, gin, out, nlev):
    """raw status of the C entry point"""
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.load().exotx_forward_set_noalloc(P._h, PREC[prec], C.c_void_p(gin.data_ptr()),
                                                 C.c_void_p(out.data_ptr()), nlev, s)


def _fields_close(a, b, tol):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    err = max(relerr(a[f], b[f]) for f in range(a.shape[0]))
    assert np.isfinite(err) and err < tol, err


@pytest.mark.parametrize("nlat,nlev,prec", [(32, 10, "fp64"), (64, 20, "fp64"), (32, 10, "fp32"),
                                            (96, 20, "fp32")])
def test_noalloc_matches_forward_set(nlat, nlev, prec):
    P = Plan(nlat)
    dt = DT[prec]
    gins = [torch.as_tensor(S.grid_tendencies(nlat, nlev, seed=sd), device="cuda").to(dt) for sd in (4, 5)]
    outs = [torch.full((4 * nlev + 1, P.nrsp), float("nan"), dtype=dt, device="cuda") for _ in gins]
    # two calls in a row on different inputs; the second must not see the first's scratch
    for g, o in zip(gins, outs):
        assert _noalloc(P, prec, g, o, nlev) == 0
    torch.cuda.synchronize()
    for g, o in zip(gins, outs):
        ref = P.forward_set(g, nlev, precision=prec)
        torch.cuda.synchronize()
        _fields_close(o, ref, TOL[prec])


def test_noalloc_alternating_grids_and_precisions():
    # the array keeps one set of twiddles; calls that switch grid length or
    # precision back and forth must each see their own
    runs = [(32, 10, "fp64"), (64, 10, "fp64"), (32, 10, "fp32"), (32, 10, "fp64"), (64, 10, "fp64")]
    plans = {n: Plan(n) for n in (32, 64)}
    for nlat, nlev, prec in runs:
        P = plans[nlat]
        g = torch.as_tensor(S.grid_tendencies(nlat, nlev, seed=nlat + nlev), device="cuda").to(DT[prec])
        o = torch.full((4 * nlev + 1, P.nrsp), float("nan"), dtype=DT[prec], device="cuda")
        assert _noalloc(P, prec, g, o, nlev) == 0
        ref = P.forward_set(g, nlev, precision=prec)
        torch.cuda.synchronize()
        _fields_close(o, ref, TOL[prec])


def test_noalloc_rejects_oversized_and_mixed():
    nlev = 20
    P = Plan(96)  # T63 L20 FP64 needs ~17.8 MB of scratch, above the 16 MiB array
    gin = torch.zeros((9 * nlev + 1, P.nlat, P.nlon), dtype=torch.float64, device="cuda")
    out = torch.full((4 * nlev + 1, P.nrsp), 7.0, dtype=torch.float64, device="cuda")
    assert _noalloc(P, "fp64", gin, out, nlev) == BAD_DIM
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())  # rejected before any work
    g32 = gin.float()
    o32 = out.float()
    assert _noalloc(P, "mixed", g32, o32, nlev) == BAD_ARG
    assert _noalloc(P, "fp64", gin, out, 0) == BAD_ARG


def test_noalloc_allocates_no_device_memory():
    nlat, nlev = 32, 10
    gin = torch.as_tensor(S.grid_tendencies(nlat, nlev, seed=6), device="cuda")
    A = Plan(nlat)
    ref = A.forward_set(gin, nlev, precision="fp64")   # loads the kernels the set launches
    out = torch.empty_like(ref)
    A.forward_set_noalloc(gin, nlev, out, precision="fp64")  # per-device set-up
    B = Plan(nlat)                                     # work buffer never grown
    out2 = torch.empty_like(ref)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    B.forward_set_noalloc(gin, nlev, out2, precision="fp64")
    B.forward_set_noalloc(gin, nlev, out2, precision="fp64")
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    _fields_close(out2, ref, TOL["fp64"])

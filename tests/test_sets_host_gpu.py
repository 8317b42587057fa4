"""exotx_sets_host: both transform sets for states in host memory, streamed
through device slots with copies and transforms overlapping.  Bar: the same
kernels run on the same data as the device-resident _batch calls, so the
outputs must be bit-identical to them, for every precision, for more groups
than device slots, for one half alone, and across repeated calls."""
import pytest
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200._lib import ExotxError
from exoplasim_b200.transforms import Plan

pytestmark = pytest.mark.gpu

DT = {"fp64": torch.float64, "fp32": torch.float32, "mixed": torch.float32}


def _host_states(P, nlev, ninst, dt, seed):
    spin = torch.stack([torch.as_tensor(S.transform_state(P.ntru, nlev, seed=seed + i, kind="nn1"))
                        for i in range(ninst)]).to(dt).contiguous().pin_memory()
    gin = torch.stack([torch.as_tensor(S.grid_tendencies(P.nlat, nlev, seed=seed + 50 + i))
                       for i in range(ninst)]).to(dt).contiguous().pin_memory()
    return spin, gin


@pytest.mark.parametrize("nlat,nlev,ninst,prec", [(32, 10, 5, "mixed"), (64, 20, 7, "mixed"), (32, 10, 4, "fp64"),
                                                  (64, 10, 3, "fp32")])
def test_host_sets_equal_device_batches(nlat, nlev, ninst, prec):
    P = Plan(nlat)
    dt = DT[prec]
    spin, gin = _host_states(P, nlev, ninst, dt, seed=nlat + ninst)
    gout = torch.full((ninst, 6 * nlev + 3, P.nlat, P.nlon), float("nan"), dtype=dt).pin_memory()
    sout = torch.full((ninst, 4 * nlev + 1, P.nrsp), float("nan"), dtype=dt).pin_memory()
    for _ in range(2):   # the second call reuses the slots
        P.sets_host(nlev, spin, gout, gin, sout, precision=prec)
        torch.cuda.current_stream().synchronize()
        ref_g = P.inverse_set_batch(spin.cuda(), nlev, precision=prec)
        ref_s = P.forward_set_batch(gin.cuda(), nlev, precision=prec)
        torch.cuda.synchronize()
        assert torch.equal(gout, ref_g.cpu())
        assert torch.equal(sout, ref_s.cpu())


def test_one_half_and_bad_arguments():
    P = Plan(32)
    nlev, ninst = 10, 3
    spin, gin = _host_states(P, nlev, ninst, torch.float32, seed=3)
    sout = torch.zeros((ninst, 4 * nlev + 1, P.nrsp)).pin_memory()
    P.sets_host(nlev, gpin=gin, spout=sout)
    torch.cuda.current_stream().synchronize()
    assert torch.equal(sout, P.forward_set_batch(gin.cuda(), nlev).cpu())
    with pytest.raises(TypeError):
        P.sets_host(nlev, spin.cuda(), None, None, None)
    gout = torch.zeros((ninst, 6 * nlev + 3, P.nlat, P.nlon)).pin_memory()
    with pytest.raises(ExotxError):   # a half with only one of its arrays
        P.sets_host(nlev, spin, None, gin, sout)
    P.sets_host(nlev, spin, gout)       # inverse half alone
    torch.cuda.current_stream().synchronize()
    assert torch.equal(gout, P.inverse_set_batch(spin.cuda(), nlev).cpu())


@pytest.mark.parametrize("nlat,nlev,ninst,prec", [(32, 10, 5, "mixed"), (64, 20, 3, "fp32"), (32, 10, 2, "fp64")])
def test_fp64_host_arrays(nlat, nlev, ninst, prec):
    # an 8-byte model's arrays: FP64 on the host whatever the transforms'
    # precision; the conversion on the device rounds to nearest, as torch does
    P = Plan(nlat)
    spin, gin = _host_states(P, nlev, ninst, torch.float64, seed=nlat + 7)
    gout = torch.full((ninst, 6 * nlev + 3, P.nlat, P.nlon), float("nan"), dtype=torch.float64).pin_memory()
    sout = torch.full((ninst, 4 * nlev + 1, P.nrsp), float("nan"), dtype=torch.float64).pin_memory()
    for _ in range(2):
        P.sets_host(nlev, spin, gout, gin, sout, precision=prec, host_fp64=True)
        torch.cuda.current_stream().synchronize()
        dt = DT[prec]
        ref_g = P.inverse_set_batch(spin.cuda().to(dt), nlev, precision=prec).double()
        ref_s = P.forward_set_batch(gin.cuda().to(dt), nlev, precision=prec).double()
        torch.cuda.synchronize()
        assert torch.equal(gout, ref_g.cpu())
        assert torch.equal(sout, ref_s.cpu())

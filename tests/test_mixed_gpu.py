"""Mixed precision (tcgen05, 3-term BF16 splits, FP32 accumulation) transform
sets against the FP64 oracle, through the C ABI.

Tolerance: <= 5e-6 norm-wise relative error per field (max|x-ref|/max|ref|)
and <= 1e-6 in the L2 norm (||x-ref||/||ref||), the same bars the FP32 SIMT
path meets; the tensor-core error word must stay 0.
"""
import numpy as np
import pytest
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200.transforms import Plan, tc_error
from tests._util import relerr

pytestmark = pytest.mark.gpu

FFTMOD_N = (8, 16, 32, 64, 96, 128, 256, 384, 512)


def _l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def plans():
    return {}


def _plan(plans, nlat):
    if nlat not in plans:
        plans[nlat] = Plan(nlat)
    return plans[nlat]


@pytest.mark.parametrize("nlat,nlev", [(32, 10), (64, 20), (96, 10), (192, 20), (256, 25)])
def test_mixed_sets_vs_oracle(plans, oracle, nlat, nlev):
    P = _plan(plans, nlat)
    L = oracle.Leg(nlat)
    use991 = 2 * nlat not in FFTMOD_N
    kind = "steep" if nlat >= 192 else "nn1"
    spin = S.transform_state(P.ntru, nlev, seed=3, kind=kind)
    gp = P.inverse_set(torch.as_tensor(spin, device="cuda").float(), nlev, precision="mixed")
    gp = gp.cpu().numpy().reshape(6 * nlev + 3, -1)
    ref = L.inverse_set(spin, nlev, plavor=S.EZ, use991=use991)
    e_max = max(relerr(gp[f], ref[f]) for f in range(6 * nlev + 3))
    e_l2 = max(_l2(gp[f], ref[f]) for f in range(6 * nlev + 3))
    assert e_max < 5e-6 and e_l2 < 1e-6, (e_max, e_l2)
    gin = S.grid_tendencies(nlat, nlev, seed=4)
    sp = P.forward_set(torch.as_tensor(gin, device="cuda").float(), nlev, precision="mixed").cpu().numpy()
    refs = L.forward_set(gin.reshape(9 * nlev + 1, -1), nlev, use991=use991)
    e_max = max(relerr(sp[f], refs[f]) for f in range(4 * nlev + 1))
    e_l2 = max(_l2(sp[f], refs[f]) for f in range(4 * nlev + 1))
    assert e_max < 5e-6 and e_l2 < 1e-6, (e_max, e_l2)
    assert tc_error() == 0


def test_mixed_batch_matches_single(plans):
    P = _plan(plans, 64)
    nlev, ninst = 10, 3
    spin = np.stack([S.transform_state(P.ntru, nlev, seed=10 + i) for i in range(ninst)])
    gin = np.stack([S.grid_tendencies(64, nlev, seed=20 + i) for i in range(ninst)])
    ts = torch.as_tensor(spin, device="cuda").float()
    tg = torch.as_tensor(gin, device="cuda").float()
    gb = P.inverse_set_batch(ts, nlev)
    sb = P.forward_set_batch(tg, nlev)
    for i in range(ninst):
        g1 = P.inverse_set(ts[i].contiguous(), nlev, precision="mixed")
        s1 = P.forward_set(tg[i].contiguous(), nlev, precision="mixed")
        assert torch.equal(gb[i], g1)
        assert torch.equal(sb[i], s1)
    assert tc_error() == 0

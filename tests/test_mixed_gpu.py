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


def _fp64_rounded_once(x, ref):
    # x is the FP64 value ref rounded once to the float32 output: within half
    # a float32 ulp of it (plus FP64 summation-order noise), where a sum in
    # FP32 or on the tensor cores lands several ulps away
    return abs(x - ref) <= 0.5 * float(np.spacing(np.float32(abs(ref)))) + 1e-14 * abs(ref)


@pytest.mark.parametrize("nlat", [64, 192])
def test_mixed_global_means_are_fp64(oracle, nlat):
    # the n = 0 coefficients of the forward set (temperature, humidity, ln ps
    # tendencies) are summed in FP64 on the mixed path and rounded once to the
    # float32 output; at NLON 384 from the row sums the forward FFT forms,
    # elsewhere from the grid
    nlev = 10
    P = Plan(nlat)
    L = oracle.Leg(nlat)
    gin = S.grid_tendencies(nlat, nlev, seed=21)
    gin[:nlev] += 0.3          # tn with a global mean well above its variance
    gin[7 * nlev] += 0.02      # gvpp
    g32 = torch.as_tensor(gin, device="cuda").float()
    refs = L.forward_set(g32.double().cpu().numpy().reshape(9 * nlev + 1, -1), nlev)
    sp = P.forward_set(g32, nlev, precision="mixed").double().cpu().numpy()
    for f in list(range(nlev, 2 * nlev)) + list(range(3 * nlev, 4 * nlev)) + [4 * nlev]:
        assert _fp64_rounded_once(sp[f][0], refs[f][0]), (f, sp[f][0], refs[f][0])
        assert sp[f][1] == 0.0
    # the vorticity and divergence have no n = 0 mode
    for f in list(range(0, nlev)) + list(range(2 * nlev, 3 * nlev)):
        assert sp[f][0] == 0.0 and sp[f][1] == 0.0


def test_mixed_d_set_global_means_are_fp64(oracle):
    # the gridpointd forward set's temperature and humidity tendencies
    # (fc2sp of gtdt, gqdt) carry FP64 n = 0 coefficients as well
    nlat, nlev = 64, 10
    P = Plan(nlat)
    L = oracle.Leg(nlat)
    rng = np.random.default_rng(22)
    gin = rng.standard_normal((4 * nlev, nlat, 2 * nlat)) * 1e-5
    gin[:nlev] += 2e-5          # gtdt with a nonzero global mean
    gin[3 * nlev:] += 1e-6      # gqdt
    g32 = torch.as_tensor(gin, device="cuda").float()
    refs = L.forward_set_d(g32.double().cpu().numpy().reshape(4 * nlev, -1), nlev)
    sp = P.forward_set_d(g32, nlev, precision="mixed").double().cpu().numpy()
    for f in list(range(nlev, 2 * nlev)) + list(range(3 * nlev, 4 * nlev)):
        assert _fp64_rounded_once(sp[f][0], refs[f][0]), (f, sp[f][0], refs[f][0])
        assert sp[f][1] == 0.0


def test_mixed_mass_drift_over_round_trips():
    # 1000 round trips of ln ps through the mixed sets (inverse: sp -> grid,
    # forward: grid as gvpp -> spf): the global mean drifts only by the float32
    # rounding of the grid values, as FP64 sums of them carry it
    nlat, nlev = 32, 1
    P = Plan(nlat)
    spin = torch.zeros((4 * nlev + 1, P.nrsp), device="cuda")
    rng = np.random.default_rng(4)
    sp0 = S.spectral_field(rng, P.ntru, 1, "nn1")[0]
    sp0[0] = 11.5 * np.sqrt(2.0)     # ln(1e5 Pa) in the n = 0 mode
    spin[4 * nlev] = torch.as_tensor(sp0, device="cuda").float()
    gin = torch.zeros((9 * nlev + 1, nlat, 2 * nlat), device="cuda")
    start = float(spin[4 * nlev, 0])
    for _ in range(1000):
        g = P.inverse_set(spin, nlev, precision="mixed")
        gin[7 * nlev] = g[6 * nlev + 2]
        out = P.forward_set(gin, nlev, precision="mixed")
        spin[4 * nlev] = out[4 * nlev]
    drift = abs(float(spin[4 * nlev, 0]) - start) / abs(start)
    assert drift < 2e-7, drift

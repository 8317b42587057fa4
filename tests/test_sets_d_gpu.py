"""The gridpointd transform sets (plasim.f90:3142-3149, :3415-3428) through
the C ABI against the FP64 oracle's composition of invlegd, fc2gp, gp2fc,
fc2sp and uv2dv.

Bars, per field (max|x-ref|/max|ref|): FP64 <= 1e-12, FP32 <= 1e-5, mixed
(tensor cores, 3-term BF16 splits) <= 5e-6 max and <= 1e-6 in the L2 norm."""
import numpy as np
import pytest
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200.transforms import Plan
from tests._util import relerr

pytestmark = pytest.mark.gpu

DT = {"fp64": torch.float64, "fp32": torch.float32, "mixed": torch.float32}
TOL = {"fp64": 1e-12, "fp32": 1e-5, "mixed": 5e-6}
DIRECT = (8, 16, 32, 64, 96, 128, 256, 384, 512)   # fftmod lengths; others FFT991


def _l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _tend(nlat, nlev, seed):
    g = S.grid_tendencies(nlat, nlev, seed=seed)      # (9L+1, nlat, nlon)
    return np.ascontiguousarray(g[:4 * nlev])


@pytest.mark.parametrize("nlat,nlev,prec", [(32, 10, "fp64"), (64, 20, "fp64"), (96, 10, "fp64"),
                                            (32, 10, "fp32"), (64, 20, "fp32"),
                                            (32, 10, "mixed"), (64, 20, "mixed"), (96, 15, "mixed"),
                                            (192, 20, "mixed"), (256, 25, "mixed")])
def test_sets_d_match_oracle(oracle, nlat, nlev, prec):
    P = Plan(nlat)
    L = oracle.Leg(nlat)
    use991 = 2 * nlat not in DIRECT
    dt = DT[prec]
    kind = "steep" if nlat >= 192 else "nn1"
    ninst = 2
    spins = [S.transform_state(P.ntru, nlev, seed=40 + i, kind=kind) for i in range(ninst)]
    gins = [_tend(nlat, nlev, 60 + i) for i in range(ninst)]
    sp_t = torch.as_tensor(np.stack(spins), device="cuda").to(dt)
    gi_t = torch.as_tensor(np.stack(gins), device="cuda").to(dt)
    gp = P.inverse_set_d_batch(sp_t, nlev, precision=prec).double().cpu().numpy()
    so = P.forward_set_d_batch(gi_t, nlev, precision=prec).double().cpu().numpy()
    for i in range(ninst):
        ref = L.inverse_set_d(spins[i], nlev, plavor=S.EZ, use991=use991)
        refs = L.forward_set_d(gins[i].reshape(4 * nlev, -1), nlev, use991=use991)
        g = gp[i].reshape(4 * nlev + 1, -1)
        for f in range(4 * nlev + 1):
            assert relerr(g[f], ref[f]) < TOL[prec], (i, f)
            if prec == "mixed":
                assert _l2(g[f], ref[f]) < 1e-6, (i, f)
        for f in range(4 * nlev):
            assert relerr(so[i][f], refs[f]) < TOL[prec], (i, f)
            if prec == "mixed":
                assert _l2(so[i][f], refs[f]) < 1e-6, (i, f)
    # the forward set leaves its input alone
    assert torch.equal(gi_t.cpu(), torch.as_tensor(np.stack(gins)).to(dt))


def test_single_state_forms_equal_batch():
    P = Plan(64)
    nlev = 5
    sp = torch.as_tensor(S.transform_state(P.ntru, nlev, seed=3), device="cuda")
    gi = torch.as_tensor(_tend(64, nlev, 4), device="cuda")
    for prec in ("fp64", "mixed"):
        dt = DT[prec]
        a = P.inverse_set_d(sp.to(dt), nlev, precision=prec)
        b = P.inverse_set_d_batch(sp.to(dt).unsqueeze(0), nlev, precision=prec)[0]
        assert torch.equal(a, b)
        c = P.forward_set_d(gi.to(dt), nlev, precision=prec)
        d = P.forward_set_d_batch(gi.to(dt).unsqueeze(0), nlev, precision=prec)[0]
        assert torch.equal(c, d)

"""The grid-point step of gridpointa (plasim.f90:2441-2455: exp of ln ps,
calcgp :2587-2755, the flux products) through the C ABI against the FP64
oracle (oracle/exo_oracle_gp.c), and the whole gridpointa transform path
inverse set -> grid-point step -> forward set against the oracle's chain.

Bars: the constants of the semi-implicit scheme (initsi) equal the oracle's
to rounding (CPU).  FP64 grid-point step <= 1e-12 per output field
(max|x-ref|/max|ref|); FP32 <= 1e-4 (it subtracts nearly equal terms, e.g.
(gt + t0)(1 + ...) - t0).  The chained FP64 path <= 1e-11."""
import numpy as np
import pytest
import torch

from exoplasim_b200 import gridpoint as GP
from exoplasim_b200 import synthetic as S
from tests._util import relerr


def test_initsi_constants_match_oracle(oracle):
    for nlev in (5, 10, 20, 25):
        p = GP.default_params(nlev)
        L = nlev
        t0 = np.array(p.t0[:L])
        g, c, tkp, t01s2, rdsig = oracle.initsi(np.array(p.sigmah[:L]), np.array(p.dsigma[:L]), t0, p.akap)
        gg = np.array(p.g[:L * L]).reshape(L, L, order="F")
        cc = np.array(p.c[:L * L]).reshape(L, L, order="F")
        assert np.allclose(gg, g, rtol=1e-15, atol=0) and np.allclose(cc, c, rtol=1e-15, atol=0)
        assert np.allclose(np.array(p.tkp[:L]), tkp, rtol=1e-15, atol=0)
        assert np.allclose(np.array(p.t01s2[:L]), t01s2, rtol=0, atol=1e-16)
        assert np.allclose(np.array(p.rdsig[:L]), rdsig, rtol=1e-15, atol=0)
        # t0 is a positive decreasing-upward profile in model units
        assert np.all(t0 > 0)


def _inputs(oracle, P, nlev, seed):
    """grid fields from the FP64 inverse set of a synthetic state: (6L+3, nhor)"""
    L = oracle.Leg(P.nlat)
    spin = S.transform_state(P.ntru, nlev, seed=seed)
    spin[4 * nlev, 0] = 0.1          # ln(ps/psurf)-like mean for the exp
    return L.inverse_set(spin, nlev, plavor=S.EZ), spin


def _oracle_step(oracle, p, gin, nlat, nlev, sid, nqspec=1, dq=None):
    rcsq = 1.0 / (1.0 - sid * sid)
    L = nlev
    return oracle.gridpoint(gin, L, 2 * nlat, np.array(p.sigmah[:L]), np.array(p.dsigma[:L]), np.array(p.t0[:L]),
                            p.akap, p.rdbrv, p.adv, p.psurf, p.ww, rcsq, nqspec=nqspec, dq=dq)


@pytest.mark.gpu
@pytest.mark.parametrize("nlat,nlev,nqspec", [(32, 10, 1), (64, 20, 1), (32, 10, 0), (96, 15, 1), (32, 25, 1)])
def test_gridpoint_fp64_fp32(oracle, nlat, nlev, nqspec):
    from exoplasim_b200.transforms import Plan
    P = Plan(nlat)
    p = GP.default_params(nlev, nqspec=nqspec)
    const = GP.GpConst(p)
    gin, _ = _inputs(oracle, P, nlev, seed=nlat + nlev)
    sid, _ = P.gauss()
    dq = np.abs(np.random.default_rng(2).standard_normal((nlev, gin.shape[1]))) * 1e-3 if nqspec == 0 else None
    ref, ref_dw = _oracle_step(oracle, p, gin, nlat, nlev, sid, nqspec, dq)
    gt = torch.as_tensor(gin.reshape(1, 6 * nlev + 3, nlat, 2 * nlat), device="cuda")
    dqt = None if dq is None else torch.as_tensor(dq.reshape(1, nlev, nlat, 2 * nlat), device="cuda")
    dw = torch.zeros((1, nlev, nlat, 2 * nlat), dtype=torch.float64, device="cuda")
    out = GP.gridpoint(P, const, gt, dw=dw, dq=dqt).cpu().numpy().reshape(9 * nlev + 1, -1)
    for f in range(9 * nlev + 1):
        assert relerr(out[f], ref[f]) < 1e-12, f
    assert relerr(dw.cpu().numpy().reshape(nlev, -1), ref_dw) < 1e-12
    out32 = GP.gridpoint(P, const, gt.float(), dq=None if dqt is None else dqt.float()).double().cpu().numpy()
    out32 = out32.reshape(9 * nlev + 1, -1)
    errs = [relerr(out32[f], ref[f]) for f in range(9 * nlev + 1)]
    assert max(errs) < 1e-4, int(np.argmax(errs))


@pytest.mark.gpu
def test_gridpointa_transform_path_fp64(oracle):
    # inverse set -> grid-point step -> forward set, all on the device, against
    # the oracle's inverse_set -> gridpoint -> forward_set
    from exoplasim_b200.transforms import Plan
    nlat, nlev = 64, 10
    P = Plan(nlat)
    p = GP.default_params(nlev)
    const = GP.GpConst(p)
    L = oracle.Leg(nlat)
    spin = S.transform_state(P.ntru, nlev, seed=5)
    spin[4 * nlev, 0] = 0.1
    sid, _ = P.gauss()
    g_ref = L.inverse_set(spin, nlev, plavor=S.EZ)
    t_ref, _ = _oracle_step(oracle, p, g_ref, nlat, nlev, sid)
    s_ref = L.forward_set(t_ref, nlev)
    sp = torch.as_tensor(spin, device="cuda")
    g = P.inverse_set(sp, nlev)
    t = GP.gridpoint(P, const, g)
    s_out = P.forward_set(t, nlev).cpu().numpy()
    for f in range(4 * nlev + 1):
        assert relerr(s_out[f], s_ref[f]) < 1e-11, f

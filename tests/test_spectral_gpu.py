"""The semi-implicit spectral step (plasim.f90 spectrala :2757-2918,
spectrald :3645-3999) through the C ABI against the FP64 oracle
(oracle/exo_oracle_spec.c), on a synthetic model state.

Bars: FP64 <= 1e-12 per updated array (max|x-ref|/max|ref|; bm1 is
inverted by different methods on the two sides); FP32 <= 1e-4 (the implicit
solve and the time filter subtract nearly equal terms).  The surface
pressure's mass-carrying coefficients stay exactly zero."""
import numpy as np
import pytest
import torch

from exoplasim_b200 import spectral as SP
from exoplasim_b200 import synthetic as S
from tests._util import relerr

pytestmark = pytest.mark.gpu


def _state(ntru, nlev, seed):
    rng = np.random.default_rng(seed)
    f = lambda k=1: S.spectral_field(rng, ntru, k, "nn1")  # noqa: E731
    st = {}
    for k in ("sdp", "szp", "stp", "sqp", "sdm", "szm", "stm", "sqm", "srp"):
        st[k] = f(nlev)
    for k in ("sdt", "szt", "stt", "sqt"):
        st[k] = f(nlev) * 0.05
    for k in ("spp", "spm", "sop"):
        st[k] = f(1)[0]
    st["spt"] = f(1)[0] * 0.05
    return st


def _pdict(p):
    d = {k: getattr(p, k) for k in ("nlev", "nqspec", "nsponge", "nhdiff", "delt", "delt2", "pnu", "pnu21",
                                    "plavor", "dampsp", "akap")}
    for k in ("t0", "sigmah", "dsigma", "damp", "tdisst", "tdissq", "tdissd", "tdissz", "tfrc"):
        d[k] = np.array(getattr(p, k)[:p.nlev])
    d["ndel"] = list(p.ndel[:p.nlev])
    return d


@pytest.mark.parametrize("nlat,nlev,over", [(32, 10, {}), (64, 20, {}),
                                            (32, 10, {"nsponge": 1, "dampsp": 0.3, "nqspec": 0}),
                                            (32, 10, {"damp": [0.05] * 10})])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_spectral_step_matches_oracle(oracle, nlat, nlev, over, prec):
    from exoplasim_b200.transforms import Plan
    P = Plan(nlat)
    p = SP.default_params(nlev, **over)
    const = SP.SpecConst(P, p)
    st = _state(P.ntru, nlev, seed=nlat + nlev)
    dt = torch.float64 if prec == "fp64" else torch.float32
    tol = 1e-12 if prec == "fp64" else 1e-4
    dev = {k: torch.as_tensor(v, device="cuda").to(dt).contiguous() for k, v in st.items()}
    ref_a = oracle.spectral_step("a", _pdict(p), P.ntru, st)
    SP.spectrala(const, dev)
    got = {k: v.double().cpu().numpy() for k, v in dev.items()}
    for k in ("sdp", "szp", "stp", "spp", "sdm", "szm", "stm", "spm", "sdt", "stt", "spt") + \
            (("sqp", "sqm") if p.nqspec == 1 else ()):
        assert relerr(got[k], ref_a[k]) < tol, ("a", k)
    assert got["spp"][0] == 0.0 and got["spp"][1] == 0.0
    # the diabatic part on the updated state, with new tendencies
    rng = np.random.default_rng(7)
    for k in ("sdt", "szt", "stt", "sqt"):
        ref_a[k] = S.spectral_field(rng, P.ntru, nlev, "nn1") * 0.05
        dev[k].copy_(torch.as_tensor(ref_a[k]).to(dt))
    ref_d = oracle.spectral_step("d", _pdict(p), P.ntru, ref_a)
    SP.spectrald(const, dev)
    got = {k: v.double().cpu().numpy() for k, v in dev.items()}
    for k in ("sdp", "szp", "stp", "spp", "sdm", "szm", "stm", "spm", "sdt", "szt", "stt") + \
            (("sqp", "sqm", "sqt") if p.nqspec == 1 else ()):
        assert relerr(got[k], ref_d[k]) < tol, ("d", k)
    assert got["spp"][0] == 0.0 and got["spp"][1] == 0.0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_spectral_batch_equals_single_calls(prec):
    # exotx_spectrala_batch / exotx_spectrald_batch over 13 states (two
    # launches of up to 12) give each state what a single call gives
    from exoplasim_b200.transforms import Plan
    P = Plan(32)
    nlev, n = 10, 13
    const = SP.SpecConst(P, SP.default_params(nlev, nsponge=1, dampsp=0.3))
    dt = torch.float64 if prec == "fp64" else torch.float32
    states = [{k: torch.as_tensor(v, device="cuda").to(dt).contiguous() for k, v in _state(P.ntru, nlev, 50 + i).items()}
              for i in range(n)]
    single = [{k: v.clone() for k, v in st.items()} for st in states]
    SP.spectrala_batch(const, states)
    SP.spectrald_batch(const, states)
    for st in single:
        SP.spectrala(const, st)
        SP.spectrald(const, st)
    torch.cuda.synchronize()
    for a, b in zip(states, single):
        for k in a:
            assert torch.equal(a[k], b[k]), k

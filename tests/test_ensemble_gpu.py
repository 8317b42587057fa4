"""Uneven ensembles (T21/T42/T63 x 10/15/20 levels) in one tensor-core launch
and one FFT launch per half of the round trip.

Bars: every instance equals the single-resolution batched path bit for bit
(the same jobs on the same kernels); one instance per resolution meets the
mixed-precision bars against the FP64 oracle (5e-6 max-norm, 1e-6 L2 per
field); a round trip is four kernel launches and replays as a CUDA graph;
the autotuner keeps the 3-term split (the 2-term split misses 1e-6).
"""
import numpy as np
import pytest
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200.ensemble import Ensemble, draw
from exoplasim_b200.transforms import Plan, launch_count
from tests._util import relerr

pytestmark = pytest.mark.gpu

FFTMOD_N = (8, 16, 32, 64, 96, 128, 256, 384, 512)


def _inputs(E, seed):
    spins, gins = [], []
    for i, (nlat, L) in enumerate(zip(E.nlat, E.nlev)):
        ntru = (2 * nlat - 1) // 3
        spins.append(torch.as_tensor(S.transform_state(ntru, L, seed=seed + i, kind="nn1"), device="cuda").float())
        gins.append(torch.as_tensor(S.grid_tendencies(nlat, L, seed=seed + 100 + i), device="cuda").float())
    return spins, gins


@pytest.fixture(scope="module")
def ens():
    nlat, nlev = draw(12, seed=4)
    nlat[:3], nlev[:3] = [32, 64, 96], [10, 15, 20]   # every resolution and level count appears
    E = Ensemble(nlat, nlev)
    spins, gins = _inputs(E, 10)
    spin, gin = E.pack("spec", spins), E.pack("gin", gins)
    _, gout, _, spout = E.buffers()
    E.inverse(spin, gout)
    E.forward(gin, spout)
    torch.cuda.synchronize()
    return E, spins, gins, spin, gin, gout.clone(), spout.clone()


def test_ensemble_equals_single_resolution_batches(ens):
    E, spins, gins, _, _, gout, spout = ens
    gouts, spouts = E.unpack("gout", gout), E.unpack("spec", spout)
    plans = {}
    for i, (nlat, L) in enumerate(zip(E.nlat, E.nlev)):
        P = plans.setdefault(nlat, Plan(nlat))
        g = P.inverse_set_batch(spins[i].unsqueeze(0).contiguous(), L, precision="mixed")[0]
        s = P.forward_set_batch(gins[i].unsqueeze(0).contiguous(), L, precision="mixed")[0]
        torch.cuda.synchronize()
        assert torch.equal(gouts[i], g), i
        assert torch.equal(spouts[i], s), i


def test_ensemble_vs_oracle(ens, oracle):
    E, spins, gins, _, _, gout, spout = ens
    gouts, spouts = E.unpack("gout", gout), E.unpack("spec", spout)
    for i in range(3):  # one instance of each resolution
        nlat, L = E.nlat[i], E.nlev[i]
        Lg = oracle.Leg(nlat)
        use991 = 2 * nlat not in FFTMOD_N
        ref = Lg.inverse_set(spins[i].double().cpu().numpy(), L, plavor=S.EZ, use991=use991)
        got = gouts[i].cpu().numpy().reshape(6 * L + 3, -1)
        assert max(relerr(got[f], ref[f]) for f in range(6 * L + 3)) < 5e-6
        refs = Lg.forward_set(gins[i].double().cpu().numpy().reshape(9 * L + 1, -1), L, use991=use991)
        gots = spouts[i].cpu().numpy()
        assert max(relerr(gots[f], refs[f]) for f in range(4 * L + 1)) < 5e-6
        l2 = max(float(np.linalg.norm(gots[f] - refs[f]) / max(np.linalg.norm(refs[f]), 1e-300))
                 for f in range(4 * L + 1))
        assert l2 < 1e-6


def test_ensemble_is_four_launches_and_replays_as_graph(ens):
    E, _, _, spin, gin, gout_ref, spout_ref = ens
    _, gout, _, spout = E.buffers()
    n0 = launch_count()
    E.inverse(spin, gout)
    E.forward(gin, spout)
    torch.cuda.synchronize()
    assert launch_count() - n0 == 5
    gout.zero_()
    spout.zero_()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            E.inverse(spin, gout)
            E.forward(gin, spout)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(gout, gout_ref) and torch.equal(spout, spout_ref)
    del g


def test_autotuner_keeps_the_three_term_split(ens):
    E, _, _, spin, gin, gout_ref, spout_ref = ens
    _, gout, _, spout = E.buffers()
    ch = E.tune(spin, gout, gin, spout, reps=2)
    assert ch["nprod"] == 6 and ch["ms"] > 0
    gout.zero_()
    spout.zero_()
    E.inverse(spin, gout)
    E.forward(gin, spout)
    torch.cuda.synchronize()
    assert torch.equal(gout, gout_ref) and torch.equal(spout, spout_ref)
    E.configure()


def test_ensemble_with_a_t127_segment():
    # a T127 segment runs the register-resident FFT bodies in a launch of their
    # own (seven launches per round trip); its instances still equal the
    # single-resolution batched path bit for bit
    E = Ensemble([192, 32, 64], [20, 10, 15])
    spins, gins = _inputs(E, 40)
    spin, gin = E.pack("spec", spins), E.pack("gin", gins)
    _, gout, _, spout = E.buffers()
    n0 = launch_count()
    E.inverse(spin, gout)
    E.forward(gin, spout)
    torch.cuda.synchronize()
    assert launch_count() - n0 == 7
    gouts, spouts = E.unpack("gout", gout), E.unpack("spec", spout)
    for i, (nlat, L) in enumerate(zip(E.nlat, E.nlev)):
        P = Plan(nlat)
        g = P.inverse_set_batch(spins[i].unsqueeze(0).contiguous(), L, precision="mixed")[0]
        s = P.forward_set_batch(gins[i].unsqueeze(0).contiguous(), L, precision="mixed")[0]
        torch.cuda.synchronize()
        assert torch.equal(gouts[i], g), i
        assert torch.equal(spouts[i], s), i

"""Radiation surrogate: training kernels against the FP64 numpy oracle, the
tensor-core inference against the FP32 network, the out-of-range fallback
against plain radstep, and what the trained network gains over baselines.

Tolerances: FP32 forward and gradients vs FP64 within 1e-4 relative
(max-norm); one Adam step within 1e-5; BF16 tensor-core inference within
0.05 (max) and 0.01 (RMS) of the FP32 network in normalised output units;
fallback columns equal to plain radstep to 1e-12.
"""
import os

import numpy as np
import pytest
import torch

from exoplasim_b200 import radiation as R
from exoplasim_b200 import surrogate as SG

pytestmark = pytest.mark.gpu

L = 20
NIN, NOUT = SG.nin_for(L), SG.nout_for(L)


def _relmax(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def chunk():
    params, dev = SG.column_chunk(L, seed=77)
    X = SG.features(params, dev)
    Y, cols, out = SG.plain_targets(params, dev)
    return params, dev, X, Y, cols, out


def test_features_match_numpy(chunk):
    """exotx_surr_features against the feature list restated in numpy."""
    params, dev, X, _, _, _ = chunk
    c = {k: v.cpu().numpy() for k, v in dev.items()}
    n = params.nhor
    lq = np.log(np.maximum(c["dq"][:L + 1], 1e-12))
    ref = np.concatenate([
        c["dt"][:L + 1],
        lq,
        c["dcc"][:L],
        np.log(np.maximum(c["dp"], 1.0))[None],
        c["dalb"][None], c["gmu0"][None],
        np.log(np.maximum(c["dqco2"][0], 1e-6))[None],
        c["zsol"][0][None], c["zsol"][2][None],
        c["sid"][np.arange(n) // params.nlon][None],
    ]).T
    assert ref.shape == (n, NIN)
    np.testing.assert_allclose(X.double().cpu().numpy(), ref, rtol=2e-6, atol=5e-5)


@pytest.mark.parametrize("width,nhid,n", [(32, 2, 64), (256, 6, 256), (64, 2, 1100)])
def test_forward_and_gradients_vs_oracle(width, nhid, n):
    from oracle import mlp_oracle as MO
    net = SG.Mlp(NIN, NOUT, width=width, nhidden=nhid, max_batch=n)
    net.init(seed=3)
    g = np.random.default_rng(5)
    X = g.standard_normal((n, NIN)).astype(np.float32)
    T = g.standard_normal((n, NOUT)).astype(np.float32)
    Xd = torch.as_tensor(X, device="cuda")
    Td = torch.as_tensor(T, device="cuda")
    params = net.params.cpu().numpy()
    Yref, _, _ = MO.forward(params, net.layers, X)
    Y = net.forward(Xd).cpu().numpy()
    assert _relmax(Y, Yref) < 1e-4
    loss = torch.zeros(1, device="cuda")
    net.backward(Xd, Td, loss)
    lref, gref = MO.loss_and_grads(params, net.layers, X, T)
    torch.cuda.synchronize()
    assert abs(loss.item() - lref) / lref < 1e-4
    G = net.grads.cpu().numpy()
    for wo, bo, di, do in net.layers:   # per tensor, so small layers are not hidden by large ones
        assert _relmax(G[wo:wo + di * do], gref[wo:wo + di * do]) < 1e-4
        assert _relmax(G[bo:bo + do], gref[bo:bo + do]) < 1e-4
    # one Adam step
    m0 = np.zeros_like(params)
    pref, _, _ = MO.adam(params, G.astype(np.float64), m0, m0.copy(), 1e-3, 1)
    net.adam(1e-3, 1)
    assert _relmax(net.params.cpu().numpy(), pref) < 1e-5


def test_weighted_gradients_vs_oracle():
    # the loss in judged units: every element's squared error weighted
    from oracle import mlp_oracle as MO
    n = 128
    net = SG.Mlp(NIN, NOUT, width=32, nhidden=2, max_batch=n)
    net.init(seed=4)
    g = np.random.default_rng(6)
    X = g.standard_normal((n, NIN)).astype(np.float32)
    T = g.standard_normal((n, NOUT)).astype(np.float32)
    W = g.uniform(0.1, 10.0, (n, NOUT)).astype(np.float32)
    params = net.params.cpu().numpy()
    loss = torch.zeros(1, device="cuda")
    net.backward(torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda"), loss,
                 torch.as_tensor(W, device="cuda"))
    lref, gref = MO.loss_and_grads(params, net.layers, X, T, W)
    torch.cuda.synchronize()
    assert abs(loss.item() - lref) / lref < 1e-4
    G = net.grads.cpu().numpy()
    for wo, bo, di, do in net.layers:
        assert _relmax(G[wo:wo + di * do], gref[wo:wo + di * do]) < 1e-4
        assert _relmax(G[bo:bo + do], gref[bo:bo + do]) < 1e-4


def test_training_reduces_loss(chunk):
    params, dev, X, Y, _, _ = chunk
    net = SG.Mlp(NIN, NOUT, max_batch=1024)
    net.init(seed=0)
    net.set_norm(*SG.norm_stats(X, Y))
    hist = SG.train(net, X, Y, epochs=10, batch=1024, lr=1e-3)
    assert hist[-1] < 0.75 * hist[0] and all(b < a for a, b in zip(hist, hist[1:])), hist


def test_tensor_core_inference_matches_fp32_network(chunk):
    params, dev, X, Y, _, _ = chunk
    net = SG.Mlp(NIN, NOUT, max_batch=params.nhor)
    net.init(seed=11)
    net.set_norm(*SG.norm_stats(X, Y))
    net.prepare()
    cols = {k: v.clone() for k, v in dev.items()}
    cols["dtdt"].zero_()
    out = R.alloc_outputs(params, torch.float64)
    nfb = SG.surrogate_step(net, params, cols, out, count=True)
    assert nfb == 0  # the ranges come from these very columns
    n = net.norm
    Xn = (X - torch.as_tensor(n["xm"], device="cuda")) / torch.as_tensor(n["xs"], device="cuda")
    Yn = net.forward(Xn.contiguous())
    ref = Yn.double() * torch.as_tensor(n["ys"], device="cuda").double() + torch.as_tensor(n["ym"], device="cuda").double()
    hs = SG.heating_scale(X, L, params.adv)
    got = torch.cat([cols["dtdt"].T * 86400.0 * hs,
                     torch.stack([out["dfd"][L], out["dfu"][L], out["dftd"][L], out["dftu"][L]], 1)], 1)
    err = (got - ref) / torch.as_tensor(n["ys"], device="cuda").double()
    assert float(err.abs().max()) < 0.05 and float(err.pow(2).mean().sqrt()) < 0.01
    # net surface fluxes are the sums of the predicted components
    assert torch.allclose(out["dswfl"][L], out["dfd"][L] + out["dfu"][L], rtol=1e-6, atol=1e-9)


def test_out_of_range_columns_fall_back_to_radstep(chunk):
    params, dev, X, Y, pcols, pout = chunk
    net = SG.Mlp(NIN, NOUT, max_batch=64)
    net.init(seed=2)
    net.set_norm(*SG.norm_stats(X, Y))
    net.prepare()
    cols = {k: v.clone() for k, v in dev.items()}
    hot = torch.arange(5, params.nhor, 997, device="cuda")
    cols["dt"][:, hot] = 400.0          # outside the 150-350 K training range
    plain = {k: v.clone() for k, v in cols.items()}
    plain["dtdt"].zero_()
    pout2 = R.radstep(params, plain)
    cols["dtdt"].zero_()
    out = R.alloc_outputs(params, torch.float64)
    nfb = SG.surrogate_step(net, params, cols, out, count=True)
    assert nfb == hot.numel()
    for k in ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux", "dtdtswr", "dtdtlwr", "dconv"):
        a, b = out[k][:, hot], pout2[k][:, hot]
        assert float((a - b).abs().max()) <= 1e-12 * max(float(b.abs().max()), 1.0), k
    assert float((cols["dtdt"][:, hot] - plain["dtdt"][:, hot]).abs().max()) <= 1e-15


@pytest.mark.skipif(not os.path.exists(SG.DEFAULT_NET), reason="no trained network in the package")
def test_trained_network_beats_baselines():
    """Ablation: the trained network against what one gets without it -- the
    per-level mean heating rate of the training set, and a linear least-squares
    model of the same features fitted on 32768 training columns."""
    net = SG.Mlp.load(SG.DEFAULT_NET)
    net.prepare()
    ev = SG.evaluate(net, L, nchunk=2)
    Xt, Yt = SG.dataset(4 * 8192, L, seed=1000)
    Xe, Ye = SG.dataset(2 * 8192, L, seed=900000)
    # baselines predict the network's target; compare all in heating rate (K/day)
    adv = R.default_params(L, 8192, 128).adv
    st = SG.heating_scale(Xt, L, adv).cpu().numpy()
    se = SG.heating_scale(Xe, L, adv).cpu().numpy()
    xt = Xt.double().cpu().numpy()
    yt = Yt[:, :L].double().cpu().numpy()
    xe = Xe.double().cpu().numpy()
    ye = Ye[:, :L].double().cpu().numpy() / se
    mean_rms = float(np.sqrt(((ye - yt.mean(0) / se) ** 2).mean()))
    A = np.hstack([xt, np.ones((xt.shape[0], 1))])
    coef, *_ = np.linalg.lstsq(A, yt, rcond=None)
    lin = (np.hstack([xe, np.ones((xe.shape[0], 1))]) @ coef) / se
    lin_rms = float(np.sqrt(((ye - lin) ** 2).mean()))
    print(f"heating RMS K/day: network {ev['heating_rms_K_per_day']:.4f}  linear {lin_rms:.4f}  "
          f"mean {mean_rms:.4f}; fallback {ev['fallback_fraction']:.4f}")
    assert ev["heating_rms_K_per_day"] < 0.5 * lin_rms
    assert ev["heating_rms_K_per_day"] < 0.2 * mean_rms
    # the evaluation columns (drawn level by level, as the radiation benchmark
    # specifies them) are all inside the training ranges
    assert ev["fallback_fraction"] == 0.0

"""Host-side pieces of the radiation surrogate that need no GPU: the heating
scale recovered from the raw features, the per-element weights of the K/day
loss, and the normalisation ranges that the out-of-range test uses."""
import numpy as np
import torch

from exoplasim_b200 import surrogate as SG
from exoplasim_b200 import synthetic as S

L = 10
ADV = 0.6078


def _raw_features(cols):
    """The feature layout of exotx_surr_features, restated for host arrays
    (T, ln q, cc per level, then ln ps, albedo, cos zenith, ln CO2, two star
    constants, sin latitude)."""
    n = cols["dp"].size
    nlon = n // cols["sid"].size
    lq = np.log(np.maximum(cols["dq"][:L + 1], 1e-12))
    return np.concatenate([
        cols["dt"][:L + 1], lq, cols["dcc"][:L],
        np.log(np.maximum(cols["dp"], 1.0))[None], cols["dalb"][None], cols["gmu0"][None],
        np.log(np.maximum(cols["dqco2"][0], 1e-6))[None], np.full((1, n), 0.8), np.full((1, n), 0.01),
        cols["sid"][np.arange(n) // nlon][None],
    ]).T


def test_heating_scale_from_features():
    cols, _ = S.radiation_columns(8, L, seed=41)
    X = torch.as_tensor(_raw_features(cols), dtype=torch.float32)
    assert X.shape[1] == SG.nin_for(L)
    hs = SG.heating_scale(X, L, ADV).numpy()
    ref = (cols["dp"] / 1e5)[:, None] * (1.0 + ADV * cols["dq"][:L].T)
    np.testing.assert_allclose(hs, ref, rtol=2e-6)


def test_judged_weights_are_the_kday_factors():
    cols, _ = S.radiation_columns(8, L, seed=42)
    X = torch.as_tensor(_raw_features(cols), dtype=torch.float32)
    ys = torch.linspace(0.5, 2.0, SG.nout_for(L))
    W = SG.judged_weights(X, L, ys, ADV)
    assert W.shape == (X.shape[0], SG.nout_for(L))
    assert abs(float(W.mean()) - 1.0) < 1e-5
    hs = SG.heating_scale(X, L, ADV).float()
    raw = torch.cat([(ys[:L] / hs) ** 2, (0.1 * ys[L:]).expand(X.shape[0], 4) ** 2], 1)
    # the weights are these factors, scaled to mean 1
    np.testing.assert_allclose((W / raw).numpy(), float((W / raw)[0, 0]), rtol=2e-5)


def test_norm_ranges_enclose_the_training_columns():
    rng = np.random.default_rng(3)
    X = torch.as_tensor(rng.normal(size=(500, 7)), dtype=torch.float32)
    Y = torch.as_tensor(rng.normal(size=(500, 3)), dtype=torch.float32)
    xm, xs, lo, hi, ym, ys = SG.norm_stats(X, Y)
    x = X.numpy()
    assert np.all(lo < x.min(0)) and np.all(hi > x.max(0))
    np.testing.assert_allclose(hi - lo, (x.max(0) - x.min(0)) * 1.04 + 2e-6, rtol=1e-5)
    np.testing.assert_allclose(xm, x.mean(0), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(ys, Y.numpy().std(0, ddof=1), rtol=1e-5)

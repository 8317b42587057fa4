"""CPU checks of the FP64 oracle: known answers and independent implementations.

The reference ships no golden vectors for these routines and no Fortran
compiler exists here, so the oracle is pinned by (a) mathematical identities
the reference's algorithms must satisfy, (b) fixtures from numpy/scipy
(tests/golden/, made by tests/golden/make_golden.py) and (c) for the
longwave scheme, a second restatement written separately in numpy
(oracle/lwr_numpy.py).
"""
import math
import os

import numpy as np
import pytest

from exoplasim_b200 import synthetic as S
from tests._util import relerr

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_v1.npz")


@pytest.mark.parametrize("nlat", [8, 32, 64, 96, 192])
def test_gauss_identities(oracle, nlat):
    sid, gwd = oracle.inigau(nlat)
    assert abs(gwd.sum() - 2.0) < 1e-13
    assert np.all(np.diff(sid) < 0)          # north first
    assert np.allclose(sid, -sid[::-1], atol=0, rtol=0)
    x, w = np.polynomial.legendre.leggauss(nlat)
    assert np.max(np.abs(np.sort(sid) - x)) < 1e-14
    assert np.max(np.abs(gwd[np.argsort(sid)] - w)) < 5e-14


@pytest.mark.parametrize("nlat", [32, 64])
def test_legendre_orthonormality(oracle, nlat):
    L = oracle.Leg(nlat)
    qi = L.table("qi").reshape(nlat, L.ncsp)
    gwd = L.table("gwd")
    w = 0
    for m in range(L.ntru + 1):
        k = L.ntru + 1 - m
        P = qi[:, w:w + k]
        G = (P * gwd[:, None]).T @ P
        assert np.max(np.abs(G - np.eye(k))) < 1e-12
        w += k


def test_tables_vs_golden(oracle):
    g = np.load(GOLDEN)
    L = oracle.Leg(32)
    for name in ("qi", "qj"):
        assert relerr(L.table(name).reshape(32, L.ncsp), g[f"t21_{name}"]) < 1e-12


def test_fft_vs_golden(oracle):
    g = np.load(GOLDEN)
    for n in (64, 128, 384, 512):
        x = g[f"fft_x_{n}"]
        assert relerr(oracle.gp2fc(x), g[f"fft_c_{n}"]) < 1e-14
    for n in (192,):
        x = g[f"fft_x_{n}"]
        assert relerr(oracle.gp2fc(x, use991=True), g[f"fft_c_{n}"]) < 1e-14


def test_sp2gp_vs_golden(oracle):
    # spectral -> grid at T21 with scipy Legendre functions and numpy's FFT
    g = np.load(GOLDEN)
    L = oracle.Leg(32)
    sp = g["t21_sp"]
    grid = oracle.fc2gp(L.sp2fc(sp))
    assert relerr(grid, g["t21_grid"]) < 1e-12


def test_fftmod_n48_is_not_a_dft(oracle):
    # documented reference defect: fftmod.f90 lists n=48 but its radix
    # schedule cannot factor 48/8 = 6.  The restatement reproduces it.
    x = np.random.default_rng(0).standard_normal((2, 48))
    ref = np.fft.rfft(x, axis=-1) / 48
    out = oracle.gp2fc(x)
    assert np.max(np.abs(out[:, 2] - ref.real[:, 1])) > 1e-3


def test_fft_roundtrip_and_impulse(oracle):
    n = 64
    x = np.zeros((1, n))
    x[0, 5] = 1.0
    c = oracle.gp2fc(x)
    k = np.arange(n // 2)
    assert np.allclose(c[0, 2::2], np.cos(2 * np.pi * 5 * k[1:] / n) / n, atol=1e-16)
    assert np.allclose(c[0, 3::2], -np.sin(2 * np.pi * 5 * k[1:] / n) / n, atol=1e-16)
    y = np.random.default_rng(1).standard_normal((3, n))
    assert relerr(oracle.fc2gp(oracle.gp2fc(y)), y - (y @ ((-1.0) ** np.arange(n)))[:, None] * ((-1.0) ** np.arange(n)) / n) < 1e-14


def test_folded_and_unfolded_fc2sp_agree(oracle):
    L = oracle.Leg(32)
    fc = np.random.default_rng(3).standard_normal((32, 64))
    assert relerr(L.fc2sp(fc, folded=True), L.fc2sp(fc, folded=False)) < 1e-13


def test_filters(oracle):
    # pyfft physics filter is exp(-8 (n/NTRU)^8) in 4-byte reals (pyfft.f90:152-156)
    L = oracle.Leg(32, pyfft_nfs=1)
    f = L.table("skspgp")
    n = np.arange(1, L.ntru + 2, dtype=np.float32)
    assert np.allclose(f, np.exp(np.float32(-8) * (n / np.float32(L.ntru)) ** 8), rtol=1e-6)
    L4 = oracle.Leg(32, nfilter=4, ngptfilter=1, nspvfilter=0)
    g = L4.table("skgpsp")
    assert np.allclose(g, (1 - np.arange(1, L4.ntru + 2) / (L4.ntru + 1)) ** 2)
    assert np.all(L4.table("skspgp") == 1.0)


def test_solarini_sun(oracle):
    # the 5772 K blackbody gives the model's default split 0.517/0.483 (radmod.f90:197-198)
    z1, z2, rc = oracle.solarini(5772.0)
    assert abs(z1 - 0.517) < 2e-3
    assert abs(z1 + z2 - 1) < 1e-15
    # rcoeff is normalised to the 5772 K spectrum with the module default 0.517
    assert abs(rc - 0.517 / z1) < 1e-9
    z1c, _, rcc = oracle.solarini(3000.0)
    assert z1c < z1 and rcc < rc


def _rad_case(oracle, nlev=10, **over):
    from exoplasim_b200 import synthetic as S
    cols, g = S.radiation_columns(8, nlev, seed=11)
    p = oracle.radpar(nlev, g["nhor"], g["nlon"], g["sigma"], g["sigmah"], g["dsigma"], nsol=0, **over)
    return oracle.radstep(p, cols["sid"], cols["cola"], cols), cols, p


def test_radstep_zero_insolation(oracle):
    out, cols, _ = _rad_case(oracle)
    dark = cols["gmu0"] <= 0
    assert dark.any()
    assert np.all(out["dswfl"][:, dark] == 0) and np.all(out["dfd"][:, dark] == 0)


def test_radstep_energy_closure(oracle):
    out, cols, p = _rad_case(oracle)
    ds = np.array([p.dsigma[i] for i in range(10)])[:, None]
    cp = p.acpd * (1 + p.adv * cols["dq"][:10])
    heat = np.sum(out["dtdt"] * ds * cols["dp"][None, :] * cp / p.ga, axis=0)
    assert relerr(heat, out["dflux"][0] - out["dflux"][10]) < 1e-12


def test_structured_columns(oracle):
    """The vertically coherent columns the surrogate is trained on: the same
    ranges as the level-by-level columns, humidity log-gradients bounded (the
    level-by-level columns reach jumps of ~17), one cloud layer, and radstep's
    energy closure on them."""
    from exoplasim_b200 import synthetic as S
    nlev = 10
    cols, g = S.radiation_columns(8, nlev, seed=13, profiles="structured")
    ind, _ = S.radiation_columns(8, nlev, seed=13)
    assert {k: v.shape for k, v in cols.items()} == {k: v.shape for k, v in ind.items()}
    assert cols["dt"].min() >= 150.0 and cols["dt"].max() <= 350.0
    assert cols["dq"].min() > 0 and cols["dq"][nlev].max() <= 3e-2
    assert cols["dcc"].min() >= 0 and cols["dcc"].max() <= 1 and np.all(cols["dcc"][nlev] == 0)
    assert cols["dp"].min() >= 1e4 and cols["dp"].max() <= 1e6
    grad = np.abs(np.diff(np.log(cols["dq"]), axis=0))
    assert grad.max() < 12 < np.abs(np.diff(np.log(ind["dq"]), axis=0)).max()
    p = oracle.radpar(nlev, g["nhor"], g["nlon"], g["sigma"], g["sigmah"], g["dsigma"], nsol=0)
    out = oracle.radstep(p, cols["sid"], cols["cola"], cols)
    ds = np.array([p.dsigma[i] for i in range(nlev)])[:, None]
    cp = p.acpd * (1 + p.adv * cols["dq"][:nlev])
    heat = np.sum(out["dtdt"] * ds * cols["dp"][None, :] * cp / p.ga, axis=0)
    assert relerr(heat, out["dflux"][0] - out["dflux"][nlev]) < 1e-12
    with pytest.raises(ValueError):
        S.radiation_columns(8, nlev, profiles="smooth")


def test_radstep_transparent_isothermal_lw(oracle):
    # no absorbers, no clouds, isothermal black surface-like column: the
    # longwave downward flux at the top is zero and the upward flux at the
    # surface is eps*sigma*T^4
    from exoplasim_b200 import synthetic as S
    cols, g = S.radiation_columns(8, 10, seed=12)
    nhor = g["nhor"]
    cols["dq"][:] = 0
    cols["dcc"][:] = 0
    cols["dql"][:] = 0
    cols["dqco2"][:] = 0
    cols["dt"][:] = 250.0
    p = oracle.radpar(10, nhor, g["nlon"], g["sigma"], g["sigmah"], g["dsigma"], nsol=0, no3=0, th2oc=0.0)
    cols["dqo3"][:] = 0
    out = oracle.radstep(p, cols["sid"], cols["cola"], cols)
    assert np.all(out["dftd"][0] == 0)
    assert np.allclose(out["dftu"][10], -0.98 * 5.67e-8 * 250.0 ** 4, rtol=1e-12)


def test_pyfft_compositions(oracle):
    """The pyfft restatement (oracle/pyfft_oracle.py): sp2gp against the scipy
    golden grid times pyfft's sqrt(2), and the identities pyfft's pairs obey
    for band-limited fields (gp2sp o sp2gp, gpvsp o spvgp with reciprocal
    radius factors, uv2dv o dv2uv); f2py's Fortran-ordered shapes."""
    from exoplasim_b200 import synthetic as S
    from oracle import pyfft_oracle as PO
    g = np.load(GOLDEN)
    sp = g["t21_sp"]
    gp = PO.sp2gp(sp[:, None], 32, 64, 21)
    assert gp.shape == (64, 32, 1)
    assert relerr(gp[:, :, 0].T, g["t21_grid"] * PO.SQRT2) < 1e-13
    assert relerr(PO.gp2sp(gp, 32, 64, 21)[:, 0], sp) < 1e-13
    rng = np.random.default_rng(7)
    sd = S.spectral_field(rng, 21, 3, "nn1").T.copy()
    sz = S.spectral_field(rng, 21, 3, "nn1").T.copy()
    sd[0:2] = sz[0:2] = 0.0                 # no n=0 divergence or vorticity
    sid, _ = PO.inigau(32)
    cs = np.sqrt(1.0 - sid ** 2)
    gu, gv = PO.spvgp(sd, sz, 6.371e6 / cs, 64, 21)
    assert gu.shape == gv.shape == (64, 32, 3)
    d2, z2 = PO.gpvsp(gu, gv, cs / 6.371e6, 21)
    assert relerr(d2, sd) < 1e-12 and relerr(z2, sz) < 1e-12
    pu, pv = PO.dv2uv(sd, sz, 32, 64, 21)
    assert pu.shape == (2, 32, 32, 3)
    pd, pz = PO.uv2dv(pu, pv, 32, 64, 21)
    assert pd.shape == (2, 253, 3)
    assert relerr(pd.transpose(1, 0, 2).reshape(-1, 3), sd) < 1e-12
    fc = PO.sp3fc(sp[:, None], 32, 64, 21)
    assert fc.shape == (2, 32, 32, 1)
    # gp3fc is fftmod's packing of numpy's DFT, scaled by 1/n
    a = rng.standard_normal((64, 32, 2))
    c = PO.gp3fc(a)
    X = np.fft.rfft(a, axis=0) / 64
    assert relerr(c[2::2], X.real[1:32]) < 1e-14 and relerr(c[3::2], X.imag[1:32]) < 1e-14
    # the FFT991 variant (pyfft991 for NLAT 192 and 320) agrees with fftmod
    assert relerr(PO.gp3fc(a, use991=True), c) < 1e-14


# ---- an independent second restatement of lwr pins the C oracle's fits ----
def _lwr_pair(O, nlat, nlev, seed, **over):
    from oracle import lwr_numpy as LN
    cols, g = S.radiation_columns(nlat, nlev, seed=seed)
    sig = O.default_sigma(nlev)
    p = O.radpar(nlev, g["nhor"], g["nlon"], *sig, nsol=0, nswr=0, **over)
    ref = O.radstep(p, cols["sid"], cols["cola"], cols)
    pd = dict(nlev=nlev, sigma=sig[0], sigmah=sig[1], dsigma=sig[2], ga=p.ga, acllwr=p.acllwr, clgray=p.clgray,
              th2oc=p.th2oc, tpofmt=p.tpofmt, npbroaden=p.npbroaden)
    got = LN.lwr(pd, cols["dt"], cols["dq"], cols["dcc"], cols["dql"], ref["dqo3"], cols["dqco2"], cols["dp"],
                 cols["dls"])
    return got, ref


@pytest.mark.parametrize("over", [{}, {"clgray": 0.5}, {"npbroaden": 0}, {"th2oc": 0.0}, {"tpofmt": 0.9}])
def test_lwr_matches_independent_numpy_restatement(oracle, over):
    # lwr_numpy.py restates radmod.f90:2122-2456 in numpy from the Fortran, apart
    # from exo_oracle_rad.c: the two agree to rounding on every flux
    (u, d, l), ref = _lwr_pair(oracle, 16, 20, seed=31, **over)
    for k, v in (("dftu", u), ("dftd", d), ("dlwfl", l)):
        assert relerr(v, ref[k]) < 1e-12, k


def test_lwr_fits_branches_and_continuity():
    # the synthetic columns reach both sides of every absorptivity fit's switch,
    # and the printed continuity constants make each fit continuous there
    # (radmod.f90:2207-2218); a slipped coefficient breaks one of the two
    from oracle import lwr_numpy as LN
    eps = 1e-9
    for name, x0 in (("h2o", 0.01), ("co2", 1.0), ("o3", 0.01), ("th2o", 2.0)):
        lo = np.array([x0 - eps]); hi = np.array([x0 + eps]); z = np.array([1e-3])
        args = {"h2o": (lo, z, z), "co2": (z, z, lo), "o3": (z, lo, z), "th2o": (lo, z, z)}[name]
        argh = {"h2o": (hi, z, z), "co2": (z, z, hi), "o3": (z, hi, z), "th2o": (hi, z, z)}[name]
        a = LN.absorptivities(*args, th2oc=0.0)
        b = LN.absorptivities(*argh, th2oc=0.0)
        idx = {"h2o": 0, "co2": 1, "th2o": 2, "o3": 3}[name]
        assert abs(a[idx][0] - b[idx][0]) < 1e-6, name
    # absorber paths of the test columns straddle the switches
    from oracle import oracle as O
    nlev = 20
    cols, g = S.radiation_columns(16, nlev, seed=31)
    sig = O.default_sigma(nlev)
    zps2 = cols["dp"] ** 2
    uwv = np.cumsum([0.1 * sig[0][j] * sig[2][j] / 9.80665 / 1e5 * zps2 * cols["dq"][j] for j in range(nlev)], axis=0)
    assert (uwv <= 0.01).any() and (uwv > 2.0).any()


@pytest.mark.parametrize("over", [{}, {"nswrcl": 0}, {"necham": 0, "necham6": 1}, {"newrsc": 1}, {"nrscat": 0},
                                  {"nclouds": 0}, {"rcoeff": 2.5, "zsolar1": 0.6, "zsolar2": 0.4}])
def test_swr_matches_independent_numpy_restatement(oracle, over):
    # swr_numpy.py restates radmod.f90:1530-2116 in numpy from the Fortran, apart
    # from exo_oracle_rad.c: fluxes and updated albedos agree to rounding
    from oracle import swr_numpy as SN
    nlev = 20
    cols, g = S.radiation_columns(16, nlev, seed=37)
    sig = oracle.default_sigma(nlev)
    p = oracle.radpar(nlev, g["nhor"], g["nlon"], *sig, nsol=0, nlwr=0, **over)
    ref = oracle.radstep(p, cols["sid"], cols["cola"], cols)
    pd = {f[0]: getattr(p, f[0]) for f in oracle.RadPar._fields_}
    pd.update(sigma=sig[0], sigmah=sig[1], dsigma=sig[2], rcl1=list(p.rcl1), rcl2=list(p.rcl2),
              acl2=list(p.acl2))
    mu = cols["gmu0"]
    got = SN.swr(pd, mu, mu, cols["dt"], cols["dq"], cols["dcc"], cols["dql"], ref["dqo3"], cols["dp"],
                 cols["dalb"], cols["dsalb"], cols["dls"], cols["dicec"])
    for k, v in zip(("dfu", "dfd", "dswfl", "dalb", "dsalb"), got):
        assert np.all(np.isfinite(v)), k
        assert relerr(v, ref[k]) < 1e-12, k
    assert (mu > 0).any() and (mu == 0).any()

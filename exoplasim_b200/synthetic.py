"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no datasets are involved; every workload is
synthetic).  All generators return float64 numpy arrays in the reference's
layouts; callers move them to the device.

Spectral fields: coefficients of the m-major triangle (m=0..NTRU, n=m..NTRU),
re and im ~ N(0, A(n)^2), imaginary part 0 at m=0, mode n=0 zero except
ln(ps) = ln(1e5 Pa); vorticity mode (0,1) carries the planetary vorticity
(the model stores absolute vorticity).
"""
import math

import numpy as np

EZ = 1.63299310207


def mode_mn(ntru):
    """(m, n) of every complex mode in the m-major triangle."""
    ms, ns = [], []
    for m in range(ntru + 1):
        for n in range(m, ntru + 1):
            ms.append(m)
            ns.append(n)
    return np.array(ms), np.array(ns)


def amplitude(n, kind="nn1", power=1.0):
    """A(n): 'nn1' -> (1/(n(n+1)))^power; 'steep' -> same for n <= 10, n^-3 beyond (continuous)."""
    n = np.asarray(n, dtype=np.float64)
    a = np.zeros_like(n)
    pos = n >= 1
    a[pos] = (1.0 / (n[pos] * (n[pos] + 1.0))) ** power
    if kind == "steep":
        hi = n > 10
        a10 = (1.0 / (10.0 * 11.0)) ** power
        a[hi] = a10 * (n[hi] / 10.0) ** -3
    return a


def spectral_field(rng, ntru, nlev, kind="nn1", power=1.0):
    """(nlev, 2*NCSP) coefficients with spectrum A(n)."""
    m, n = mode_mn(ntru)
    a = amplitude(n, kind, power)
    re = rng.standard_normal((nlev, m.size)) * a
    im = rng.standard_normal((nlev, m.size)) * a
    im[:, m == 0] = 0.0
    out = np.empty((nlev, 2 * m.size))
    out[:, 0::2] = re
    out[:, 1::2] = im
    return out


def transform_state(ntru, nlev, seed=0, kind="nn1"):
    """Spectral input of the gridpointa transform set: (4L+1, NRSP) = sd, st, sz, sq, sp."""
    rng = np.random.default_rng(seed)
    sd = spectral_field(rng, ntru, nlev, kind)
    st = spectral_field(rng, ntru, nlev, kind)
    sz = spectral_field(rng, ntru, nlev, kind)
    sz[:, 2] += EZ  # mode (0,1) real part: planetary vorticity
    sq = spectral_field(rng, ntru, nlev, kind, power=1.5)
    sp = spectral_field(rng, ntru, 1, kind)
    sp[0, 0] = math.log(1.0e5)
    return np.concatenate([sd, st, sz, sq, sp], axis=0)


def grid_tendencies(nlat, nlev, seed=1, scale=1e-5):
    """Grid input of the forward transform set: (9L+1, NLAT, NLON) ~ N(0, scale^2)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((9 * nlev + 1, nlat, 2 * nlat)) * scale


def sigma_levels(nlev):
    """Default sigma (full, half, delta) levels (plasim.f90:1554-1564)."""
    z = np.arange(1, nlev + 1) / nlev
    sigmah = 0.75 * z + 1.75 * z ** 3 - 1.5 * z ** 4
    dsigma = np.diff(np.concatenate([[0.0], sigmah]))
    sigma = 0.5 * (np.concatenate([[0.0], sigmah[:-1]]) + sigmah)
    return sigma, sigmah, dsigma


def radiation_columns(nlat, nlev, seed=2, teff=False, profiles="independent"):
    """Synthetic radiation columns on an NLAT x 2NLAT grid (nhor = 2 NLAT^2).

    profiles="independent" (every level drawn on its own):
    T(surface) ~ U(150,350) K, lapse rate ~ U(0,9) K/km over heights
    z = -(R T_s/g) ln(sigma) plus N(0, 5 K) noise, clipped to [150,350];
    q log-uniform [1e-7, 3e-2] kg/kg; cloud cover U(0,1); cloud water
    0.1*q*cc; ps log-uniform [1e4, 1e6] Pa; albedo U(0.05, 0.7); CO2
    log-uniform [1e-5, 1e-1] vmr (as ppmv); cos zenith from a tidally locked
    substellar point at (0 N, 180 E) scaled by U(0.5, 1) (zero on the night
    side); optional Teff U(2500, 6000) K per column.

    profiles="structured" (vertically coherent columns, as a model state has
    them; the same ranges of surface temperature, humidity, ps, albedo, CO2,
    zenith angle and Teff): T as above with N(0, 1 K) level noise and an
    isothermal stratosphere at U(150, 230) K below which T does not fall;
    q = q_s sigma^lambda exp(N(0, 0.2)) with q_s log-uniform [1e-7, 3e-2] and
    lambda ~ U(1, 4) (q_s at the surface level); cloud cover one Gaussian
    layer in sigma, amplitude U(0, 1) (none in 30% of columns), centre
    U(0.2, 0.95), half-width U(0.05, 0.25).
    """
    if profiles not in ("independent", "structured"):
        raise ValueError(f"profiles must be 'independent' or 'structured', not {profiles!r}")
    rng = np.random.default_rng(seed)
    nlon = 2 * nlat
    nhor = nlat * nlon
    nlep = nlev + 1
    sigma, sigmah, dsigma = sigma_levels(nlev)
    # Gaussian latitudes (cheap numpy equivalent is fine for input generation)
    x, _ = np.polynomial.legendre.leggauss(nlat)
    sid = -x  # north first
    cola = np.sqrt(1.0 - sid ** 2)
    ts = rng.uniform(150.0, 350.0, nhor)
    gam = rng.uniform(0.0, 9.0, nhor)
    zlev = -(287.0 * ts[None, :] / 9.80665) * np.log(sigma[:, None])
    if profiles == "independent":
        t = ts[None, :] - gam[None, :] * zlev / 1000.0 + rng.normal(0.0, 5.0, (nlev, nhor))
        t = np.clip(t, 150.0, 350.0)
        dq = np.exp(rng.uniform(np.log(1e-7), np.log(3e-2), (nlep, nhor)))
        dcc = rng.uniform(0.0, 1.0, (nlep, nhor))
    else:
        t = ts[None, :] - gam[None, :] * zlev / 1000.0 + rng.normal(0.0, 1.0, (nlev, nhor))
        t = np.clip(np.maximum(t, rng.uniform(150.0, 230.0, nhor)[None, :]), 150.0, 350.0)
        qs = np.exp(rng.uniform(np.log(1e-7), np.log(3e-2), nhor))
        lam = rng.uniform(1.0, 4.0, nhor)
        dq = np.empty((nlep, nhor))
        dq[:nlev] = qs[None, :] * sigma[:, None] ** lam[None, :] * np.exp(rng.normal(0.0, 0.2, (nlev, nhor)))
        dq[nlev] = qs
        amp = rng.uniform(0.0, 1.0, nhor) * (rng.uniform(0.0, 1.0, nhor) >= 0.3)
        sc = rng.uniform(0.2, 0.95, nhor)
        wd = rng.uniform(0.05, 0.25, nhor)
        dcc = np.zeros((nlep, nhor))
        dcc[:nlev] = amp[None, :] * np.exp(-((sigma[:, None] - sc[None, :]) / wd[None, :]) ** 2)
    dt = np.concatenate([t, ts[None, :]], axis=0)
    dcc[nlev] = 0.0
    dql = 0.1 * dq * dcc
    dp = np.exp(rng.uniform(np.log(1e4), np.log(1e6), nhor))
    dalb = rng.uniform(0.05, 0.7, nhor)
    dsalb = np.stack([dalb, dalb], axis=1).copy()
    co2 = np.exp(rng.uniform(np.log(1e-5), np.log(1e-1), nhor)) * 1e6
    dqco2 = np.repeat(co2[None, :], nlev, axis=0)
    lat = np.repeat(np.arcsin(sid), nlon)
    lon = np.tile(np.arange(nlon) * 2 * np.pi / nlon, nlat)
    cosd = np.cos(lat) * np.cos(lon - np.pi)
    gmu0 = np.maximum(0.0, cosd) * rng.uniform(0.5, 1.0, nhor)
    cols = dict(sid=sid, cola=cola, dt=dt, dq=dq, dcc=dcc, dql=dql, dqco2=dqco2, dp=dp,
                dls=np.zeros(nhor), dicec=np.zeros(nhor), dqo3=np.zeros((nlev, nhor)), gmu0=gmu0,
                dalb=dalb, dsalb=dsalb, dtdt=np.zeros((nlev, nhor)))
    if teff:
        cols["teff"] = rng.uniform(2500.0, 6000.0, nhor)
    return cols, dict(sigma=sigma, sigmah=sigmah, dsigma=dsigma, nlon=nlon, nhor=nhor)

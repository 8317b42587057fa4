"""A second, independent restatement of radmod's shortwave scheme (test
infrastructure only).

SUBROUTINE SWR, radmod.f90:1530-2116, rewritten in vectorised numpy straight
from the Fortran (without the aerosol branch, l_aerorad = 0, and for
nstartemp = 0), apart from the C oracle (exo_oracle_rad.c), so that a slip in
either transcription of the O3 and H2O transmissivity fits (:1899-1906,
:1937-1963), the cloud optics (:1685-1766), Rayleigh scattering (:1907-1915)
or the adding method (:1917-2112) shows up as a disagreement.  Only tests use
it.
"""
import numpy as np

ZERO = 1.0e-6
ZBETTA, ZMBAR = 1.66, 1.9
ZRO3 = 2.14
ZFO3 = 100.0 / ZRO3
AA, BB, C0 = 0.2542857142857143, 0.8229693877551021, 0.14997959183673468


def o3_absorption(x):
    """Lacis and Hansen's ozone absorption of an effective path x (cm STP), the
    bracket of radmod.f90:1900-1902."""
    return 0.02118 * x / (1.0 + 0.042 * x + 0.000323 * x ** 2) + 1.082 * x / ((1.0 + 138.6 * x) ** 0.805) \
        + 0.0658 * x / (1.0 + (103.6 * x) ** 3)


def h2o_absorption(y):
    """Water-vapour absorption of an effective path y, radmod.f90:1905-1906."""
    return 2.9 * y / ((1.0 + 141.5 * y) ** 0.635 + 5.925 * y)


def swr(p, zmu0, zmu1, dt, dq, dcc, dql, dqo3, dp, dalb, dsalb, dls, dicec):
    """Shortwave fluxes of columns (reference layouts: dt, dq, dcc, dql (NLEP, n);
    dqo3 (NLEV, n); the rest (n,), dsalb (n, 2)).  zmu0, zmu1: the cloud and
    insolation cos zenith of each column.  p: mapping of the radmod scalars.
    Returns dfu, dfd, dswfl (NLEP, n) and the updated dalb, dsalb."""
    L = int(p["nlev"])
    E = L + 1
    sigma, dsigma = (np.asarray(p[k], dtype=np.float64)[:L] for k in ("sigma", "dsigma"))
    ga = p["ga"]
    n = dp.shape[0]
    nclouds, nrscat, newrsc = p["nclouds"], p["nrscat"], p["newrsc"]
    assert p["nstartemp"] == 0
    zftop1 = p["zsolar1"] * p["gsol0"] * p["gdist2"] * zmu1
    zftop2 = p["zsolar2"] * p["gsol0"] * p["gdist2"] * zmu1
    losun = zftop1 + zftop2 > ZERO
    dfu, dfd, dsw = np.zeros((E, n)), np.zeros((E, n)), np.zeros((E, n))
    dalb, dsalb = dalb.copy(), dsalb.copy()
    if not losun.any():
        return dfu, dfd, dsw, dalb, dsalb
    s = losun   # work on the sunlit columns only, as the Fortran's where blocks do
    mu0, mu1 = zmu0[s], zmu1[s]
    dt_, dq_, dcc_, dql_, dqo3_ = dt[:, s], dq[:, s], dcc[:, s], dql[:, s], dqo3[:, s]
    dp_, dls_, dicec_ = dp[s], dls[s], dicec[s]
    ns = mu0.shape[0]
    f1, f2 = zftop1[s], zftop2[s]
    zmu00 = 0.5
    zb3 = p["tswr1"] * np.sqrt(zmu00) / zmu00
    zb4 = p["tswr2"] * np.sqrt(zmu00)
    zb5 = p["tswr3"] * zmu00 * zmu00
    # cloud optics (:1685-1766)
    rcl1, rcl1s, rcl2, rcl2s, tcl2, tcl2s = (np.zeros((L, ns)) for _ in range(6))
    tcl2[:] = 1.0
    tcl2s[:] = 1.0
    zcs = np.ones(ns)
    if nclouds == 1:
        if p["nswrcl"] == 0:
            for j in range(L):
                b = 0 if sigma[j] <= 1.0 / 3.0 else (1 if sigma[j] <= 2.0 / 3.0 else 2)
                r1, r2, a2 = p["rcl1"][b], p["rcl2"][b], p["acl2"][b]
                rcl1s[j] = r1 / (r1 + zmu00)
                rcl1[j] = zcs * r1 / (r1 + mu0) + (1.0 - zcs) * rcl1s[j]
                rcl2s[j] = min(1.0 - a2, r2 / (r2 + zmu00))
                rcl2[j] = np.minimum(1.0 - a2, zcs * r2 / (r2 + mu0) + (1.0 - zcs) * rcl2s[j])
                tcl2s[j] = 1.0 - rcl2s[j] - a2
                tcl2[j] = 1.0 - rcl2[j] - a2
                zcs = zcs * (1.0 - dcc_[j])
        else:
            for j in range(L):
                c = dcc_[j] > 0.0
                if c.any():
                    m0 = mu0[c]
                    lwp = np.minimum(1000.0, 1000.0 * dql_[j][c] * dp_[c] / ga * dsigma[j])
                    tau = 2.0 * np.log10(lwp + 1.5) ** 3.9
                    zlog = np.log(1000.0 / tau)

                    def two_stream(b1, b2, om_, mu):
                        un = 1.0 - om_
                        uz = un + 2.0 * b2 * om_
                        u = np.sqrt(uz / un)
                        ex = np.exp(np.minimum(25.0, tau * np.sqrt(uz * un) / mu))
                        r = (u + 1.0) ** 2 * ex - (u - 1.0) ** 2 / ex
                        return 1.0 - 1.0 / (1.0 + b1 * tau / mu), 4.0 * u / r, (u * u - 1.0) / r * (ex - 1.0 / ex)

                    r1s, t2s, r2s = two_stream(zb3 * zmu00, zb4 / np.log(3.0 + 0.1 * tau),
                                               np.minimum(0.9999, 1.0 - zb5 * zlog), zmu00)
                    r1, t2, r2 = two_stream(p["tswr1"] * np.sqrt(m0),
                                            p["tswr2"] * np.sqrt(m0) / np.log(3.0 + 0.1 * tau),
                                            np.minimum(0.9999, 1.0 - p["tswr3"] * m0 * m0 * zlog), m0)
                    cs = zcs[c]
                    rcl1s[j][c], tcl2s[j][c], rcl2s[j][c] = r1s, t2s, r2s
                    rcl1[j][c] = cs * r1 + (1.0 - cs) * r1s
                    tcl2[j][c] = cs * t2 + (1.0 - cs) * t2s
                    rcl2[j][c] = cs * r2 + (1.0 - cs) * r2s
                zcs = zcs * (1.0 - dcc_[j])
    # absorber paths with the magnification factor (:1767-1797)
    zm = 35.0 / np.sqrt(1.0 + 1224.0 * mu0 * mu0)
    zcs = np.ones(ns)
    o3t, xo3t, wvt, ywvt = (np.zeros(ns) for _ in range(4))
    o3l, xo3l, wvl, ywvl, rcs, rcsu = (np.zeros((L, ns)) for _ in range(6))
    scl = (dp_ / 101100.0) * (9.80665 / ga) * nrscat * newrsc
    for j in range(L):
        o3 = ZFO3 * dsigma[j] * dp_ * dqo3_[j] / ga
        o3t = o3t + o3
        xo3t = zcs * (xo3t + zm * o3) + (1.0 - zcs) * (xo3t + ZMBAR * o3)
        o3l[j], xo3l[j] = o3t, xo3t
        wv = 0.1 * dsigma[j] * dq_[j] * dp_ / ga * np.sqrt(273.0 / dt_[j]) * sigma[j] * dp_ / 100000.0
        wvt = wvt + wv
        ywvt = zcs * (ywvt + zm * wv) + (1.0 - zcs) * (ywvt + ZBETTA * wv)
        wvl[j], ywvl[j] = wvt, ywvt
        zcs = zcs * (1.0 - dcc_[j] * nclouds)
        rcs[j] = (AA / (1.0 + BB * mu0) * zcs + C0 * (1.0 - zcs - dcc_[L - 1] * nclouds)) * dsigma[j] * scl
        rcsu[j] = C0 * (1.0 - dcc_[L - 1]) * dsigma[j] * scl
    ta1, ta1s, ta2, ta2s = np.ones(ns), np.ones(ns), np.ones(ns), np.ones(ns)
    ra1, ra1s, ra2, ra2s = np.zeros(ns), np.zeros(ns), np.zeros(ns), np.zeros(ns)
    to3t = np.ones(ns)
    to3tu = 1.0 - o3_absorption(xo3t + ZMBAR * o3t) / p["zsolar1"]
    twvt = np.ones(ns)
    twvtu = 1.0 - h2o_absorption(ywvt + ZBETTA * wvt) / p["zsolar2"]
    # Rayleigh scattering in the lowest layer (:1907-1915)
    rcs[L - 1] = rcs[L - 1] * newrsc
    rcsu[L - 1] = rcsu[L - 1] * newrsc
    zscf = p["rcoeff"] * dp_ / 101100.0 * 9.80665 / ga
    rcsu[L - 1] = rcsu[L - 1] + (1.0 - np.exp(zscf * np.log(1.0 - 0.144))) * (1 - newrsc) * nrscat \
        * (1 - dcc_[L - 1] * nclouds)
    rcs[L - 1] = rcs[L - 1] + (1.0 - np.exp(zscf * np.log(1.0 - (0.219 / (1.0 + 0.816 * mu0))))) * zcs \
        * (1 - newrsc) * nrscat + (1.0 - np.exp(zscf * np.log(1.0 - 0.144))) * (1.0 - zcs - dcc_[L - 1]) \
        * nrscat * (1 - newrsc)
    # downward adding (:1917-1989)
    t1, t2, r1s, r2s = (np.zeros((E, ns)) for _ in range(4))
    rb1, rb1s, rb2, rb2s, tb1, tb1u, tb2, tb2u = (np.zeros((L, ns)) for _ in range(8))
    for j in range(L):
        t1[j], t2[j], r1s[j], r2s[j] = ta1, ta2, ra1s, ra2s
        rb1[j] = rcs[j] + rcl1[j] * dcc_[j] * nclouds
        rb1s[j] = rcsu[j] + rcl1s[j] * dcc_[j] * nclouds
        to3 = (1.0 - o3_absorption(xo3l[j]) / p["zsolar1"]) / to3t
        to3t = to3t * to3
        to3u = to3tu / (1.0 - o3_absorption(xo3t + ZMBAR * (o3t - o3l[j])) / p["zsolar1"])
        to3tu = to3tu / to3u
        tb1[j] = 1.0 - (1.0 - to3) * (1.0 - dcc_[j]) - rb1[j]
        tb1u[j] = 1.0 - (1.0 - to3u) * (1.0 - dcc_[j]) - rb1s[j]
        k = 1.0 / (1.0 - ra1s * rb1s[j])
        ra1 = ra1 + ta1 * rb1[j] * ta1s * k
        ta1 = ta1 * tb1[j] * k
        ra1s = rb1s[j] + tb1u[j] * ra1s * tb1[j] * k
        ta1s = tb1u[j] * ta1s * k
        rb2[j] = rcl2[j] * dcc_[j] * nclouds
        rb2s[j] = rcl2s[j] * dcc_[j] * nclouds
        twv = (1.0 - h2o_absorption(ywvl[j]) / p["zsolar2"]) / twvt
        twvt = twvt * twv
        twvu = twvtu / (1.0 - h2o_absorption(ywvt + ZBETTA * (wvt - wvl[j])) / p["zsolar2"])
        twvtu = twvtu / twvu
        tb2[j] = 1.0 - (1.0 - twv) * (1.0 - dcc_[j] * nclouds) - (1.0 - tcl2[j]) * dcc_[j] * nclouds
        tb2u[j] = 1.0 - (1.0 - twvu) * (1.0 - dcc_[j] * nclouds) - (1.0 - tcl2s[j]) * dcc_[j] * nclouds
        k = 1.0 / (1.0 - ra2s * rb2s[j])
        ra2 = ra2 + ta2 * rb2[j] * ta2s * k
        ta2 = ta2 * tb2[j] * k
        ra2s = rb2s[j] + tb2u[j] * ra2s * tb2[j] * k
        ta2s = tb2u[j] * ta2s * k
    t1[L], t2[L], r1s[L], r2s[L] = ta1, ta2, ra1s, ra2s
    # surface albedo (:2000-2036), nstartemp = 0
    sal = dsalb[s].copy()
    alb = dalb[s].copy()
    ra1s = alb.copy()
    ra2s = alb.copy()
    ocean = np.minimum(0.05 / (mu0 + 0.15), 0.15) * p["necham"] * (1 - p["necham6"]) \
        + (1 - p["necham"]) * p["necham6"] * (0.026 / (mu0 ** 1.7 + 0.065)
                                             + 0.15 * (mu0 - 1) * (mu0 - 0.5) * (mu0 - 0.1) + 0.0082)
    keep = (1.0 - p["necham"]) * (1 - p["necham6"])
    wet = (1.0 - dls_) * (1.0 - dicec_)
    for b in range(2):
        sal[:, b] = dls_ * sal[:, b] + (1.0 - dls_) * dicec_ * sal[:, b] + wet * ocean + wet * keep * sal[:, b]
    alb = dls_ * alb + (1.0 - dls_) * dicec_ * alb + wet * ocean + wet * keep * alb
    ra1 = alb.copy()
    ra2 = alb.copy()
    # upward adding (:2039-2057)
    rl1, rl2, rl1s, rl2s = (np.zeros((E, ns)) for _ in range(4))
    for j in range(L - 1, -1, -1):
        rl1[j + 1], rl2[j + 1], rl1s[j + 1], rl2s[j + 1] = ra1, ra2, ra1s, ra2s
        ra1 = rb1[j] + tb1[j] * ra1 * tb1u[j] / (1.0 - ra1s * rb1s[j])
        ra1s = rb1s[j] + tb1u[j] * ra1s * tb1u[j] / (1.0 - ra1s * rb1s[j])
        ra2 = rb2[j] + tb2[j] * ra2 * tb2u[j] / (1.0 - ra2s * rb2s[j])
        ra2s = rb2s[j] + tb2u[j] * ra2s * tb2u[j] / (1.0 - ra2s * rb2s[j])
    rl1[0], rl2[0], rl1s[0], rl2s[0] = ra1, ra2, ra1s, ra2s
    # interface fluxes (:2099-2112)
    u_ = np.zeros((E, ns))
    d_ = np.zeros((E, ns))
    for j in range(E):
        k = 1.0 / (1.0 - r1s[j] * rl1s[j])
        fd1, fu1 = t1[j] * k, -t1[j] * rl1[j] * k
        k = 1.0 / (1.0 - r2s[j] * rl2s[j])
        fd2, fu2 = t2[j] * k, -t2[j] * rl2[j] * k
        u_[j] = fu1 * f1 + fu2 * f2
        d_[j] = fd1 * f1 + fd2 * f2
    dfu[:, s], dfd[:, s] = u_, d_
    dsw[:, s] = u_ + d_
    dalb[s] = alb
    dsalb[s] = sal
    return dfu, dfd, dsw, dalb, dsalb

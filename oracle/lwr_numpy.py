"""A second, independent restatement of radmod's longwave scheme (test
infrastructure only).

SUBROUTINE LWR, radmod.f90:2122-2456, rewritten in vectorised numpy straight
from the Fortran (constants as printed there, Stefan-Boltzmann SBK from
radmod.f90:18), in a different language and a different loop structure from
the C oracle (exo_oracle_rad.c), so that a slip in a fit coefficient or an
exponent in either transcription shows up as a disagreement between the two.
It covers the clear-sky absorptivity fits of H2O (6.3 micron band and
continuum), CO2 (with the Boer et al. H2O overlap) and O3 (:2306-2346), the
random-overlap cloud transmissivity (:2279-2292, :2349-2354), the effective
layer emission (:2357-2391) and the flux sums with the surface emissivity
correction (:2393-2452).  Only tests use it.
"""
import numpy as np

SBK = 5.67e-8                        # radmod.f90:18
ZMMAIR, ZMMCO2 = 0.0289644, 0.0440098
ZPV2PM = ZMMCO2 / ZMMAIR             # co2 ppvol -> ppmass
ZRCO2, ZRO3 = 1.9635, 2.14
ZTTOP = 0.0
ZFH2O, ZFCO2, ZFO3 = 0.1, 100.0 / ZRCO2, 100.0 / ZRO3
ZERO = 1.0e-6


def fit_constants():
    """The continuity offsets of the absorptivity fits (radmod.f90:2207-2218)."""
    c = {}
    c["zao30"] = 0.209 * (7.0e-5) ** 0.436
    c["zco20"] = 0.0676 * (0.01022) ** 0.421
    c["zh2o0a"] = 0.846 * (3.59e-5) ** 0.243
    c["zh2o0"] = 0.832 * 0.0286 ** 0.26
    c["zao3c"] = 0.209 * (0.01 + 7.0e-5) ** 0.436 - c["zao30"] - 0.0212 * np.log10(0.01)
    c["zaco2c"] = 0.0676 * (1.01022) ** 0.421 - c["zco20"]
    c["zah2oc"] = 0.846 * (0.01 + 3.59e-5) ** 0.243 - c["zh2o0a"] - 0.24 * np.log10(0.02)
    c["zth2oc"] = 1.0 - (0.832 * (2.0 + 0.0286) ** 0.26 - c["zh2o0"]) + 0.1196 * np.log(2.0 - 0.6931)
    return c


def absorptivities(uwv, uo3, uco2, th2oc, c=None):
    """a(H2O), a(CO2), t(H2O at the CO2 overlap), a(O3) of absorber paths
    (g/cm2 water vapour, cm-STP ozone and CO2), radmod.f90:2306-2341."""
    c = c or fit_constants()
    uwv, uo3, uco2 = (np.asarray(x, dtype=np.float64) for x in (uwv, uo3, uco2))
    with np.errstate(divide="ignore", invalid="ignore"):
        ah2o = np.where(uwv <= 0.01, 0.846 * (uwv + 3.59e-5) ** 0.243 - c["zh2o0a"],
                        0.24 * np.log10(uwv + 0.01) + c["zah2oc"])
        if th2oc > 0.0:
            ah2o = np.minimum(ah2o + (1.0 - np.exp(-th2oc * uwv)), 1.0)
        aco2 = np.where(uco2 <= 1.0, 0.0676 * (uco2 + 0.01022) ** 0.421 - c["zco20"],
                        0.0546 * np.log10(uco2) + c["zaco2c"])
        th2o = np.where(uwv <= 2.0, 1.0 - (0.832 * (uwv + 0.0286) ** 0.26 - c["zh2o0"]),
                        np.maximum(0.0, c["zth2oc"] - 0.1196 * np.log(uwv - 0.6931)))
        ao3 = np.where(uo3 <= 0.01, 0.209 * (uo3 + 7.0e-5) ** 0.436 - c["zao30"],
                       0.0212 * np.log10(uo3) + c["zao3c"])
    return ah2o, aco2, th2o, ao3


def lwr(p, dt, dq, dcc, dql, dqo3, dqco2, dp, dls):
    """Longwave fluxes of columns given as reference-layout arrays
    (dt, dq, dcc, dql: (NLEP, n); dqo3, dqco2: (NLEV, n); dp, dls: (n,)).
    p: mapping with nlev, sigma, sigmah, dsigma, ga, acllwr, clgray, th2oc,
    tpofmt, npbroaden.  Returns (dftu, dftd, dlwfl), each (NLEP, n)."""
    L = int(p["nlev"])
    E = L + 1
    sigma, sigmah, dsigma = (np.asarray(p[k], dtype=np.float64)[:L] for k in ("sigma", "sigmah", "dsigma"))
    ga = p["ga"]
    n = dp.shape[0]
    c = fit_constants()
    zps2 = dp * dp if p["npbroaden"] > 0.5 else np.full(n, 101100.0 * 101100.0)
    # sigma T^4 on full levels (and surface) and half levels (:2226-2245)
    zst4 = SBK * dt[:E] ** 4
    zst4h = np.zeros((E, n))
    zst4h[0] = zst4[0] - (zst4[0] - zst4[1]) * sigma[0] / (sigma[0] - sigma[1])
    for jl in range(1, L):
        zst4h[jl] = (zst4[jl] * (sigma[jl - 1] - sigmah[jl - 1]) + zst4[jl - 1] * (sigmah[jl - 1] - sigma[jl])) \
            / (sigma[jl - 1] - sigma[jl])
    keep = (zst4[L - 1] - zst4h[L - 1]) * (zst4[L - 1] - zst4[L]) > 0.0
    zst4h[L] = np.where(keep, zst4[L], zst4[L - 1] + (zst4[L - 1] - zst4[L - 2]) * (1.0 - sigma[L - 1])
                        / (sigma[L - 1] - sigma[L - 2]))
    # indices of zbu/zbd run 0..NLEP as in the Fortran
    zbd = np.zeros((E + 1, n))
    zbu = np.zeros((E + 1, n))
    zbd[0] = SBK * ZTTOP ** 4
    zeps = dls + 0.98 * (1.0 - dls)
    zbu[E] = zeps * zst4[L]
    # absorber amounts and layer cloud transmissivities (:2263-2279)
    zq, zqo3, zqco2, ztaucc0 = (np.zeros((L, n)) for _ in range(4))
    for jl in range(L):
        zzf1 = sigma[jl] * dsigma[jl] / ga / 100000.0
        zzf2 = ZPV2PM * 1.0e-6
        zzf3 = -1.66 * p["acllwr"] * 1000.0 * dsigma[jl] / ga
        zsfac = zzf1 * zps2
        zq[jl] = ZFH2O * zsfac * dq[jl]
        zqo3[jl] = ZFO3 * zsfac * dqo3[jl]
        zqco2[jl] = ZFCO2 * zzf2 * zsfac * dqco2[jl]
        if p["clgray"] > 0:
            ztaucc0[jl] = 1.0 - dcc[jl] * p["clgray"]
        else:
            ztaucc0[jl] = 1.0 - dcc[jl] * (1.0 - np.exp(zzf3 * dql[jl] * dp))
    dftu = np.zeros((E, n))
    dftd = np.zeros((E, n))
    ztaucs = np.zeros((L, n))
    ztau = np.zeros((L, n))
    ztausf = np.zeros((L, n))
    for jl in range(L):                   # Fortran jlev = jl + 1
        ztaucc = np.ones(n)
        swv, so3, sco2 = np.zeros(n), np.zeros(n), np.zeros(n)
        for j2 in range(jl, L):
            swv = swv + zq[j2]
            so3 = so3 + zqo3[j2]
            sco2 = sco2 + zqco2[j2]
            ah2o, aco2, th2o, ao3 = absorptivities(swv, so3, sco2, p["th2oc"], c)
            ztaucs[j2] = np.minimum(1.0 - ZERO, np.maximum(ZERO, 1.0 - ah2o - ao3 - aco2 * th2o))
            ztaucc = ztaucc * ztaucc0[j2]
            ztau[j2] = ztaucs[j2] * ztaucc
        if jl == 0:
            # effective emission of each layer (:2357-2391)
            ztau0 = np.full(n, 1.0 - ZERO)
            for j2 in range(L):
                ztau0 = ztaucs[j2] / ztau0 * ztaucc0[j2] * p["tpofmt"]
                ztau0 = np.minimum(1.0 - ZERO, np.maximum(ZERO, ztau0))
                iso = (zst4[j2] - zst4h[j2]) * (zst4[j2] - zst4h[j2 + 1]) > 0.0
                with np.errstate(divide="ignore", invalid="ignore"):
                    bd = (zst4h[j2 + 1] - ztau0 * zst4h[j2]) / (1.0 - ztau0) \
                        - (zst4h[j2] - zst4h[j2 + 1]) / np.log(ztau0)
                bdi = 0.5 * zst4[j2] + 0.25 * (zst4h[j2] + zst4h[j2 + 1])
                zbd[j2 + 1] = np.where(iso, bdi, bd)
                zbu[j2 + 1] = np.where(iso, bdi, zst4h[j2] + zst4h[j2 + 1] - bd)
                ztau0 = ztaucs[j2]
        dftu[jl] = dftu[jl] - zbu[jl + 1]
        dftd[jl] = dftd[jl] + zbd[jl]
        zbdl = zbd[jl] - zbd[jl + 1]
        for j2 in range(jl, L):
            dftu[jl] = dftu[jl] - (zbu[j2 + 2] - zbu[j2 + 1]) * ztau[j2]
            dftd[j2 + 1] = dftd[j2 + 1] + zbdl * ztau[j2]
        ztausf[jl] = ztau[L - 1]
    dftu[L] = dftu[L] - zbu[E]
    dftd[L] = dftd[L] + zbd[L]
    zepsd = (1.0 - zeps) * dftd[L]
    for jl in range(L):
        dftu[jl] = dftu[jl] - ztausf[jl] * zepsd
    return dftu, dftd, dftu + dftd

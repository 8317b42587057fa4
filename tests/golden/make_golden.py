"""Generate tests/golden/golden_v1.npz from independent implementations.

The reference ships no golden vectors for its transforms and its Fortran
cannot be compiled here, so these fixtures come from numpy (FFT) and scipy
(normalised associated Legendre functions) using the reference's
conventions:
  - P(m,n) normalised to integrate to 1 over mu in [-1,1], with the
    Condon-Shortley phase (legmod.f90:61-89); Q = (1 - mu^2) dP/dmu;
  - forward FFT c_k = (1/n) sum x_j e^{-2 pi i jk/n} stored (A0,0,A1,B1,...);
  - spectral -> grid = sum_n P*sp per m, then x_j = A0 + 2 sum Re(c_k e^{ijk..}).
Run:  python tests/golden/make_golden.py
"""
import math
import os

import numpy as np
from scipy.special import lpmv

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_v1.npz")


def main():
    nlat, ntru = 32, 21
    x, w = np.polynomial.legendre.leggauss(nlat)
    sid = -x  # north first
    cols_p, cols_q = [], []
    for m in range(ntru + 1):
        for n in range(m, ntru + 1):
            c = math.sqrt((2 * n + 1) / 2 * math.factorial(n - m) / math.factorial(n + m))
            cols_p.append(lpmv(m, n, sid) * c)
            dp = (n + 1) * sid * lpmv(m, n, sid) - (n - m + 1) * lpmv(m, n + 1, sid)
            cols_q.append(dp * c)
    qi = np.stack(cols_p, axis=1)
    qj = np.stack(cols_q, axis=1)
    rng = np.random.default_rng(2024)
    out = {"t21_qi": qi, "t21_qj": qj}
    for n in (64, 128, 192, 384, 512):
        xx = rng.standard_normal((4, n))
        c = np.fft.rfft(xx, axis=-1) / n
        f = np.zeros_like(xx)
        f[:, 0::2] = c.real[:, : n // 2]
        f[:, 1::2] = c.imag[:, : n // 2]
        f[:, 1] = 0.0
        out[f"fft_x_{n}"] = xx
        out[f"fft_c_{n}"] = f
    ncsp = qi.shape[1]
    sp = rng.standard_normal(2 * ncsp)
    ms = np.concatenate([[m] * (ntru + 1 - m) for m in range(ntru + 1)])
    sp[1::2][ms == 0] = 0.0
    fc = np.zeros((nlat, 2 * nlat))
    spc = sp[0::2] + 1j * sp[1::2]
    for m in range(ntru + 1):
        sel = ms == m
        v = qi[:, sel] @ spc[sel]
        fc[:, 2 * m] = v.real
        fc[:, 2 * m + 1] = v.imag
    nlon = 2 * nlat
    cc = fc[:, 0::2] + 1j * fc[:, 1::2]
    cc[:, 0] = cc[:, 0].real
    full = np.zeros((nlat, nlon // 2 + 1), dtype=complex)
    full[:, : nlon // 2] = cc
    grid = np.fft.irfft(full * nlon, n=nlon, axis=-1)
    out["t21_sp"] = sp
    out["t21_grid"] = grid
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()

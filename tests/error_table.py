"""Per-field error table of the transform sets against the FP64 oracle.

Runs the gridpointa inverse and forward sets (plasim.f90:2396-2486) through
the C ABI in FP64, FP32 and mixed precision at T21 L10, T42 L20, T63 L10,
T127 L20 and T170 L25 on the synthetic inputs the parity tests use, and prints
one markdown table per set: for each field group the largest, over its levels,
norm-wise relative error max|x-ref|/max|ref| and L2 relative error
||x-ref||/||ref||.  Needs a CUDA GPU; not collected by pytest.

    python -m tests.error_table > error_table.md
"""
import sys

import numpy as np
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200.transforms import Plan
from oracle import oracle as O

FFTMOD_N = (8, 16, 32, 64, 96, 128, 256, 384, 512)
CASES = [(32, 10), (64, 20), (96, 10), (192, 20), (256, 25)]
PRECS = ["fp64", "fp32", "mixed"]


def inverse_groups(L):
    g = {n: range(i * L, (i + 1) * L) for i, n in enumerate(["u", "v", "T", "D", "zeta", "q"])}
    g.update({"dlnps/dmu": [6 * L], "dlnps/dlambda": [6 * L + 1], "lnps": [6 * L + 2]})
    return g


def forward_groups(L):
    g = {n: range(i * L, (i + 1) * L) for i, n in enumerate(["sdf", "stf", "szf", "sqf"])}
    g["spf"] = [4 * L]
    return g


def errs(x, ref, fields):
    emax = el2 = 0.0
    for f in fields:
        a, b = x[f].astype(np.float64).ravel(), ref[f].ravel()
        nb = np.max(np.abs(b))
        if nb == 0.0:
            continue
        emax = max(emax, float(np.max(np.abs(a - b)) / nb))
        el2 = max(el2, float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    return emax, el2


def main():
    O.lib()
    rows_inv, rows_fwd = [], []
    for nlat, nlev in CASES:
        P = Plan(nlat)
        L = O.Leg(nlat)
        use991 = 2 * nlat not in FFTMOD_N
        kind = "steep" if nlat >= 192 else "nn1"
        spin = S.transform_state(P.ntru, nlev, seed=3, kind=kind)
        gin = S.grid_tendencies(nlat, nlev, seed=4)
        ref_g = L.inverse_set(spin, nlev, plavor=S.EZ, use991=use991)
        ref_s = L.forward_set(gin.reshape(9 * nlev + 1, -1), nlev, use991=use991)
        for prec in PRECS:
            dt = torch.float64 if prec == "fp64" else torch.float32
            g = P.inverse_set(torch.as_tensor(spin, device="cuda", dtype=dt), nlev, precision=prec)
            g = g.cpu().numpy().reshape(6 * nlev + 3, -1)
            s = P.forward_set(torch.as_tensor(gin, device="cuda", dtype=dt), nlev, precision=prec).cpu().numpy()
            tag = f"T{P.ntru} L{nlev}"
            rows_inv.append((tag, prec, {k: errs(g, ref_g, v) for k, v in inverse_groups(nlev).items()}))
            rows_fwd.append((tag, prec, {k: errs(s, ref_s, v) for k, v in forward_groups(nlev).items()}))
        del P
        torch.cuda.empty_cache()
    for title, rows in (("inverse set (spectral -> grid)", rows_inv), ("forward set (grid -> spectral)", rows_fwd)):
        names = list(rows[0][2])
        print(f"\n{title}: max-norm / L2 relative error, worst level of each field\n")
        print("| case | precision | " + " | ".join(names) + " |")
        print("|---|---|" + "---|" * len(names))
        for tag, prec, e in rows:
            print(f"| {tag} | {prec} | " + " | ".join(f"{e[n][0]:.1e} / {e[n][1]:.1e}" for n in names) + " |")
    sys.stdout.flush()


if __name__ == "__main__":
    main()

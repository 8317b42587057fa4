"""Make tests/golden/pyburn_T21.npz: a small PlaSim raw output file and what
the reference's own postprocessor makes of it.

Run where the reference source tree is readable (it is imported, never
copied):

    python tests/golden/make_pyburn_golden.py /path/to/ExoPlaSim

1. Synthetic T21 fields (3 output steps; temperature, vorticity and
   divergence on 2 levels, ln ps, and a grid field) are written as raw
   records by oracle/rawfmt.py (outmod.f90 writegp/writesp).
2. The reference's pyburn reads them back (readallvariables, refactorvariable,
   pyburn.py:453-551) -- this pins the byte layout to the reference's reader.
3. The reference's _transformvar (modes grid, spectral, fourier) and
   _transformvectorvar (grid) run on the decoded variables (pyburn.py:623-1348),
   with the f2py module exoplasim.pyfft (which needs a Fortran compiler) stood
   in for by oracle/pyfft_oracle.py, the FP64 restatement of pyfft.f90 -- this
   pins the reshapes, transposes, scalings and longitude roll to the
   reference's code.
The fixture holds the source fields, the file's bytes, the decoded variables
and the transformed arrays.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NLAT, NLEV, NTIMES = 32, 2, 3
NLON = 2 * NLAT
NTRU = (NLON - 1) // 3
NRSP = (NTRU + 1) * (NTRU + 2)
DAYS = 360


def fields(seed=11):
    from exoplasim_b200 import synthetic as S
    rng = np.random.default_rng(seed)
    out = {}
    for t in range(NTIMES):
        out[("sp", 130, t)] = S.spectral_field(rng, NTRU, NLEV, "nn1") * 50.0     # temperature
        out[("sp", 138, t)] = S.spectral_field(rng, NTRU, NLEV, "nn1") * 1e-4     # vorticity
        out[("sp", 155, t)] = S.spectral_field(rng, NTRU, NLEV, "nn1") * 1e-5     # divergence
        out[("sp", 152, t)] = S.spectral_field(rng, NTRU, 1, "nn1")               # ln ps
        out[("gp", 139, t)] = 250.0 + 30.0 * rng.standard_normal((1, NLAT * NLON))  # surface temperature
    return out


def records(src):
    """(raw bytes, per-record (kind, code, level, step, scale, offset)) in the model's write order."""
    from oracle import oracle as O
    from oracle import rawfmt as RF
    sig = O.default_sigma(NLEV)[1]
    blob = RF.params_block(NLON, NLAT, NLEV, NTRU, sig, DAYS, 1 + 100 * 1)
    meta = []
    for t in range(NTIMES):
        d3, d4 = 1 + 100 * 1 + 10000 * 0, 100 * 6 * t
        for code in (130, 138, 155):
            for lev in range(NLEV):
                pscale = {130: 1.0, 138: 1.0 / 2.0, 155: 2.0}[code]
                head = [code, lev + 1, d3, d4, NRSP, 1, 6 * t, DAYS]
                blob += RF.writesp(src[("sp", code, t)][lev], head, NTRU, pscale, 0.0)
                meta.append(("sp", code, lev + 1, 6 * t, pscale, 0.0))
        head = [152, 0, d3, d4, NRSP, 1, 6 * t, DAYS]
        blob += RF.writesp(src[("sp", 152, t)][0], head, NTRU, 1.0, np.log(1e5))
        meta.append(("sp", 152, 0, 6 * t, 1.0, float(np.log(1e5))))
        head = [139, 0, d3, d4, NLON, NLAT, 6 * t, DAYS]
        blob += RF.writegp(src[("gp", 139, t)][0], head)
        meta.append(("gp", 139, 0, 6 * t, 1.0, 0.0))
    return blob, meta


def main(refroot):
    sys.path.insert(0, refroot)
    from oracle import pyfft_oracle
    import exoplasim.pyburn as pb       # the reference's postprocessor
    src = fields()
    blob, meta = records(src)
    headers, variables = pb.readallvariables(blob)
    time = variables["time"]
    ntimes = len(time)
    dec = {k: pb.refactorvariable(variables[k], headers[k], ntimes=ntimes, nlev=NLEV)
           for k in variables if k not in ("main", "sigmah", "time")}
    # the f2py module, stood in for by the FP64 restatement of pyfft.f90
    shim = types.ModuleType("exoplasim.pyfft")
    for name in ("inigau", "sp2gp", "gp2sp", "sp3fc", "gp3fc", "fc3gp", "spvgp", "gpvsp"):
        setattr(shim, name, getattr(pyfft_oracle, name))
    sys.modules["exoplasim.pyfft"] = shim
    import exoplasim
    exoplasim.pyfft = shim
    sid, _ = pyfft_oracle.inigau(NLAT)
    lat = np.arcsin(sid) * 180.0 / np.pi
    lon = np.arange(NLON) / float(NLON) * 360.0
    out = {}
    for code in ("130", "152", "139"):
        for mode in ("grid", "spectral", "fourier"):
            if code == "139" and mode == "spectral":
                # the reference raises NameError here: a single-level grid field
                # reaches the misspelt `vairable` test (pyburn.py:798)
                continue
            meta_l = ["x", "x", "x"]
            r = pb._transformvar(lon, lat, dec[code].copy(), meta_l, NLAT, NLON, NLEV, NTRU, ntimes, mode=mode)
            out[f"tv_{code}_{mode}"] = np.asarray(r[0] if isinstance(r, tuple) else r)
    gu, gv, *_ = pb._transformvectorvar(lon, dec["155"].copy(), dec["138"].copy(), ["u"], ["v"], lat, NLON, NLEV,
                                        NTRU, ntimes, mode="grid")
    out["tvv_u_grid"] = np.asarray(gu)
    out["tvv_v_grid"] = np.asarray(gv)
    save = {"raw": np.frombuffer(blob, dtype=np.uint8), "time": np.asarray(time),
            "meta_kind": np.array([m[0] for m in meta]), "meta_num": np.array([m[1:] for m in meta], dtype=np.float64)}
    for (kind, code, t), v in src.items():
        save[f"src_{kind}_{code}_{t}"] = v
    for k, v in dec.items():
        save[f"dec_{k}"] = v
        save[f"head_{k}"] = np.asarray(headers[k])
    save["head_main"] = np.asarray(headers["main"])
    save.update(out)
    np.savez_compressed(os.path.join(HERE, "pyburn_T21.npz"), **save)
    print({k: v.shape for k, v in save.items() if k.startswith(("tv", "dec"))})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

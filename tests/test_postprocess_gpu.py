"""The raw output writer on the GPU and pyburn's transforms on the GPU,
against what the reference's own pyburn made of the same data
(tests/golden/pyburn_T21.npz, made by tests/golden/make_pyburn_golden.py
with the reference's readallvariables / refactorvariable / _transformvar /
_transformvectorvar and the FP64 pyfft restatement in place of the f2py
module).

Bars: the written bytes equal the golden file exactly; the transforms are
within 1e-12 (norm-wise relative, per output array) of the golden outputs,
both being FP64 transforms of the same float32 data."""
import os

import numpy as np
import pytest
import torch

from exoplasim_b200 import outfmt as OF
from exoplasim_b200 import postprocess as PP
from tests._util import relerr

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "pyburn_T21.npz"))
NLAT, NLEV, NTIMES = 32, 2, 3
NLON, NTRU = 64, 21


def _src(kind, code, t):
    return G[f"src_{kind}_{code}_{t}"]


def test_device_writer_reproduces_the_file(tmp_path):
    from oracle import oracle as O
    path = tmp_path / "out.raw"
    sig = O.default_sigma(NLEV)[1]
    with OF.RawWriter(str(path), NLAT, NLEV, sig, days_per_year=360, date=(0, 1, 1)) as w:
        for t in range(NTIMES):
            fields = []
            for code, scale in ((130, 1.0), (138, 0.5), (155, 2.0)):
                sp = torch.as_tensor(_src("sp", code, t), device="cuda")
                for lev in range(NLEV):
                    fields.append(("sp", code, lev + 1, sp[lev].contiguous(), scale, 0.0))
            fields.append(("sp", 152, 0, torch.as_tensor(_src("sp", 152, t)[0], device="cuda"), 1.0,
                           float(np.log(1e5))))
            fields.append(("gp", 139, 0, torch.as_tensor(_src("gp", 139, t)[0], device="cuda"), 1.0, 0.0))
            w.write_step(fields, nstep=6 * t, date=(0, 1, 1, 6 * t, 0))
    assert path.read_bytes() == G["raw"].tobytes()


def test_device_writer_float32_fields_match_restatement():
    # a 4-byte model: spnorm and the scale in float32, as writesp runs there
    from oracle import rawfmt as RF
    rng = np.random.default_rng(3)
    pf = rng.standard_normal(506).astype(np.float32)
    head = [130, 1, 101, 0, 506, 1, 0, 360]
    ref = RF.writesp(pf, head, NTRU, 0.37, 2.5)
    recs = (OF.RawRec * 1)()
    r = recs[0]
    t = torch.as_tensor(pf, device="cuda")
    r.head[:] = head
    r.src, r.n, r.prec, r.kind, r.ntru, r.pscale, r.poff = t.data_ptr(), 506, 1, 1, NTRU, 0.37, 2.5
    from exoplasim_b200._lib import call
    import ctypes as C
    buf = torch.empty(48 + 4 * 506, dtype=torch.uint8, device="cuda")
    call("exotx_raw_pack", recs, 1, C.c_void_p(buf.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert buf.cpu().numpy().tobytes() == ref


@pytest.mark.parametrize("code", ["130", "152", "139"])
@pytest.mark.parametrize("mode", ["grid", "spectral", "fourier"])
def test_transformvar_matches_reference(code, mode):
    key = f"tv_{code}_{mode}"
    dec = G["dec_" + code]
    got = PP.transformvar(dec, NLAT, NLON, NLEV, NTRU, mode=mode)
    if key not in G.files:
        # the reference raises NameError on this case (pyburn.py:798); the
        # transform itself is pyfft's gp2sp of every output step
        from oracle import pyfft_oracle as PO
        gp = np.asfortranarray(np.transpose(dec.reshape(NTIMES, NLAT, NLON)))
        ref = np.transpose(PO.gp2sp(gp, NLAT, NLON, NTRU, 0)).reshape(NTIMES, -1, 2)
    else:
        ref = G[key]
    assert got.shape == ref.shape, (got.shape, ref.shape)
    assert relerr(got, ref) < 1e-12


def test_transformvectorvar_matches_reference():
    from oracle import pyfft_oracle as PO
    sid, _ = PO.inigau(NLAT)
    lat = np.arcsin(sid) * 180.0 / np.pi
    gu, gv = PP.transformvectorvar(G["dec_155"], G["dec_138"], lat, NLON, NLEV, NTRU, mode="grid")
    assert gu.shape == G["tvv_u_grid"].shape
    assert relerr(gu, G["tvv_u_grid"]) < 1e-12 and relerr(gv, G["tvv_v_grid"]) < 1e-12


def test_transformvar_keeps_device_tensors():
    dec = torch.as_tensor(G["dec_130"], device="cuda")
    out = PP.transformvar(dec, NLAT, NLON, NLEV, NTRU, mode="grid")
    assert isinstance(out, torch.Tensor) and out.is_cuda
    assert relerr(out.cpu().numpy(), G["tv_130_grid"]) < 1e-12

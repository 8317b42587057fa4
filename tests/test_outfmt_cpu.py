"""PlaSim's raw output format on the host side: the reader parses the golden
file the way the reference's pyburn reader did when the fixture was made
(tests/golden/make_pyburn_golden.py), and the byte-level restatement of
outmod.f90 (oracle/rawfmt.py) reproduces the file.  Exact equality: the
format is bytes, not arithmetic."""
import os
import struct

import numpy as np

from exoplasim_b200 import outfmt as OF
from exoplasim_b200.postprocess import refactor

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "pyburn_T21.npz"))
NLEV = 2


def _blob():
    return G["raw"].tobytes()


def test_reader_matches_reference_reader():
    headers, variables = OF.read_variables(_blob())
    assert tuple(headers["main"]) == tuple(G["head_main"])
    assert list(variables["time"]) == list(G["time"])
    for code in ("130", "138", "155", "152", "139"):
        assert tuple(headers[code]) == tuple(G["head_" + code])
        got = refactor(variables[code], headers[code], ntimes=len(variables["time"]), nlev=NLEV)
        ref = G["dec_" + code]
        assert got.shape == ref.shape and np.array_equal(got, ref), code


def test_restated_writer_reproduces_the_file():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mk", os.path.join(os.path.dirname(__file__), "golden", "make_pyburn_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    src = {}
    for k in G.files:
        if k.startswith("src_"):
            _, kind, code, t = k.split("_")
            src[(kind, int(code), int(t))] = G[k]
    blob, _ = mk.records(src)
    assert blob == _blob()


def test_spnorm_signs():
    s = OF.spnorm(21)
    assert s.size == 22 * 23
    assert np.all(s[:44] > 0) and np.all(s[44:86] < 0) and abs(s[0] - 0.7071067811865475) == 0.0


def _reframe(blob, ml, en):
    """the same records with ml-byte markers in byte order en"""
    out, n = b"", 0
    while n < len(blob):
        ln = struct.unpack("<i", blob[n:n + 4])[0]
        body = blob[n + 4:n + 4 + ln]
        words = np.frombuffer(body, dtype="<i4" if ln == 32 else "<f4").astype(en + ("i4" if ln == 32 else "f4"))
        m = struct.pack(en + ("i" if ml == 4 else "q"), ln)
        out += m + words.tobytes() + m
        n += 8 + ln
    return out


def test_reader_byte_orders_and_marker_lengths():
    ref = OF.read_raw(_blob())
    for ml, en in ((4, ">"), (8, "<")):
        got = OF.read_raw(_reframe(_blob(), ml, en))
        assert len(got) == len(ref)
        for (h1, d1), (h2, d2) in zip(got, ref):
            assert tuple(h1) == tuple(h2) and np.array_equal(d1.astype(np.float32), d2)

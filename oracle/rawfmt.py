"""Byte-level restatement of PlaSim's raw output records (test infrastructure only).

outmod.f90 outini :5-42 (code-333 parameter block), writegp :97-134 and
writesp :140-169 with spnorm (plasim.f90:1637-1650), as numpy producing the
bytes gfortran writes: every record framed by 4-byte little-endian length
markers, headers int32, data float32.  The product forms the same bytes on
the GPU (exotx_raw_pack); tests compare the two and read both back with
pyburn's readers.
"""
import struct

import numpy as np


def spnorm(ntru, dtype=np.float64):
    z = dtype(1.0) / np.sqrt(dtype(2.0))
    out = []
    for m in range(ntru + 1):
        out += [z] * (2 * (ntru + 1 - m))
        z = -z
    return np.array(out, dtype=dtype)


def record(payload):
    m = struct.pack("<i", len(payload))
    return m + payload + m


def params_block(nlon, nlat, nlev, ntru, sigmah, days_per_year, date_word):
    head = np.array([333, 0, date_word, 0, nlon, nlat, nlev, ntru], dtype=np.int32)
    zsig = np.zeros(nlon * nlat, dtype=np.float32)
    zsig[:nlev] = np.asarray(sigmah)[:nlev]
    zsig[nlev] = days_per_year
    return record(head.tobytes()) + record(zsig.tobytes())


def writegp(pf, head):
    return record(np.asarray(head, dtype=np.int32).tobytes()) + record(np.asarray(pf).astype(np.float32).tobytes())


def writesp(pf, head, ntru, pscale=1.0, poff=0.0):
    """zf = pf * spnorm * pscale rounded to float32, then zf(1) += poff in the
    model's real kind (outmod.f90:163-164); pf's dtype is the model's kind."""
    pf = np.asarray(pf)
    kind = pf.dtype.type
    zf = (pf * spnorm(ntru, kind) * kind(pscale)).astype(np.float32)
    zf[0] = np.float32(kind(zf[0]) + kind(poff))
    return record(np.asarray(head, dtype=np.int32).tobytes()) + record(zf.tobytes())

"""PlaSim's raw output format: writer on the GPU, reader on the host.

The model writes its output as Fortran unformatted sequential records
(outmod.f90): a parameter block (code 333: NLON, NLAT, NLEV, NTRU in the
header, the half-level sigmas and the days per year in a float32 block of
NLON*NLAT values, outini :5-42), then for every field an 8-word int32 header
(code, level, date, time, two dimensions, step, days per year) and the field
as float32 -- grid fields as NLON*NLAT values (writegp :97-134), spectral
fields as NRSP coefficients normalised by spnorm = (-1)^m/sqrt(2) times a
scale, plus an offset on the first (writesp :140-169).  pyburn reads these
files (pyburn.py:221-553).

``RawWriter`` forms each output step's records on the device in one launch
(exotx_raw_pack) and appends the bytes to the file; ``read_raw`` and
``read_variables`` parse a file the way pyburn's readrecord and
readallvariables do.
"""
import ctypes as C
import struct

import numpy as np
import torch

from . import _lib
from ._lib import FP32, FP64, call



class RawRec(C.Structure):
    _fields_ = [("head", C.c_int * 8), ("src", C.c_void_p), ("n", C.c_longlong), ("prec", C.c_int),
                ("kind", C.c_int), ("ntru", C.c_int), ("pscale", C.c_double), ("poff", C.c_double)]


def spnorm(ntru):
    """ECHAM output normalisation of the NRSP spectral reals (plasim.f90:1637-1650):
    1/sqrt(2) with the sign (-1)^m."""
    out = []
    z = 1.0 / np.sqrt(2.0)
    for m in range(ntru + 1):
        out += [z] * (2 * (ntru + 1 - m))
        z = -z
    return np.array(out)


def date_words(nyear=0, nmonth=1, nday=1, nhour=0, nmin=0):
    """Header words 3 and 4 of a record (outmod.f90:118-119)."""
    return nday + 100 * nmonth + 10000 * nyear, nmin + 100 * nhour


class RawWriter:
    """Append PlaSim raw records to a file.

    ``fields`` of a step are (kind, code, level, tensor, pscale, poff) with kind
    "gp" (NLAT x NLON grid, north first, longitude fastest) or "sp" (NRSP
    coefficients); tensors are float64 or float32 CUDA tensors."""

    def __init__(self, path, nlat, nlev, sigmah, days_per_year=360, date=(0, 1, 1)):
        self.nlat, self.nlon = nlat, 2 * nlat
        self.ntru = (self.nlon - 1) // 3
        self.nrsp = (self.ntru + 1) * (self.ntru + 2)
        self.nlev, self.days = nlev, int(days_per_year)
        self.f = open(path, "wb")
        # the parameter block is host data written once (outini, outmod.f90:5-42)
        head = [333, 0, date_words(*date)[0], 0, self.nlon, self.nlat, nlev, self.ntru]
        zsig = np.zeros(self.nlon * self.nlat, dtype=np.float32)
        zsig[:nlev] = np.asarray(sigmah, dtype=np.float64)[:nlev]
        zsig[nlev] = days_per_year
        self._record(np.asarray(head, dtype=np.int32).tobytes())
        self._record(zsig.tobytes())
        self._buf = None

    def _record(self, payload):
        m = struct.pack("<i", len(payload))
        self.f.write(m + payload + m)

    def write_step(self, fields, nstep=0, nstep1=0, date=(0, 1, 1, 0, 0)):
        """One output step: every field's header and data record, formed on the device."""
        d3, d4 = date_words(*date)
        recs = (RawRec * len(fields))()
        keep = []
        for r, (kind, code, lev, t, pscale, poff) in zip(recs, fields):
            if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
                raise TypeError("fields must be contiguous CUDA tensors")
            if t.dtype not in (torch.float64, torch.float32):
                raise TypeError("fields must be float64 or float32")
            sp = kind == "sp"
            n = self.nrsp if sp else self.nlat * self.nlon
            if t.numel() != n:
                raise ValueError(f"a {kind} field of this grid has {n} values, got {t.numel()}")
            dims = (self.nrsp, 1) if sp else (self.nlon, self.nlat)
            r.head[:] = [int(code), int(lev), d3, d4, dims[0], dims[1], int(nstep - nstep1), self.days]
            r.src = t.data_ptr()
            r.n = n
            r.prec = FP64 if t.dtype == torch.float64 else FP32
            r.kind = 1 if sp else 0
            r.ntru = self.ntru
            r.pscale = float(pscale)
            r.poff = float(poff)
            keep.append(t)
        nbytes = C.c_size_t()
        call("exotx_raw_size", recs, len(fields), C.byref(nbytes))
        if self._buf is None or self._buf.numel() < nbytes.value:
            self._buf = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
        call("exotx_raw_pack", recs, len(fields), C.c_void_p(self._buf.data_ptr()),
             C.c_void_p(torch.cuda.current_stream().cuda_stream))
        self.f.write(self._buf[:nbytes.value].cpu().numpy().tobytes())

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_raw(path_or_bytes):
    """Every record pair of a raw file as (header tuple, float32 array), the
    parameter block first.  4- and 8-byte markers in either byte order
    (pyburn.py:221-366 reads the same files; its marker test recognises 8-byte
    markers only when they are big-endian)."""
    buf = path_or_bytes if isinstance(path_or_bytes, (bytes, bytearray)) else open(path_or_bytes, "rb").read()
    # the first record is the 8-word header of the parameter block: the framing
    # whose leading and trailing markers both read 32 is the file's
    for ml, en in ((4, "<"), (4, ">"), (8, "<"), (8, ">")):
        mf = en + ("i" if ml == 4 else "q")
        if len(buf) >= 2 * ml + 32 and struct.unpack(mf, buf[:ml])[0] == 32 \
                and struct.unpack(mf, buf[ml + 32:2 * ml + 32])[0] == 32:
            break
    else:
        raise ValueError("not a PlaSim raw output file: no 8-word header record at the start")
    out, n = [], 0
    while n < len(buf):
        hl = struct.unpack(mf, buf[n:n + ml])[0]
        n += ml
        head = struct.unpack(en + "%di" % (hl // 4), buf[n:n + hl])
        n += hl + ml
        dl = struct.unpack(mf, buf[n:n + ml])[0]
        n += ml
        words = head[4] * head[5]
        wl = dl // words if words else 4
        data = np.frombuffer(buf[n:n + dl], dtype=np.dtype(en + ("f4" if wl == 4 else "f8"))).copy()
        n += dl + ml
        out.append((head, data))
    return out


def read_variables(path_or_bytes):
    """(headers, variables) by code, as pyburn.readallvariables (pyburn.py:453-495):
    the fields of one code concatenated over levels and steps, the sigma
    levels, and the step of every code-139 record."""
    recs = read_raw(path_or_bytes)
    main, zsig = recs[0]
    headers = {"main": main}
    variables = {"main": zsig, "sigmah": zsig[:main[6]], "time": []}
    for head, data in recs[1:]:
        k = str(head[0])
        if int(k) == 139:
            variables["time"].append(head[6])
        if k not in variables:
            variables[k] = data.astype(np.float64)
            headers[k] = head
        else:
            variables[k] = np.append(variables[k], data)
    return headers, variables

"""Uneven ensembles of transform sets on one GPU (exotx_ensemble_*).

Instances of different truncations (NLAT) and level counts run together:
each half of the gridpointa round trip (plasim.f90 :2396-2486) is one
tensor-core Legendre launch plus one FFT launch over every instance, in
MIXED precision (3-term BF16 splits, FP32 accumulation).  Data live in
packed float32 buffers; `pack`/`unpack` convert per-instance tensors.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Ensemble:
    def __init__(self, nlat, nlev):
        nlat = np.ascontiguousarray(nlat, dtype=np.int32)
        nlev = np.ascontiguousarray(nlev, dtype=np.int32)
        assert nlat.shape == nlev.shape and nlat.ndim == 1
        self._lib = _lib.load()
        h = C.c_void_p()
        call("exotx_ensemble_create", len(nlat), nlat.ctypes.data_as(C.c_void_p), nlev.ctypes.data_as(C.c_void_p),
             C.byref(h))
        self._h = h
        self.nlat, self.nlev = nlat.tolist(), nlev.tolist()
        n = len(nlat)
        so, gi, go = (np.zeros(n, np.int64) for _ in range(3))
        tot = np.zeros(3, np.int64)
        call("exotx_ensemble_layout", h, so.ctypes.data_as(C.c_void_p), gi.ctypes.data_as(C.c_void_p),
             go.ctypes.data_as(C.c_void_p), tot.ctypes.data_as(C.c_void_p))
        self.spec_off, self.gin_off, self.gout_off, self.totals = so, gi, go, tot
        self.choice = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.exotx_ensemble_destroy(h)
            except Exception:
                pass
            self._h = None

    def dims(self, i):
        nlat = self.nlat[i]
        nlon = 2 * nlat
        ntru = (nlon - 1) // 3
        return nlat, nlon, (ntru + 1) * (ntru + 2)

    def buffers(self):
        """Zeroed packed buffers (spec_in, gout, gin, spec_out)."""
        z = lambda k: torch.zeros(int(self.totals[k]), dtype=torch.float32, device="cuda")
        return z(0), z(2), z(1), z(0)

    def pack(self, kind, tensors, buf=None):
        """kind 'spec' | 'gin' | 'gout': per-instance tensors -> packed buffer."""
        off, tot = {"spec": (self.spec_off, 0), "gin": (self.gin_off, 1), "gout": (self.gout_off, 2)}[kind]
        if buf is None:
            buf = torch.zeros(int(self.totals[tot]), dtype=torch.float32, device="cuda")
        for i, t in enumerate(tensors):
            buf[int(off[i]):int(off[i]) + t.numel()] = t.reshape(-1).to(torch.float32)
        return buf

    def unpack(self, kind, buf):
        off = {"spec": self.spec_off, "gin": self.gin_off, "gout": self.gout_off}[kind]
        out = []
        for i in range(len(self.nlat)):
            nlat, nlon, nrsp = self.dims(i)
            L = self.nlev[i]
            shape = {"spec": (4 * L + 1, nrsp), "gin": (9 * L + 1, nlat, nlon), "gout": (6 * L + 3, nlat, nlon)}[kind]
            n = int(np.prod(shape))
            out.append(buf[int(off[i]):int(off[i]) + n].view(*shape))
        return out

    def inverse(self, spin, gout):
        call("exotx_ensemble_inverse", self._h, C.c_void_p(spin.data_ptr()), C.c_void_p(gout.data_ptr()), _s())
        return gout

    def forward(self, gin, spout):
        call("exotx_ensemble_forward", self._h, C.c_void_p(gin.data_ptr()), C.c_void_p(spout.data_ptr()), _s())
        return spout

    def configure(self, nc_qi=128, nc_uv=64, sorted=True, nprod=6):
        call("exotx_ensemble_configure", self._h, nc_qi, nc_uv, 1 if sorted else 0, nprod)

    def tune(self, spin, gout, gin, spout, reps=3):
        ch = np.zeros(4, np.int32)
        ms = C.c_float()
        call("exotx_ensemble_tune", self._h, C.c_void_p(spin.data_ptr()), C.c_void_p(gout.data_ptr()),
             C.c_void_p(gin.data_ptr()), C.c_void_p(spout.data_ptr()), reps, _s(), ch.ctypes.data_as(C.c_void_p),
             C.byref(ms))
        self.choice = dict(nc_qi=int(ch[0]), nc_uv=int(ch[1]), sorted=bool(ch[2]), nprod=int(ch[3]),
                           ms=float(ms.value))
        return self.choice


def draw(ninst, seed=0, nlats=(32, 64, 96), nlevs=(10, 15, 20)):
    """Seeded uneven ensemble: resolutions and level counts uniform over the sets."""
    g = np.random.default_rng(seed)
    return g.choice(nlats, ninst).tolist(), g.choice(nlevs, ninst).tolist()

"""PyTorch-facing spectral-transform API over libexotx.

A `Plan` holds the device tables for one resolution (NLAT Gaussian latitudes,
NLON = 2 NLAT, triangular truncation NTRU = (NLON-1)//3).  Every method takes
and returns CUDA tensors in the reference's layouts:

  spectral  (nfld, NRSP)        re/im pairs, m-major triangle   (legmod sp(2,NCSP))
  Fourier   (nfld, NLAT, NLON)  NLON/2 complex per latitude     (legmod fc(2,NLON/2,NLAT))
  grid      (nfld, NLAT, NLON)  same storage as Fourier rows

Precision "fp64" works on float64 tensors; "fp32" and "mixed" on float32
("mixed" = tensor-core Legendre with 3-term BF16 splits, FP32 accumulation).
Kernels run on torch's current CUDA stream.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import FP32, FP64, MIXED, PRECISIONS, call

EZ = 1.63299310207  # 1/sqrt(3/8): planetary vorticity in model units (plasimmod.f90:118,227)
TABLES = ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv")


def _prec(precision):
    if isinstance(precision, int):
        return precision
    return PRECISIONS[precision]


def _dtype(prec):
    return torch.float64 if prec == FP64 else torch.float32


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _check(t, dtype, shape, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


class Plan:
    """Device tables for one resolution; replaces inigau + legini (gaussmod.f90:5, legmod.f90:30)."""

    def __init__(self, nlat, nfilter=0, ngptfilter=0, nspvfilter=0, landhoskn0=15.0, filterkappa=8.0,
                 nfilterexp=8, pyfft_nfs=-1, plavor=EZ):
        lib = _lib.load()
        d = _lib.GridDesc()
        call("exotx_grid_desc_default", nlat, C.byref(d))
        d.nfilter, d.ngptfilter, d.nspvfilter = nfilter, ngptfilter, nspvfilter
        d.landhoskn0, d.filterkappa, d.nfilterexp = landhoskn0, filterkappa, nfilterexp
        d.pyfft_nfs, d.plavor = pyfft_nfs, plavor
        torch.cuda.init()
        h = C.c_void_p()
        call("exotx_plan_create", C.byref(d), C.byref(h))
        self._h = h
        self._lib = lib
        dims = [C.c_int() for _ in range(4)]
        call("exotx_plan_dims", h, *[C.byref(x) for x in dims])
        self.nlat, self.nlon, self.ntru, self.ncsp = (x.value for x in dims)
        self.nrsp = 2 * self.ncsp
        self.nhor = self.nlat * self.nlon

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.exotx_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def tune(self, chunk_inv=None, chunk_fwd=None, inv_half=None):
        """exotx_plan_tune: bytes of Fourier intermediate per tensor-core launch,
        and whether the inverse kernel may run two CTAs per SM."""
        if chunk_inv is not None:
            call("exotx_plan_tune", self._h, 0, int(chunk_inv))
        if chunk_fwd is not None:
            call("exotx_plan_tune", self._h, 1, int(chunk_fwd))
        if inv_half is not None:
            call("exotx_plan_tune", self._h, 2, int(bool(inv_half)))

    # ---------------------------------------------------------------- tables
    def gauss(self):
        """(sid, gwd) as float64 numpy arrays, north first (inigau outputs)."""
        sid = np.zeros(self.nlat)
        gwd = np.zeros(self.nlat)
        call("exotx_plan_gauss", self._h, sid.ctypes.data_as(C.c_void_p), gwd.ctypes.data_as(C.c_void_p))
        return sid, gwd

    def table(self, name):
        """One FP64 legini table as (NLAT, NCSP) numpy, i.e. Fortran q(NCSP,NLAT)."""
        out = np.zeros((self.nlat, self.ncsp))
        call("exotx_plan_table", self._h, TABLES.index(name), out.ctypes.data_as(C.c_void_p))
        return out

    # -------------------------------------------------------- allocation helpers
    def spectral(self, nfld, precision="fp64", device="cuda"):
        return torch.zeros((nfld, self.nrsp), dtype=_dtype(_prec(precision)), device=device)

    def grid(self, nfld, precision="fp64", device="cuda"):
        return torch.zeros((nfld, self.nlat, self.nlon), dtype=_dtype(_prec(precision)), device=device)

    # ---------------------------------------------------------- Legendre ops
    def _inv(self, fn, precision, ins, outs):
        p = _prec(precision)
        dt = _dtype(p)
        nlev = ins[0].shape[0]
        for i, t in enumerate(ins):
            _check(t, dt, (nlev, self.nrsp), f"input {i}")
        if outs is None:
            outs = [self.grid(nlev, p) for _ in range(len(ins))]
        for i, t in enumerate(outs):
            _check(t, dt, (nlev, self.nlat, self.nlon), f"output {i}")
        call(fn, self._h, p, *[_ptr(t) for t in ins], *[_ptr(t) for t in outs], nlev, _stream())
        return outs

    def sp2fc(self, sp, precision="fp64", out=None):
        """legmod.f90:230 sp2fc for a stack of fields."""
        return self._inv("exotx_sp2fc", precision, [sp], None if out is None else [out])[0]

    def sp2fcdmu(self, sp, precision="fp64", out=None):
        """legmod.f90:262 sp2fcdmu (d/dmu table qj)."""
        return self._inv("exotx_sp2fcdmu", precision, [sp], None if out is None else [out])[0]

    def dv2uv(self, pd, pz, precision="fp64", out=None):
        """legmod.f90:312 dv2uv: (divergence, vorticity) -> (u cos(phi), v cos(phi)) Fourier."""
        u, v = self._inv("exotx_dv2uv", precision, [pd, pz], out)
        return u, v

    def _fwd(self, fn, precision, ins, nout, outs):
        p = _prec(precision)
        dt = _dtype(p)
        nlev = ins[0].shape[0]
        for i, t in enumerate(ins):
            _check(t, dt, (nlev, self.nlat, self.nlon), f"input {i}")
        if outs is None:
            outs = [self.spectral(nlev, p) for _ in range(nout)]
        for i, t in enumerate(outs):
            _check(t, dt, (nlev, self.nrsp), f"output {i}")
        return p, nlev, outs

    def fc2sp(self, fc, precision="fp64", out=None):
        """legmod.f90:178 fc2sp (symmetric branch)."""
        p, nlev, outs = self._fwd("exotx_fc2sp", precision, [fc], 1, None if out is None else [out])
        call("exotx_fc2sp", self._h, p, _ptr(fc), _ptr(outs[0]), nlev, _stream())
        return outs[0]

    def uv2dv(self, pu, pv, precision="fp64", out=None):
        """legmod.f90:356 uv2dv: (u, v) Fourier -> (divergence, vorticity)."""
        p, nlev, outs = self._fwd("exotx_uv2dv", precision, [pu, pv], 2, out)
        call("exotx_uv2dv", self._h, p, _ptr(pu), _ptr(pv), _ptr(outs[0]), _ptr(outs[1]), nlev, _stream())
        return outs[0], outs[1]

    def mktend(self, tn, fu, fv, ke, ut, vt, precision="fp64", out=None):
        """legmod.f90:505 mktend -> (d, t, z) tendencies."""
        p, nlev, outs = self._fwd("exotx_mktend", precision, [tn, fu, fv, ke, ut, vt], 3, out)
        call("exotx_mktend", self._h, p, *[_ptr(o) for o in outs], *[_ptr(t) for t in (tn, fu, fv, ke, ut, vt)],
             nlev, _stream())
        return tuple(outs)

    def qtend(self, qn, uq, vq, precision="fp64", out=None):
        """legmod.f90:433 qtend -> q tendency."""
        p, nlev, outs = self._fwd("exotx_qtend", precision, [qn, uq, vq], 1, None if out is None else [out])
        call("exotx_qtend", self._h, p, _ptr(outs[0]), _ptr(qn), _ptr(uq), _ptr(vq), nlev, _stream())
        return outs[0]

    # ----------------------------------------------------------------- FFTs
    @staticmethod
    def gp2fc(a, precision=None):
        """fftmod.f90:29 gp2fc, in place on rows of the last axis."""
        return gp2fc(a, precision)

    @staticmethod
    def fc2gp(a, precision=None):
        """fftmod.f90:64 fc2gp, in place on rows of the last axis."""
        return fc2gp(a, precision)

    # ------------------------------------------------------- transform sets
    def inverse_set(self, spin, nlev, precision="fp64", out=None):
        """gridpointa inverse half: (4L+1, NRSP) -> (6L+3, NLAT, NLON)."""
        p = _prec(precision)
        dt = _dtype(p)
        _check(spin, dt, (4 * nlev + 1, self.nrsp), "spin")
        if out is None:
            out = self.grid(6 * nlev + 3, p)
        _check(out, dt, (6 * nlev + 3, self.nlat, self.nlon), "gpout")
        call("exotx_inverse_set", self._h, p, _ptr(spin), _ptr(out), nlev, _stream())
        return out

    def forward_set(self, gpin, nlev, precision="fp64", out=None):
        """gridpointa forward half: (9L+1, NLAT, NLON) -> (4L+1, NRSP); gpin unchanged."""
        p = _prec(precision)
        dt = _dtype(p)
        _check(gpin, dt, (9 * nlev + 1, self.nlat, self.nlon), "gpin")
        if out is None:
            out = self.spectral(4 * nlev + 1, p)
        _check(out, dt, (4 * nlev + 1, self.nrsp), "spout")
        call("exotx_forward_set", self._h, p, _ptr(gpin), _ptr(out), nlev, _stream())
        return out

    # size of the library's fixed scratch array used by forward_set_noalloc
    STATIC_WORK_BYTES = 16 << 20

    def forward_set_noalloc(self, gpin, nlev, out, precision="fp64"):
        """forward_set for callers that cannot allocate device memory: the
        Fourier intermediate and FFT twiddles live in a fixed array of
        STATIC_WORK_BYTES inside the library (shared by all calls on a device;
        calls that overlap on the GPU race).  `out` must be given.  Sets that
        need more scratch than the array holds raise ExotxError (BAD_DIM)."""
        p = _prec(precision)
        dt = _dtype(p)
        _check(gpin, dt, (9 * nlev + 1, self.nlat, self.nlon), "gpin")
        _check(out, dt, (4 * nlev + 1, self.nrsp), "spout")
        call("exotx_forward_set_noalloc", self._h, p, _ptr(gpin), _ptr(out), nlev, _stream())
        return out


    def inverse_set_batch(self, spin, nlev, precision="mixed", out=None):
        """inverse_set for ninst states stored back to back: (ninst, 4L+1, NRSP) -> (ninst, 6L+3, NLAT, NLON)."""
        p = _prec(precision)
        dt = _dtype(p)
        ninst = spin.shape[0]
        _check(spin, dt, (ninst, 4 * nlev + 1, self.nrsp), "spin")
        if out is None:
            out = torch.zeros((ninst, 6 * nlev + 3, self.nlat, self.nlon), dtype=dt, device=spin.device)
        _check(out, dt, (ninst, 6 * nlev + 3, self.nlat, self.nlon), "gpout")
        call("exotx_inverse_set_batch", self._h, p, _ptr(spin), _ptr(out), nlev, ninst, _stream())
        return out

    def forward_set_batch(self, gpin, nlev, precision="mixed", out=None):
        """forward_set for ninst states: (ninst, 9L+1, NLAT, NLON) -> (ninst, 4L+1, NRSP)."""
        p = _prec(precision)
        dt = _dtype(p)
        ninst = gpin.shape[0]
        _check(gpin, dt, (ninst, 9 * nlev + 1, self.nlat, self.nlon), "gpin")
        if out is None:
            out = torch.zeros((ninst, 4 * nlev + 1, self.nrsp), dtype=dt, device=gpin.device)
        _check(out, dt, (ninst, 4 * nlev + 1, self.nrsp), "spout")
        call("exotx_forward_set_batch", self._h, p, _ptr(gpin), _ptr(out), nlev, ninst, _stream())
        return out

    # ---------------------------------------------- gridpointd transform sets
    def inverse_set_d_batch(self, spin, nlev, precision="mixed", out=None):
        """gridpointd inverse half (invlegd + fc2gp, plasim.f90:3142-3149) for ninst
        states: (ninst, 4L+1, NRSP) sd, st, sz, sq, sp -> (ninst, 4L+1, NLAT, NLON)
        gu, gv, gt, gq, gp."""
        p = _prec(precision)
        dt = _dtype(p)
        ninst = spin.shape[0]
        _check(spin, dt, (ninst, 4 * nlev + 1, self.nrsp), "spin")
        if out is None:
            out = torch.zeros((ninst, 4 * nlev + 1, self.nlat, self.nlon), dtype=dt, device=spin.device)
        _check(out, dt, (ninst, 4 * nlev + 1, self.nlat, self.nlon), "gpout")
        call("exotx_inverse_set_d_batch", self._h, p, _ptr(spin), _ptr(out), nlev, ninst, _stream())
        return out

    def forward_set_d_batch(self, gpin, nlev, precision="mixed", out=None):
        """gridpointd forward half (gp2fc, fc2sp, uv2dv, plasim.f90:3415-3428) for
        ninst states: (ninst, 4L, NLAT, NLON) gtdt, gudt, gvdt, gqdt -> (ninst, 4L, NRSP)
        sdf, stf, szf, sqf; gpin is not modified."""
        p = _prec(precision)
        dt = _dtype(p)
        ninst = gpin.shape[0]
        _check(gpin, dt, (ninst, 4 * nlev, self.nlat, self.nlon), "gpin")
        if out is None:
            out = torch.zeros((ninst, 4 * nlev, self.nrsp), dtype=dt, device=gpin.device)
        _check(out, dt, (ninst, 4 * nlev, self.nrsp), "spout")
        call("exotx_forward_set_d_batch", self._h, p, _ptr(gpin), _ptr(out), nlev, ninst, _stream())
        return out

    def inverse_set_d(self, spin, nlev, precision="fp64", out=None):
        """inverse_set_d_batch of one state: (4L+1, NRSP) -> (4L+1, NLAT, NLON)."""
        o = None if out is None else out.unsqueeze(0)
        return self.inverse_set_d_batch(spin.unsqueeze(0), nlev, precision, o)[0]

    def forward_set_d(self, gpin, nlev, precision="fp64", out=None):
        """forward_set_d_batch of one state: (4L, NLAT, NLON) -> (4L, NRSP)."""
        o = None if out is None else out.unsqueeze(0)
        return self.forward_set_d_batch(gpin.unsqueeze(0), nlev, precision, o)[0]

    def sets_host(self, nlev, spin=None, gpout=None, gpin=None, spout=None, precision="mixed", host_fp64=False):
        """Both transform sets for states held in HOST tensors (page-locked for
        overlap): spin (ninst, 4L+1, NRSP) -> gpout (ninst, 6L+3, NLAT, NLON) and
        gpin (ninst, 9L+1, NLAT, NLON) -> spout (ninst, 4L+1, NRSP); leave out a
        half by passing None for both of its tensors.  The copies and transforms
        of neighbouring states overlap; the current stream waits for the last
        copy out, so synchronise it before reading the outputs.  host_fp64: the
        host tensors are float64 whatever the precision (an 8-byte model's
        arrays), converted on the device (exotx_sets_host_f64)."""
        p = _prec(precision)
        dt = torch.float64 if host_fp64 else _dtype(p)
        ninst = (spin if spin is not None else gpin).shape[0]
        shapes = {"spin": (ninst, 4 * nlev + 1, self.nrsp), "gpout": (ninst, 6 * nlev + 3, self.nlat, self.nlon),
                  "gpin": (ninst, 9 * nlev + 1, self.nlat, self.nlon), "spout": (ninst, 4 * nlev + 1, self.nrsp)}
        ptrs = []
        for name, t in (("spin", spin), ("gpout", gpout), ("gpin", gpin), ("spout", spout)):
            if t is None:
                ptrs.append(None)
                continue
            if not isinstance(t, torch.Tensor) or t.is_cuda:
                raise TypeError(f"{name} must be a host tensor")
            if t.dtype != dt or tuple(t.shape) != shapes[name] or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous {dt} tensor of shape {shapes[name]}")
            ptrs.append(_ptr(t))
        call("exotx_sets_host_f64" if host_fp64 else "exotx_sets_host", self._h, p, *ptrs, nlev, ninst, _stream())


def tc_error():
    """Read and reset the tensor-core kernels' error word (0 = no bounded wait gave up)."""
    code = C.c_int(0)
    call("exotx_tc_error", C.byref(code), _stream())
    return code.value


def _fft_args(a, precision):
    if not isinstance(a, torch.Tensor) or not a.is_cuda or not a.is_contiguous():
        raise TypeError("FFT input must be a contiguous CUDA tensor")
    p = (FP64 if a.dtype == torch.float64 else FP32) if precision is None else _prec(precision)
    if a.dtype != _dtype(p):
        raise TypeError(f"FFT input dtype {a.dtype} does not match precision")
    n = a.shape[-1]
    lot = a.numel() // n if n else 0
    return p, n, lot


def gp2fc(a, precision=None):
    """Real forward FFT of every row (last axis) in place: (A0, 0, A1, B1, ...) scaled by 1/n."""
    p, n, lot = _fft_args(a, precision)
    call("exotx_gp2fc", p, _ptr(a), n, lot, _stream())
    return a


def fc2gp(a, precision=None):
    """Inverse real FFT of every row in place (the m=0 imaginary slot is ignored)."""
    p, n, lot = _fft_args(a, precision)
    call("exotx_fc2gp", p, _ptr(a), n, lot, _stream())
    return a


def fft_supported(n):
    return bool(_lib.load().exotx_fft_supported(int(n)))


def inigau(nlat, device="cuda"):
    """Gaussian latitudes (sin) and weights on the device (gaussmod.f90:5-40)."""
    sid = torch.empty(nlat, dtype=torch.float64, device=device)
    gwd = torch.empty(nlat, dtype=torch.float64, device=device)
    call("exotx_inigau", nlat, _ptr(sid), _ptr(gwd), _stream())
    return sid, gwd


def launch_count():
    """Kernel launches issued by libexotx in this process so far."""
    return int(_lib.load().exotx_launch_count())


KERNELS = {"tc_forward": 0, "tc_inverse": 1, "fft_forward": 2, "fft_inverse": 3, "leg_forward": 4,
           "leg_inverse": 5, "radstep": 6, "surrogate": 7}


def kernel_timing(enable):
    """Bracket the library's main kernel launches (outside stream capture)
    with CUDA events on their launching stream while enabled."""
    call("exotx_kernel_timing", 1 if enable else 0)


def kernel_time(name):
    """(summed milliseconds, launches) recorded for one kernel since the last
    read; clears that kernel's record."""
    ms = C.c_double()
    n = C.c_longlong()
    call("exotx_kernel_time", KERNELS[name], C.byref(ms), C.byref(n))
    return ms.value, n.value

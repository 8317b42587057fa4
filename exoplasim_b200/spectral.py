"""The semi-implicit spectral time step on the GPU (plasim.f90 spectrala
:2757-2918 and spectrald :3645-3999, one model state).

A state is a dict of CUDA tensors: sdp szp stp sqp (L, NRSP), spp (NRSP) at
time t; sdm szm stm sqm spm at t - dt; the tendencies sdt szt stt sqt spt;
sop (NRSP) and srp (L, NRSP).  spectrala advances the adiabatic part from
gridpointa's tendencies, spectrald adds gridpointd's diabatic tendencies
with the implicit drag, restoration and diffusion, updating in place.
"""
import ctypes as C

import torch

from . import _lib
from ._lib import FP32, FP64, call

STATE = ("sdp", "szp", "stp", "sqp", "spp", "sdm", "szm", "stm", "sqm", "spm",
         "sdt", "szt", "stt", "sqt", "spt", "sop", "srp")


class SpecParams(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("nlev", "nqspec", "nsponge", "nhdiff")] +
                [(n, C.c_double) for n in ("delt", "delt2", "pnu", "pnu21", "plavor", "dampsp", "akap")] +
                [(n, C.c_double * 64) for n in ("t0", "sigmah", "dsigma", "damp", "tdisst", "tdissq", "tdissd",
                                               "tdissz", "tfrc")] +
                [("ndel", C.c_int * 64)])


class SpecState(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in STATE]


def default_params(nlev, **over):
    p = SpecParams()
    call("exotx_spec_params_default", nlev, C.byref(p))
    for k, v in over.items():
        if isinstance(getattr(p, k), (int, float)):
            setattr(p, k, v)
        else:
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = x
    return p


class SpecConst:
    """bm1, the level matrices and sak of one plan and parameter set, on the device."""

    def __init__(self, plan, params):
        self.params, self.plan = params, plan
        self._lib = _lib.load()
        h = C.c_void_p()
        call("exotx_specconst_create", plan.handle, C.byref(params), C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.exotx_specconst_destroy(h)
            except Exception:
                pass
            self._h = None


def _state(st):
    s = SpecState()
    dtype = st["spp"].dtype
    for k in STATE:
        t = st.get(k)
        if t is None:
            continue
        if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
            raise TypeError(f"{k} must be a contiguous CUDA tensor of {dtype}")
        setattr(s, k, t.data_ptr())
    return s, (FP64 if dtype == torch.float64 else FP32)


def spectrala(const, st):
    s, prec = _state(st)
    call("exotx_spectrala", const._h, prec, C.byref(s), C.c_void_p(torch.cuda.current_stream().cuda_stream))


def spectrald(const, st):
    s, prec = _state(st)
    call("exotx_spectrald", const._h, prec, C.byref(s), C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _states(sts):
    arr = (SpecState * len(sts))()
    prec = None
    for i, st in enumerate(sts):
        s, p = _state(st)
        if prec is not None and p != prec:
            raise TypeError("every state of a batch has one precision")
        prec = p
        arr[i] = s
    return arr, prec


def spectrala_batch(const, states):
    """spectrala of several states in one launch per 12 (exotx_spectrala_batch)."""
    arr, prec = _states(states)
    call("exotx_spectrala_batch", const._h, prec, arr, len(states), C.c_void_p(torch.cuda.current_stream().cuda_stream))


def spectrald_batch(const, states):
    """spectrald of several states in one launch per 12 (exotx_spectrald_batch)."""
    arr, prec = _states(states)
    call("exotx_spectrald_batch", const._h, prec, arr, len(states), C.c_void_p(torch.cuda.current_stream().cuda_stream))

"""The gfortran-named, by-reference entry points (include/exotx_fortran.h):
sp2fc_, sp2fcdmu_, fc2sp_, dv2uv_, uv2dv_, mktend_, qtend_, gp2fc_, fc2gp_,
inigau_ and radstep_ called through ctypes the way a Fortran caller calls
them -- every argument by reference, the model's own host arrays in the
reference's column-major layouts -- against the FP64 oracle.

Tolerances: 8-byte arrays with FP64 transforms <= 1e-12 norm-wise relative
error per field (radiation <= 1e-11); FP32 transforms (4- or 8-byte arrays)
<= 2e-5.  The CPU tests check the argument handling that runs before any
device work.
"""
import ctypes as C

import numpy as np
import pytest

from exoplasim_b200 import _lib
from exoplasim_b200 import synthetic as S
from tests._util import relerr

FP64, FP32, MIXED = 0, 1, 2
BAD_ARG, UNSUPPORTED_N = 3, 2
_ip = lambda v: C.byref(C.c_int(v))
_dp = lambda v: C.byref(C.c_double(v))


def _f():
    lib = _lib.load()
    for name in ("exotx_legini_", "exotx_legfree_", "exotx_fortran_status_", "exotx_stop_on_error_", "inigau_",
                 "sp2fc_", "sp2fcdmu_", "fc2sp_", "dv2uv_", "uv2dv_", "qtend_", "mktend_", "gp2fc_", "fc2gp_",
                 "radstep_"):
        getattr(lib, name).restype = None
    return lib


def _status(lib):
    st = C.c_int(-1)
    lib.exotx_fortran_status_(C.byref(st))
    return st.value


def _legini(lib, nlat, nlev, real_bytes, prec, nfilter=0):
    ierr = C.c_int(-1)
    lib.exotx_legini_(_ip(nlat), _ip(nlev), _ip(real_bytes), _ip(prec), _ip(nfilter), _ip(0), _ip(0),
                      _dp(15.0), _dp(8.0), _ip(8), _dp(S.EZ), C.byref(ierr))
    return ierr.value


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def test_fortran_arguments_checked_before_device_work():
    lib = _f()
    off = C.c_int(0)
    lib.exotx_stop_on_error_(C.byref(off))
    assert _status(lib) == 0
    lib.exotx_legfree_()
    buf = np.zeros(64)
    lib.sp2fc_(_p(buf), _p(buf))                      # nothing registered
    assert _status(lib) == BAD_ARG and _status(lib) == 0
    assert _legini(lib, 32, 10, 6, FP64) == BAD_ARG   # real kind 6
    assert _legini(lib, 32, 0, 8, FP64) == BAD_ARG
    assert _legini(lib, 32, 10, 8, 9) == BAD_ARG
    assert _status(lib) == BAD_ARG
    lib.gp2fc_(_p(buf), _ip(14), _ip(1))              # n = 14 is not a supported length
    assert _status(lib) == UNSUPPORTED_N
    lib.fc2gp_(None, _ip(64), _ip(1))
    assert _status(lib) == BAD_ARG
    lib.radstep_(None, None)
    assert _status(lib) == BAD_ARG


def _fields(nlat, nlev, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nlev, nlat, 2 * nlat))


@pytest.mark.gpu
@pytest.mark.parametrize("real_bytes,prec", [(8, FP64), (8, MIXED), (4, FP32)])
def test_fortran_legendre_and_fft(oracle, real_bytes, prec):
    lib = _f()
    lib.exotx_stop_on_error_(_ip(0))
    nlat, nlev = 64, 3
    assert _legini(lib, nlat, nlev, real_bytes, prec) == 0
    L = oracle.Leg(nlat)
    hdt = np.float64 if real_bytes == 8 else np.float32
    tol = 1e-12 if prec == FP64 else 2e-5
    h = lambda a: np.ascontiguousarray(a, dtype=hdt)
    sp = S.spectral_field(np.random.default_rng(1), L.ntru, nlev, "nn1")
    # single-field routines
    for name in ("sp2fc", "sp2fcdmu"):
        fc = np.zeros((nlat, 2 * nlat), dtype=hdt)
        getattr(lib, name + "_")(_p(h(sp[0])), _p(fc))
        assert relerr(fc, getattr(L, name)(sp[0])) < tol, name
    fcin = _fields(nlat, 1, 2)[0]
    out = np.zeros(L.nrsp, dtype=hdt)
    lib.fc2sp_(_p(h(fcin)), _p(out))
    assert relerr(out, L.fc2sp(fcin)) < tol
    # NLEV-level routines
    pz = sp.copy()
    pz[:, 2] += S.EZ
    pu, pv = np.zeros((nlev, nlat, 2 * nlat), dtype=hdt), np.zeros((nlev, nlat, 2 * nlat), dtype=hdt)
    pzh = h(pz)
    pz_before = pzh.copy()
    lib.dv2uv_(_p(h(sp)), _p(pzh), _p(pu), _p(pv))
    ru, rv = L.dv2uv(sp, pz, plavor=S.EZ)
    assert relerr(pu, ru) < tol and relerr(pv, rv) < tol
    assert np.array_equal(pzh, pz_before)
    u, v = _fields(nlat, nlev, 3), _fields(nlat, nlev, 4)
    pd, pzo = np.zeros((nlev, L.nrsp), dtype=hdt), np.zeros((nlev, L.nrsp), dtype=hdt)
    lib.uv2dv_(_p(h(u)), _p(h(v)), _p(pd), _p(pzo))
    rd, rz = L.uv2dv(u, v)
    assert relerr(pd, rd) < tol and relerr(pzo, rz) < tol
    qn, uq, vq = (_fields(nlat, nlev, s) for s in (5, 6, 7))
    q = np.zeros((nlev, L.nrsp), dtype=hdt)
    lib.qtend_(_p(q), _p(h(qn)), _p(h(uq)), _p(h(vq)))
    assert relerr(q, L.qtend(qn, uq, vq)) < tol
    ins = [_fields(nlat, nlev, s) for s in range(10, 16)]   # tn fu fv ke ut vt
    d, t, z = (np.zeros((nlev, L.nrsp), dtype=hdt) for _ in range(3))
    lib.mktend_(_p(d), _p(t), _p(z), *[_p(h(a)) for a in ins])
    for got, ref in zip((d, t, z), L.mktend(*ins)):
        assert relerr(got, ref) < tol
    # FFTs in place on lot rows of length n
    rows = _fields(nlat, 1, 8)[0]
    ref = oracle.gp2fc(rows)
    a = np.array(rows, dtype=hdt)   # a copy: the routine works in place
    lib.gp2fc_(_p(a), _ip(2 * nlat), _ip(nlat))
    assert relerr(a, ref) < (1e-13 if prec == FP64 else 2e-6)
    lib.fc2gp_(_p(a), _ip(2 * nlat), _ip(nlat))
    assert relerr(a, oracle.fc2gp(ref)) < (1e-13 if prec == FP64 else 2e-6)
    assert _status(lib) == 0
    lib.exotx_legfree_()


@pytest.mark.gpu
def test_fortran_inigau(oracle):
    lib = _f()
    lib.exotx_stop_on_error_(_ip(0))
    for nlat in (32, 192):
        z0, zw = np.zeros(nlat), np.zeros(nlat)
        lib.inigau_(_ip(nlat), _p(z0), _p(zw))
        r0, rw = oracle.inigau(nlat)
        assert relerr(z0, r0) < 1e-14 and relerr(zw, rw) < 1e-12
    assert _status(lib) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("real_bytes,prec", [(8, FP64), (4, FP32)])
def test_fortran_radstep(oracle, real_bytes, prec):
    from exoplasim_b200 import radiation as R
    lib = _f()
    lib.exotx_stop_on_error_(_ip(0))
    nlat, nlev = 32, 10
    assert _legini(lib, nlat, nlev, real_bytes, prec) == 0
    cols, g = S.radiation_columns(nlat, nlev, seed=21)
    over = dict(nsol=1, zdecl=0.2, zmins=500.0)
    par = R.default_params(nlev, g["nhor"], g["nlon"], **over)
    sig = [np.array(getattr(par, k)[:nlev]) for k in ("sigma", "sigmah", "dsigma")]
    ref = oracle.radstep(oracle.radpar(nlev, g["nhor"], g["nlon"], *sig, **over), cols["sid"], cols["cola"], cols)
    hdt = np.float64 if real_bytes == 8 else np.float32
    host = {k: np.ascontiguousarray(v, dtype=hdt) for k, v in cols.items()}
    nlep = nlev + 1
    for k in ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux"):
        host[k] = np.zeros((nlep, g["nhor"]), dtype=hdt)
    for k in ("dtdtswr", "dtdtlwr", "dconv"):
        host[k] = np.zeros((nlev, g["nhor"]), dtype=hdt)
    io = _lib.RadIO()
    for name in _lib.RAD_IO_FIELDS:
        if name in host:
            setattr(io, name, host[name].ctypes.data)
    lib.radstep_(C.byref(par), C.byref(io))
    assert _status(lib) == 0
    if prec == FP64:
        for k in ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux", "dtdt", "dtdtswr", "dtdtlwr", "dconv",
                  "gmu0", "dqo3", "dalb", "dsalb"):
            assert relerr(host[k], ref[k]) < 1e-11, k
    else:
        assert np.max(np.abs(host["gmu0"] - ref["gmu0"])) < 1e-5
        col = np.max(np.abs(host["dflux"] - ref["dflux"]), axis=0) / np.max(np.abs(ref["dflux"]))
        assert np.median(col) < 1e-5
    lib.exotx_legfree_()

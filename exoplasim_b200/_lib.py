"""ctypes binding of libexotx.so (the C ABI declared in include/exotx.h).

The library is built in-tree by exoplasim_b200.build.  There is no fallback:
if the shared library is missing or does not load, every entry point raises.
"""
import ctypes as C
import os
import re

from . import build as _build

FP64, FP32, MIXED = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32": FP32, "mixed": MIXED}

STATUS = {0: "ok", 1: "unsupported dimension", 2: "FFT length not supported", 3: "bad argument",
          4: "CUDA error", 5: "out of device memory", 6: "device wait timed out",
          7: "path not available in this build"}


class ExotxError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: {STATUS.get(code, code)} (status {code})")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("nlat", C.c_int), ("nfilter", C.c_int), ("ngptfilter", C.c_int), ("nspvfilter", C.c_int),
                ("landhoskn0", C.c_double), ("filterkappa", C.c_double), ("nfilterexp", C.c_int),
                ("pyfft_nfs", C.c_int), ("plavor", C.c_double)]


class RadParams(C.Structure):
    _fields_ = ([("nlev", C.c_int), ("nhor", C.c_int), ("nlon", C.c_int)] +
                [(n, C.c_double) for n in ("ga", "gascon", "acpd", "adv", "gsol0", "gdist2", "zsolar1",
                                           "zsolar2", "rcoeff", "tswr1", "tswr2", "tswr3", "tpofmt", "acllwr",
                                           "th2oc", "clgray", "a0o3", "a1o3", "aco3", "bo3", "co3", "toffo3",
                                           "o3scale")] +
                [("rcl1", C.c_double * 3), ("rcl2", C.c_double * 3), ("acl2", C.c_double * 3)] +
                [(n, C.c_int) for n in ("ndcycle", "no3", "nswrcl", "nclouds", "nrscat", "newrsc", "necham",
                                        "necham6", "nstartemp", "npbroaden", "nswr", "nlwr", "nsol", "nfixed",
                                        "ncstsol", "ngenkeplerian")] +
                [(n, C.c_double) for n in ("zdecl", "zmins", "zrtim", "rasc", "dawn", "solclat", "solcdec",
                                           "zcday")] +
                [("sigma", C.c_double * 64), ("sigmah", C.c_double * 64), ("dsigma", C.c_double * 64)])


RAD_IO_FIELDS = ("sid", "cola", "dt", "dq", "dcc", "dql", "dqco2", "dp", "dls", "dicec", "dqo3", "gmu0",
                 "dalb", "dsalb", "dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux", "dtdt", "dtdtswr",
                 "dtdtlwr", "dconv", "zsol")


class RadIO(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in RAD_IO_FIELDS]


_lib = None

_P, _I, _D, _S = C.c_void_p, C.c_int, C.c_double, C.c_void_p
SIGNATURES = {
    "exotx_grid_desc_default": [_I, C.POINTER(GridDesc)],
    "exotx_plan_create": [C.POINTER(GridDesc), C.POINTER(C.c_void_p)],
    "exotx_plan_destroy": [_P],
    "exotx_plan_dims": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "exotx_plan_gauss": [_P, _P, _P],
    "exotx_plan_table": [_P, _I, _P],
    "exotx_inigau": [_I, _P, _P, _S],
    "exotx_sp2fc": [_P, _I, _P, _P, _I, _S],
    "exotx_sp2fcdmu": [_P, _I, _P, _P, _I, _S],
    "exotx_fc2sp": [_P, _I, _P, _P, _I, _S],
    "exotx_dv2uv": [_P, _I, _P, _P, _P, _P, _I, _S],
    "exotx_uv2dv": [_P, _I, _P, _P, _P, _P, _I, _S],
    "exotx_mktend": [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _S],
    "exotx_qtend": [_P, _I, _P, _P, _P, _P, _I, _S],
    "exotx_gp2fc": [_I, _P, _I, _I, _S],
    "exotx_fc2gp": [_I, _P, _I, _I, _S],
    "exotx_inverse_set": [_P, _I, _P, _P, _I, _S],
    "exotx_forward_set": [_P, _I, _P, _P, _I, _S],
    "exotx_rad_params_default": [_I, _I, _I, C.POINTER(RadParams)],
    "exotx_solarini": [_D, _D, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)],
    "exotx_radstep": [C.POINTER(RadParams), _I, C.POINTER(RadIO), _S],
    "exotx_tc_selftest": [_P, _P, _P, _I, _I, _I, _S],
    "exotx_inverse_set_batch": [_P, _I, _P, _P, _I, _I, _S],
    "exotx_forward_set_batch": [_P, _I, _P, _P, _I, _I, _S],
    "exotx_inverse_set_d": [_P, _I, _P, _P, _I, _S],
    "exotx_forward_set_d": [_P, _I, _P, _P, _I, _S],
    "exotx_inverse_set_d_batch": [_P, _I, _P, _P, _I, _I, _S],
    "exotx_forward_set_d_batch": [_P, _I, _P, _P, _I, _I, _S],
    "exotx_raw_size": [_P, _I, C.POINTER(C.c_size_t)],
    "exotx_gp_params_default": [_I, _P],
    "exotx_gp_params_derive": [_P],
    "exotx_gpconst_create": [_P, C.POINTER(C.c_void_p)],
    "exotx_gpconst_destroy": [_P],
    "exotx_gridpoint": [_P, _P, _I, _P, _P, _P, _P, _I, _S],
    "exotx_spec_params_default": [_I, _P],
    "exotx_plan_tune": [_P, _I, C.c_longlong],
    "exotx_specconst_create": [_P, _P, C.POINTER(C.c_void_p)],
    "exotx_specconst_destroy": [_P],
    "exotx_spectrala": [_P, _I, _P, _S],
    "exotx_spectrald": [_P, _I, _P, _S],
    "exotx_spectrala_batch": [_P, _I, _P, _I, _S],
    "exotx_spectrald_batch": [_P, _I, _P, _I, _S],
    "exotx_raw_pack": [_P, _I, _P, _S],
    "exotx_sets_host": [_P, _I, _P, _P, _P, _P, _I, _I, _S],
    "exotx_sets_host_f64": [_P, _I, _P, _P, _P, _P, _I, _I, _S],
    "exotx_forward_set_noalloc": [_P, _I, _P, _P, _I, _S],
    "exotx_kernel_timing": [_I],
    "exotx_ensemble_create": [_I, _P, _P, C.POINTER(C.c_void_p)],
    "exotx_ensemble_destroy": [_P],
    "exotx_ensemble_layout": [_P, _P, _P, _P, _P],
    "exotx_ensemble_inverse": [_P, _P, _P, _S],
    "exotx_ensemble_forward": [_P, _P, _P, _S],
    "exotx_ensemble_configure": [_P, _I, _I, _I, _I],
    "exotx_ensemble_tune": [_P, _P, _P, _P, _P, _I, _S, _P, _P],
    "exotx_mlp_create": [_I, _I, _I, _I, _I, C.POINTER(C.c_void_p)],
    "exotx_mlp_destroy": [_P],
    "exotx_mlp_params": [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_longlong)],
    "exotx_mlp_layer": [_P, _I, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(_I), C.POINTER(_I)],
    "exotx_mlp_set_norm": [_P, _P],
    "exotx_mlp_forward": [_P, _P, _P, _I, _S],
    "exotx_mlp_backward": [_P, _P, _P, _I, _P, _S],
    "exotx_mlp_backward_weighted": [_P, _P, _P, _P, _I, _P, _S],
    "exotx_mlp_check": [_P, _S],
    "exotx_mlp_adam": [_P, C.c_float, C.c_float, C.c_float, C.c_float, _I, _S],
    "exotx_mlp_prepare": [_P, _S],
    "exotx_surr_features": [C.POINTER(RadParams), _I, C.POINTER(RadIO), _P, _S],
    "exotx_surr_targets": [C.POINTER(RadParams), _I, C.POINTER(RadIO), _P, _S],
    "exotx_rad_surrogate": [_P, C.POINTER(RadParams), _I, C.POINTER(RadIO), C.POINTER(_I), _S],
    "exotx_kernel_time": [_I, C.POINTER(_D), C.POINTER(C.c_longlong)],
    "exotx_tc_error": [C.POINTER(_I), _S],
}
RESTYPES = {"exotx_fft_supported": C.c_int, "exotx_launch_count": C.c_ulonglong,
            "exotx_status_string": C.c_char_p}


def lib_path():
    return _build.LIB


def load(build_if_missing=True):
    """Load libexotx.so; build it first if it is missing and nvcc exists."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"libexotx.so not built ({path}); run python -m exoplasim_b200.build")
        _build.build()
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    for name, rt in RESTYPES.items():
        getattr(lib, name).restype = rt
    lib.exotx_fft_supported.argtypes = [_I]
    lib.exotx_status_string.argtypes = [_I]
    _lib = lib
    return lib


def check(fn, code):
    if code != 0:
        raise ExotxError(fn, code)


def call(name, *args):
    """Call an exotx entry point and raise ExotxError on a non-OK status."""
    f = getattr(load(), name)
    check(name, f(*args))


def declared_symbols():
    """Function names declared in include/*.h (for the ABI export test)."""
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    names = []
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(inc, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(exotx_\w+|\w+_)\s*\(", txt, flags=re.M)
    return sorted(set(names))

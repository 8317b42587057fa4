"""The C-ABI library loads, exports every function include/*.h declares, and
its host-side logic (argument validation, FFT length support, parameter
defaults, the solarini band split) behaves -- all without a GPU."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from exoplasim_b200 import _lib
from exoplasim_b200 import radiation as R


def test_library_exports_declared_symbols():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 24
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.lib_path()], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        assert hasattr(lib, s)


def test_fft_supported_lengths():
    lib = _lib.load()
    for n in (4, 8, 16, 32, 48, 64, 96, 128, 192, 256, 320, 384, 512, 1024, 4096, 60, 160):
        assert lib.exotx_fft_supported(n) == 1, n
    for n in (0, 2, 7, 14, 28, 4098, 8192, 44):
        assert lib.exotx_fft_supported(n) == 0, n


def test_host_validation_without_gpu():
    lib = _lib.load()
    d = _lib.GridDesc()
    assert lib.exotx_grid_desc_default(32, C.byref(d)) == 0
    assert abs(d.plavor - 1.63299310207) < 1e-15 and d.pyfft_nfs == -1
    h = C.c_void_p()
    d.nlat = 7
    assert lib.exotx_plan_create(C.byref(d), C.byref(h)) == 1          # BAD_DIM
    d.nlat = 14
    assert lib.exotx_plan_create(C.byref(d), C.byref(h)) == 2          # NLON=28 unsupported
    d.nlat = 32
    d.nfilter = 9
    assert lib.exotx_plan_create(C.byref(d), C.byref(h)) == 3          # bad filter
    assert lib.exotx_sp2fc(None, 0, None, None, 1, None) == 3
    assert lib.exotx_gp2fc(0, None, 64, 1, None) == 3
    assert lib.exotx_gp2fc(7, C.c_void_p(16), 64, 1, None) == 3        # bad precision
    assert lib.exotx_radstep(None, 0, None, None) == 3
    assert lib.exotx_status_string(2) == b"FFT length not supported"


def test_rad_params_default():
    p = R.default_params(20, 8192, 128)
    assert p.nlev == 20 and p.no3 == 1 and p.ndcycle == 1 and p.nswrcl == 1
    sh = np.array(p.sigmah[:20])
    z = np.arange(1, 21) / 20
    assert np.allclose(sh, 0.75 * z + 1.75 * z ** 3 - 1.5 * z ** 4, rtol=0, atol=1e-15)
    assert abs(sum(p.dsigma[:20]) - 1.0) < 1e-15
    with pytest.raises(_lib.ExotxError):
        R.default_params(65, 10, 10)


@pytest.mark.parametrize("teff", [2500.0, 3300.0, 5772.0, 6000.0])
def test_solarini_matches_oracle(oracle, teff):
    a = R.solarini(teff)
    b = oracle.solarini(teff)
    assert np.allclose(a, b, rtol=1e-13, atol=0)

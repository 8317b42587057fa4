"""exoplasim_b200.pyfft / pyfft991 (the drop-in for the f2py modules pyburn
imports) against the FP64 restatement of pyfft.f90 in oracle/pyfft_oracle.py.

Called the way pyburn calls them (pyburn.py:711, 810, 840, 867, 1067, 1172):
Fortran-ordered numpy arrays in, f2py-shaped numpy arrays out; torch CUDA
tensors in give the same values as CUDA tensors.  Tolerance: FP64,
max|x-ref|/max|ref| below 1e-12 per output.
"""
import numpy as np
import pytest
import torch

from exoplasim_b200 import pyfft as PF
from exoplasim_b200 import pyfft991 as PF991
from exoplasim_b200 import synthetic as S
from tests._util import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-12
NLEV = 3
# (nlat, the oracle FFT): T21 and T42 use fftmod; T63's NLON=192 is FFT991-only
RES = [(32, False), (64, False), (96, True)]


def _sp(ntru, seed):
    """(NRSP, nlev) Fortran-ordered, as pyburn builds it"""
    return np.asfortranarray(S.spectral_field(np.random.default_rng(seed), ntru, NLEV, "nn1").T)


def _po():
    from oracle import pyfft_oracle as PO
    return PO


@pytest.mark.parametrize("nfs", [0, 1])
@pytest.mark.parametrize("nlat,use991", RES)
def test_scalar_transforms(nlat, use991, nfs):
    PO = _po()
    nlon, ntru = 2 * nlat, (2 * nlat - 1) // 3
    sp = _sp(ntru, nlat + nfs)
    gp = PF.sp2gp(sp, nlat, nlon, ntru, nfs)
    ref = PO.sp2gp(sp, nlat, nlon, ntru, nfs, use991=use991)
    assert isinstance(gp, np.ndarray) and gp.shape == (nlon, nlat, NLEV)
    assert relerr(gp, ref) < TOL
    grid = np.asfortranarray(np.random.default_rng(nlat).standard_normal((nlon, nlat, NLEV)))
    s2 = PF.gp2sp(grid, nlat, nlon, ntru, nfs)
    assert s2.shape == (2 * (ntru + 1) * (ntru + 2) // 2, NLEV)
    assert relerr(s2, PO.gp2sp(grid, nlat, nlon, ntru, nfs, use991=use991)) < TOL
    fc = PF.sp3fc(sp, nlat, nlon, ntru, nfs)
    assert fc.shape == (2, nlon // 2, nlat, NLEV)
    assert relerr(fc, PO.sp3fc(sp, nlat, nlon, ntru, nfs)) < TOL


@pytest.mark.parametrize("nfs", [0, 1])
@pytest.mark.parametrize("nlat,use991", RES)
def test_vector_transforms(nlat, use991, nfs):
    PO = _po()
    nlon, ntru = 2 * nlat, (2 * nlat - 1) // 3
    sd, sz = _sp(ntru, 5), _sp(ntru, 6)
    sid, _ = PF.inigau(nlat)
    cs = np.sqrt(1.0 - sid ** 2)
    rdc = 6.371e6 / cs
    gu, gv = PF.spvgp(sd, sz, rdc, nlon, ntru, nfs)
    ru, rv = PO.spvgp(sd, sz, rdc, nlon, ntru, nfs, use991=use991)
    assert gu.shape == gv.shape == (nlon, nlat, NLEV)
    assert relerr(gu, ru) < TOL and relerr(gv, rv) < TOL
    grid = np.random.default_rng(nlat + 1).standard_normal((2, nlon, nlat, NLEV))
    d, z = PF.gpvsp(grid[0], grid[1], cs / 6.371e6, ntru, nfs)
    rd, rz = PO.gpvsp(grid[0], grid[1], cs / 6.371e6, ntru, nfs, use991=use991)
    assert relerr(d, rd) < TOL and relerr(z, rz) < TOL
    pu, pv = PF.dv2uv(sd, sz, nlat, nlon, ntru, NLEV, nfs)
    qu, qv = PO.dv2uv(sd, sz, nlat, nlon, ntru, nfs)
    assert pu.shape == (2, nlon // 2, nlat, NLEV)
    assert relerr(pu, qu) < TOL and relerr(pv, qv) < TOL
    pd, pz = PF.uv2dv(qu, qv, nlat, nlon, ntru, NLEV, nfs)
    qd, qz = PO.uv2dv(qu, qv, nlat, nlon, ntru, nfs)
    assert pd.shape == (2, (ntru + 1) * (ntru + 2) // 2, NLEV)
    assert relerr(pd, qd) < TOL and relerr(pz, qz) < TOL


@pytest.mark.parametrize("nlat,use991", RES)
def test_fourier_levels_and_gauss(nlat, use991):
    PO = _po()
    nlon = 2 * nlat
    a = np.asfortranarray(np.random.default_rng(2).standard_normal((nlon, nlat, NLEV)))
    c = PF.gp3fc(a)
    assert c.shape == a.shape and relerr(c, PO.gp3fc(a, use991=use991)) < TOL
    g = PF.fc3gp(c)
    assert relerr(g, PO.fc3gp(c, use991=use991)) < TOL
    sid, gwd = PF.inigau(nlat)
    rs, rw = PO.inigau(nlat)
    assert relerr(sid, rs) < 1e-14 and relerr(gwd, rw) < 1e-12


def test_torch_tensors_stay_on_device_and_pyfft991_is_the_same():
    nlat, nlon, ntru = 64, 128, 42
    sp = _sp(ntru, 9)
    gp = PF.sp2gp(sp, nlat, nlon, ntru, 0)
    gt = PF.sp2gp(torch.as_tensor(sp, device="cuda"), nlat, nlon, ntru, 0)
    assert isinstance(gt, torch.Tensor) and gt.is_cuda
    assert np.array_equal(gt.cpu().numpy(), gp)
    assert np.array_equal(PF991.sp2gp(sp, nlat, nlon, ntru, 0), gp)
    assert PF991.spvgp is PF.spvgp


def test_t127_sp2gp_for_pyfft991():
    """NLAT 192 is where pyburn switches to pyfft991 (pyburn.py:594-602)."""
    PO = _po()
    nlat, nlon, ntru = 192, 384, 127
    sp = _sp(ntru, 11)[:, :1]
    gp = PF991.sp2gp(sp, nlat, nlon, ntru, 1)
    assert relerr(gp, PO.sp2gp(sp, nlat, nlon, ntru, 1)) < TOL


def test_wrong_truncation_is_rejected():
    sp = _sp(21, 1)
    with pytest.raises(ValueError):
        PF.sp2gp(sp, 32, 64, 20, 0)
    with pytest.raises(ValueError):
        PF.sp2gp(sp, 32, 96, 21, 0)

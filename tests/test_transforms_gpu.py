"""Parity of the CUDA transform path (through the C ABI) against the FP64 oracle.

Tolerances: FP64 path <= 1e-12 norm-wise relative error (max|gpu-oracle| /
max|oracle| per field); FP32 path <= 2e-5; FFT alone <= 1e-13 (FP64).
"""
import numpy as np
import pytest
import torch

from exoplasim_b200 import synthetic as S
from exoplasim_b200._lib import ExotxError
from exoplasim_b200.transforms import TABLES, Plan, fc2gp, gp2fc
from tests._util import relerr

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5
RES = [32, 64, 96, 192]   # T21, T42, T63 (NLON=192), T127


@pytest.fixture(scope="module")
def plans():
    return {n: Plan(n) for n in RES + [256, 8]}


def _spec(ntru, nlev, seed, kind="nn1"):
    return S.spectral_field(np.random.default_rng(seed), ntru, nlev, kind)


def _cuda(a, dt=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


@pytest.mark.parametrize("nlat", RES + [256])
def test_gauss_and_tables(plans, oracle, nlat):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    sid, gwd = P.gauss()
    # the Newton iteration converges to the same roots; the weights carry the
    # last-ulp differences of acos/cos through 1/P'(mu)^2 (gaussmod.f90:35-36)
    assert relerr(sid, L.table("sid")) < 1e-14
    assert relerr(gwd, L.table("gwd")) < 1e-12
    for t in TABLES:
        ref = L.table(t).reshape(nlat, L.ncsp)
        assert relerr(P.table(t), ref) < 1e-12, t


@pytest.mark.parametrize("nlat", RES)
@pytest.mark.parametrize("op", ["sp2fc", "sp2fcdmu"])
def test_inverse_single(plans, oracle, nlat, op):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    sp = _spec(P.ntru, 3, seed=nlat)
    out = getattr(P, op)(_cuda(sp)).cpu().numpy()
    for v in range(3):
        ref = getattr(L, op)(sp[v])
        assert relerr(out[v], ref) < FP64_TOL
    out32 = getattr(P, op)(_cuda(sp, torch.float32), precision="fp32").cpu().numpy()
    for v in range(3):
        assert relerr(out32[v], getattr(L, op)(sp[v])) < FP32_TOL


@pytest.mark.parametrize("nlat", RES)
def test_dv2uv(plans, oracle, nlat):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    nlev = 4
    pd = _spec(P.ntru, nlev, 1)
    pz = _spec(P.ntru, nlev, 2)
    pz[:, 2] += S.EZ
    u, v = P.dv2uv(_cuda(pd), _cuda(pz))
    ru, rv = L.dv2uv(pd, pz, plavor=S.EZ)
    assert relerr(u.cpu().numpy(), ru) < FP64_TOL
    assert relerr(v.cpu().numpy(), rv) < FP64_TOL
    u32, v32 = P.dv2uv(_cuda(pd, torch.float32), _cuda(pz, torch.float32), precision="fp32")
    assert relerr(u32.cpu().numpy(), ru) < FP32_TOL
    assert relerr(v32.cpu().numpy(), rv) < FP32_TOL


def _fourier(nlat, nlev, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nlev, nlat, 2 * nlat))


@pytest.mark.parametrize("nlat", RES)
def test_fc2sp(plans, oracle, nlat):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    fc = _fourier(nlat, 3, 5)
    out = P.fc2sp(_cuda(fc)).cpu().numpy()
    for v in range(3):
        assert relerr(out[v], L.fc2sp(fc[v], folded=True)) < FP64_TOL
        # the unfolded (parallel) branch agrees too
        assert relerr(out[v], L.fc2sp(fc[v], folded=False)) < FP64_TOL
    out32 = P.fc2sp(_cuda(fc, torch.float32), precision="fp32").cpu().numpy()
    assert relerr(out32[1], L.fc2sp(fc[1])) < FP32_TOL


@pytest.mark.parametrize("nlat", RES)
def test_uv2dv_qtend_mktend(plans, oracle, nlat):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    nlev = 2
    f = [_fourier(nlat, nlev, 10 + i) for i in range(6)]
    pd, pz = P.uv2dv(_cuda(f[0]), _cuda(f[1]))
    rd, rz = L.uv2dv(f[0], f[1])
    assert relerr(pd.cpu().numpy(), rd) < FP64_TOL
    assert relerr(pz.cpu().numpy(), rz) < FP64_TOL
    q = P.qtend(_cuda(f[0]), _cuda(f[1]), _cuda(f[2]))
    assert relerr(q.cpu().numpy(), L.qtend(f[0], f[1], f[2])) < FP64_TOL
    d, t, z = P.mktend(*[_cuda(x) for x in f])
    rd, rt, rz = L.mktend(*f)
    for a, b in ((d, rd), (t, rt), (z, rz)):
        assert relerr(a.cpu().numpy(), b) < FP64_TOL
    d32, t32, z32 = P.mktend(*[_cuda(x, torch.float32) for x in f], precision="fp32")
    for a, b in ((d32, rd), (t32, rt), (z32, rz)):
        assert relerr(a.cpu().numpy(), b) < FP32_TOL


FFT_N = [16, 32, 64, 96, 128, 256, 384, 512, 1024]


def test_fft_n8_follows_the_contract():
    # For n = 8 fftmod.f90 runs dfft8 alone (:44) and never inserts the zero
    # imaginary slot of m=0 that dfft4 adds when la = 1 (:310-315), so its
    # output packs (A0,A1,B1,...,A4).  This library keeps the layout of every
    # other length, (A0,0,A1,B1,A2,B2,A3,B3), checked against numpy here.
    x = np.random.default_rng(8).standard_normal((3, 8))
    a = _cuda(x)
    gp2fc(a)
    c = np.fft.rfft(x, axis=-1) / 8
    exp = np.zeros_like(x)
    exp[:, 0::2] = c.real[:, :4]
    exp[:, 1::2] = c.imag[:, :4]
    assert relerr(a.cpu().numpy(), exp) < 1e-14


@pytest.mark.parametrize("n", FFT_N)
def test_fft_fp64_vs_fftmod(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((7, n))
    a = _cuda(x)
    gp2fc(a)
    ref = oracle.gp2fc(x)
    assert relerr(a.cpu().numpy(), ref) < 1e-13
    fc2gp(a)
    assert relerr(a.cpu().numpy(), oracle.fc2gp(ref)) < 1e-13
    # round trip recovers the grid when the Nyquist term is zero
    back = oracle.fc2gp(oracle.gp2fc(x))
    assert relerr(a.cpu().numpy(), back) < 1e-13


@pytest.mark.parametrize("n", [64, 96, 128, 192, 256, 320, 384])
def test_fft_fp64_vs_fft991(oracle, n):
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal((5, n))
    a = _cuda(x)
    gp2fc(a)
    ref = oracle.gp2fc(x, use991=True)
    assert relerr(a.cpu().numpy(), ref) < 1e-13
    f = rng.standard_normal((5, n))
    b = _cuda(f)
    fc2gp(b)
    assert relerr(b.cpu().numpy(), oracle.fc2gp(f, use991=True)) < 1e-13


def test_fft_n48_is_a_true_dft():
    # fftmod.f90 lists n=48 but its radix schedule (8, then 4 while la >= 4)
    # cannot factor 48/8 = 6, so the reference does not return a DFT there;
    # this library computes the transform the contract defines.
    rng = np.random.default_rng(48)
    x = rng.standard_normal((3, 48))
    a = _cuda(x)
    gp2fc(a)
    ref = np.fft.rfft(x, axis=-1) / 48
    exp = np.zeros_like(x)
    exp[:, 0::2] = ref.real[:, :24]
    exp[:, 1::2] = ref.imag[:, :24]
    exp[:, 1] = 0
    assert relerr(a.cpu().numpy(), exp) < 1e-14


@pytest.mark.parametrize("n", [64, 192, 384])
def test_fft_fp32(oracle, n):
    rng = np.random.default_rng(n + 7)
    x = rng.standard_normal((9, n))
    a = _cuda(x, torch.float32)
    gp2fc(a)
    ref = oracle.gp2fc(x, use991=(n == 192))
    assert relerr(a.cpu().numpy(), ref) < 2e-6


@pytest.mark.parametrize("rows", [1, 9, 32, 70])
def test_fft_fp32_384_rows(oracle, rows):
    # n = 384 runs the register-resident kernels: 32 rows per block, bulk copies
    # of even row runs and a plain-load path otherwise; partial blocks, odd
    # counts and the row-major Fourier side (k fastest across threads)
    rng = np.random.default_rng(rows + 384)
    x = rng.standard_normal((rows, 384))
    a = _cuda(x, torch.float32)
    gp2fc(a)
    ref = oracle.gp2fc(x)
    assert relerr(a.cpu().numpy(), ref) < 2e-6
    f = rng.standard_normal((rows, 384))
    b = _cuda(f, torch.float32)
    fc2gp(b)
    assert relerr(b.cpu().numpy(), oracle.fc2gp(f)) < 2e-6


def test_fft_bad_lengths():
    for n in (14, 7, 5000, 2):
        a = torch.zeros((2, n), dtype=torch.float64, device="cuda")
        with pytest.raises(ExotxError) as e:
            gp2fc(a)
        assert e.value.code in (2, 3)


def test_bad_args(plans):
    P = plans[32]
    with pytest.raises(TypeError):
        P.sp2fc(torch.zeros((1, P.nrsp), dtype=torch.float32, device="cuda"))  # dtype mismatch
    with pytest.raises(ValueError):
        P.sp2fc(torch.zeros((1, P.nrsp + 2), dtype=torch.float64, device="cuda"))
    with pytest.raises(ExotxError):
        Plan(7)    # odd NLAT
    with pytest.raises(ExotxError):
        Plan(14)   # NLON = 28 = 4*7: no radix-7 pass


def test_zero_levels_is_a_noop(plans):
    P = plans[32]
    sp = torch.zeros((0, P.nrsp), dtype=torch.float64, device="cuda")
    out = P.sp2fc(sp)
    assert out.shape == (0, 32, 64)


def test_smallest_resolution(plans, oracle):
    P = plans[8]  # NLON=16, NTRU=5
    L = oracle.Leg(8)
    sp = _spec(P.ntru, 2, 3)
    out = P.sp2fc(_cuda(sp)).cpu().numpy()
    assert relerr(out[0], L.sp2fc(sp[0])) < FP64_TOL


@pytest.mark.parametrize("nlat,nlev", [(32, 10), (64, 20), (96, 10), (192, 20), (256, 25)])
def test_transform_sets_fp64(plans, oracle, nlat, nlev):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    spin = S.transform_state(P.ntru, nlev, seed=3)
    gp = P.inverse_set(_cuda(spin), nlev).cpu().numpy().reshape(6 * nlev + 3, -1)
    ref = L.inverse_set(spin, nlev, plavor=S.EZ, use991=(2 * nlat not in (8, 16, 32, 64, 96, 128, 256, 384, 512)))
    for f in range(6 * nlev + 3):
        assert relerr(gp[f], ref[f]) < FP64_TOL, f
    gin = S.grid_tendencies(nlat, nlev, seed=4)
    gin_t = _cuda(gin)
    spout = P.forward_set(gin_t, nlev).cpu().numpy()
    refs = L.forward_set(gin.reshape(9 * nlev + 1, -1), nlev,
                         use991=(2 * nlat not in (8, 16, 32, 64, 96, 128, 256, 384, 512)))
    for f in range(4 * nlev + 1):
        assert relerr(spout[f], refs[f]) < FP64_TOL, f
    # the forward set leaves its input unchanged
    assert np.array_equal(gin_t.cpu().numpy(), gin)


@pytest.mark.parametrize("nlat,nlev", [(64, 20), (192, 20), (256, 25)])
def test_transform_sets_fp32(plans, oracle, nlat, nlev):
    P = plans[nlat]
    L = oracle.Leg(nlat)
    spin = S.transform_state(P.ntru, nlev, seed=5, kind="steep" if nlat >= 192 else "nn1")
    gp = P.inverse_set(_cuda(spin, torch.float32), nlev, precision="fp32").cpu().numpy().reshape(6 * nlev + 3, -1)
    ref = L.inverse_set(spin, nlev, plavor=S.EZ)
    errs = [relerr(gp[f], ref[f]) for f in range(6 * nlev + 3)]
    assert max(errs) < 1e-5
    gin = S.grid_tendencies(nlat, nlev, seed=6)
    spout = P.forward_set(_cuda(gin, torch.float32), nlev, precision="fp32").cpu().numpy()
    refs = L.forward_set(gin.reshape(9 * nlev + 1, -1), nlev)
    errs = [relerr(spout[f], refs[f]) for f in range(4 * nlev + 1)]
    assert max(errs) < 1e-5


def test_roundtrip_identity_t127(plans):
    # size-independent property at full size: sp -> grid -> sp recovers a
    # truncated field (FP64), through the C ABI.
    P = plans[192]
    sp = _spec(P.ntru, 2, 9, kind="steep")
    g = P.sp2fc(_cuda(sp))
    fc2gp(g)
    gp2fc(g)
    back = P.fc2sp(g).cpu().numpy()
    assert relerr(back, sp) < 1e-10


# the model's spectral filters (legmod.f90:124-155): Cesaro, exponential,
# Lander-Hoskins and Riesz-2, applied grid->spectral (ngptfilter) and
# spectral->grid (nspvfilter), through the plan the GPU builds
FILTERS = [dict(nfilter=1, ngptfilter=1, nspvfilter=1),
           dict(nfilter=2, ngptfilter=1, nspvfilter=1, filterkappa=6.0, nfilterexp=6),
           dict(nfilter=3, ngptfilter=1, nspvfilter=1, landhoskn0=12.0),
           dict(nfilter=4, ngptfilter=1, nspvfilter=0),
           dict(nfilter=2, ngptfilter=0, nspvfilter=1)]


@pytest.mark.parametrize("filt", range(len(FILTERS)))
def test_model_filters(oracle, filt):
    kw = FILTERS[filt]
    nlat, nlev = 64, 4
    P = Plan(nlat, **kw)
    L = oracle.Leg(nlat, **kw)
    for t in TABLES:
        assert relerr(P.table(t), L.table(t).reshape(nlat, L.ncsp)) < 1e-12, t
    sp = _spec(P.ntru, 2, seed=17)
    fc = P.sp2fc(_cuda(sp)).cpu().numpy()
    for v in range(2):
        assert relerr(fc[v], L.sp2fc(sp[v])) < FP64_TOL
    gin = np.random.default_rng(18).standard_normal((2, nlat, 2 * nlat))
    fsp = P.fc2sp(_cuda(gin)).cpu().numpy()
    for v in range(2):
        assert relerr(fsp[v], L.fc2sp(gin[v])) < FP64_TOL
    # whole sets in FP64 and on the tensor cores (the filter is folded into
    # the split tables there)
    spin = S.transform_state(P.ntru, nlev, seed=19)
    ref = L.inverse_set(spin, nlev, plavor=S.EZ)
    gp = P.inverse_set(_cuda(spin), nlev).cpu().numpy().reshape(6 * nlev + 3, -1)
    gpm = P.inverse_set(_cuda(spin, torch.float32), nlev, precision="mixed").cpu().numpy().reshape(6 * nlev + 3, -1)
    g4 = S.grid_tendencies(nlat, nlev, seed=20)
    refs = L.forward_set(g4.reshape(9 * nlev + 1, -1), nlev)
    spo = P.forward_set(_cuda(g4), nlev).cpu().numpy()
    spm = P.forward_set(_cuda(g4, torch.float32), nlev, precision="mixed").cpu().numpy()
    for f in range(6 * nlev + 3):
        assert relerr(gp[f], ref[f]) < FP64_TOL, f
        assert relerr(gpm[f], ref[f]) < 5e-6, f
    for f in range(4 * nlev + 1):
        assert relerr(spo[f], refs[f]) < FP64_TOL, f
        assert relerr(spm[f], refs[f]) < 5e-6, f

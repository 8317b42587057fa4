"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

The oracle restates ExoPlaSim's gaussmod.f90, legmod.f90, fftmod.f90,
fft991mod.f90 and radmod.f90 in C (exo_oracle_*.c, built by oracle/Makefile).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the exoplasim_b200 package never does.

All arrays use the reference's memory layouts (see exo_oracle.h).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)


def build():
    """Compile the oracle with its Makefile (gcc, no Fortran needed)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class LegTables(C.Structure):
    _fields_ = [("ntru", C.c_int), ("nlat", C.c_int), ("nlon", C.c_int), ("ncsp", C.c_int),
                ("sid", _dp), ("gwd", _dp),
                ("qi", _dp), ("qj", _dp), ("qc", _dp), ("qe", _dp),
                ("qm", _dp), ("qq", _dp), ("qu", _dp), ("qv", _dp),
                ("skgpsp", _dp), ("skspgp", _dp)]


class RadPar(C.Structure):
    _fields_ = [("nlev", C.c_int), ("nhor", C.c_int), ("nlon", C.c_int),
                ("sigma", _dp), ("sigmah", _dp), ("dsigma", _dp),
                ("ga", C.c_double), ("gascon", C.c_double), ("acpd", C.c_double), ("adv", C.c_double),
                ("gsol0", C.c_double), ("gdist2", C.c_double), ("zsolar1", C.c_double),
                ("zsolar2", C.c_double), ("rcoeff", C.c_double),
                ("tswr1", C.c_double), ("tswr2", C.c_double), ("tswr3", C.c_double),
                ("tpofmt", C.c_double), ("acllwr", C.c_double), ("th2oc", C.c_double), ("clgray", C.c_double),
                ("a0o3", C.c_double), ("a1o3", C.c_double), ("aco3", C.c_double), ("bo3", C.c_double),
                ("co3", C.c_double), ("toffo3", C.c_double), ("o3scale", C.c_double),
                ("rcl1", C.c_double * 3), ("rcl2", C.c_double * 3), ("acl2", C.c_double * 3),
                ("ndcycle", C.c_int), ("no3", C.c_int), ("nswrcl", C.c_int), ("nclouds", C.c_int),
                ("nrscat", C.c_int), ("newrsc", C.c_int), ("necham", C.c_int), ("necham6", C.c_int),
                ("nstartemp", C.c_int), ("npbroaden", C.c_int), ("nswr", C.c_int), ("nlwr", C.c_int),
                ("nsol", C.c_int),
                ("nfixed", C.c_int), ("ncstsol", C.c_int), ("ngenkeplerian", C.c_int),
                ("zdecl", C.c_double), ("zmins", C.c_double), ("zrtim", C.c_double), ("rasc", C.c_double),
                ("dawn", C.c_double), ("solclat", C.c_double), ("solcdec", C.c_double),
                ("zcday", C.c_double)]


class RadIO(C.Structure):
    _fields_ = [(n, _dp) for n in (
        "sid", "cola", "dt", "dq", "dcc", "dql", "dqco2", "dp", "dls", "dicec",
        "dqo3", "gmu0", "dalb", "dsalb",
        "dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux",
        "dtdt", "dtdtswr", "dtdtlwr", "dconv")]


def _declare(L):
    P = C.POINTER
    L.oracle_inigau.argtypes = [C.c_int, _dp, _dp]
    L.oracle_legini.argtypes = [P(LegTables), C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_double, C.c_double, C.c_int, C.c_int]
    L.oracle_legfree.argtypes = [P(LegTables)]
    for f in ("oracle_sp2fc", "oracle_sp2fcdmu"):
        getattr(L, f).argtypes = [P(LegTables), _dp, _dp]
    L.oracle_fc2sp.argtypes = [P(LegTables), _dp, _dp, C.c_int]
    L.oracle_dv2uv.argtypes = [P(LegTables), _dp, _dp, _dp, _dp, C.c_int, C.c_double]
    L.oracle_uv2dv.argtypes = [P(LegTables), _dp, _dp, _dp, _dp, C.c_int, C.c_int]
    L.oracle_qtend.argtypes = [P(LegTables), _dp, _dp, _dp, _dp, C.c_int, C.c_int]
    L.oracle_mktend.argtypes = [P(LegTables)] + [_dp] * 9 + [C.c_int, C.c_int]
    for f in ("oracle_gp2fc", "oracle_fc2gp", "oracle_gp2fc_991", "oracle_fc2gp_991"):
        getattr(L, f).argtypes = [_dp, C.c_int, C.c_int]
        getattr(L, f).restype = C.c_int
    L.oracle_radpar_default.argtypes = [P(RadPar), C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
    L.oracle_solarini.argtypes = [C.c_double, C.c_double, _dp, _dp, _dp]
    L.oracle_radstep.argtypes = [P(RadPar), P(RadIO)]
    L.oracle_radstep_par.argtypes = [P(RadPar), P(RadIO)]
    L.oracle_num_threads.restype = C.c_int
    L.oracle_inverse_set.argtypes = [P(LegTables), C.c_int, _dp, _dp, C.c_double, C.c_int]
    L.oracle_forward_set.argtypes = [P(LegTables), C.c_int, _dp, _dp, C.c_int]
    L.oracle_gridpoint.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    L.oracle_initsi.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp, _dp]
    L.oracle_tau.argtypes = [C.c_int] + [_dp] * 7
    L.oracle_makebm.argtypes = [C.c_int, C.c_int, C.c_double] + [_dp] * 5
    L.oracle_sak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, _dp]
    L.oracle_spectrala.argtypes = [C.c_void_p, C.c_void_p]
    L.oracle_spectrald.argtypes = [C.c_void_p, C.c_void_p]
    L.oracle_inverse_set_d.argtypes = [P(LegTables), C.c_int, _dp, _dp, C.c_double, C.c_int]
    L.oracle_forward_set_d.argtypes = [P(LegTables), C.c_int, _dp, _dp, C.c_int]


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "oracle arrays are C-contiguous float64"
    return a.ctypes.data_as(_dp)


def inigau(nlat):
    sid = np.zeros(nlat)
    gwd = np.zeros(nlat)
    lib().oracle_inigau(nlat, _ptr(sid), _ptr(gwd))
    return sid, gwd


class Leg:
    """legini tables for one resolution (legmod.f90:30-171)."""

    def __init__(self, nlat, nfilter=0, ngptfilter=0, nspvfilter=0, landhoskn0=15.0,
                 filterkappa=8.0, nfilterexp=8, pyfft_nfs=-1):
        self.t = LegTables()
        lib().oracle_legini(C.byref(self.t), nlat, nfilter, ngptfilter, nspvfilter,
                            landhoskn0, filterkappa, nfilterexp, pyfft_nfs)
        self.nlat, self.nlon, self.ntru, self.ncsp = nlat, self.t.nlon, self.t.ntru, self.t.ncsp
        self.nrsp = 2 * self.ncsp

    def __del__(self):
        try:
            lib().oracle_legfree(C.byref(self.t))
        except Exception:
            pass

    def table(self, name):
        p = getattr(self.t, name)
        n = self.nlat * self.ncsp if name.startswith("q") else (self.nlat if name in ("sid", "gwd") else self.ntru + 1)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def _fc(self, nlev=1):
        return np.zeros((nlev, self.nlat, self.nlon))

    def sp2fc(self, sp):
        fc = self._fc()[0]
        lib().oracle_sp2fc(C.byref(self.t), _ptr(np.ascontiguousarray(sp)), _ptr(fc))
        return fc

    def sp2fcdmu(self, sp):
        fc = self._fc()[0]
        lib().oracle_sp2fcdmu(C.byref(self.t), _ptr(np.ascontiguousarray(sp)), _ptr(fc))
        return fc

    def fc2sp(self, fc, folded=True):
        sp = np.zeros(self.nrsp)
        lib().oracle_fc2sp(C.byref(self.t), _ptr(np.ascontiguousarray(fc)), _ptr(sp), int(folded))
        return sp

    def dv2uv(self, pd, pz, plavor=0.0):
        nlev = pd.shape[0]
        pu, pv = self._fc(nlev), self._fc(nlev)
        pz = np.array(pz, dtype=np.float64, order="C")
        lib().oracle_dv2uv(C.byref(self.t), _ptr(np.ascontiguousarray(pd)), _ptr(pz), _ptr(pu), _ptr(pv),
                           nlev, plavor)
        return pu, pv

    def uv2dv(self, pu, pv, folded=True):
        nlev = pu.shape[0]
        pd, pz = np.zeros((nlev, self.nrsp)), np.zeros((nlev, self.nrsp))
        lib().oracle_uv2dv(C.byref(self.t), _ptr(np.ascontiguousarray(pu)), _ptr(np.ascontiguousarray(pv)),
                           _ptr(pd), _ptr(pz), nlev, int(folded))
        return pd, pz

    def qtend(self, qn, uq, vq, folded=True):
        nlev = qn.shape[0]
        q = np.zeros((nlev, self.nrsp))
        lib().oracle_qtend(C.byref(self.t), _ptr(q), *[_ptr(np.ascontiguousarray(a)) for a in (qn, uq, vq)],
                           nlev, int(folded))
        return q

    def mktend(self, tn, fu, fv, ke, ut, vt, folded=True):
        nlev = tn.shape[0]
        d, t, z = (np.zeros((nlev, self.nrsp)) for _ in range(3))
        lib().oracle_mktend(C.byref(self.t), _ptr(d), _ptr(t), _ptr(z),
                            *[_ptr(np.ascontiguousarray(a)) for a in (tn, fu, fv, ke, ut, vt)],
                            nlev, int(folded))
        return d, t, z

    def inverse_set(self, spin, nlev, plavor, use991=False):
        gpout = np.zeros(((6 * nlev + 3), self.nlat * self.nlon))
        lib().oracle_inverse_set(C.byref(self.t), nlev, _ptr(np.ascontiguousarray(spin)), _ptr(gpout),
                                 plavor, int(use991))
        return gpout

    def inverse_set_d(self, spin, nlev, plavor, use991=False):
        """gridpointd inverse half: (4L+1, NRSP) -> (4L+1, NHOR) gu, gv, gt, gq, gp."""
        gpout = np.zeros(((4 * nlev + 1), self.nlat * self.nlon))
        lib().oracle_inverse_set_d(C.byref(self.t), nlev, _ptr(np.ascontiguousarray(spin)), _ptr(gpout),
                                   plavor, int(use991))
        return gpout

    def forward_set_d(self, gpin, nlev, use991=False):
        """gridpointd forward half: (4L, NHOR) gtdt, gudt, gvdt, gqdt -> (4L, NRSP) sdf, stf, szf, sqf."""
        work = np.array(gpin, dtype=np.float64, order="C", copy=True).reshape(4 * nlev, -1)
        spout = np.zeros((4 * nlev, self.nrsp))
        lib().oracle_forward_set_d(C.byref(self.t), nlev, _ptr(work), _ptr(spout), int(use991))
        return spout

    def forward_set(self, gpin, nlev, use991=False):
        work = np.array(gpin, dtype=np.float64, order="C", copy=True)
        spout = np.zeros((4 * nlev + 1, self.nrsp))
        lib().oracle_forward_set(C.byref(self.t), nlev, _ptr(work), _ptr(spout), int(use991))
        return spout


def gp2fc(a, use991=False):
    """In-place real forward FFT of rows (fftmod.f90:29-58); returns a copy."""
    a = np.array(a, dtype=np.float64, order="C", copy=True)
    n = a.shape[-1]
    lot = a.size // n
    f = lib().oracle_gp2fc_991 if use991 else lib().oracle_gp2fc
    if f(_ptr(a), n, lot) != 0:
        raise ValueError(f"FFT does not support n = {n}")
    return a


def fc2gp(a, use991=False):
    """Inverse real FFT of rows (fftmod.f90:64-87); returns a copy."""
    a = np.array(a, dtype=np.float64, order="C", copy=True)
    n = a.shape[-1]
    lot = a.size // n
    f = lib().oracle_fc2gp_991 if use991 else lib().oracle_fc2gp
    if f(_ptr(a), n, lot) != 0:
        raise ValueError(f"FFT does not support n = {n}")
    return a


def solarini(starbbtemp, minwavel_nm=316.036116751):
    z1, z2, rc = C.c_double(), C.c_double(), C.c_double()
    lib().oracle_solarini(starbbtemp, minwavel_nm * 1e-9, C.byref(z1), C.byref(z2), C.byref(rc))
    return z1.value, z2.value, rc.value


def default_sigma(nlev):
    """Default sigma half/full levels (plasim.f90:1554-1564)."""
    zsk = np.arange(1, nlev + 1) / nlev
    sigmah = 0.75 * zsk + 1.75 * zsk ** 3 - 1.5 * zsk ** 4
    dsigma = np.empty(nlev)
    dsigma[0] = sigmah[0]
    dsigma[1:] = sigmah[1:] - sigmah[:-1]
    sigma = np.empty(nlev)
    sigma[0] = 0.5 * sigmah[0]
    sigma[1:] = 0.5 * (sigmah[:-1] + sigmah[1:])
    return sigma, sigmah, dsigma


RAD_INPUTS = ("dt", "dq", "dcc", "dql", "dqco2", "dp", "dls", "dicec", "dqo3", "gmu0", "dalb", "dsalb", "dtdt")
RAD_OUTPUTS = ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux", "dtdt", "dtdtswr", "dtdtlwr",
               "dconv", "dqo3", "gmu0", "dalb", "dsalb")


def radpar(nlev, nhor, nlon, sigma, sigmah, dsigma, **over):
    p = RadPar()
    keep = [np.ascontiguousarray(sigma, dtype=np.float64), np.ascontiguousarray(sigmah, dtype=np.float64),
            np.ascontiguousarray(dsigma, dtype=np.float64)]
    lib().oracle_radpar_default(C.byref(p), nlev, nhor, nlon, *[_ptr(k) for k in keep])
    for k, v in over.items():
        if k in ("rcl1", "rcl2", "acl2"):
            getattr(p, k)[:] = list(v)
        else:
            setattr(p, k, v)
    p._keep = keep
    return p


def radstep(p, sid, cola, cols, parallel=False):
    """Run radstep on columns given as a dict of reference-layout arrays.

    cols: dt, dq, dcc, dql [nlep][nhor]; dqco2, dqo3, dtdt [nlev][nhor];
    dp, dls, dicec, gmu0, dalb [nhor]; dsalb [nhor][2].  Returns a dict with
    the outputs (and the in/out arrays after the call)."""
    nlev, nhor = p.nlev, p.nhor
    nlep = nlev + 1
    arr = {k: np.array(cols[k], dtype=np.float64, order="C", copy=True) for k in
           ("dt", "dq", "dcc", "dql", "dqco2", "dp", "dls", "dicec", "dqo3", "gmu0", "dalb", "dsalb")}
    arr["dtdt"] = np.array(cols.get("dtdt", np.zeros((nlev, nhor))), dtype=np.float64, order="C", copy=True)
    for k in ("dfu", "dfd", "dftu", "dftd", "dswfl", "dlwfl", "dflux"):
        arr[k] = np.zeros((nlep, nhor))
    for k in ("dtdtswr", "dtdtlwr", "dconv"):
        arr[k] = np.zeros((nlev, nhor))
    sid = np.ascontiguousarray(sid, dtype=np.float64)
    cola = np.ascontiguousarray(cola, dtype=np.float64)
    io = RadIO()
    io.sid, io.cola = _ptr(sid), _ptr(cola)
    for k, v in arr.items():
        setattr(io, k, _ptr(v))
    (lib().oracle_radstep_par if parallel else lib().oracle_radstep)(C.byref(p), C.byref(io))
    return arr


class GpPar(C.Structure):
    _fields_ = [("nlev", C.c_int), ("nhor", C.c_int), ("nlon", C.c_int), ("nqspec", C.c_int)] + \
               [(n, _dp) for n in ("dsigma", "sigmah", "rdsig", "t0", "t01s2", "tkp", "g", "c")] + \
               [(n, C.c_double) for n in ("akap", "rdbrv", "adv", "psurf", "ww")] + [("dq", _dp)]


def initsi(sigmah, dsigma, t0, akap):
    """g, c (nlev x nlev, [i, j] = g(i+1, j+1)), tkp, t01s2, rdsig (plasim.f90:1709-1745, :1564)."""
    L = len(sigmah)
    g, c = np.zeros(L * L), np.zeros(L * L)
    tkp, t01s2, rdsig = np.zeros(L), np.zeros(L), np.zeros(L)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (sigmah, dsigma, t0)]
    lib().oracle_initsi(L, *[_ptr(x) for x in a], akap, _ptr(g), _ptr(c), _ptr(tkp), _ptr(t01s2), _ptr(rdsig))
    return g.reshape(L, L, order="F"), c.reshape(L, L, order="F"), tkp, t01s2, rdsig


def gridpoint(gin, nlev, nlon, sigmah, dsigma, t0, akap, rdbrv, adv, psurf, ww, rcsq, nqspec=1, dq=None):
    """The grid-point step of gridpointa (plasim.f90:2441-2455) on gin
    ((6L+3, nhor): gu gv gt gd gz gq gpj gpmt gp); returns (gout (9L+1, nhor), dw (L, nhor))."""
    L = nlev
    gin = np.ascontiguousarray(gin, dtype=np.float64).reshape(6 * L + 3, -1)
    nhor = gin.shape[1]
    g, c, tkp, t01s2, rdsig = initsi(sigmah, dsigma, t0, akap)
    keep = [np.ascontiguousarray(x, dtype=np.float64) for x in (dsigma, sigmah, rdsig, t0, t01s2, tkp)]
    gF, cF = np.ascontiguousarray(g.ravel(order="F")), np.ascontiguousarray(c.ravel(order="F"))
    p = GpPar()
    p.nlev, p.nhor, p.nlon, p.nqspec = L, nhor, nlon, nqspec
    for name, arr in zip(("dsigma", "sigmah", "rdsig", "t0", "t01s2", "tkp"), keep):
        setattr(p, name, _ptr(arr))
    p.g, p.c = _ptr(gF), _ptr(cF)
    p.akap, p.rdbrv, p.adv, p.psurf, p.ww = akap, rdbrv, adv, psurf, ww
    dqa = None if dq is None else np.ascontiguousarray(dq, dtype=np.float64)
    p.dq = _ptr(dqa) if dqa is not None else None
    gout = np.zeros((9 * L + 1, nhor))
    dw = np.zeros((L, nhor))
    rc = np.ascontiguousarray(rcsq, dtype=np.float64)
    lib().oracle_gridpoint(C.byref(p), _ptr(gin), _ptr(gout), _ptr(dw), _ptr(rc))
    return gout, dw


SPEC_STATE = ("sdp", "szp", "stp", "sqp", "spp", "sdm", "szm", "stm", "sqm", "spm",
              "sdt", "szt", "stt", "sqt", "spt", "sop", "srp")


class SpecPar(C.Structure):
    _fields_ = [("nlev", C.c_int), ("ntru", C.c_int), ("nqspec", C.c_int), ("nsponge", C.c_int)] + \
               [(n, C.c_double) for n in ("delt", "delt2", "pnu", "pnu21", "plavor", "dampsp")] + \
               [(n, _dp) for n in ("t0", "dsigma", "g", "tau", "bm1", "damp", "tdisst", "tdissq", "tdissd",
                                   "tdissz", "tfrc", "sak")]


class SpecState(C.Structure):
    _fields_ = [(n, _dp) for n in SPEC_STATE]


def spec_setup(ntru, nlev, sigmah, dsigma, t0, akap, delt, ndel, nhdiff):
    """(g, tau, bm1, sak) of initsi, makebm and the diffusion (plasim.f90:1709-1760, :1683-1704, :1617-1633)."""
    L = nlev
    g, c, tkp, t01s2, rdsig = initsi(sigmah, dsigma, t0, akap)
    gF, cF = np.ascontiguousarray(g.ravel(order="F")), np.ascontiguousarray(c.ravel(order="F"))
    tau = np.zeros(L * L)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (sigmah, dsigma, rdsig, tkp, t01s2)]
    lib().oracle_tau(L, *[_ptr(x) for x in a], _ptr(cF), _ptr(tau))
    bm1 = np.zeros((ntru + 1) * L * L)
    t0a, dsa = np.ascontiguousarray(t0, dtype=np.float64), np.ascontiguousarray(dsigma, dtype=np.float64)
    lib().oracle_makebm(L, ntru, delt, _ptr(t0a), _ptr(dsa), _ptr(gF), _ptr(tau), _ptr(bm1))
    nrsp = (ntru + 1) * (ntru + 2)
    sak = np.zeros(L * nrsp)
    nd = (C.c_int * L)(*[int(x) for x in ndel[:L]])
    lib().oracle_sak(L, ntru, nd, nhdiff, _ptr(sak))
    return gF, tau, bm1, sak


def spectral_step(part, p, ntru, state):
    """spectrala ("a") or spectrald ("d") on a dict of [L][NRSP] arrays (copies
    returned).  p: mapping with nlev, nqspec, nsponge, delt, delt2, pnu, pnu21,
    plavor, dampsp, t0, sigmah, dsigma, damp, tdiss*, tfrc, akap, ndel, nhdiff."""
    L = p["nlev"]
    gF, tau, bm1, sak = spec_setup(ntru, L, p["sigmah"][:L], p["dsigma"][:L], p["t0"][:L], p["akap"], p["delt"],
                                   p["ndel"], p["nhdiff"])
    P = SpecPar()
    P.nlev, P.ntru, P.nqspec, P.nsponge = L, ntru, p["nqspec"], p["nsponge"]
    for k in ("delt", "delt2", "pnu", "pnu21", "plavor", "dampsp"):
        setattr(P, k, p[k])
    keep = {k: np.ascontiguousarray(np.asarray(p[k], dtype=np.float64)[:L]) for k in
            ("t0", "dsigma", "damp", "tdisst", "tdissq", "tdissd", "tdissz", "tfrc")}
    keep.update(g=gF, tau=tau, bm1=bm1, sak=sak)
    for k, v in keep.items():
        setattr(P, k, _ptr(v))
    out = {k: np.array(v, dtype=np.float64, order="C", copy=True) for k, v in state.items()}
    S = SpecState()
    for k in SPEC_STATE:
        if k in out:
            setattr(S, k, _ptr(out[k]))
    (lib().oracle_spectrala if part == "a" else lib().oracle_spectrald)(C.byref(P), C.byref(S))
    return out

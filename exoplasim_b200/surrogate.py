"""Learned radiation surrogate over libexotx (no counterpart in the reference).

An MLP (3L+9 inputs -> 6 hidden layers of 256, SiLU -> L+4 outputs) learns
radmod's column map (radmod.f90 radstep :927-1110): the heating-rate profile
(K/day) and the four surface fluxes (dfd, dfu, dftd, dftu at NLEP).  Its
training columns come from the plain GPU radstep kernel in FP64; training
runs on the library's FP32 kernels (exotx_mlp_backward / exotx_mlp_adam);
inference (exotx_rad_surrogate) runs the network in BF16 on the tensor cores
and computes every column whose inputs leave the training ranges with the
plain radstep kernel.

    python -m exoplasim_b200.surrogate --train OUT.npz [--columns 2000000] [--epochs 400]

The packaged network (data/rad_surrogate_L20.npz) was trained this way with
the defaults: 2M columns drawn level by level as the radiation benchmark's
configuration specifies (synthetic.radiation_columns), 400 epochs of Adam with
cosine decay from 1e-3, the loss in normalised output units.  With
--profiles structured the columns are vertically coherent instead.
"""
import argparse
import ctypes as C
import math
import os
import time

import numpy as np
import torch

from . import _lib
from . import radiation as R
from . import synthetic as S
from ._lib import FP32, FP64, call

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_NET = os.path.join(DATA, "rad_surrogate_L20.npz")
GRID_NLAT = 64            # training columns are laid out on T42 grids (64 x 128 = 8192 columns)
PROFILES = "independent"  # training columns as the radiation benchmark draws them (synthetic.radiation_columns)


def nin_for(nlev):
    return 3 * nlev + 9


def nout_for(nlev):
    return nlev + 4


class _DevArray:
    """A view of library-owned device memory for torch (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Mlp:
    """An exotx_mlp: FP32 parameters, gradients and Adam state on the device."""

    def __init__(self, nin, nout, width=256, nhidden=6, max_batch=4096):
        lib = _lib.load()
        h = C.c_void_p()
        call("exotx_mlp_create", nin, width, nhidden, nout, max_batch, C.byref(h))
        self._h, self._lib = h, lib
        self.nin, self.nout, self.width, self.nhidden, self.max_batch = nin, nout, width, nhidden, max_batch
        p, g, n = C.c_void_p(), C.c_void_p(), C.c_longlong()
        call("exotx_mlp_params", h, C.byref(p), C.byref(g), C.byref(n))
        self.nparams = n.value
        self.params = torch.as_tensor(_DevArray(p.value, n.value), device="cuda")
        self.grads = torch.as_tensor(_DevArray(g.value, n.value), device="cuda")
        self.layers = []
        for l in range(nhidden + 1):
            wo, bo, di, do = C.c_longlong(), C.c_longlong(), C.c_int(), C.c_int()
            call("exotx_mlp_layer", h, l, C.byref(wo), C.byref(bo), C.byref(di), C.byref(do))
            self.layers.append((wo.value, bo.value, di.value, do.value))
        self.norm = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.exotx_mlp_destroy(h)
            except Exception:
                pass
            self._h = None

    def weights(self, l):
        """(W, b) views of layer l: W (dout x din), b (dout)."""
        wo, bo, di, do = self.layers[l]
        return self.params[wo:wo + di * do].view(do, di), self.params[bo:bo + do]

    def grad(self, l):
        wo, bo, di, do = self.layers[l]
        return self.grads[wo:wo + di * do].view(do, di), self.grads[bo:bo + do]

    def init(self, seed=0):
        """He-normal weights (SiLU), zero biases; the output layer scaled down."""
        g = np.random.default_rng(seed)
        with torch.no_grad():
            for l, (wo, bo, di, do) in enumerate(self.layers):
                s = math.sqrt(2.0 / di) * (0.1 if l == len(self.layers) - 1 else 1.0)
                W, b = self.weights(l)
                W.copy_(torch.as_tensor(g.standard_normal((do, di)) * s, dtype=torch.float32))
                b.zero_()

    def set_norm(self, xm, xs, xlo, xhi, ym, ys):
        v = np.concatenate([xm, xs, xlo, xhi, ym, ys]).astype(np.float32)
        assert v.size == 4 * self.nin + 2 * self.nout
        self.norm = dict(xm=np.asarray(xm, np.float32), xs=np.maximum(np.asarray(xs, np.float32), 1e-6),
                         xlo=np.asarray(xlo, np.float32), xhi=np.asarray(xhi, np.float32),
                         ym=np.asarray(ym, np.float32), ys=np.maximum(np.asarray(ys, np.float32), 1e-6))
        call("exotx_mlp_set_norm", self._h, v.ctypes.data_as(C.c_void_p))

    def forward(self, X):
        """FP32 forward of normalised rows (n <= max_batch) -> normalised outputs."""
        n = X.shape[0]
        Y = torch.empty((n, self.nout), dtype=torch.float32, device="cuda")
        call("exotx_mlp_forward", self._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), n, _stream())
        return Y

    def backward(self, X, T, loss, W=None):
        """Gradients of the mean squared error of rows X against T, each element's
        squared error weighted by W (same shape) when given; loss (device) += it."""
        if W is None:
            call("exotx_mlp_backward", self._h, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), X.shape[0],
                 C.c_void_p(loss.data_ptr()), _stream())
        else:
            call("exotx_mlp_backward_weighted", self._h, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()),
                 C.c_void_p(W.data_ptr()), X.shape[0], C.c_void_p(loss.data_ptr()), _stream())

    def adam(self, lr, step, b1=0.9, b2=0.999, eps=1e-8):
        call("exotx_mlp_adam", self._h, C.c_float(lr), C.c_float(b1), C.c_float(b2), C.c_float(eps), step,
             _stream())

    def prepare(self):
        call("exotx_mlp_prepare", self._h, _stream())

    def check(self):
        """Raise if a bounded wait of the tensor-core training GEMMs gave up."""
        call("exotx_mlp_check", self._h, _stream())

    def save(self, path, **meta):
        np.savez(path, params=self.params.cpu().numpy(), nin=self.nin, nout=self.nout, width=self.width,
                 nhidden=self.nhidden, **{k: v for k, v in (self.norm or {}).items()}, **meta)

    @classmethod
    def load(cls, path, max_batch=4096):
        d = np.load(path)
        net = cls(int(d["nin"]), int(d["nout"]), int(d["width"]), int(d["nhidden"]), max_batch)
        with torch.no_grad():
            net.params.copy_(torch.as_tensor(d["params"], dtype=torch.float32))
        net.set_norm(d["xm"], d["xs"], d["xlo"], d["xhi"], d["ym"], d["ys"])
        net.meta = {k: d[k] for k in d.files if k not in ("params",)}
        net.prepare()   # a loaded network is ready for exotx_rad_surrogate
        return net


# ------------------------------------------------------------------ data
def _solar_table():
    teff = np.arange(2400.0, 6101.0, 10.0)
    tab = np.array([R.solarini(t) for t in teff])
    return teff, tab


_SOLAR = None


def zsol_for(teff):
    """(3, n) zsolar1, zsolar2, rcoeff for per-column stellar Teff (linear in a 10 K table)."""
    global _SOLAR
    if _SOLAR is None:
        _SOLAR = _solar_table()
    t, tab = _SOLAR
    return np.stack([np.interp(teff, t, tab[:, k]) for k in range(3)])


def column_chunk(nlev, seed, dtype=torch.float64, profiles=PROFILES):
    """One T42 grid of synthetic columns on the device with per-column stars."""
    cols, g = S.radiation_columns(GRID_NLAT, nlev, seed=seed, teff=True, profiles=profiles)
    zsol = zsol_for(cols.pop("teff"))
    dev = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=dtype, device="cuda") for k, v in cols.items()}
    dev["zsol"] = torch.as_tensor(np.ascontiguousarray(zsol), dtype=dtype, device="cuda")
    params = R.default_params(nlev, g["nhor"], g["nlon"], nsol=0)
    return params, dev


def features(params, dev, precision="fp64"):
    prec = FP64 if precision == "fp64" else FP32
    io = R.make_io(dev, R.alloc_outputs(params, dev["dt"].dtype), prec)
    X = torch.empty((params.nhor, nin_for(params.nlev)), dtype=torch.float32, device="cuda")
    call("exotx_surr_features", C.byref(params), prec, C.byref(io), C.c_void_p(X.data_ptr()), _stream())
    return X


def plain_targets(params, dev, precision="fp64"):
    """radstep on a copy of the columns; returns (targets Y, outputs dict)."""
    prec = FP64 if precision == "fp64" else FP32
    cols = {k: v.clone() for k, v in dev.items()}
    cols["dtdt"].zero_()
    out = R.radstep(params, cols, precision=precision)
    io = R.make_io(cols, out, prec)
    Y = torch.empty((params.nhor, nout_for(params.nlev)), dtype=torch.float32, device="cuda")
    call("exotx_surr_targets", C.byref(params), prec, C.byref(io), C.c_void_p(Y.data_ptr()), _stream())
    return Y, cols, out


def dataset(ncols, nlev=20, seed=1000, profiles=PROFILES):
    """Features and targets of ncols synthetic columns (a multiple of 8192)."""
    nchunk = max(1, ncols // (2 * GRID_NLAT * GRID_NLAT))
    Xs, Ys = [], []
    for i in range(nchunk):
        params, dev = column_chunk(nlev, seed + i, profiles=profiles)
        Xs.append(features(params, dev))
        Ys.append(plain_targets(params, dev)[0])
    return torch.cat(Xs), torch.cat(Ys)


def norm_stats(X, Y, margin=0.02):
    xm, xs = X.mean(0), X.std(0)
    lo, hi = X.min(0).values, X.max(0).values
    pad = margin * (hi - lo) + 1e-6
    return (xm.cpu().numpy(), xs.cpu().numpy(), (lo - pad).cpu().numpy(), (hi + pad).cpu().numpy(),
            Y.mean(0).cpu().numpy(), Y.std(0).cpu().numpy())


# ------------------------------------------------------------------ training
def judged_weights(X, nlev, ys, adv, flux_k_per_day_per_w=0.1):
    """Per-element loss weights that make the training loss the squared error in
    the units the surrogate is judged in: a normalised heating output's error e
    is e * ys / ((ps / 1e5)(1 + ADV q)) K/day, so its weight is that factor
    squared; a surface flux's error of 1 W/m2 counts as flux_k_per_day_per_w
    K/day.  Scaled to mean 1."""
    L = nlev
    hs = heating_scale(X, L, adv).float()
    W = torch.empty((X.shape[0], L + 4), dtype=torch.float32, device=X.device)
    W[:, :L] = (ys[:L] / hs) ** 2
    W[:, L:] = (flux_k_per_day_per_w * ys[L:]) ** 2
    return (W / W.mean()).contiguous()


def train(net, X, Y, epochs=16, batch=4096, lr=1e-3, lr_min=1e-5, seed=0, log=None, weighted=False, adv=None):
    """Adam over normalised (X, Y) on the device; cosine learning-rate decay.
    weighted: the loss of judged_weights (needs the radiation constant adv)."""
    n = X.shape[0]
    xm = torch.as_tensor(net.norm["xm"], device="cuda")
    xs = torch.as_tensor(net.norm["xs"], device="cuda")
    ym = torch.as_tensor(net.norm["ym"], device="cuda")
    ys = torch.as_tensor(net.norm["ys"], device="cuda")
    Wt = judged_weights(X, net.nout - 4, ys, adv) if weighted else None
    Xn = ((X - xm) / xs).contiguous()
    Yn = ((Y - ym) / ys).contiguous()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    step = 0
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        loss.zero_()
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            xb = Xn.index_select(0, idx)
            yb = Yn.index_select(0, idx)
            wb = Wt.index_select(0, idx) if Wt is not None else None
            step += 1
            rate = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * step / total))
            net.backward(xb, yb, loss, wb)
            net.adam(rate, step)
        ep_loss = loss.item() / steps_per_epoch
        net.check()
        hist.append(ep_loss)
        if log:
            log(f"epoch {ep + 1}/{epochs}  loss {ep_loss:.5f}  {time.time() - t0:.1f} s")
    net.prepare()
    return hist


# ------------------------------------------------------------------ inference
def surrogate_step(net, params, cols, out, precision="fp64", count=False):
    """exotx_rad_surrogate on device columns (in place, like radstep); returns the
    number of fallback columns when count is True."""
    prec = FP64 if precision == "fp64" else FP32
    io = R.make_io(cols, out, prec)
    nfb = C.c_int(0)
    call("exotx_rad_surrogate", net._h, C.byref(params), prec, C.byref(io), C.byref(nfb) if count else None,
         _stream())
    return nfb.value if count else None


def heating_scale(X, nlev, adv):
    """Per column and level, (ps / 1e5 Pa)(1 + ADV q): the heating-rate target
    divided by this is the heating rate in K/day (X holds raw features)."""
    L = nlev
    ps = torch.exp(X[:, 3 * L + 2].double())
    q = torch.exp(X[:, L + 1:2 * L + 1].double())
    return (ps / 1e5)[:, None] * (1.0 + adv * q)


def heating_rms(pred_dtdt, ref_dtdt):
    """RMS heating-rate difference in K/day over all columns and levels."""
    return float(torch.sqrt(torch.mean(((pred_dtdt - ref_dtdt) * 86400.0) ** 2)))


def evaluate(net, nlev=20, seed=900000, nchunk=4, precision="fp64", profiles=PROFILES):
    """Surrogate vs plain radstep on fresh columns: heating RMS (K/day), surface-flux
    RMS (W/m2) and the fallback fraction."""
    se, sf, ncol, nfb = 0.0, 0.0, 0, 0
    for i in range(nchunk):
        params, dev = column_chunk(nlev, seed + i, profiles=profiles)
        Y, pcols, _ = plain_targets(params, dev)
        cols = {k: v.clone() for k, v in dev.items()}
        cols["dtdt"].zero_()
        out = R.alloc_outputs(params, cols["dt"].dtype)
        nfb += surrogate_step(net, params, cols, out, precision, count=True)
        L = nlev
        pred_h = cols["dtdt"].T * 86400.0
        se += float(((pred_h - pcols["dtdt"].T * 86400.0) ** 2).sum())
        fl = torch.stack([out["dfd"][L], out["dfu"][L], out["dftd"][L], out["dftu"][L]], 1)
        sf += float(((fl - Y[:, L:].double()) ** 2).sum())
        ncol += params.nhor
    return {"heating_rms_K_per_day": math.sqrt(se / (ncol * nlev)),
            "surface_flux_rms_W_m2": math.sqrt(sf / (ncol * 4)), "fallback_fraction": nfb / ncol,
            "columns": ncol}


def fallback_curve(net, ps_min_list, nlev=20, seed=900000, nchunk=4, profiles=PROFILES):
    """Heating RMS against the fallback fraction when columns with surface
    pressure below ps_min go to the plain radstep kernel: the range test of
    exotx_rad_surrogate with the lower bound of the ln ps feature raised to
    ln(ps_min).  Returns [(ps_min, fallback fraction, heating RMS K/day,
    surface-flux RMS W/m2)]; the network's own ranges are restored after."""
    nrm = {k: v.copy() for k, v in net.norm.items()}
    ips = 3 * nlev + 2
    rows = []
    try:
        for pmin in ps_min_list:
            xlo = nrm["xlo"].copy()
            xlo[ips] = max(xlo[ips], math.log(pmin)) if pmin > 0 else xlo[ips]
            net.set_norm(nrm["xm"], nrm["xs"], xlo, nrm["xhi"], nrm["ym"], nrm["ys"])
            ev = evaluate(net, nlev, seed, nchunk, profiles=profiles)
            rows.append((pmin, ev["fallback_fraction"], ev["heating_rms_K_per_day"], ev["surface_flux_rms_W_m2"]))
    finally:
        net.set_norm(nrm["xm"], nrm["xs"], nrm["xlo"], nrm["xhi"], nrm["ym"], nrm["ys"])
    return rows


def main():
    a = argparse.ArgumentParser()
    a.add_argument("--train", required=True, help="output .npz")
    a.add_argument("--columns", type=int, default=2_000_000)
    a.add_argument("--epochs", type=int, default=400)
    a.add_argument("--batch", type=int, default=4096)
    a.add_argument("--lr", type=float, default=1e-3)
    a.add_argument("--nlev", type=int, default=20)
    a.add_argument("--seed", type=int, default=0)
    a.add_argument("--loss", default="normalised", choices=("kday", "normalised"),
                   help="squared error in K/day (and W/m2, judged_weights) or in normalised output units")
    a.add_argument("--profiles", default=PROFILES, choices=("structured", "independent"),
                   help="column generator of the training and evaluation columns")
    args = a.parse_args()
    t0 = time.time()
    X, Y = dataset(args.columns, args.nlev, seed=1000, profiles=args.profiles)
    print(f"dataset {X.shape[0]} columns in {time.time() - t0:.1f} s", flush=True)
    net = Mlp(nin_for(args.nlev), nout_for(args.nlev), max_batch=args.batch)
    net.init(args.seed)
    net.set_norm(*norm_stats(X, Y))
    adv = R.default_params(args.nlev, 2 * GRID_NLAT * GRID_NLAT, 2 * GRID_NLAT).adv
    hist = train(net, X, Y, epochs=args.epochs, batch=args.batch, lr=args.lr,
                 log=lambda s: print(s, flush=True), weighted=args.loss == "kday", adv=adv)
    ev = evaluate(net, args.nlev, profiles=args.profiles)
    print(ev, flush=True)
    other = "independent" if args.profiles == "structured" else "structured"
    print(f"{other} columns:", evaluate(net, args.nlev, profiles=other), flush=True)
    net.save(args.train, loss=np.array(hist), columns=X.shape[0], epochs=args.epochs,
             heating_rms=ev["heating_rms_K_per_day"], profiles=args.profiles)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark: T127 L20 spectral-transform round trips/s and radiation columns/s.

One step = one pass of the gridpointa transform set (plasim.f90:2396-2486)
over a batch of B independent T127 L20 model states (the inverse set:
dv2uv + sp2fc x4L + sp2fc/sp2fcdmu(ln ps) + i*m d/dlambda + fc2gp of 6L+3
fields; then the forward set: gp2fc of 9L+1 fields + fc2sp + mktend + qtend),
on synthetic seeded inputs already resident in HBM.  value = round trips/s
summed over all ranks (weak scaling: every rank runs its own B instances;
the instances are independent, so there is no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The reference arm (--impl reference) times the FP64 CPU restatement of the
reference's legmod/fftmod (the Fortran itself cannot be compiled on these
hosts) on all host cores, on the same workload, and prints the same line.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NLAT, NLEV = 192, 20           # T127 L20: 192 x 384 Gaussian grid
RAD_NLAT, RAD_NLEV = 64, 20    # radiation: T42 grid, 8192 columns, L20
WORKLOAD = "T127 L20 gridpointa transform round trip (inverse + forward set)"
# one metric string for both arms, so that their lines compare
METRIC = "T127 L20 transform round-trips/s (mixed vs FP32 @\u22641e-6 rel); radiation cols/s"
BATCH = 8                      # T127 L20 instances per step and rank, in both arms


def fp32_round_trip_bytes(nlat, nlev):
    """Algorithmic bytes of one round trip at FP32: spectral in+out and grid out+in."""
    ntru = (2 * nlat - 1) // 3
    nrsp = (ntru + 1) * (ntru + 2)
    nhor = nlat * 2 * nlat
    return 2 * (4 * nlev + 1) * nrsp * 4 + (15 * nlev + 4) * nhor * 4


def legendre_flops(nlat, nlev, half="both"):
    """Algorithmic folded Legendre flops of one instance: F_leg = 2 NLAT NCSP per
    complex field-level; (8L+2) products in the inverse set, (11L+1) in the forward."""
    ntru = (2 * nlat - 1) // 3
    ncsp = (ntru + 1) * (ntru + 2) // 2
    nprod = {"inverse": 8 * nlev + 2, "forward": 11 * nlev + 1, "both": 19 * nlev + 3}[half]
    return nprod * 2 * nlat * ncsp


def fft_bytes(nlat, nlev, half, esz):
    """Algorithmic bytes of one instance's FFT stage: grid rows of NLON reals on
    one side, NTRU+1 complex Fourier coefficients per row on the other."""
    ntru = (2 * nlat - 1) // 3
    nlon = 2 * nlat
    rows = ((6 * nlev + 3) if half == "inverse" else (9 * nlev + 1)) * nlat
    return rows * (nlon * esz + (ntru + 1) * 2 * esz)


def legendre_bytes(nlat, nlev, half, esz):
    """Algorithmic bytes of one instance's Legendre stage in the mixed path: the
    spectral fields on one side, the m-major Fourier intermediate (NTRU+1
    complex coefficients per grid row) on the other.  At 17 flops per byte the
    stage sits far below the tensor cores' ridge point, so HBM is its roofline."""
    ntru = (2 * nlat - 1) // 3
    nrsp = (ntru + 1) * (ntru + 2)
    spec = (4 * nlev + 1) * nrsp * esz
    rows = ((6 * nlev + 3) if half == "inverse" else (9 * nlev + 1)) * nlat
    return spec + rows * (ntru + 1) * 2 * esz


# DRAM bytes per INSTANCE of the dominant kernel from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch over a known number
# of instances, divided by it), keyed by (kernel, workload); scaled to a launch by
# the instances it processes (the traffic grows in proportion: the intermediate
# is read once per instance, the tables once per launch are small beside it).
# k_tc_forward_pipe over eight T127 L20 instances (one launch of the default
# step), one ncu capture: 312.3 MB read + 42.1 MB written.  The summary with its
# command is in profiles/.
NCU_TRAFFIC_PER_INST = {("tc_forward", WORKLOAD): (312293376 + 42070272) / 8}


def traffic_per_launch(kernel, inst_per_launch):
    t = NCU_TRAFFIC_PER_INST.get((kernel, WORKLOAD))
    return None if t is None else t * inst_per_launch


def args_():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=20)
    a.add_argument("--warmup", type=int, default=5)
    a.add_argument("--impl", default="ours", choices=["ours", "reference"])
    a.add_argument("--batch", type=int, default=BATCH, help="T127 L20 instances per step and rank")
    a.add_argument("--no-cpu-baseline", action="store_true")
    a.add_argument("--precisions", default="mixed,fp32,fp64",
                   help="transform paths to time, first = headline (profiling runs pass one)")
    a.add_argument("--skip-radiation", action="store_true")
    a.add_argument("--skip-ensemble", action="store_true")
    return a.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: begin timing once it is sampling
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_sample(rounds=1):
    """FP64 oracle (C restatement of legmod/fftmod, OpenMP) on the same workload."""
    from oracle import oracle as O
    from exoplasim_b200 import synthetic as S
    L = O.Leg(NLAT)
    spin = S.transform_state(L.ntru, NLEV, seed=3, kind="steep")
    gin = S.grid_tendencies(NLAT, NLEV, seed=4).reshape(9 * NLEV + 1, -1)
    t0 = time.perf_counter()
    for _ in range(rounds):
        L.inverse_set(spin, NLEV, plavor=S.EZ)
        L.forward_set(gin, NLEV)
    dt = time.perf_counter() - t0
    return rounds / dt, dt, O.lib().oracle_num_threads()


def run_reference(a, rank):
    """The CPU arm: the FP64 restatement of legmod/fftmod on all host cores, one
    step = the same B round trips as the GPU arm's step."""
    if rank != 0:
        return
    B = a.batch
    for _ in range(a.warmup):
        cpu_baseline_sample(B)
    times = []
    for _ in range(a.steps):
        _, dt, threads = cpu_baseline_sample(B)
        times.append(dt)
    med = statistics.median(times)
    value = B / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "round-trips/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000.0 * med, "ms_per_step_mean": 1000.0 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, BASELINE config shapes)",
        "config": config_block(B, "fp64 (CPU)", 1),
        "cpu_baseline": {"value": value, "unit": "round-trips/s", "cores": threads, "kind": "port",
                         "sample": f"{B} T127 L20 round trips per step (median of {a.steps} steps), FP64 C "
                                   f"restatement of legmod/fftmod (gfortran absent), OpenMP over levels and rows"},
        "e2e": {"value": value, "unit": "round-trips/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(B, precision, world):
    """config of both arms' lines: the same workload keys, batch stated alike"""
    return {"workload": WORKLOAD, "batch": B, "precision": precision, "nlat": NLAT, "nlon": 2 * NLAT,
            "ntru": (2 * NLAT - 1) // 3, "nlev": NLEV,
            "l2": f"inputs larger than L2: {B} instances x {fp32_round_trip_bytes(NLAT, NLEV) / 1e6:.0f} MB",
            "parallelism": f"replicas x{world} (independent instances)"}


def relerr_fields(a, b):
    a = a.double().reshape(a.shape[0], -1)
    b = b.double().reshape(b.shape[0], -1)
    num = (a - b).abs().amax(dim=1)
    den = b.abs().amax(dim=1).clamp_min(1e-300)
    return float((num / den).max())


def dynamics_step(a, plan, spin64, gin64, B, world, time_graph, dev):
    """A whole dynamics timestep of B states on the device, in FP32 with the
    mixed transforms: the inverse gridpointa set -> the grid-point step
    (exp ln ps, calcgp, flux products) -> the forward set -> spectrala per
    state -> the inverse gridpointd set -> the forward gridpointd set (its grid
    tendencies, the physics' output, synthetic here) -> spectrald per state
    (plasim.f90 gridpointa :2396-2486, spectrala :2757-2918, gridpointd
    :3142-3433, spectrald :3645-3999).  The states advance in place."""
    import torch

    from exoplasim_b200 import gridpoint as GP
    from exoplasim_b200 import spectral as SP
    from exoplasim_b200.replicas import max_over_ranks

    from exoplasim_b200 import synthetic as S

    L, nrsp = NLEV, plan.nrsp
    gpc = GP.GpConst(GP.default_params(L))
    # a T127 time step: 256 per rotation (about 5.6 minutes of an Earth day)
    dt = 2.0 * math.pi / 256.0
    spc = SP.SpecConst(plan, SP.default_params(L, delt=dt, delt2=2.0 * dt))
    # the synthetic spectra scaled to atmospheric amplitudes (winds of about
    # 10 m/s, temperature anomalies of tens of K, surface-pressure anomalies of
    # about 1%) so the states stay finite over the timed steps; the planetary
    # vorticity kept, and ln(ps / psurf) with a zero global mean, as the model
    # holds it (spectrala keeps spp(1:2) = 0)
    s0 = spin64.clone()
    s0 *= 0.01
    s0[2 * L:3 * L, 2] += 0.99 * S.EZ
    s0[4 * L, 0:2] = 0.0
    state = s0.float().unsqueeze(0).repeat(B, 1, 1).contiguous()          # sd st sz sq sp at t
    prev = state.clone()                                                  # at t - dt
    ga = torch.empty((B, 6 * L + 3, NLAT, 2 * NLAT), device=dev)
    gf = torch.empty((B, 9 * L + 1, NLAT, 2 * NLAT), device=dev)
    tend_a = torch.empty((B, 4 * L + 1, nrsp), device=dev)
    gd = torch.empty((B, 4 * L + 1, NLAT, 2 * NLAT), device=dev)
    phys = gin64[:4 * L].float().unsqueeze(0).repeat(B, 1, 1, 1).contiguous() * 1e-2
    tend_d = torch.empty((B, 4 * L, nrsp), device=dev)
    sop = torch.zeros(nrsp, device=dev)
    srp = state[0, L:2 * L].clone()

    def views(x, i, nf):
        v = x[i]
        return {"d": v[0:L], "t": v[L:2 * L], "z": v[2 * L:3 * L], "q": v[3 * L:4 * L],
                "p": v[4 * L] if nf > 4 * L else None}

    states_a, states_d = [], []
    for i in range(B):
        sp_, sm_, ta, td = views(state, i, 4 * L + 1), views(prev, i, 4 * L + 1), views(tend_a, i, 4 * L + 1), \
            views(tend_d, i, 4 * L)
        base = {"sdp": sp_["d"], "szp": sp_["z"], "stp": sp_["t"], "sqp": sp_["q"], "spp": sp_["p"],
                "sdm": sm_["d"], "szm": sm_["z"], "stm": sm_["t"], "sqm": sm_["q"], "spm": sm_["p"],
                "sop": sop, "srp": srp}
        states_a.append({**base, "sdt": ta["d"], "szt": ta["z"], "stt": ta["t"], "sqt": ta["q"], "spt": ta["p"]})
        states_d.append({**base, "sdt": td["d"], "szt": td["z"], "stt": td["t"], "sqt": td["q"],
                         "spt": ta["p"]})

    def step():
        plan.inverse_set_batch(state, L, precision="mixed", out=ga)
        GP.gridpoint(plan, gpc, ga, gf)
        plan.forward_set_batch(gf, L, precision="mixed", out=tend_a)
        SP.spectrala_batch(spc, states_a)
        plan.inverse_set_d_batch(state, L, "mixed", out=gd)
        plan.forward_set_d_batch(phys, L, "mixed", out=tend_d)
        SP.spectrald_batch(spc, states_d)

    ms, nl, st_ms = time_graph(step, a.steps, a.warmup, with_steps=True)
    med = max_over_ranks(statistics.median(st_ms))
    return {"chain": "inverse set, calcgp, forward set, spectrala, inverse d-set, forward d-set, spectrald",
            "precision": "mixed transforms, FP32 grid-point and spectral steps", "ms_per_step": med,
            "timesteps_per_s": world * B / (med / 1000.0), "launches_per_step": nl,
            "finite": bool(torch.isfinite(state).all())}


def run_ours(a, rank, world, local_rank):
    import torch

    from exoplasim_b200 import radiation as R
    from exoplasim_b200 import synthetic as S
    from exoplasim_b200.replicas import barrier, max_over_ranks, unit_seed
    from exoplasim_b200.transforms import Plan, kernel_time, kernel_timing, launch_count

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    B = a.batch
    plan = Plan(NLAT)
    spin64 = torch.as_tensor(S.transform_state(plan.ntru, NLEV, seed=unit_seed(3, rank), kind="steep"), device=dev)
    gin64 = torch.as_tensor(S.grid_tendencies(NLAT, NLEV, seed=unit_seed(4, rank)), device=dev)

    def make(dtype):
        pr = "fp64" if dtype == torch.float64 else "fp32"
        spin = spin64.to(dtype).unsqueeze(0).repeat(B, 1, 1).contiguous()
        gin = gin64.to(dtype).unsqueeze(0).repeat(B, 1, 1, 1).contiguous()
        gout = torch.zeros((B, 6 * NLEV + 3, NLAT, 2 * NLAT), dtype=dtype, device=dev)
        sout = torch.zeros((B, 4 * NLEV + 1, plan.nrsp), dtype=dtype, device=dev)
        return spin, gin, gout, sout

    def step_fn(prec, bufs):
        spin, gin, gout, sout = bufs

        def f():
            plan.inverse_set_batch(spin, NLEV, precision=prec, out=gout)
            plan.forward_set_batch(gin, NLEV, precision=prec, out=sout)
        return f

    def time_graph(fn, steps, warmup, with_steps=False):
        fn()  # eager call: allocates work buffers and FFT tables outside capture
        torch.cuda.synchronize()
        n0 = launch_count()
        fn()
        torch.cuda.synchronize()
        per_step = launch_count() - n0
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                fn()
        torch.cuda.current_stream().wait_stream(s)
        for _ in range(warmup):
            g.replay()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        # one event between consecutive steps: the region's total and every
        # step's own duration come from the same K replays
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record()
        for i in range(steps):
            g.replay()
            ev[i + 1].record()
        torch.cuda.synchronize()
        barrier()
        ms = ev[0].elapsed_time(ev[-1])
        step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
        del g
        if with_steps:
            return ms, per_step, step_ms
        return ms, per_step

    results = {}
    # FP64 reference outputs for the error columns
    b64 = make(torch.float64)
    step_fn("fp64", b64)()
    torch.cuda.synchronize()
    ref_gout, ref_sout = b64[2][0].clone(), b64[3][0].clone()
    precisions = [p for p in a.precisions.split(",") if p]
    # clocks are sampled over the timed regions of every precision (each region
    # alone is shorter than a few sampling intervals)
    clocks = Clocks(local_rank)
    clocks.start()
    for prec in precisions:
        bufs = b64 if prec == "fp64" else make(torch.float32)
        fn = step_fn(prec, bufs)
        ms, per_step, step_ms = time_graph(fn, a.steps, a.warmup, with_steps=True)
        ms = max_over_ranks(ms)
        med = max_over_ranks(statistics.median(step_ms))
        err_g = relerr_fields(bufs[2][0], ref_gout) if prec != "fp64" else 0.0
        err_s = relerr_fields(bufs[3][0], ref_sout) if prec != "fp64" else 0.0
        # headline: the median of the K event-timed steps (slowest rank's)
        results[prec] = {"ms_per_step": med, "round_trips_per_s": world * B / (med / 1000.0),
                         "ms_per_step_mean": ms / a.steps,
                         "round_trips_per_s_mean": world * B * a.steps / (ms / 1000.0),
                         "launches_per_step": per_step, "max_rel_err_vs_fp64": max(err_g, err_s)}
        del bufs
    clk = clocks.stop()
    primary = precisions[0]

    # a whole dynamics timestep's transforms: the gridpointa round trip above
    # plus the gridpointd one (invlegd + fc2gp, then gp2fc + fc2sp + uv2dv,
    # plasim.f90:3142-3149, :3415-3428), same states, same precision
    timestep = None
    if primary != "fp64":
        sd_in = spin64.float().unsqueeze(0).repeat(B, 1, 1).contiguous()
        gd_in = gin64[:4 * NLEV].float().unsqueeze(0).repeat(B, 1, 1, 1).contiguous()
        gd_out = torch.zeros((B, 4 * NLEV + 1, NLAT, 2 * NLAT), device=dev)
        sd_out = torch.zeros((B, 4 * NLEV, plan.nrsp), device=dev)
        ba = make(torch.float32)

        def full_step():
            step_fn(primary, ba)()
            plan.inverse_set_d_batch(sd_in, NLEV, primary, out=gd_out)
            plan.forward_set_d_batch(gd_in, NLEV, primary, out=sd_out)
        ms_t, nl_t, st_t = time_graph(full_step, a.steps, a.warmup, with_steps=True)
        med_t = max_over_ranks(statistics.median(st_t))
        timestep = {"sets": "gridpointa + gridpointd round trips", "precision": primary,
                    "ms_per_step": med_t, "timesteps_per_s": world * B / (med_t / 1000.0),
                    "launches_per_step": nl_t}
        del ba, sd_in, gd_in, gd_out, sd_out
        timestep["dynamics_step"] = dynamics_step(a, plan, spin64, gin64, B, world, time_graph, dev)

    # per-stage timing of the primary precision
    bufs = make(torch.float32) if primary != "fp64" else make(torch.float64)
    inv_ms, _ = time_graph(lambda: plan.inverse_set_batch(bufs[0], NLEV, primary, out=bufs[2]), a.steps, a.warmup)
    fwd_ms, _ = time_graph(lambda: plan.forward_set_batch(bufs[1], NLEV, primary, out=bufs[3]), a.steps, a.warmup)
    hbm, tc, peak_kind = peaks()
    esz = 4 if primary != "fp64" else 8

    # per-kernel device time: each launch bracketed by CUDA events on its own
    # stream (the library's kernel timer), over K eager steps of the same work
    fn = step_fn(primary, bufs)
    for _ in range(a.warmup):
        fn()
    torch.cuda.synchronize()
    kernel_timing(True)
    for _ in range(a.steps):
        fn()
    torch.cuda.synchronize()
    leg = "tc" if primary == "mixed" else "leg"
    # the mixed path's Legendre kernels are judged against HBM (their arithmetic
    # intensity, 17 flops per byte, is far below the tensor-core ridge point);
    # their tensor-core rate is reported beside it
    units = {f"{leg}_inverse": ("hbm" if leg == "tc" else "fma",
                                legendre_bytes(NLAT, NLEV, "inverse", esz) if leg == "tc"
                                else legendre_flops(NLAT, NLEV, "inverse")),
             f"{leg}_forward": ("hbm" if leg == "tc" else "fma",
                                legendre_bytes(NLAT, NLEV, "forward", esz) if leg == "tc"
                                else legendre_flops(NLAT, NLEV, "forward")),
             "fft_inverse": ("hbm", fft_bytes(NLAT, NLEV, "inverse", esz)),
             "fft_forward": ("hbm", fft_bytes(NLAT, NLEV, "forward", esz))}
    flops = {f"{leg}_inverse": legendre_flops(NLAT, NLEV, "inverse"), f"{leg}_forward": legendre_flops(NLAT, NLEV, "forward")}
    kernels = {}
    for name, (bound, per_inst) in units.items():
        kms, nl = kernel_time(name)
        if nl == 0:
            continue
        work = per_inst * B * a.steps            # algorithmic flops or bytes over the timed steps
        rate = work / (kms / 1000.0)
        if bound == "hbm":
            ach, pk, unit = rate / 1e9, hbm, "GB/s"
        elif bound == "tensor":
            ach, pk, unit = rate / 1e12, tc, "TFLOP/s"
        else:  # SIMT FMA path: no measured peak to divide by
            ach, pk, unit = rate / 1e12, None, "TFLOP/s"
        kernels[name] = {"bound": bound, "ms_total": kms, "launches": nl, "ms_per_launch": kms / nl,
                         "achieved": ach, "peak": pk, "unit": unit, "frac": ach / pk if pk else None,
                         "share": None, "algorithmic_per_launch": work / nl}
        if leg == "tc" and name in flops:
            tf = flops[name] * B * a.steps / (kms / 1000.0) / 1e12
            kernels[name].update({"tensor_tflops": tf, "tensor_frac": tf / tc})
    kernel_timing(False)
    tot = sum(k["ms_total"] for k in kernels.values())
    for k in kernels.values():
        k["share"] = k["ms_total"] / tot
    dom = max(kernels, key=lambda k: kernels[k]["ms_total"])
    D = kernels[dom]
    roof = {"bound": "tensor" if D["bound"] == "tensor" else "hbm", "kernel": dom, "achieved": D["achieved"],
            "peak": D["peak"], "unit": D["unit"], "frac": D["frac"],
            "traffic": traffic_per_launch(dom, B * a.steps / D["launches"]), "peak_kind": peak_kind,
            "algorithmic_per_launch": D["algorithmic_per_launch"],
            "algorithmic_unit": "flops" if D["unit"] == "TFLOP/s" else "bytes",
            "ms_per_launch": D["ms_per_launch"]}
    if "tensor_tflops" in D:
        roof.update({"tensor_tflops": D["tensor_tflops"], "tensor_frac": D["tensor_frac"]})
    del bufs

    # end to end through the public API with host buffers: exotx_sets_host streams
    # the B states through device slots, copies in both directions overlapping
    # the transforms.  Host arrays of the transforms' kind (a 4-byte model's for
    # FP32/mixed), and FP64 host arrays converted on the device (an 8-byte
    # model's, exotx_sets_host_f64)
    def e2e_run(host_fp64):
        dtype = torch.float64 if (host_fp64 or primary == "fp64") else torch.float32
        hsz = 8 if dtype == torch.float64 else 4
        h_spin = spin64.to(dtype).cpu().unsqueeze(0).repeat(B, 1, 1).contiguous().pin_memory()
        h_gin = gin64.to(dtype).cpu().unsqueeze(0).repeat(B, 1, 1, 1).contiguous().pin_memory()
        h_gout = torch.empty((B, 6 * NLEV + 3, NLAT, 2 * NLAT), dtype=dtype).pin_memory()
        h_sout = torch.empty((B, 4 * NLEV + 1, plan.nrsp), dtype=dtype).pin_memory()

        def e2e_step():
            plan.sets_host(NLEV, h_spin, h_gout, h_gin, h_sout, precision=primary, host_fp64=host_fp64)

        for _ in range(a.warmup):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        h2d = (h_spin.numel() + h_gin.numel()) * hsz
        d2h = (h_gout.numel() + h_sout.numel()) * hsz
        # the outputs that came back against the device-resident FP64 path
        err = max(relerr_fields(h_gout[0], ref_gout.cpu()), relerr_fields(h_sout[0], ref_sout.cpu()))
        return {"value": world * B * a.steps / (ms / 1000.0), "unit": "round-trips/s",
                "max_rel_err_vs_fp64": err, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "host_dtype": str(dtype).replace("torch.", "")}

    e2e = e2e_run(False)
    e2e["api"] = "exotx_sets_host (pinned host arrays, copies overlapping the transforms)"
    e2e64 = e2e_run(True) if primary != "fp64" else None
    if e2e64:
        e2e64["api"] = "exotx_sets_host_f64 (pinned FP64 host arrays, converted on the device)"

    # radiation column pass: 8192 columns at L20 (T42 grid), plain kernel
    cols, g = S.radiation_columns(RAD_NLAT, RAD_NLEV, seed=unit_seed(2, rank))
    rad = {}
    for rprec, rdt in (() if a.skip_radiation else (("fp64", torch.float64), ("fp32", torch.float32))):
        dev_cols = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=rdt, device=dev) for k, v in cols.items()}
        params = R.default_params(RAD_NLEV, g["nhor"], g["nlon"], nsol=0)
        outs = R.alloc_outputs(params, rdt)
        ms, _ = time_graph(lambda: R.radstep(params, dev_cols, outs, precision=rprec), a.steps, a.warmup)
        ms = max_over_ranks(ms)
        rad[rprec] = {"cols_per_s": world * g["nhor"] * a.steps / (ms / 1000.0), "ms_per_pass": ms / a.steps}

    # learned surrogate (BF16 tensor-core MLP with out-of-range fallback) on the same
    # columns, and on 16 such grids side by side (64 tiles of 128 columns cannot fill
    # 148 SMs); the plain kernel is timed again on the same columns
    from exoplasim_b200 import surrogate as SG
    if not a.skip_radiation and os.path.exists(SG.DEFAULT_NET):
        net = SG.Mlp.load(SG.DEFAULT_NET)
        net.prepare()
        rad["surrogate"] = {"net": os.path.basename(SG.DEFAULT_NET)}
        for ncopy in (1, 16):
            rep = {k: (np.tile(v, ncopy) if k in ("sid", "cola") else
                       np.ascontiguousarray(np.tile(v, (1, ncopy)) if np.ndim(v) == 2 and k != "dsalb"
                                            else np.tile(v, (ncopy, 1)) if k == "dsalb" else np.tile(v, ncopy)))
                   for k, v in cols.items()}
            nh = g["nhor"] * ncopy
            params = R.default_params(RAD_NLEV, nh, g["nlon"], nsol=0)
            dev_cols = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64, device=dev)
                        for k, v in rep.items()}
            outs = R.alloc_outputs(params, torch.float64)
            ms_p, _ = time_graph(lambda: R.radstep(params, dev_cols, outs, precision="fp64"), a.steps, a.warmup)
            scols = {k: v.clone() for k, v in dev_cols.items()}
            souts = R.alloc_outputs(params, torch.float64)
            ms_s, nlaunch = time_graph(lambda: SG.surrogate_step(net, params, scols, souts), a.steps, a.warmup)
            cols32 = {k: v.float() for k, v in dev_cols.items()}
            outs32 = R.alloc_outputs(params, torch.float32)
            ms_p32, _ = time_graph(lambda: R.radstep(params, cols32, outs32, precision="fp32"), a.steps, a.warmup)
            ms_p, ms_p32, ms_s = max_over_ranks(ms_p), max_over_ranks(ms_p32), max_over_ranks(ms_s)
            key = f"{nh}_columns"
            rad["surrogate"][key] = {"cols_per_s": world * nh * a.steps / (ms_s / 1000.0),
                                     "plain_fp64_cols_per_s": world * nh * a.steps / (ms_p / 1000.0),
                                     "plain_fp32_cols_per_s": world * nh * a.steps / (ms_p32 / 1000.0),
                                     "speedup_vs_plain_fp64": ms_p / ms_s, "speedup_vs_plain_fp32": ms_p32 / ms_s,
                                     "launches_per_pass": nlaunch}
            del cols32, outs32
            if ncopy == 1:
                # accuracy against plain FP64 radstep on fresh outputs
                pc = {k: v.clone() for k, v in dev_cols.items()}
                pc["dtdt"].zero_()
                po = R.radstep(params, pc, precision="fp64")
                sc = {k: v.clone() for k, v in dev_cols.items()}
                sc["dtdt"].zero_()
                so = R.alloc_outputs(params, torch.float64)
                nfb = SG.surrogate_step(net, params, sc, so, count=True)
                L = RAD_NLEV
                fl = lambda o: torch.stack([o["dfd"][L], o["dfu"][L], o["dftd"][L], o["dftu"][L]])
                rad["surrogate"]["heating_rms_K_per_day"] = SG.heating_rms(sc["dtdt"], pc["dtdt"])
                rad["surrogate"]["surface_flux_rms_W_m2"] = float(torch.sqrt(((fl(so) - fl(po)) ** 2).mean()))
                rad["surrogate"]["fallback_fraction"] = nfb / nh
        del net
    # uneven ensemble: 96 instances of T21/T42/T63 x 10/15/20 levels, one tensor-core
    # and one FFT launch per half of the round trip, tuned, against running the same
    # instances one at a time through the single-resolution API
    ens = None
    if not a.skip_ensemble:
        from exoplasim_b200.ensemble import Ensemble, draw
        nl_e, lv_e = draw(96, seed=0)
        E = Ensemble(nl_e, lv_e)
        sp_i, gi_i = [], []
        for i, (nlat, L) in enumerate(zip(nl_e, lv_e)):
            ntru = (2 * nlat - 1) // 3
            spi = S.transform_state(ntru, L, seed=unit_seed(7, rank, i), kind="nn1")
            sp_i.append(torch.as_tensor(spi, device=dev).float())
            gi_i.append(torch.as_tensor(S.grid_tendencies(nlat, L, seed=unit_seed(500, rank, i)), device=dev).float())
        spin_e, gin_e = E.pack("spec", sp_i), E.pack("gin", gi_i)
        _, gout_e, _, spout_e = E.buffers()
        choice = E.tune(spin_e, gout_e, gin_e, spout_e, reps=3)
        ms_e, nlch_e = time_graph(lambda: (E.inverse(spin_e, gout_e), E.forward(gin_e, spout_e)), a.steps, a.warmup)
        eplans = {n: Plan(n) for n in sorted(set(nl_e))}
        sp_b = [t.unsqueeze(0).contiguous() for t in sp_i]
        gi_b = [t.unsqueeze(0).contiguous() for t in gi_i]
        go_b = [torch.zeros((1, 6 * L + 3, n, 2 * n), device=dev) for n, L in zip(nl_e, lv_e)]
        so_b = [torch.zeros_like(t) for t in sp_b]

        def one_by_one():
            for i, (n, L) in enumerate(zip(nl_e, lv_e)):
                eplans[n].inverse_set_batch(sp_b[i], L, "mixed", out=go_b[i])
                eplans[n].forward_set_batch(gi_b[i], L, "mixed", out=so_b[i])
        ms_1, nlch_1 = time_graph(one_by_one, a.steps, a.warmup)
        ms_e, ms_1 = max_over_ranks(ms_e), max_over_ranks(ms_1)
        ens = {"instances": 96, "resolutions": {f"T{(2 * n - 1) // 3}": nl_e.count(n) for n in sorted(set(nl_e))},
               "round_trips_per_s": world * 96 * a.steps / (ms_e / 1000.0), "launches_per_step": nlch_e,
               "one_by_one_round_trips_per_s": world * 96 * a.steps / (ms_1 / 1000.0),
               "one_by_one_launches_per_step": nlch_1, "tuned": choice}
        del E, eplans
    barrier()
    if rank != 0:
        return
    cpu = None
    if not a.no_cpu_baseline and world == 1:
        r, dt, threads = cpu_baseline_sample(1)
        if dt < 10.0:
            n = max(1, int(15.0 / dt))
            r, dt, threads = cpu_baseline_sample(n)
        cpu = {"value": r, "unit": "round-trips/s", "cores": threads, "kind": "port",
               "sample": f"{max(1, round(r * dt))} T127 L20 round trip(s) in {dt:.1f} s, FP64 C restatement of "
                         f"legmod/fftmod with OpenMP (gfortran absent, reference not buildable)"}
    prim = results[primary]
    line = {
        "metric": METRIC,
        "value": prim["round_trips_per_s"], "unit": "round-trips/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": prim["ms_per_step"], "ms_per_step_mean": prim["ms_per_step_mean"],
        "timing": f"median of {a.steps} event-timed steps (CUDA graph replays)",
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if primary != "fp64" else "f64",
        "data": "synthetic (seeded spectra ~1/(n(n+1)), n^-3 beyond n=10; grid tendencies N(0,1e-5^2))",
        "config": config_block(B, primary, world),
        "precisions": results,
        "roofline": roof,
        "kernels": kernels,
        "stages_ms_per_instance": {"inverse_set": inv_ms / (a.steps * B), "forward_set": fwd_ms / (a.steps * B)},
        "full_timestep": timestep,
        "e2e": e2e,
        "e2e_fp64_host": e2e64,
        "radiation": {"metric": "radiation cols/s (T42 grid, 8192 columns, L20, plain radmod kernel)", **rad},
        "ensemble": ens,
        "clocks": clk,
        "gpu_launches": prim["launches_per_step"] * a.steps,
        "cpu_baseline": cpu,
        "legendre_gflop_per_round_trip": legendre_flops(NLAT, NLEV) / 1e9,
    }
    print(json.dumps(line), flush=True)


def main():
    a = args_()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the SPH step: particle-steps/s of block-timestep system steps on one B200.

One "step" is one system step (blocks.advance): the GN gravity flow of every particle, density
for the active rows and their neighbours, the fused force + du/dt pass for the active rows,
cooling, kicks and new levels.  value = active particles summed over the K timed system steps of
all ranks / the slowest rank's device time (CUDA events on the launching stream).

Workloads (seeded synthetic inputs; there is no dataset):
  torus   4,194,304 particles, Gaussian torus R=100 a=40 sigma=15, T=1e9 K, disc viscosity
          alpha_SS = 0.1, bremsstrahlung cooling, block steps (dt_max 256)   [default]
  streams 1,048,576 particles, two colliding cylinders at r=1664, 1e-10 g/cm^3, bremsstrahlung
  cloud   262,144-particle cloud on a GN orbit (block steps)
Inputs (~1 GB of particle state at 4M) are larger than the 126 MB L2, so no flush is needed.

--impl reference times the reference's algorithm on the host cores instead: the CPU oracle port
(oracle/, C + OpenMP, all host threads) on a bounded sample of the same workload.
Multi-GPU: replicas only (each rank runs an independent seeded run; no collective in the step).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 FP32 lanes x FMA x clock
FP64_NOMINAL_TFLOPS = FP32_NOMINAL_TFLOPS / 2.0
FLOP_PER_DENSITY_EVAL = 25.0  # distance + kernel + two sums per pair evaluation
FLOP_PER_FORCE_PAIR = 75.0  # pressure + viscosity + P dV (+20 with disc viscosity)
# DRAM bytes (read + write) per row of one launch, from ncu captures (cold caches) of the FP32
# kernels on the 1,048,576-particle torus, scaled to a launch by its rows: density 199.9 MB over
# 195,200 rows; forces (walk + pair launches) 1,347 + 1,007 MB over 1,045,504 rows; a list build
# (candidate, test and expansion passes of a build after the start, 163 entries per row)
# 1,273 MB over 1,048,576 particles
DRAM_BYTES_PER_ROW = {"forces": 2251.0, "density": 1024.0, "lists": 1214.0}
# What the ncu counters of the same captures show limits each kernel (the roofline's ceiling
# stays the HBM copy bandwidth; none of these kernels is a contraction)
LIMITER = {
    "lists": "issue: the test pass at 80 % issue active (FMA 45 %, ALU 42 %), the expansion at "
             "64 %; the candidate pass latency bound (long-scoreboard 3.2 per issue at 24 % warp "
             "occupancy); DRAM 0.1-9 % of peak",
    "cooling": "issue and shared-memory latency: 39 % issue active at 24 % warp occupancy (128 "
               "registers), tensor pipe 19.5 %, FP64 pipe 6.4 % (the check)",
    "density": "latency: long-scoreboard stalls 4.2 per issue on the gathered records, 66 % "
               "issue active at 43 % warp occupancy, DRAM 8 % of peak",
    "forces": "latency: the walk launch stalls 11.5 per issue on the gathered records (DRAM 21 %); "
              "the pair launch runs the FMA pipe at 36 % with 43 % warp occupancy",
    "flow": "FP64 pipe 69-71 % (the double-precision flow update), DRAM 25-29 %",
}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return {"hbm_gbs": p["hbm_gbs"], "bf16_tflops": p["bf16_tflops"], "source": "measured"}
    return {**PEAKS_FALLBACK, "source": "fallback"}


# Disc viscosity of the torus: alpha_AV = 1, the value of the reference's own disc-viscosity block
# test.  It gives alpha_SS = alpha_AV <h> / (10 H) (physics/disc_viscosity.py:56-58) with H = 15 M;
# alpha_SS = 0.1 would need alpha_AV = 10 alpha_SS H / <h> ~ 16 at 4,194,304 particles
# (<h> ~ 0.93 M), where a few particles heat without bound within ten system steps in FP64 and
# FP32 alike under the reference's viscous step limit 0.25 h^2 / nu.
TORUS_ALPHA_AV = 1.0
TORUS_SCALE_HEIGHT = 15.0
WEIGHTS = os.path.join(ROOT, "blackhole_nebula_simulator_b200", "data", "cooling_mlp.npy")


def cooling_network():
    """The trained cooling network (weights trained on the GPU by the library's kernels and
    saved by `python -m blackhole_nebula_simulator_b200.cooling`); trained here if absent."""
    from blackhole_nebula_simulator_b200 import cooling

    if os.path.exists(WEIGHTS):
        return cooling.load_network(WEIGHTS, cooling.mlp_params(judge=64))
    net = cooling.train_network()
    net.params = cooling.mlp_params(judge=64)
    return net


def workload(name: str, n: int | None, precision: str, seed_shift: int = 0, mlp=None,
             eos: str = "ideal", shock: bool = False):
    from blackhole_nebula_simulator_b200 import ics
    from blackhole_nebula_simulator_b200.config import BlockConfig, CoupledConfig, HydroConfig

    # shock: the reference's default shock capturing (Cullen-Dehnen switch from alpha = 0 and
    # velocity reconstruction), else constant alpha
    common = dict(kernel="cubic", eta=1.2, switch=shock, reconstruction=shock,
                  conductivity_signal=1, alpha_u=0.05, h_max=200.0, precision=precision,
                  eos=eos)  # fmt: skip
    if name == "torus":
        n = n or 4_194_304
        ic = ics.torus(n, seed=4 + seed_shift)
        hc = HydroConfig(disc_alpha_av=TORUS_ALPHA_AV, **common)
        bc = BlockConfig(coupled=CoupledConfig(hydro=hc, cooling="brems", cooling_mlp=mlp),
                         dt_max=256.0)  # fmt: skip
    elif name == "streams":
        n = n or 1_048_576
        ic = ics.streams(n, seed=3 + seed_shift)
        bc = BlockConfig(coupled=CoupledConfig(hydro=HydroConfig(**common), cooling="brems",
                                               cooling_mlp=mlp), dt_max=4096.0)  # fmt: skip
    elif name == "cloud":
        n = n or 262_144
        ic = ics.cloud(n, seed=1 + seed_shift)
        bc = BlockConfig(coupled=CoupledConfig(hydro=HydroConfig(**common)), dt_max=4096.0)
    else:
        raise ValueError(name)
    return ic, bc


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)  # fmt: skip
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 3 + k and r[3 + k].lower() == "active"})  # fmt: skip
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def profile_read(ctx):
    import ctypes

    from blackhole_nebula_simulator_b200 import _lib

    names = ["lists", "density", "forces", "flow", "marks", "levels", "cooling", "eos", "gradients"]
    out = (ctypes.c_double * (4 * len(names)))()
    _lib.check(ctx, _lib.lib().nb_profile_read(ctx, out))
    return {names[c]: {"ms": out[4 * c], "launches": int(out[4 * c + 1]), "units": out[4 * c + 2],
                       "pairs": out[4 * c + 3]} for c in range(len(names))}  # fmt: skip


def roofline(prof, precision, disc, pk):
    """Dominant kernel: its algorithmic bytes per launch over its event-timed duration."""
    dom = max(("lists", "density", "forces", "flow"), key=lambda k: prof[k]["ms"])
    d = prof[dom]
    if d["launches"] == 0:
        return None, dom
    ms = d["ms"] / d["launches"]
    rec = 112.0 if precision == "fp32" else 128.0  # packed per-particle records of a pair pass
    units = d["units"] / d["launches"]
    pairs = d["pairs"] / d["launches"]
    if dom == "forces":
        bytes_ = units * (rec + 48.0) + pairs * 4.0
        flops = pairs * (FLOP_PER_FORCE_PAIR + (20.0 if disc else 0.0))
    elif dom == "density":
        bytes_ = units * (48.0 + 40.0) + pairs * 4.0
        flops = pairs * FLOP_PER_DENSITY_EVAL
    elif dom == "lists":
        bytes_ = units * (32.0 + 8.0) + pairs * 4.0
        flops = 0.0
    else:  # flow: x_beg, p_half, n_beg, n_end, a read; x, p_flow, p_pred written
        bytes_ = units * (48.0 + 16.0 + 24.0 + 72.0 + 8.0)
        flops = 0.0
    gbs = bytes_ / (ms * 1e-3) / 1e9
    pipe_peak = FP32_NOMINAL_TFLOPS if precision == "fp32" else FP64_NOMINAL_TFLOPS
    traffic = (DRAM_BYTES_PER_ROW[dom] * units
               if (precision == "fp32" or dom == "lists") and dom in DRAM_BYTES_PER_ROW
               else None)  # fmt: skip
    rf = {"bound": "hbm", "kernel": dom, "achieved": round(gbs, 2), "peak": pk["hbm_gbs"],
          "unit": "GB/s", "frac": round(gbs / pk["hbm_gbs"], 4), "traffic": traffic,
          "peak_source": pk["source"], "ms_per_launch": round(ms, 4),
          "bytes_per_launch": bytes_, "limiter": LIMITER.get(dom)}  # fmt: skip
    if flops:
        tf = flops / (ms * 1e-3) / 1e12
        rf["pipe"] = {"unit": "TFLOP/s", "achieved": round(tf, 3), "peak": round(pipe_peak, 2),
                      "frac": round(tf / pipe_peak, 4), "peak_source": "nominal",
                      "precision": precision}  # fmt: skip
    return rf, dom


# algorithmic bytes and FLOPs of one launch of each category, from its units (rows or
# particles) and pairs (list entries written, in-support density evaluations, interacting force
# pairs) per launch; None where the category has no such model
def _category_work(cat, units, pairs, precision, disc):
    rec = 112.0 if precision == "fp32" else 128.0  # packed per-particle records of a pair pass
    if cat == "lists":  # sorted record read, offset written, 4 B per entry written
        return units * (32.0 + 8.0) + pairs * 4.0, 0.0
    if cat == "density":  # row records in, h / rho / omega out, 4 B per pair evaluation
        return units * (48.0 + 40.0) + pairs * 4.0, pairs * FLOP_PER_DENSITY_EVAL
    if cat == "forces":
        return (units * (rec + 48.0) + pairs * 4.0,
                pairs * (FLOP_PER_FORCE_PAIR + (20.0 if disc else 0.0)))  # fmt: skip
    if cat == "flow":  # x_beg, p_half, n_beg, n_end, a in; x, p_flow, p_pred out
        return units * (48.0 + 16.0 + 24.0 + 72.0 + 8.0), 0.0
    if cat == "cooling":  # u, rho, dt in; u out
        return units * 32.0, 0.0
    if cat == "eos":  # rho, u, mask in; P, c_s out
        return units * 33.0, 0.0
    return None, None


def kernel_table(prof, precision, disc, pk):
    """Every timed category: launches, ms per launch, algorithmic GB/s and FP32 (or FP64)
    TFLOP/s per launch with their fractions of the measured HBM peak and the nominal pipe."""
    pipe_peak = FP32_NOMINAL_TFLOPS if precision == "fp32" else FP64_NOMINAL_TFLOPS
    out = {}
    for cat, d in prof.items():
        if cat.startswith("_") or d["launches"] == 0:
            continue
        ms = d["ms"] / d["launches"]
        units, pairs = d["units"] / d["launches"], d["pairs"] / d["launches"]
        b, f = _category_work(cat, units, pairs, precision, disc)
        row = {"launches": d["launches"], "ms_per_launch": round(ms, 4),
               "units_per_launch": round(units), "pairs_per_launch": round(pairs)}  # fmt: skip
        if b is not None and ms > 0:
            gbs = b / (ms * 1e-3) / 1e9
            row.update(bytes_per_launch=round(b), gbs=round(gbs, 1),
                       hbm_frac=round(gbs / pk["hbm_gbs"], 4))  # fmt: skip
        if f and ms > 0:
            tf = f / (ms * 1e-3) / 1e12
            row.update(flop_per_launch=round(f), tflops=round(tf, 3),
                       pipe_frac=round(tf / pipe_peak, 4))  # fmt: skip
        if cat in LIMITER:
            row["limiter"] = LIMITER[cat]
        out[cat] = row
    return out


def combine_ranks(ms, psteps, device):
    """Replicas: the job's time is the slowest rank's, its work the sum over ranks."""
    import torch

    t = torch.tensor([ms, float(psteps)], dtype=torch.float64, device=device)
    tmax = t.clone()
    torch.distributed.all_reduce(tmax, op=torch.distributed.ReduceOp.MAX)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return float(tmax[0]), float(t[1])


def run_gpu(args, rank, world, precision=None, use_mlp=None, e2e=True):
    import torch

    from blackhole_nebula_simulator_b200 import _lib, blocks, cooling
    from blackhole_nebula_simulator_b200.device import ctx

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    precision = precision or args.precision
    use_mlp = (precision == "fp32") if use_mlp is None else use_mlp
    net = cooling_network() if use_mlp else None
    ic, bc = workload(args.workload, args.n, precision, seed_shift=rank, mlp=net, eos=args.eos,
                      shock=args.shock)
    st = blocks.initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, bc, t_stop=bc.dt_max * 2.0**20)
    led_init = blocks.ledger(st, bc)  # every particle is at a step boundary here
    for _ in range(args.warmup):
        blocks.advance(st, bc)
    c = ctx(dev)
    stream = torch.cuda.current_stream()
    snap = snapshot_state(st)
    led0 = blocks.ledger(st, bc)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    _lib.check(c, _lib.lib().nb_profile(c, 1))
    steps0 = st.particle_steps
    launches0 = _lib.lib().nb_launch_count()
    syncs0 = _lib.lib().nb_sync_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            blocks.advance(st, bc)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = _lib.lib().nb_launch_count() - launches0
    syncs = _lib.lib().nb_sync_count() - syncs0
    prof = profile_read(c)
    prof["_launches"] = launches
    prof["_syncs"] = syncs
    _lib.check(c, _lib.lib().nb_profile(c, 0))
    ms = e0.elapsed_time(e1)
    psteps = st.particle_steps - steps0
    if world > 1:
        ms, total = combine_ranks(ms, psteps, dev)
    else:
        total = float(psteps)
    mlp = cooling.mlp_stats(reset=True) if use_mlp else None
    led = blocks.ledger(st, bc)
    led["drift"] = (led["energy"] - led0["energy"]) / led0["abs_h"]
    # energy drift between full synchronisation points (the ledger is exact only when every
    # particle is at a step boundary): run, untimed, to the end of the longest open step
    if not st.synced():
        blocks.run(st, bc, st.t0 + int(st.n_end.max()) * st.tick)
    led_sync = blocks.ledger(st, bc)
    led["drift_synced"] = (led_sync["energy"] - led_init["energy"]) / led_init["abs_h"]
    led["t_synced"] = st.t
    led["sync_steps"] = len(st.active_counts) - args.warmup - args.steps
    e2e_out = run_e2e(args, st, bc, snap) if e2e else None
    return ms, total, prof, clk.summary(), st, led, e2e_out, mlp


# removal bookkeeping (original ids, starting radius and |L|, flags): neither read nor written by a
# block step without removal radii, as in every bench workload, so not part of its transfers
REMOVAL_FIELDS = ("ids", "r0", "L0", "vr_neg", "passed_peri", "doomed")


def _tensor_fields(st):
    import torch

    return [k for k, v in st.__dict__.items() if isinstance(v, torch.Tensor) and k != "_rows"
            and k not in REMOVAL_FIELDS]  # fmt: skip


def snapshot_state(st):
    """Pinned host copy of the block state and its host-side counters (before the timed steps)."""
    import copy

    host = {k: getattr(st, k).detach().to("cpu").pin_memory() for k in _tensor_fields(st)}
    scal = {k: copy.copy(v) for k, v in st.__dict__.items() if k not in host and k != "_rows"
            and not k.startswith("_")}  # fmt: skip
    return host, scal


# the block-state fields a system step reads (sim/blocks.py:502-563): the step's starts, half
# kicks and tick counters, levels, the accelerations and du/dt of the predictor, masses, smoothing
# lengths (the density's start), alpha (the neighbours' viscosity), rho (the predicted cooling of
# every particle), the heat budget (added to at every kick) and the parts of du/dt (read by the
# kicks of the particles whose steps the wake-up cuts).  x, p, u are overwritten for every
# particle by the flow, the predictor and the cooling; omega, c_s, vsig_max and nu are recomputed
# where they are read.
STEP_READS = ("x_beg", "p_half", "u_half", "n_beg", "n_end", "level", "level_offset", "a_hydro",
              "dudt", "mass", "h", "alpha", "rho", "visc_heating", "cond_heating",
              "disk_heating", "heat_visc", "heat_cond", "heat_disk", "heat_pdv",
              "heat_cool")  # fmt: skip


def run_e2e(args, st, bc, snap):
    """The same K system steps again, through the public API with the state in host memory:
    each step copies in from pinned host memory the state fields the step reads and copies the
    whole updated state back out into the same host buffers (so every step's input is the host
    copy of the previous step's result), timed with CUDA events around copies and steps.

    The copies run on their own streams, one per direction, field by field: a field's copy-in
    waits for the previous step's copy-out of that field only, so the copy-in of one field
    overlaps the copy-out of the next (the two directions of the host link are independent).
    The fields the step only writes are copied out from a device copy taken when the step ends,
    so the next step starts once its copy-ins have finished, while those copy-outs still run."""
    import torch

    from blackhole_nebula_simulator_b200 import blocks

    host, scal = snap
    for k, v in scal.items():
        setattr(st, k, v)
    names = list(host)
    reads = [k for k in names if k in STEP_READS]
    writes = [k for k in names if k not in STEP_READS]  # written by the step, never read by it
    in_bytes = sum(host[k].numel() * host[k].element_size() for k in reads)
    nbytes = sum(host[k].numel() * host[k].element_size() for k in names)
    shadow = {k: torch.empty_like(getattr(st, k)) for k in writes}
    stream = torch.cuda.current_stream()
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    s0 = st.particle_steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h2d.wait_event(e0)
    out_done = {}
    shadow_free = None
    for _ in range(args.steps):
        with torch.cuda.stream(h2d):
            for k in reads:
                if k in out_done:
                    h2d.wait_event(out_done[k])
                getattr(st, k).copy_(host[k], non_blocking=True)
        stream.wait_stream(h2d)
        blocks.advance(st, bc)
        if shadow_free is not None:
            stream.wait_event(shadow_free)  # the last step's copy-outs of the shadow are done
        for k in writes:
            shadow[k].copy_(getattr(st, k), non_blocking=True)
        d2h.wait_stream(stream)
        with torch.cuda.stream(d2h):
            for k in reads:  # the read set first: the next step's copy-ins wait for it
                host[k].copy_(getattr(st, k), non_blocking=True)
                out_done[k] = torch.cuda.Event()
                out_done[k].record(d2h)
            for k in writes:
                host[k].copy_(shadow[k], non_blocking=True)
            shadow_free = torch.cuda.Event()
            shadow_free.record(d2h)
    stream.wait_event(shadow_free)
    stream.wait_stream(h2d)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": (st.particle_steps - s0) / (ms * 1e-3), "unit": "particle-steps/s",
            "h2d_bytes_per_step": int(in_bytes), "d2h_bytes_per_step": int(nbytes),
            "steps": args.steps, "ms_per_step": ms / args.steps,
            "copies": "per field on one stream per direction; the fields a step only writes "
                      "go out from a device copy while the next step runs"}  # fmt: skip


def h_stats(st):
    h = st.h.detach().cpu().numpy()
    q = np.percentile(h, [0, 50, 99, 100])
    return {"min": float(q[0]), "median": float(q[1]), "p99": float(q[2]), "max": float(q[3])}


def cpu_reference(args, steps, warmup, sample_n=None):
    """The reference algorithm on the host cores: the CPU oracle's block step (C + OpenMP on all
    host threads), on a bounded sample of the workload (same generator and physics, fewer
    particles), so that the run stays within minutes."""
    from oracle import steps as osteps

    n_full = {"torus": 4_194_304, "streams": 1_048_576, "cloud": 262_144}[args.workload]
    n = sample_n or min(args.n or n_full, 32_768)
    ic, bc = workload(args.workload, n, "fp64", eos=args.eos, shock=args.shock)
    st = osteps.blocks_initialise(ic.x, ic.v, ic.u, ic.mass, ic.h, bc, t_stop=bc.dt_max * 2.0**20)
    for _ in range(warmup):
        osteps.blocks_advance(st, bc)
    s0 = st.particle_steps
    t0 = time.perf_counter()
    for _ in range(steps):
        osteps.blocks_advance(st, bc)
    dt = time.perf_counter() - t0
    cores = os.cpu_count()
    return {"value": (st.particle_steps - s0) / dt, "unit": "particle-steps/s", "cores": cores,
            "kind": "port", "sample": f"{args.workload} workload at {n} particles (same generator "
            f"and physics), {steps} timed system steps after {warmup} warm-up, oracle on "
            f"{cores} OpenMP threads"}  # fmt: skip


# deposition frame: the 4M torus snapshot onto the reference's default log-spherical render grid
# (192 x 96 x 192, wide particles through the coarse grid; its cells are wider than the torus
# particles' kernels, so they take the trilinear weights) and a detail box of 160^3 cells of
# 0.4 across the torus' ring at x = 100 (kernel weights over ~4^3 cells per particle)
DEPOSIT_BOX = dict(centre=(100.0, 0.0, 0.0), size=64.0, n=160)


def deposit_inputs(n, seed=4):
    from blackhole_nebula_simulator_b200 import ics, units

    ic = ics.torus(n, seed=seed)
    t = ic.u / units.gas_u_from_temperature(1.0)  # the ideal-gas temperature of u (linear in T)
    return ic.x, ic.h, ic.mass, t, ic.v


def deposit_frame(gg, x, h, m, t, v, grid, box, host=False):
    a = gg.deposit_log_split(x, h, m, t, v, grid)
    b = gg.deposit_box(x, h, m, t, v, box)
    if host:  # the renderer's float32 fields and the ledgers back on the host
        return [f.cpu() for f in (a.rho, a.t_mass, a.t_em, a.vel, b.rho, b.t_mass, b.t_em, b.vel)]
    return a, b


def cpu_deposit(n_sample, n_full=4_194_304):
    """The reference's deposition on the host cores: the oracle (C, one thread, the reference's
    two fixed chunks one after the other) on the first n_sample particles of the frame's
    snapshot (the same smoothing lengths as the whole snapshot's)."""
    from blackhole_nebula_simulator_b200 import gasgrid as gg
    from oracle import deposit as odep

    x, h, m, t, v = (a[:n_sample] for a in deposit_inputs(n_full))
    grid, box = gg.LogSphericalGrid(), gg.CartesianBox(**DEPOSIT_BOX)
    t0 = time.perf_counter()
    odep.deposit_log_split(x, h, m, t, v, grid, gg.coarse_log_grid(grid))
    odep.deposit_box(x, h, m, t, v, box)
    dt = time.perf_counter() - t0
    return {"value": n_sample / dt, "unit": "particles/s", "cores": 1, "kind": "port",
            "sample": f"the first {n_sample} particles of the {n_full}-particle torus snapshot, one "
                      "frame (log-spherical 192x96x192 split + 160^3 box), oracle in C on one "
                      "thread"}  # fmt: skip


def run_deposit(args, rank, world):
    """One step = one render frame's deposition of the whole snapshot (inputs resident)."""
    import torch

    from blackhole_nebula_simulator_b200 import _lib
    from blackhole_nebula_simulator_b200 import gasgrid as gg
    from blackhole_nebula_simulator_b200.device import ctx

    n = args.n or 4_194_304
    config = {"workload": f"deposit: torus snapshot, {n} particles -> log-spherical grid "
                          "192x96x192 (wide particles on the coarse grid) + 160^3 box",
              "particles": n, "l2_flush": "inputs and grids larger than L2",
              "parallelism": f"replicas x{world}"}  # fmt: skip
    metric = "particles deposited/s"
    if args.impl == "reference":
        if rank == 0:
            cb = cpu_deposit(min(n, 131_072), n)
            print(json.dumps({"metric": metric, "value": cb["value"], "unit": "particles/s",
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "impl": "reference", "dtype": "f64",
                              "data": "synthetic", "config": config, "cpu_baseline": cb,
                              "e2e": {"value": cb["value"], "unit": "particles/s",
                                      "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))  # fmt: skip
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    xs, hs, ms, ts, vs = deposit_inputs(n, seed=4 + rank)
    x, h, m, t, v = (torch.as_tensor(a, dtype=torch.float64, device=dev) for a in (xs, hs, ms, ts, vs))
    grid, box = gg.LogSphericalGrid(), gg.CartesianBox(**DEPOSIT_BOX)
    for _ in range(args.warmup):
        deposit_frame(gg, x, h, m, t, v, grid, box)
    stream = torch.cuda.current_stream()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.lib().nb_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev.index) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            a, b = deposit_frame(gg, x, h, m, t, v, grid, box)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = _lib.lib().nb_launch_count() - launches0
    ms_t = e0.elapsed_time(e1)
    total = float(n * args.steps)
    if world > 1:
        ms_t, total = combine_ranks(ms_t, n * args.steps, dev)
    ledger = (float(a.mass.sum()) + a.outside) / float(ms.sum())
    # the same frames through the public API from host arrays, fields back on the host
    pinned = [torch.as_tensor(q).pin_memory() for q in (xs, hs, ms, ts, vs)]
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        deposit_frame(gg, *[q.to(dev, non_blocking=True) for q in pinned], grid, box, host=True)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    ncell = grid.nr * grid.nth * grid.nph + box.n**3
    in_bytes = n * 9 * 8  # x, h, m, t, v
    out_bytes = ncell * 6 * 4  # rho, T, T_em (float32) and v (3 x float32)
    # roofline: algorithmic bytes of one frame (particle inputs read twice, one per grid; the
    # 6 FP64 sums of every cell written and read back; the float32 fields and masses written)
    alg = 2 * in_bytes + ncell * (6 * 8 * 2 + 8 + 6 * 4)
    pk = peaks()
    achieved = alg / (ms_t / args.steps * 1e-3) / 1e9
    if rank == 0:
        cb = None if args.no_cpu_baseline else cpu_deposit(min(n, 131_072), n)
        print(json.dumps({
            "metric": metric, "value": total / (ms_t * 1e-3), "unit": "particles/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded torus snapshot)",
            "config": config,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 5), "traffic": None,
                         "peak_source": pk["source"], "bytes_per_launch": alg,
                         "note": "scattered FP64 atomic adds, not a streaming kernel"},
            "clocks": clk.summary(),
            "e2e": {"value": n * args.steps / (ms_e2e * 1e-3), "unit": "particles/s",
                    "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": out_bytes},
            "gpu_launches": launches, "mass_ledger": ledger, "n_wide": a.extra["n_wide"],
            "n_trilinear": [a.n_trilinear, b.n_trilinear], "cpu_baseline": cb,
        }))  # fmt: skip


def measure(args, name, rank, world, steps=None):
    """One workload on this rank: the FP32 + MLP form (value, e2e, kernel categories, drift),
    the FP64 plain form on the same workload, and on rank 0 the roofline and the CPU baseline.
    Returns the workload's JSON object (rank 0) or None."""
    import copy

    a = copy.copy(args)
    a.workload = name
    a.n = args.n if name == args.workload else None
    if steps is not None:
        a.steps = steps
    ms, total, prof, clocks, st, led, e2e, mlp = run_gpu(a, rank, world)
    plain = None
    if a.precision == "fp32" and not a.no_plain:
        # the comparison form of the metric: FP64 pair arithmetic with the exact integrator
        p_ms, p_total, p_prof, p_clk, p_st, p_led, _, _ = run_gpu(a, rank, world, "fp64", False,
                                                                  e2e=False)  # fmt: skip
        plain = {"value": p_total / (p_ms * 1e-3), "unit": "particle-steps/s",
                 "ms_per_step": p_ms / a.steps, "dtype": "f64", "cooling": "exact integrator",
                 "energy_rel_drift": p_led["drift_synced"],
                 "kernel_ms": {k: round(v["ms"], 3) for k, v in p_prof.items()
                               if not k.startswith("_")}}  # fmt: skip
    if rank != 0:
        return None
    pk = peaks()
    launches = prof.pop("_launches")
    syncs = prof.pop("_syncs")
    rf, dom = roofline(prof, a.precision, "torus" == name, pk)
    n_full = a.n or N_FULL[name]
    out = {
        "value": total / (ms * 1e-3), "unit": "particle-steps/s", "steps": a.steps,
        "ms_per_step": ms / a.steps, "config": workload_config(a, name, n_full, world),
        "roofline": rf, "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
        "host_syncs_per_step": syncs / a.steps,
        "kernel_ms": {k: round(v["ms"], 3) for k, v in prof.items()},
        "kernel_table": kernel_table(prof, a.precision, "torus" == name, pk),
        "mean_active": total / a.steps / max(world, 1),
        "list_builds": st.builds, "list_reuses": st.reuses,
        "levels_used": sorted(set(int(v) for v in st.level.unique().tolist())),
        "mean_list_entries": (prof["lists"]["pairs"] / prof["lists"]["units"]
                              if prof["lists"]["units"] else None),
        "pairs_per_force_row": (prof["forces"]["pairs"] / prof["forces"]["units"]
                                if prof["forces"]["units"] else None),
        "h_stats": h_stats(st),
        "disc_alpha_ss": (TORUS_ALPHA_AV * float(st.h.mean()) / (10.0 * TORUS_SCALE_HEIGHT)
                          if name == "torus" else None),
        "cooling": ("network (BF16 tensor cores, exact fallback; bremsstrahlung law of this "
                    "library, parity with the reference unpinned: it has no such law)"
                    if mlp is not None else "exact integrator"),
        "cooling_network": (dict(mlp, gain=(
            "net cost: the exact integrator of this library's bremsstrahlung law is a closed "
            "form; cooling category ms per step with the network "
            f"{prof['cooling']['ms'] / a.steps:.3f} vs {plain['kernel_ms']['cooling'] / a.steps:.3f} "
            "with the exact integrator (FP64 plain)" if plain else "net cost (closed-form law)"))
                            if mlp is not None else None),
        "energy_rel_drift": led["drift_synced"],
        "energy_drift_over_time": led["t_synced"],
        "energy_drift_sync_steps": led["sync_steps"],
        "fp64_plain": plain,
        "speedup_vs_fp64_plain": (total / (ms * 1e-3)) / plain["value"] if plain else None,
    }  # fmt: skip
    if not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_reference(a, 2, 1)
    return out


N_FULL = {"torus": 4_194_304, "streams": 1_048_576, "cloud": 262_144}
# the second configuration of the metric ("at 1M & 4M"): the 1M streams, timed over more system
# steps than the torus because its steps are short (small active sets, about a millisecond each,
# bound by the host that launches them: 300 steps keep one slow host moment from moving the
# number)
STREAMS_STEPS_PER_STEP = 30


def workload_config(args, name, n_full, world):
    config = {"workload": f"{name}, {n_full} particles, block time steps",
              "particles": n_full,
              "precision": args.precision if args.impl == "ours" else "fp64 (CPU oracle)",
              "l2_flush": "inputs larger than L2",
              "parallelism": f"replicas x{world}", "eos": args.eos,
              "shock_capturing": "switch + reconstruction" if args.shock else "constant alpha"}  # fmt: skip
    if name == "torus":
        config["disc_alpha_av"] = TORUS_ALPHA_AV
        config["scale_height"] = TORUS_SCALE_HEIGHT
    return config


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=None, choices=["torus", "streams", "cloud", "deposit"],
                    help="one workload only (default: the 4M torus, then the 1M streams in the "
                         "same run as the line's streams_1m object)")  # fmt: skip
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--shock", action="store_true",
                    help="the reference's default shock capturing: Cullen-Dehnen switch and "
                         "velocity reconstruction (else constant alpha)")  # fmt: skip
    ap.add_argument("--eos", default="ideal", choices=["ideal", "gasrad", "radiation"],
                    help="equation of state (gas + radiation and the radiation limit run without "
                         "cooling: the cloud workload)")  # fmt: skip
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain comparison form")
    args = ap.parse_args()
    both = args.workload is None
    if both:
        args.workload = "torus"
    if args.eos != "ideal" and args.workload != "cloud":
        ap.error("--eos gasrad/radiation needs a workload without cooling: --workload cloud")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.workload == "deposit":
        if world > 1 and args.impl == "ours":
            import torch

            torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        run_deposit(args, rank, world)
        if world > 1 and args.impl == "ours":
            torch.distributed.destroy_process_group()
        return
    n_full = args.n or N_FULL[args.workload]
    config = workload_config(args, args.workload, n_full, world)
    metric = "particle-steps/s"
    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_reference(args, max(1, min(args.steps, 3)), max(1, min(args.warmup, 1)))
        line = {"metric": metric, "value": cb["value"], "unit": "particle-steps/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "impl": "reference", "dtype": "f64",
                "data": "synthetic", "config": config, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "particle-steps/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}  # fmt: skip
        if both:
            import copy

            a = copy.copy(args)
            a.workload, a.n = "streams", None
            sb = cpu_reference(a, max(1, min(args.steps, 3)), max(1, min(args.warmup, 1)))
            line["streams_1m"] = {"value": sb["value"], "unit": "particle-steps/s",
                                  "config": workload_config(a, "streams", N_FULL["streams"], world),
                                  "cpu_baseline": sb}  # fmt: skip
        print(json.dumps(line))
        return
    if world > 1:
        import torch

        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    head = measure(args, args.workload, rank, world)
    streams = None
    if both:
        streams = measure(args, "streams", rank, world, steps=args.steps * STREAMS_STEPS_PER_STEP)
    if rank == 0:
        out = {"metric": metric, "value": head.pop("value"), "unit": head.pop("unit"),
               "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": head.pop("ms_per_step"), "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None,
               "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic"}  # fmt: skip
        head.pop("steps")
        out.update(head)
        if streams is not None:
            out["streams_1m"] = streams
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark: converged CW-OPO solves/s of a batched parameter sweep.

Workload (the batched CW sweep): 1024 independent 2-equation MgO:PPLN cavity
instances (532 nm pump, degenerate 1064 nm signal, 5 mm crystal) with pump
ratio N ~ U[1.2, 6], detuning delta ~ U[-pi, pi] rad, intracavity GDD ~
U[-500, 500] fs^2, reflectivity R ~ U[0.90, 0.99] and grid size drawn from
{2^12, 2^13, 2^14, 2^15}; 100 slices per pass; complex64 fields seeded with
complex Gaussian noise (sigma 1e-15, seed = instance index).  Each instance
runs until the relative change of its signal power per round trip is below
1e-7 or 5000 round trips have run; a "solve" is one instance finished under
that rule.

Steps: the K timed steps together run the whole sweep to completion; step k
continues every unfinished instance by ceil(5000 / K) round trips (one
persistent launch per grid size).  The W warm-up steps do the same on a
second sweep drawn with another seed.  value = solves / device time of the K
steps; e2e adds the host->device copy of the initial fields from pinned
memory and the device->host read of every instance's result and field.

--impl reference times the reference's own crystal-pass code and cuFFT
(oracle/_ref, compiled from the reference's sources; its parameters, grids
and pump from the reference's own set-up code in the same library, without
this package) on a bounded sample: every step runs 20 round trips of one
sweep instance per grid size, and the mean time per round trip is scaled to
the sweep by the round trips each instance needs (tests/golden).

Launch: python bench.py [--gpus N --steps K --warmup W]; N > 1 under
torch.distributed.run, one rank per GPU, each rank solving its own sweep
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

COUNT = 1024
MAX_RT = 5000
TOL = 1e-7
N_Z = 100
NOISE = 1e-15
SIZES = (4096, 8192, 16384, 32768)
LAMBDA_UM = 6.970206862971646   # QPM period: dk = 0 at 26.85 C for 532 -> 1064 nm in MgO:PPLN
REF_RTS_PER_STEP = 20
RTS_RECORD = ROOT / "tests" / "golden" / "cw_sweep_rts.json"
TRAFFIC_RECORD = ROOT / "profiles" / "ssfm_traffic.json"
CPU_RTS = 4
METRIC = "converged CW-OPO solves/s at <=1e-5 rel err vs FP64; SSFM slices/s; % HBM peak"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuopo", "reference"], default="cuopo")
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--no-validate", action="store_true", help="skip the FP64 check of converged instances")
    ap.add_argument("--record", type=str, default="", help="write per-instance round trips to this file")
    ap.add_argument("--sizes", type=str, default="", help="grid sizes to draw from (default 4096,8192,16384,32768); "
                    "reduced variants are for profiling only")
    ap.add_argument("--max-rt", type=int, default=MAX_RT, help="round-trip limit (default 5000)")
    ap.add_argument("--no-autotune", action="store_true", help="the default; accepted for recorded commands")
    ap.add_argument("--autotune", action="store_true",
                    help="time each grid size's kernel configurations first (cuopo_autotune); default: the built-in "
                         "order, measured on batches of every grid size running together")
    ap.add_argument("--warm-count", type=int, default=296,
                    help="held-out instances (2^13 points) of the learned warm-start comparison (0: skip)")
    ap.add_argument("--split", action="store_true",
                    help="N > 1: split one sweep of --count instances over the ranks (strong scaling) instead of "
                         "giving every rank its own sweep (weak scaling, the default)")
    a = ap.parse_args()
    a.sizes = tuple(int(x) for x in a.sizes.split(",")) if a.sizes else SIZES
    return a


def flops_per_instance_rt(n_t: int, gdd: float) -> float:
    """Algorithmic FP32 work of one round trip (5 N log2 N per complex FFT,
    2-eq RK4 328 and linear step 12 flops per point and slice; cavity map)."""
    per_slice = n_t * (10 * 2 * math.log2(n_t) + 328 + 12)
    cav = n_t * 8 + (n_t * (10 * math.log2(n_t) + 6) if gdd != 0 else 0)
    return N_Z * per_slice + cav


def measured_hbm_gbs() -> float:
    """HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else
    the earlier measurement on the same pool (6650 GB/s)."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _cpu_sample(job):
    """One process of the CPU baseline: CPU_RTS round trips of one sweep
    instance per grid size with the FP32 C restatement; seconds per round trip."""
    insts = job
    import cuopo_b200 as cu
    from oracle import binding as ob
    from cuopo_b200 import sweep
    per_rt = {}
    for n_t in SIZES:
        k = next(i for i, x in enumerate(insts) if x["n_t"] == n_t)
        p, _ = cu.derive_params(sweep.cw_base_inputs(n_t=n_t, n_z=N_Z))
        p.Rs, p.delta, p.gdd, p.ap0 = insts[k]["Rs"], insts[k]["delta"], insts[k]["gdd"], insts[k]["ap0"]
        T, w = cu.make_grids(n_t, p.t_rt)
        As = cu.noise_host(n_t, NOISE, insts[k]["seed"])
        Ap = np.zeros(n_t, np.complex64)
        pump = np.full(n_t, p.ap0, np.complex64)
        t0 = time.perf_counter()
        ob.round_trips(p, w, T, Ap, As, None, pump, 0, 0, CPU_RTS, bits=32)
        per_rt[n_t] = (time.perf_counter() - t0) / CPU_RTS
    return per_rt


def cpu_baseline_leg(insts, rts_by_size):
    """FP32 CPU restatement (oracle, C) on a bounded sample, on the host's
    cores (up to 128): one process per core (spawned before any GPU work) runs CPU_RTS
    round trips of one sweep instance per grid size at the same time; the
    sweep's CPU time is its round trips per grid size x the measured time
    per round trip, divided over the cores (instances are independent)."""
    import multiprocessing as mp
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    cores = max(1, min(cores, 128))
    sample = [dict(x) for x in insts[:64]]
    for n_t in SIZES:
        if not any(x["n_t"] == n_t for x in sample):
            sample.append(dict(next(x for x in insts if x["n_t"] == n_t)))
    t0 = time.perf_counter()
    if cores == 1:
        results = [_cpu_sample(sample)]
    else:
        with mp.get_context("spawn").Pool(cores) as pool:
            results = pool.map(_cpu_sample, [sample] * cores)
    wall = time.perf_counter() - t0
    per_rt = {n: float(np.mean([r[n] for r in results])) for n in SIZES}
    est = sum(rts_by_size.get(n, 0) * per_rt[n] for n in SIZES) / cores
    return {"value": (len(insts) / est) if est > 0 else None, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"{CPU_RTS} round trips of one sweep instance per grid size in each of {cores} processes at "
                      f"once (FP32 C restatement, radix-2 FFT, {wall:.1f} s wall), scaled by the sweep's round trips "
                      f"per grid size and divided over the cores",
            "s_per_rt": {str(k): round(v, 4) for k, v in per_rt.items()},
            "single_cw_opo_1core": single_cw_opo_cpu(), "cpu_model": cpu_model(), "nproc": os.cpu_count()}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def single_cw_opo_cpu(n_rt_sample: int = 3) -> dict:
    """The single CW OPO (2-eq MgO:PPLN, 2^13 points, 100 slices, N = 4,
    R = 0.98, 2000 round trips) on one host core with the C restatement, in
    FP64 and FP32: a few round trips timed, scaled to the 2000 of a run."""
    import cuopo_b200 as cu
    from cuopo_b200 import sweep
    from oracle import binding as ob
    p, _ = cu.derive_params(sweep.cw_base_inputs(n_t=8192, n_z=N_Z))
    T, w = cu.make_grids(p.n_t, p.t_rt)
    out = {}
    for bits, ct in ((64, np.complex128), (32, np.complex64)):
        As = cu.noise_host(p.n_t, 1e-20, 0).astype(ct)
        Ap = np.zeros(p.n_t, ct)
        pump = cu.pump_cw(p.n_t, p.ap0).astype(ct)
        t0 = time.perf_counter()
        ob.round_trips(p, w, T, Ap, As, None, pump, 0, 0, n_rt_sample, bits=bits)
        s_rt = (time.perf_counter() - t0) / n_rt_sample
        out[f"fp{bits}"] = {"s_per_rt": round(s_rt, 4), "s_per_run_2000_rt": round(2000 * s_rt, 1)}
    out["sample"] = (f"{n_rt_sample} round trips per precision on 1 core (radix-2 C FFT; FFTW3 is not installed); "
                     "from 1e-20 noise the FP32 run computes with subnormal numbers, which the host cores "
                     "execute far more slowly than the FP64 run's normal ones")
    return out


def load_rts_record(count):
    if not RTS_RECORD.exists():
        return None
    rec = json.loads(RTS_RECORD.read_text())
    if rec.get("count") != count or rec.get("max_rt") != MAX_RT:
        return None
    return rec


def rts_by_size_from(rec, table):
    out = {n: 0 for n in SIZES}
    for n_t, r in zip(table["n_t"], rec["rts"]):
        out[int(n_t)] += int(r)
    return out


def draw_sweep_table(count: int, rng_seed: int, sizes=SIZES) -> dict:
    """The batched CW sweep's parameter draws: the generator calls of
    cuopo_b200.sweep.random_cw_sweep, repeated here so that the reference arm
    draws the same instances without importing this package."""
    rng = np.random.default_rng(rng_seed)
    N = rng.uniform(1.2, 6.0, count)
    dl = rng.uniform(-np.pi, np.pi, count)
    gd = rng.uniform(-500.0, 500.0, count)
    R = rng.uniform(0.90, 0.99, count)
    nt = rng.choice(np.asarray(sizes), count)
    return dict(n_thr=N, delta_rad=dl, gdd_fs2=gd, refl=R, n_t=nt)


def run_reference(args):
    """The reference arm: its own kernels + cuFFT (oracle/_ref) on a bounded
    sample, set up by its own host code (ref_setup_cw2); imports nothing of
    this package, so only oracle/_ref libraries are loaded."""
    from oracle import binding as ob
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    line = {"impl": "reference", "metric": METRIC, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic"}
    missing = [n for n in SIZES if not ob.ref_available("ppln", n)]
    if missing:
        line["unavailable"] = f"reference harness not built for grid sizes {missing} (oracle/build_ref.sh)"
        print(json.dumps(line))
        return 0
    table = draw_sweep_table(args.count, 0)
    rec = load_rts_record(args.count)
    rts_by_size = rts_by_size_from(rec, table) if rec else {n: MAX_RT * int(np.sum(table["n_t"] == n)) for n in SIZES}
    sample = {}
    for n_t in SIZES:
        k = int(np.flatnonzero(table["n_t"] == n_t)[0])
        rp, w, T, pump, _, _ = ob.ref_setup_cw2(n_t, 532.0, LAMBDA_UM, float(table["n_thr"][k]),
                                                float(table["refl"][k]) * 100.0,
                                                float(table["delta_rad"][k]) / np.pi,
                                                float(table["gdd_fs2"][k]) * 1e-6, 5.0, N_Z)
        rng = np.random.default_rng(k)
        As0 = (NOISE * (rng.standard_normal(n_t) + 1j * rng.standard_normal(n_t))).astype(np.complex64)
        sample[n_t] = (rp, w, T, pump, As0)

    def one_step():
        ms = {}
        for n_t, (rp, w, T, pump, As0) in sample.items():
            Ap, As = pump.copy(), As0.copy()
            _, t = ob.ref_round_trips("ppln", rp, w, T, Ap, As, None, pump, 0, 0, REF_RTS_PER_STEP)
            ms[n_t] = t / REF_RTS_PER_STEP
        return ms

    for _ in range(args.warmup):
        one_step()
    acc = {n: [] for n in SIZES}
    t_steps = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ms = one_step()
        t_steps.append(time.perf_counter() - t0)
        for n in SIZES:
            acc[n].append(ms[n])
    ms_rt = {n: float(np.mean(acc[n])) for n in SIZES}
    per_step_value = [args.count / sum(rts_by_size[n] * acc[n][k] * 1e-3 for n in SIZES) for k in range(args.steps)]
    est_s = sum(rts_by_size[n] * ms_rt[n] * 1e-3 for n in SIZES)
    value = args.count / est_s
    converged = int(np.sum(np.asarray(rec["flags"]) == 1)) if rec else None
    line.update({
        "value": value, "ms_per_step": 1e3 * float(np.mean(t_steps)),
        "converged_solves_per_s": (converged / est_s) if converged is not None else None,
        "config": {"workload": "batched CW sweep, 1024 instances (2-eq MgO:PPLN, N~U[1.2,6], delta~U[-pi,pi], "
                               "GDD~U[-500,500] fs^2, R~U[0.90,0.99], grid 2^12..2^15, 100 slices, tol 1e-7, "
                               "max 5000 rt), reference kernels + cuFFT run one instance at a time",
                   "global_batch": args.count,
                   "sample": f"{REF_RTS_PER_STEP} round trips of one sweep instance per grid size per step",
                   "ms_per_round_trip": {str(n): round(ms_rt[n], 3) for n in SIZES},
                   "ms_per_round_trip_min_max": {str(n): [round(min(acc[n]), 3), round(max(acc[n]), 3)]
                                                 for n in SIZES},
                   "value_spread_over_steps": [min(per_step_value), max(per_step_value)],
                   "round_trips_source": ("tests/golden/cw_sweep_rts.json (round trips per instance recorded by "
                                          "this project's FP32 solver under the same rule)") if rec else
                                         "5000 per instance (no record)",
                   "setup": "reference host code (ref_setup_cw2: src/cuOPO.cu:92-234 with its Sellmeier, "
                            "linspace, fftshift, input_field_T), numpy-seeded noise"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": 1, "kind": "reference",
                         "sample": "reference crystal pass + cavity kernels with cuFFT on the GPU, driven by one host "
                                   f"thread; {REF_RTS_PER_STEP} round trips per grid size per step, scaled to the "
                                   "sweep"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line))
    return 0


def run_cuopo(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from cuopo_b200 import shard, sweep
    max_rt = args.max_rt
    split = args.split and world > 1
    if split:
        # one sweep, instances dealt to the ranks by expected cost (same split on every rank)
        base, insts, table = sweep.random_cw_sweep(args.count, 0, n_t_choices=args.sizes, n_z=N_Z)
        mine = shard.partition(shard.instance_cost(table, N_Z), world)[rank]
        insts = [insts[i] for i in mine]
        table = {k: np.asarray(v)[mine] for k, v in table.items()}
        wbase, winsts, _ = sweep.random_cw_sweep(len(insts), 10_000 + rank, n_t_choices=args.sizes, n_z=N_Z)
    else:
        base, insts, table = sweep.random_cw_sweep(args.count, rank, n_t_choices=args.sizes, n_z=N_Z)
        wbase, winsts, _ = sweep.random_cw_sweep(args.count, 10_000 + rank, n_t_choices=args.sizes, n_z=N_Z)
    rec = load_rts_record(args.count) if args.sizes == SIZES and max_rt == MAX_RT and not split else None
    cpu = None
    if rank == 0 and args.sizes == SIZES and not split:  # before any GPU work
        cpu = cpu_baseline_leg(insts, rts_by_size_from(rec, table) if rec else
                               {n: MAX_RT * int(np.sum(table["n_t"] == n)) for n in SIZES})

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    import cuopo_b200 as cu
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    peak = cu.probe_fp32_peak()
    # set-up (untimed): pick each grid size's kernel configuration by timing the candidates
    kernels = {}
    for n in sorted(set(int(x["n_t"]) for x in insts)):
        if args.autotune and not args.no_autotune:
            pb, _ = cu.derive_params(sweep.cw_base_inputs(n_t=n, n_z=N_Z))
            cu.autotune(pb, cu.F32, count=max(1, sum(1 for x in insts if x["n_t"] == n)), n_rt=2)
        m, cl = cu.kernel_config(n)
        kernels[str(n)] = f"{cl} x {m}-point CTA" + ("s" if cl > 1 else "")

    # LPT order within each grid size: longest expected solves first
    order = np.argsort(-sweep.growth_estimate(table), kind="stable")
    insts_o = [insts[i] for i in order]
    batch = cu.Batch(base, insts_o)
    warm = cu.Batch(wbase, winsts)
    total = batch.total
    h_init = torch.empty(total, dtype=torch.complex64).pin_memory()
    off = 0
    for x in insts_o:
        h_init[off:off + x["n_t"]] = torch.from_numpy(cu.noise_host(x["n_t"], NOISE, x["seed"]))
        off += x["n_t"]
    w_init = torch.empty(warm.total, dtype=torch.complex64).pin_memory()
    off = 0
    for x in winsts:
        w_init[off:off + x["n_t"]] = torch.from_numpy(cu.noise_host(x["n_t"], NOISE, x["seed"]))
        off += x["n_t"]
    h_out = torch.empty(total, dtype=torch.complex64).pin_memory()

    K = max(1, args.steps)
    chunk = int(math.ceil(max_rt / K))
    # warm-up: the same kind of step on the warm-up sweep
    warm.set_signal(w_init)
    warm.reset()
    for _ in range(max(0, args.warmup)):
        warm.step(chunk, max_rt, TOL, 1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = ClockSampler(int(vis[local]) if local < len(vis) and vis[local].strip().isdigit() else local)
    clocks.start()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    e_start, e_h2d, e_steps, e_end = ev(), ev(), ev(), ev()
    torch.cuda.synchronize()
    e_start.record(stream)
    batch.set_signal(h_init)           # host -> device, pinned
    batch.reset()
    e_h2d.record(stream)
    # the K steps: each grid size runs on its own stream and starts its next
    # step as soon as its own part of the previous one is done
    for k in range(K):
        batch.step(chunk, max_rt, TOL, 1)
    batch.wait(stream)                 # every grid size's last step done
    e_steps.record(stream)
    ps, rts, flags = batch.results()   # device -> host (synchronises the stream)
    batch.get_signal(h_out)
    e_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()

    dev_ms = e_h2d.elapsed_time(e_steps)
    e2e_ms = e_start.elapsed_time(e_end)
    done = int(np.sum(flags != 0))
    conv = int(np.sum(flags == 1))
    (dev_ms, e2e_ms), (done_all, conv_all) = shard.reduce_over_ranks([dev_ms, e2e_ms], [done, conv], device=dev)

    # work accounting (algorithmic, this rank; all ranks solve equal-size sweeps)
    nt_o = np.array([x["n_t"] for x in insts_o])
    gdd_o = np.array([x["gdd"] for x in insts_o])
    flops = float(sum(r * flops_per_instance_rt(int(m), g) for r, m, g in zip(rts, nt_o, gdd_o)))
    slices = float(np.sum(rts)) * N_Z
    pt_slices = float(np.sum(rts * nt_o)) * N_Z
    # HBM bytes (algorithmic): each step loads and stores both fields of every running instance
    hbm_bytes = 2 * 2 * 8 * float(np.sum(nt_o)) * K
    achieved = flops / (dev_ms * 1e-3) / 1e12

    if args.record and rank == 0:
        inv = np.empty_like(order)
        inv[order] = np.arange(len(order))
        Path(args.record).write_text(json.dumps({"count": args.count, "max_rt": MAX_RT, "tol": TOL,
                                                 "rts": rts[inv].tolist(), "flags": flags[inv].tolist(),
                                                 "ps": ps[inv].tolist()}))

    # per-grid-size kernel timing (untimed for `value`): each grid size's instances of the sweep alone
    per_size = time_per_size(cu, base, insts_o, peak, stream) if rank == 0 else None
    fp64 = None
    if rank == 0 and per_size:
        # the FP64 solver on the same per-size batches, and the sweep rate it implies (same round trips)
        peak64 = cu.probe_fp64_peak()
        per64 = time_per_size(cu, base, insts_o, peak64, stream, precision=cu.F64)
        t64 = 0.0
        for n in per64:
            rts_n = float(np.sum(rts[nt_o == int(n)]))
            t64 += rts_n * per64[n]["ms"] * 1e-3 / (per64[n]["round_trips"] * per64[n]["instances"])
        fp64 = {"per_size": {n: {k: v for k, v in d.items() if k in ("kernel", "ms", "tflops", "frac")}
                             for n, d in per64.items()},
                "fp64_peak_tflops": peak64,
                "peak_source": "measured live: fma.rn.f64-chain probe over every SM (cuopo_probe_fp64_peak)",
                "sweep_solves_per_s_estimate": len(insts_o) / t64 if t64 > 0 else None,
                "note": "FP64 fields and arithmetic (the FP64 plan kernels, FP64 rate counted against the same "
                        "algorithmic work); the sweep estimate scales each grid size's per-instance round-trip "
                        "time by the FP32 sweep's round trips (one grid size at a time, no overlap of sizes)"}

    validation = None
    if not args.no_validate and rank == 0:
        validation = validate_fp64(cu, base, insts_o, h_init, ps, rts, flags)
    warm_leg = warm_start_leg(args) if rank == 0 and args.warm_count > 0 else None

    traffic = None
    if TRAFFIC_RECORD.exists():
        # DRAM bytes per instance-point and launch from one ncu capture; a step is one launch per grid size
        rate = json.loads(TRAFFIC_RECORD.read_text()).get("dram_bytes_per_instance_point")
        traffic = rate * float(np.sum(nt_o)) if rate else None
    dom = None
    if per_size:
        # the dominant kernel: the grid size with the largest share of the sweep's algorithmic work
        work = {n: float(sum(r * flops_per_instance_rt(int(m), g) for r, m, g in zip(rts, nt_o, gdd_o) if m == n))
                for n in set(nt_o.tolist())}
        n_dom = max(work, key=work.get)
        dom = dict(per_size[str(n_dom)], n_t=n_dom, share_of_sweep_flops=work[n_dom] / flops)
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": done_all / (dev_ms * 1e-3),
            "converged_solves_per_s": conv_all / (dev_ms * 1e-3),
            "unit": "solves/s",
            "n_gpus": world,
            "steps": K,
            "warmup": args.warmup,
            "ms_per_step": dev_ms / K,
            "higher_is_better": True,
            "scaling": "strong" if split else "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded parameter draws and seeded noise)",
            "config": {"workload": "batched CW sweep: 1024 instances of 2-eq MgO:PPLN (532->1064 nm, 5 mm), "
                                   "N~U[1.2,6], delta~U[-pi,pi] rad, GDD~U[-500,500] fs^2, R~U[0.90,0.99], "
                                   "grid 2^12..2^15, 100 slices/pass, tol 1e-7, max 5000 rt, noise 1e-15",
                       "global_batch": args.count if split else args.count * world, "per_rank_batch": len(insts),
                       "grid_sizes": list(args.sizes), "max_rt": max_rt,
                       "round_trips_per_step": chunk, "kernels": kernels,
                       "kernel_choice": "autotuned (cuopo_autotune)" if args.autotune and not args.no_autotune else "built-in order",
                       "parallelism": (f"one sweep split over {world} ranks by expected cost" if split else
                                       f"own sweep per rank, {world} rank(s)") + ", no collective on the data path",
                       "l2": "working set (fields of 1024 instances, 252 MB) larger than L2",
                       "solves_converged": conv_all, "solves_total": done_all,
                       "converged_decayed": int(np.sum((flags == 1) & (ps <= 1e-20))) if world == 1 else None},
            "slices_per_s": slices * world / (dev_ms * 1e-3),
            "point_slices_per_s": pt_slices * world / (dev_ms * 1e-3),
            "hbm_frac": (hbm_bytes / (dev_ms * 1e-3)) / (measured_hbm_gbs() * 1e9),
            "roofline": ({"bound": "fp32", "achieved": dom["tflops"], "peak": peak, "unit": "TFLOP/s",
                          "frac": dom["frac"], "traffic": dom["traffic_bytes"],
                          "traffic_per": "launch (ncu-measured DRAM bytes per instance-point x instance-points)",
                          "peak_source": "measured live: best of scalar and packed f32x2 FMA-chain probes "
                                         "(cuopo_probe_fp32_peak); fields stay in shared memory, so neither HBM nor "
                                         "tensor cores bound it",
                          "kernel": f"ssfm_kernel, grid 2^{int(math.log2(dom['n_t']))} ({dom['kernel']}), "
                                    f"{dom['share_of_sweep_flops']:.0%} of the sweep's algorithmic work; "
                                    "CUDA events around its launch on the launching stream"} if dom else None),
            "sweep_roofline": {"achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                               "frac": achieved / peak if peak else None, "traffic": traffic,
                               "traffic_per": "step (one launch per grid size; ncu-measured bytes per instance-point)",
                               "kernel": "ssfm_kernel (fused round trips, all grid sizes at once)"},
            "per_size": per_size,
            "fp64_solver": fp64,
            "cpu_baseline": cpu,
            "e2e": {"value": done_all / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(total * 8 / K), "d2h_bytes_per_step": int((total * 8 + len(insts) * 16) / K)},
            "gpu_launches": K * len(set(nt_o.tolist())),
            "clocks": clk,
            "validation_fp64": validation,
            "warm_start": warm_leg,
        }
        print(json.dumps(line))
    batch.close()
    warm.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def time_per_size(cu, base, insts_o, peak, stream, n_rt: int = 20, precision=None) -> dict:
    """Each grid size's kernel alone: a batch of that size's sweep instances
    runs n_rt round trips from noise (one launch) between CUDA events on the
    launching stream; algorithmic TFLOP/s and fraction of `peak` (the FP32
    probe; with precision F64 the FP64 solver's kernels, same work counted,
    against the FP64 probe)."""
    import torch
    prec = cu.F32 if precision is None else precision
    rate = None
    if TRAFFIC_RECORD.exists() and prec == cu.F32:
        rate = json.loads(TRAFFIC_RECORD.read_text()).get("dram_bytes_per_instance_point")
    out = {}
    for n in sorted(set(int(x["n_t"]) for x in insts_o)):
        sub = [x for x in insts_o if x["n_t"] == n]
        m, cl = cu.kernel_config(n, precision=prec)
        with cu.Batch(base, sub, precision=prec) as b:
            if prec == cu.F32:
                b.seed_noise(NOISE)
            else:
                b.set_signal(np.concatenate([cu.noise_host(n, NOISE, x["seed"]) for x in sub]).astype(np.complex128))
            b.reset()
            b.step(n_rt, n_rt, 0.0, 1)     # warm-up launch
            b.reset()
            b.wait(stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            b.step(n_rt, n_rt, 0.0, 1)
            b.wait(stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            _, r, _ = b.results()
        fl = float(sum(int(rr) * flops_per_instance_rt(n, x["gdd"]) for rr, x in zip(r, sub)))
        tf = fl / (ms * 1e-3) / 1e12
        out[str(n)] = {"kernel": f"{cl} x {m}-point CTA" + ("s" if cl > 1 else ""), "instances": len(sub),
                       "round_trips": n_rt, "ms": round(ms, 3), "tflops": tf, "frac": tf / peak if peak else None,
                       "point_slices_per_s": float(np.sum(r)) * n * N_Z / (ms * 1e-3),
                       "traffic_bytes": rate * n * len(sub) if rate else None}
    return out


def measured_bf16_tflops() -> float | None:
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"])
    except (OSError, ValueError, KeyError):
        return None


def warm_start_leg(args, seed: int = 7) -> dict:
    """The learned warm start (cuopo_b200/data/warmstart_mlp.npz): held-out
    instances of the sweep's distribution at 2^13 points solved from noise
    and from the network's prediction by the same batched solver and rule
    (warmstart.evaluate); plus the network's tensor-core kernels timed alone:
    one training step (forward, backward, Adam; CUDA graph) at batch 4096 and
    inference, against the measured BF16 peak."""
    import torch
    from cuopo_b200 import warmstart as ws
    if not ws.MODEL_PATH.exists():
        return {"unavailable": f"no trained model at {ws.MODEL_PATH.relative_to(ROOT)}"}
    model = ws.WarmStartModel.load()
    out = ws.evaluate(model, args.warm_count, seed, n_t=8192, max_rt=args.max_rt, tol=TOL)
    out["model"] = model.meta
    # the network's kernels alone
    mlp = ws.MLP(max_batch=4096, seed=1)
    x = torch.rand(4096, ws.N_FEATURES, device="cuda") * 2 - 1
    t = torch.randn(4096, 2 * ws.N_MODES, device="cuda")
    for _ in range(5):
        mlp.train_step(x, t, 1e-4)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    n = 50
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(n):
        mlp.train_step(x, t, 1e-4)
    ev[1].record()
    for _ in range(n):
        mlp.forward(x)
    ev[2].record()
    torch.cuda.synchronize()
    mlp.status()
    mlp.close()
    train_ms = ev[0].elapsed_time(ev[1]) / n
    fwd_ms = ev[1].elapsed_time(ev[2]) / n
    w, d, k0 = ws.WIDTH, ws.DEPTH, 64
    fwd_flops = 2.0 * 4096 * (k0 * w + (d - 1) * w * w + w * 2 * ws.N_MODES)
    train_flops = 3.0 * fwd_flops - 2.0 * 4096 * k0 * w      # forward, dW of every layer, dX of all but the first
    peak = measured_bf16_tflops()
    out["tensor_cores"] = {
        "train_step_us": 1e3 * train_ms, "train_tflops": train_flops / (train_ms * 1e-3) / 1e12,
        "forward_us": 1e3 * fwd_ms, "forward_tflops": fwd_flops / (fwd_ms * 1e-3) / 1e12,
        "bf16_peak_tflops": peak, "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS burst)",
        "train_frac": (train_flops / (train_ms * 1e-3) / 1e12) / peak if peak else None,
        "note": "batch 4096, 4 -> 512 x 4 (GELU) -> 512; layer 0 padded to K = 64; the training step is one "
                "CUDA graph (14 tcgen05 GEMM launches, loss and Adam) after an input-packing kernel"}
    model.close()
    return out


def validate_fp64(cu, base, insts_o, h_init, ps, rts, flags, per_class: int = 1):
    """FP64 check of the output signal power, stratified: for every grid size,
    `per_class` converged (non-trivial power) and `per_class` round-trip-limit
    instances are re-run with an FP64 plan from the same initial noise for the
    same number of round trips (all at once, one stream each); reports the
    relative error of the FP32 final signal power per grid size and class."""
    import torch
    idx = []
    for n in sorted(set(x["n_t"] for x in insts_o)):
        for flag in (1, 2):
            cand = [k for k, x in enumerate(insts_o) if x["n_t"] == n and flags[k] == flag and ps[k] > 1e-20]
            cand.sort(key=lambda k: rts[k])
            if cand:
                # the median-round-trip member of the class (deterministic)
                idx += [cand[len(cand) // 2]] if per_class == 1 else cand[:: max(1, len(cand) // per_class)][:per_class]
    if not idx:
        return {"checked": 0}
    offs = np.concatenate([[0], np.cumsum([x["n_t"] for x in insts_o])])
    t0 = time.perf_counter()
    runs = []
    for k in idx:
        x = insts_o[k]
        p = cu.Params(**base.to_dict())
        p.n_t, p.Rs, p.delta, p.gdd, p.ap0 = x["n_t"], x["Rs"], x["delta"], x["gdd"], x["ap0"]
        plan = cu.Plan(p, precision=cu.F64)
        As = h_init[offs[k]:offs[k + 1]].to("cuda", torch.complex128)
        Ap = torch.zeros_like(As)
        hist = torch.zeros(int(rts[k]), dtype=torch.float64, device="cuda")
        # the inputs were made on the current stream: the instance's own stream waits for them
        st = torch.cuda.Stream()
        st.wait_stream(torch.cuda.current_stream())
        plan.round_trips(Ap, As, None, None, 0, 0, int(rts[k]), ps_hist=hist, stream=st)
        # the fields stay referenced until the streams are done: torch's allocator
        # does not see the library's use of them on `st`
        runs.append((plan, hist, As, Ap))
    torch.cuda.synchronize()
    ps64 = np.array([r[1][-1].item() for r in runs])
    for r in runs:
        r[0].close()
    err = np.abs(ps[idx] - ps64) / np.abs(ps64)
    cases = [{"n_t": int(insts_o[k]["n_t"]), "class": "converged" if flags[k] == 1 else "rt_limit",
              "rts": int(rts[k]), "rel_err_ps": float(e)} for k, e in zip(idx, err)]
    return {"checked": len(idx), "rule": "FP64 plan, same initial noise, same round trips; per grid size the "
                                         "median-round-trip converged and round-trip-limit instance",
            "max_rel_err_ps": float(np.max(err)), "median_rel_err_ps": float(np.median(err)),
            "frac_within_1e-5": float(np.mean(err <= 1e-5)), "cases": cases,
            "seconds": round(time.perf_counter() - t0, 1)}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_cuopo(args)


if __name__ == "__main__":
    sys.exit(main())

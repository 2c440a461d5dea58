"""FIM report-step throughput on one B200 (cell-steps/s), plus the reference CPU arm.

One bench step is one report step of the fully implicit controller (Newton iterations with
assembly, well Schur elimination, CPR-FGMRES and the update, including any substeps and retries)
on a seeded synthetic waterflood deck, run through the C ABI (`rf_step`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ensemble|72k|72k-bo|adjoint|2m|1d] [--variants V] [--precision fp64|mixed]
                    [--dt DAYS] [--no-cpu-baseline]

The default workload is the sensitivity ensemble: 256 two-phase waterflood variants of uneven
size (3,300 to 64,512 cells, 4.9M cells in all) per GPU, all advanced together one report step at
a time (rf_batch_step).  `--workload 72k-bo` is the single 60x60x20 three-phase black-oil deck of
the plain FP64 form; `--workload 72k` is the same grid and wells with two-phase oil-water physics.

Legs of the `--impl ours` run:
  value     device time of K report steps with the state resident in HBM, L2 flushed (256 MB
            write) between steps.  Single deck: CUDA events recorded by the library on its own
            stream around each `rf_step`.  Ensemble: CUDA events on the caller's stream around each
            `rf_batch_step`, which returns when every variant's stream has finished;
  e2e       the same metric through the public API with host buffers: every step uploads each
            state from pinned host memory (`rf_set_state`), steps, and reads it back
            (`rf_get_state`), timed from before the uploads to after the read-backs, on the same K
            report steps as `value` (a second simulator or ensemble after the same warm-up);
  roofline  the pressure BiCGStab kernel (the dominant kernel): algorithmic bytes of one launch /
            that launch's duration (CUDA events on the launching stream, averaged over the
            launches), against the measured HBM copy bandwidth;
  cpu_baseline  the CPU restatement (C++, single thread, like the reference, built with
            -march=native on this host) on the same deck (ensemble: variant 0) and the same report
            steps after the same warm-up, in a spawned process beside the GPU legs;
  matched_comparison  (ensemble) the batched mixed form over all variants against the plain FP64
            path one variant at a time, both with Newton accepted at CNV 1e-8 / MB 1e-10 and every
            CPR-FGMRES solve refined to 1e-10 relative, and the field error between them.

The reference arm (`--impl reference`) times the CPU restatement on the host cores: the single
deck on one core (the reference is single-threaded), the ensemble as one single-threaded process
per core, each on a variant of a sample spread over the size range, their throughputs summed.

Multi-GPU (torchrun): a single deck does not shard, so each rank runs a replica; the ensemble
shards by variant, every rank stepping its own `--variants` variants.  Both are weak scaling with
no collective on the data path; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
# many contexts' streams at once: give them their own hardware queues (read at CUDA start-up)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

HBM_FALLBACK_GBS = 6650.0

WORKLOADS = {
    # name: (nx, ny, nz, dt_days, description)
    "72k": (60, 60, 20, 10.0,
            "waterflood_3d 60x60x20 (72,000 cells), two-phase oil-water, log-normal kh (ln-mean ln 100 mD, "
            "sigma 1, 5-cell correlation), kv/kh 0.1, inverted five-spot (4 rate injectors, 1 BHP producer), "
            "no gravity, dt 10 d report steps, FP64"),
    "72k-bo": (60, 60, 20, 10.0,
               "black_oil_3d 60x60x20 (72,000 cells), three-phase black-oil (PVT table with bubble point 200 bar, "
               "Stone II, regime switching, gas flash), log-normal kh (ln-mean ln 100 mD, sigma 1, 5-cell correlation), "
               "kv/kh 0.1, phi from ln k, gravity on, p_init 250 bar, inverted five-spot (4 water rate injectors, "
               "1 BHP producer at 150 bar), dt 10 d report steps, FP64"),
    "adjoint": (60, 60, 20, 2.0,
                "discrete adjoint on black_oil_3d 60x60x20 (72,000 cells, the three-phase deck of --workload 72k-bo): "
                "forward report steps recorded with per-report-step checkpoints, then the backward pass (substeps "
                "replayed from the checkpoints, transposed well-Schur / CPR-FGMRES solves in reverse time); objective "
                "cumulative surface oil, gradient in 72,000 per-cell ln k and 5 well controls; one substep per report "
                "step, Newton to CNV 1e-9 / MB 1e-11, dt 2 d, FP64"),
    "2m": (200, 200, 50, 10.0,
           "waterflood_3d 200x200x50 (2,000,000 cells), same statistics and wells, dt 10 d report steps, FP64"),
    "1d": (200, 1, 1, 10.0, "waterflood_1d 200x1x1, rate injector cell 0, BHP producer cell 199, dt 10 d, FP64"),
    "ensemble": (0, 0, 0, 10.0,
                 "sensitivity ensemble: {nv} two-phase waterflood variants per GPU (decks.ensemble_variant: nx, ny "
                 "in 20..64, nz in 5..16, sigma ln k 0.5..1.5, mobility ratio 0.5..10, Corey exponents 1.5..4, kv/kh "
                 "0.01..1, quarter five-spot), one context per variant stepped concurrently (rf_batch_step), "
                 "dt 10 d report steps"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="ensemble")
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="linear-solver precision of the device path (mixed: FP32 ILU and pressure stage)")
    ap.add_argument("--variants", type=int, default=256, help="ensemble variants per GPU (--workload ensemble)")
    ap.add_argument("--cluster-table", default=None,
                    help="ensemble: JSON table of tuned cluster sizes (ressim_b200.autotune) applied per variant")
    ap.add_argument("--tune-variants", type=int, default=0,
                    help="ensemble: first tune this many variants spread over the size range into --cluster-table")
    ap.add_argument("--host-threads", type=int, default=0,
                    help="ensemble: host threads, one per group of variants (0: the library's default)")
    ap.add_argument("--batch-mode", choices=["groups", "threads"], default="groups",
                    help="ensemble: fiber groups with batched level-scheduled launches, or a thread per variant")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-matched", action="store_true",
                    help="ensemble: skip the matched-profile comparison (batched mixed vs plain FP64)")
    ap.add_argument("--cpu-sample-s", type=float, default=20.0, help="wall budget of the CPU baseline sample")
    return ap.parse_args()


def make_deck(workload):
    from ressim_b200 import decks

    nx, ny, nz, dt, desc = WORKLOADS[workload]
    if workload == "ensemble":  # the CPU legs time variant 0 of the ensemble
        return decks.ensemble_variant(0), dt, desc
    if workload == "1d":
        deck, _, _ = decks.waterflood_1d()
    elif workload in ("72k-bo", "adjoint"):
        deck = decks.black_oil_3d(nx, ny, nz, seed=7)
    else:
        deck = decks.waterflood_3d(nx, ny, nz, seed=7)
    return deck, dt, desc


def dist_setup(args):
    """Rank/world from torchrun's environment; each rank sees only its own GPU."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        visible = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        os.environ["CUDA_VISIBLE_DEVICES"] = visible[local] if local < len(visible) else str(local)
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm, smax, power = [], [], []
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "power_w_max": max(power) if power else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of `value` over all ranks of the default process group (identity when `dist`
    is None); every rank takes the same collective step."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def partition_by_cells(sizes, world):
    """Greedy longest-first assignment of independent variants (cell counts `sizes`) to `world`
    ranks; returns one index list per rank.  Deterministic for given inputs."""
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += sizes[i]
    return parts


def measured_hbm_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


def bicgstab_bytes_per_iteration(n_cells, nnzb):
    """Algorithmic bytes of one BiCGStab iteration of the pressure stage (FP64 values, int32 indices):
    two ILU0 applications (forward + backward: L/U values and columns once, 12 B per entry; per row
    rhs, y written and read, out, inverse pivot, level row ids and row pointers = 64 B), two SpMVs
    (12 B per entry; row pointer, x, y = 20 B per row) and the vector updates and dot products
    (160 B per row)."""
    return 2 * (12 * nnzb + 64 * n_cells) + 2 * (12 * nnzb + 20 * n_cells) + 160 * n_cells


def use_native_oracle():
    """Builds the CPU oracle for this host (-O3 -march=native) and points the CPU legs, which run in
    spawned processes started after this call, at that build.  Returns the compiler flags used."""
    from oracle import oracle_py

    so = oracle_py.build_native()
    if so:
        os.environ["RESSIM_ORACLE_SO"] = so
        return "g++ -O3 -march=native -ffp-contract=off"
    return "g++ -O3 -ffp-contract=off (the -march=native build failed on this host)"


def spread_sample(sizes, k):
    """k indices spread over the size order of `sizes` (smallest to largest, evenly), so a sample of
    the ensemble has its size distribution."""
    order = sorted(range(len(sizes)), key=lambda i: (sizes[i], i))
    k = max(1, min(k, len(sizes)))
    if k == 1:
        return [order[len(order) // 2]]
    return sorted({order[round(j * (len(order) - 1) / (k - 1))] for j in range(k)})


def cpu_leg(workload, dt, warmup, steps, budget_s):
    """The CPU restatement of the reference FIM (C++, one thread, like the reference) on the same
    deck and the same report steps as the GPU legs: `warmup` untimed report steps from the initial
    state, then up to `steps` timed ones (stopping once `budget_s` of wall time is spent, after at
    least one).  Returns (cell-steps/s, timed steps, seconds, Newton iterations, [(p, sw) after
    each timed step])."""
    sys.path.insert(0, HERE)
    from oracle.oracle_py import OracleSimulator

    deck, dt_default, _ = make_deck(workload)
    dt = dt if dt is not None else dt_default
    sim = OracleSimulator(deck)
    for _ in range(warmup):
        sim.step(dt)
    n = deck.n_cells
    k = 0
    newton = 0
    el = 0.0
    states = []
    while k < steps:
        t0 = time.perf_counter()
        _, rep = sim.step(dt)
        el += time.perf_counter() - t0
        newton += rep.newton_iterations
        st = sim.state()
        states.append((st["pressure"], st["sat_water"], st["sat_gas"]))
        k += 1
        if el >= budget_s:
            break
    sim.close()
    return n * k / el, k, el, newton, states


def _ref_variant_worker(index, dt, warmup, steps):
    """One reference-arm worker: variant `index` stepped `warmup` untimed and `steps` timed report
    steps by the CPU restatement, single-threaded.  Returns (cells, seconds, Newton iterations)."""
    sys.path.insert(0, HERE)
    from oracle.oracle_py import OracleSimulator
    from ressim_b200 import decks

    d = decks.ensemble_variant(index)
    sim = OracleSimulator(d)
    for _ in range(warmup):
        sim.step(dt)
    t0 = time.perf_counter()
    newton = 0
    for _ in range(steps):
        _, rep = sim.step(dt)
        newton += rep.newton_iterations
    el = time.perf_counter() - t0
    sim.close()
    return d.n_cells, el, newton


def run_reference_ensemble(args):
    """Reference arm of the ensemble: the reference steps one deck per simulator, single-threaded,
    so a multi-core host runs one variant per core.  One process per host core (spawned) steps one
    variant of a sample spread over the ensemble's size range (a bounded sample: W untimed and K
    timed report steps each).  Each core's throughput is its variant's cells x K / its own timed
    seconds; the host's throughput is their sum (every core kept busy with variants like its
    sample)."""
    import multiprocessing as mp

    from ressim_b200 import decks

    flags = use_native_oracle()
    cores = max(1, min(os.cpu_count() or 1, args.variants))
    dt = args.dt if args.dt is not None else WORKLOADS["ensemble"][3]
    k = max(1, args.steps)
    sizes = [decks.ensemble_variant(i).n_cells for i in range(args.variants)]
    sample = spread_sample(sizes, cores)
    with mp.get_context("spawn").Pool(len(sample)) as pool:
        res = pool.starmap(_ref_variant_worker, [(i, dt, args.warmup, k) for i in sample])
    cells = sum(r[0] for r in res)
    newton = sum(r[2] for r in res)
    v = sum(r[0] * k / r[1] for r in res)
    desc = WORKLOADS["ensemble"][4].format(nv=args.variants)
    line = {
        "metric": "FIM cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * cells / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded deck generator)",
        "config": {"workload": desc, "sample_variants": sample, "sample_cells": cells, "dt_days": dt,
                   "newton_iterations": newton},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": len(sample), "kind": "port",
                         "sample": f"{len(sample)} variants spread over the size range ({cells} cells), one "
                                   f"single-threaded process per core, report steps {args.warmup}.."
                                   f"{args.warmup + k - 1} after {args.warmup} untimed ones; throughput summed "
                                   f"over the cores; C++ restatement of the reference FIM, {flags}"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """Reference arm: the reference's FIM path on the host cores.  The reference (Rust/WASM) cannot
    be built in this image (no cargo, rustc or node), so its C++ restatement (oracle) is timed, one
    thread, as the reference's FIM runs, on the same deck and the same report steps as the GPU arm
    (W untimed warm-up steps from the initial state, then K timed steps).  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "ensemble":
        return run_reference_ensemble(args)
    if args.workload == "adjoint":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint (no backward pass to time)"}),
              flush=True)
        return 0
    _, dt_default, desc = make_deck(args.workload)
    dt = args.dt if args.dt is not None else dt_default
    flags = use_native_oracle()
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(1) as pool:
        v, k, el, newton, _ = pool.apply(cpu_leg, (args.workload, dt, args.warmup, args.steps, float("inf")))
    n = make_deck(args.workload)[0].n_cells
    if args.workload == "ensemble":
        desc = desc.format(nv=args.variants) + "; the reference steps one deck per simulator, so its arm times " \
               "variant 0 (" + str(n) + " cells)"
    line = {
        "metric": "FIM cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * el / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded deck generator)",
        "config": {"workload": desc, "cells": n, "dt_days": dt, "newton_iterations": newton},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                         "sample": f"report steps {args.warmup}..{args.warmup + k - 1} of the deck "
                                   f"({newton} Newton iterations), C++ restatement of the reference FIM, 1 thread, "
                                   f"{flags}"},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


MATCHED_CNV, MATCHED_MB = 1e-8, 1e-10
MATCHED_LIN_RTOL, MATCHED_LIN_PASSES = 1e-10, 12


# DRAM bytes (read + write) per algorithmic byte of one batched level-order pressure launch, from
# an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, one pass, caches flushed before the
# launch) of the first k_bicgstab_level_batch launch of `bench.py --variants 2 --host-threads 1
# --steps 1 --warmup 0`: variants 0 and 1 (18,705 and 39,480 cells), 50 iterations each, 11.03 MB
# of DRAM traffic against 1,901 MB of algorithmic bytes.  The solves' working set is read from
# DRAM about once and every later pass hits L2.
LEVEL_BATCH_DRAM_PER_ALG_BYTE = 11.03e6 / 1901.47e6
# DRAM bytes per launch of the one-cluster pressure BiCGStab on the 60x60x20 black-oil deck
# (k_bicgstab_dsmem, ncu dram__bytes_read.sum + dram__bytes_write.sum, caches flushed).
CLUSTER_DRAM_PER_LAUNCH = {"72k-bo": 15.71e6}


def ensemble_roofline(ds, profs, peak, peak_kind, batch=None):
    """Roofline of the dominant kernel (the pressure BiCGStab): algorithmic bytes of one launch / its
    duration (CUDA events on the launching stream), averaged over the launches (bytes and time
    pooled, then divided by the launches).  With batched stepping one launch carries a whole
    group's solves and `batch` holds those launches' count and time; otherwise every variant's own
    launches are timed by its profile."""
    from ressim_b200 import _lib

    it = sum(p["bicgstab_iterations"] for p in profs)
    byts = sum(bicgstab_bytes_per_iteration(d.n_cells, p["nnzb"]) * p["bicgstab_iterations"] for d, p in zip(ds, profs))
    if batch is not None and batch.get("pressure_launches", 0) > 0 and batch.get("pressure_ms", 0) > 0:
        nl, kms = batch["pressure_launches"], batch["pressure_ms"]
        kernel = "k_bicgstab_level_batch (one launch = a group's pressure solves, one thread block each)"
        solves = batch["pressure_items"]
    else:
        nl = sum(p["bicgstab_launches"] for p in profs)
        kms = sum(p["bicgstab_kernel"] for p in profs)
        kernel = "k_bicgstab_level (one launch = one variant's pressure solve, one thread block)"
        solves = nl
    if nl <= 0 or kms <= 0:
        return None
    phase_ms = sum(sum(p[k] for k in _lib.PHASES if k != "bicgstab_kernel") for p in profs)
    achieved = (byts / nl) / (kms / nl / 1e3) / 1e9
    traffic = LEVEL_BATCH_DRAM_PER_ALG_BYTE * byts / nl
    return {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_basis": "ncu DRAM bytes per algorithmic byte of one batched launch (caches flushed), "
                             "scaled to this run's bytes per launch", "bytes_per_launch": byts / nl,
            "ms_per_launch": kms / nl, "launches": nl, "solves": solves, "iterations_per_solve": it / max(solves, 1),
            "share_of_phase_time": sum(p["bicgstab_kernel"] for p in profs) / max(phase_ms, 1e-9)}


def matched_comparison(ds, dt, sample):
    """Batched mixed against plain FP64 on the ensemble at the matched profile (Newton accepted at
    CNV 1e-8 / MB 1e-10 and every CPR-FGMRES solve refined to 1e-10 relative on both paths, the
    reference's controller otherwise): the batched mixed form over all variants against the plain
    FP64 path stepping variants one at a time through rf_step.  One
    untimed and one timed report step each; the plain path runs on `sample` (variants spread over
    the size range), the batched path on all of them; field error of the batched mixed states
    against the plain FP64 ones on the sample."""
    import numpy as np
    import torch

    from ressim_b200 import Ensemble, ReservoirSimulator

    seq_cells = seq_ms = 0.0
    fp64_states = {}
    for i in sample:
        sim = ReservoirSimulator.from_deck(ds[i])
        sim.set_controller_options(False, MATCHED_CNV, MATCHED_MB)
        sim.set_linear_refinement(MATCHED_LIN_RTOL, MATCHED_LIN_PASSES)
        sim.step(dt)
        r = sim.step(dt)
        seq_ms += r["device_ms"]
        seq_cells += ds[i].n_cells
        fp64_states[i] = sim.state()
        sim.close()
    ens = Ensemble(ds, precision="mixed")
    ens.set_controller_options(False, MATCHED_CNV, MATCHED_MB)
    ens.set_linear_refinement(MATCHED_LIN_RTOL, MATCHED_LIN_PASSES)
    ens.step(dt)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    reps = ens.step(dt)
    ev1.record()
    ev1.synchronize()
    batch_ms = ev0.elapsed_time(ev1)
    ep = es = 0.0
    for i in sample:
        st = ens.state(i)
        ep = max(ep, float(np.max(np.abs(st["pressure"] - fp64_states[i]["pressure"]) /
                                  np.maximum(np.abs(fp64_states[i]["pressure"]), 1.0))))
        es = max(es, float(np.max(np.abs(st["sat_water"] - fp64_states[i]["sat_water"]))))
    ens.close()
    cells = sum(d.n_cells for d in ds)
    v_batch = cells / (batch_ms / 1e3)
    v_seq = seq_cells / (seq_ms / 1e3)
    return {"profile": "matched: reference controller, Newton accepted at CNV 1e-8 / MB 1e-10, every CPR-FGMRES "
                       "solve refined to 1e-10 relative, on both paths",
            "batched_mixed": v_batch, "plain_fp64_one_at_a_time": v_seq, "ratio": v_batch / v_seq,
            "plain_sample_variants": list(sample), "report_step": "the second report step (one untimed before it)",
            "newton_iterations_batched": sum(r["newton_iterations"] for r in reps),
            "field_error_mixed_vs_fp64": {"pressure_rel": ep, "sat_water_abs": es, "variants": list(sample)}}


def run_ensemble(args, rank, world):
    """`--workload ensemble`: every rank steps its own `--variants` variants (weak scaling, no
    collective on the data path); value = all ranks' cells x K / the slowest rank's device time."""
    cpu_job = None
    flags = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import multiprocessing as mp

        flags = use_native_oracle()
        pool = mp.get_context("spawn").Pool(1)
        cpu_job = (pool, pool.apply_async(cpu_leg, ("ensemble", args.dt, args.warmup, 1, args.cpu_sample_s)))
    import ctypes as C

    import torch

    import numpy as np

    from ressim_b200 import Ensemble, _lib, decks

    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}))
        return 1
    torch.cuda.set_device(0)
    dev_index = (os.environ.get("CUDA_VISIBLE_DEVICES", "") or "0").split(",")[0].strip() or "0"
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", 0))
        pg = dist
    dt_default, desc = WORKLOADS["ensemble"][3], WORKLOADS["ensemble"][4]
    dt = args.dt if args.dt is not None else dt_default
    nv = args.variants
    ds = [decks.ensemble_variant(rank * nv + i) for i in range(nv)]
    cells = sum(d.n_cells for d in ds)
    tuned = None
    if args.cluster_table and args.tune_variants > 0 and rank == 0:
        from ressim_b200 import autotune

        order = sorted(range(nv), key=lambda i: ds[i].n_cells)
        pick = sorted({order[int(round(q * (nv - 1)))] for q in np.linspace(0.0, 1.0, args.tune_variants)})
        autotune.tune([ds[i] for i in pick], dt, args.precision, path=args.cluster_table)
    if pg:
        pg.barrier()

    def make_ensemble():
        e = Ensemble(ds, precision=args.precision, host_threads=args.host_threads)
        e.set_mode(args.batch_mode)
        nonlocal tuned
        if args.cluster_table and os.path.exists(args.cluster_table):
            from ressim_b200 import autotune

            table = autotune.load(args.cluster_table)
            sizes = autotune.apply(e, table, args.precision,
                                   autotune.plan(table, ds, args.precision, host_threads=32,
                                                 sms=torch.cuda.get_device_properties(0).multi_processor_count))
            tuned = {"table": os.path.basename(args.cluster_table),
                     "sizes": {str(k): sizes.count(k) for k in sorted(set(sizes))}}
        return e

    ens = make_ensemble()
    L = _lib.load()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def l2_flush():
        flush.zero_()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ens.step(dt)
    for i in range(nv):
        ens.profile(i, enable=True, reset=True)
    batch_prof = hasattr(ens, "batch_profile")
    if batch_prof:
        ens.batch_profile(enable=True, reset=True)
    launches0 = ens.kernel_launches()
    l2_flush()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev_index)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_ms = 0.0
    newton = 0
    first_state = None
    for k in range(args.steps):
        ev0.record()
        reps = ens.step(dt)  # returns once every variant's stream has finished the report step
        ev1.record()
        ev1.synchronize()
        dev_ms += ev0.elapsed_time(ev1)
        newton += sum(r["newton_iterations"] for r in reps)
        if k == 0 and rank == 0:
            first_state = ens.state(0)  # outside the timed region: variant 0 after report step W
        l2_flush()
    clk = clocks.stop()
    launches = ens.kernel_launches() - launches0
    profs = [ens.profile(i, enable=False, reset=True) for i in range(nv)]
    batch = ens.batch_profile(enable=False, reset=True) if batch_prof else None
    if batch:  # the batched launches carry the filed solves; the contexts count their own launches
        launches += batch["pressure_launches"] + batch["block_sweep_launches"] + batch["factor_launches"]
    dev_ms_max = max_over_ranks(dev_ms, pg, "cuda")
    value = world * cells * args.steps / (dev_ms_max / 1e3)
    ens.close()

    # e2e: a second ensemble takes the same warm-up (the path is deterministic), then the same K
    # report steps are timed on the host clock with every variant's state uploaded from pinned host
    # memory before each step and read back after it
    ens = make_ensemble()
    for _ in range(args.warmup):
        reps = ens.step(dt)
    times = [r["time_days"] for r in reps] if args.warmup else [0.0] * nv
    hosts = []
    for i, d in enumerate(ds):
        st = ens.state(i)
        p_h = torch.tensor(st["pressure"]).pin_memory()
        s_h = torch.tensor(st["sat_water"]).pin_memory()
        hosts.append((p_h, s_h, C.cast(p_h.data_ptr(), C.POINTER(C.c_double)),
                      C.cast(s_h.data_ptr(), C.POINTER(C.c_double))))
    tt = C.c_double()
    l2_flush()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for i in range(nv):
            if L.rf_set_state(ens._ctx[i], hosts[i][2], hosts[i][3], None, None, C.c_double(times[i])) != 0:
                raise RuntimeError(f"rf_set_state failed for variant {i}")
        reps = ens.step(dt)
        times = [r["time_days"] for r in reps]
        for i in range(nv):
            if L.rf_get_state(ens._ctx[i], hosts[i][2], hosts[i][3], None, None, None, C.byref(tt)) != 0:
                raise RuntimeError(f"rf_get_state failed for variant {i}")
        e2e_s += time.perf_counter() - t0
        l2_flush()
    e2e_s = max_over_ranks(e2e_s, pg, "cuda")
    e2e_value = world * cells * args.steps / e2e_s
    ens.close()

    peak, peak_kind = measured_hbm_peak()
    roof = ensemble_roofline(ds, profs, peak, peak_kind, batch)
    matched = None
    if rank == 0 and world == 1 and not args.no_matched:
        sample = spread_sample([d.n_cells for d in ds], 16)
        matched = matched_comparison(ds, dt, sample)
    cpu = None
    field_err = None
    if cpu_job is not None:
        pool, job = cpu_job
        try:
            v, k, el, cnewton, cstates = job.get(timeout=900)
            cpu = {"value": v, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                   "sample": f"variant 0 ({ds[0].n_cells} cells), report step(s) {args.warmup}..{args.warmup + k - 1} "
                             f"after {args.warmup} untimed ones ({cnewton} Newton iterations, {el:.1f} s), C++ "
                             f"restatement of the reference FIM, 1 thread, {flags}"}
            if first_state is not None and cstates:
                cp_, cs_ = cstates[0][0], cstates[0][1]
                field_err = {"variant": 0, "report_step": args.warmup,
                             "pressure_rel": float(np.max(np.abs(first_state["pressure"] - cp_) /
                                                          np.maximum(np.abs(cp_), 1.0))),
                             "sat_water_abs": float(np.max(np.abs(first_state["sat_water"] - cs_))),
                             "against": "FP64 oracle (C++ restatement of the reference), the reference's tolerances"}
        except Exception as e:  # noqa: BLE001 - reported in the line
            cpu = {"value": None, "unit": "cell-steps/s", "cores": 1, "kind": "port", "sample": f"failed: {e}"}
        pool.terminate()
    if rank == 0:
        line = {
            "metric": "FIM cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64+f32",
            "data": "synthetic (seeded deck generator)",
            "config": {"workload": desc.format(nv=nv), "variants_per_gpu": nv, "cells_per_gpu": cells,
                       "dt_days": dt, "parallelism": f"variants sharded over {world} GPU(s)",
                       "l2": "flushed (256 MB write) between timed report steps; state alone exceeds L2",
                       "newton_iterations": newton,
                       "e2e_steps": "the same K report steps, on a second ensemble after the same warm-up",
                       "cluster_sizes": tuned or "automatic", "batch_mode": args.batch_mode},
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 2 * 8 * cells,
                    "d2h_bytes_per_step": 2 * 8 * cells},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "precision": args.precision, "field_error_vs_oracle": field_err, "matched_comparison": matched,
            "batch": batch,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


ADJ_CNV, ADJ_MB = 1e-9, 1e-11


def adjoint_objective(deck, dt, steps):
    """Cumulative surface oil of a forward run (controller options as the adjoint leg's)."""
    from ressim_b200 import ReservoirSimulator

    sim = ReservoirSimulator.from_deck(deck)
    sim.set_controller_options(True, ADJ_CNV, ADJ_MB)
    for _ in range(steps):
        r = sim.step(dt)
        if r["warning"]:
            raise RuntimeError(f"forward warning {r['warning']}")
    t0, J = 0.0, 0.0
    for h in sim.get_rate_history():
        J += (h["time"] - t0) * h["total_production_oil"]
        t0 = h["time"]
    sim.close()
    return J


def run_adjoint(args, rank, world):
    """`--workload adjoint`: a warm-up of W recorded report steps and a backward pass on a separate
    simulator; then, from the initial state, K recorded forward report steps and the backward pass
    over them, timed together with CUDA events (value) and by the host clock through the public
    API with the state uploaded from host memory and the gradient read back (e2e).  One rank per GPU runs a replica (the backward pass does not shard).  A directional
    derivative along a seeded random direction is checked against central differences (step 1e-4
    in ln k) of two more forward runs."""
    import copy

    import numpy as np
    import torch

    from ressim_b200 import ReservoirSimulator

    torch.cuda.set_device(0)
    dev_index = (os.environ.get("CUDA_VISIBLE_DEVICES", "") or "0").split(",")[0].strip() or "0"
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", 0))
        pg = dist
    deck, dt_default, desc = make_deck("adjoint")
    dt = args.dt if args.dt is not None else dt_default
    n, K, W = deck.n_cells, args.steps, args.warmup
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # warm-up: W recorded report steps and a backward pass on a separate simulator (untimed)
    warm = ReservoirSimulator.from_deck(deck)
    warm.set_controller_options(True, ADJ_CNV, ADJ_MB)
    warm.adjoint_record(True)
    for _ in range(W):
        warm.step(dt)
    if W:
        warm.backward()
    warm.close()
    sim = ReservoirSimulator.from_deck(deck)
    sim.set_controller_options(True, ADJ_CNV, ADJ_MB)
    st0 = sim.state()
    t_state = sim.time_days
    flush.zero_()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(dev_index)
    clocks.start()
    launches0 = sim.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    t0 = time.perf_counter()
    # the public API from host buffers: upload the state, record K steps, backward, read back
    from ressim_b200 import _abi, _lib
    import ctypes as C

    L = _lib.load()
    h = sim._context()
    bufs = [np.ascontiguousarray(st0[k]) for k in ("pressure", "sat_water", "sat_gas", "rs")]
    ptrs = [b.ctypes.data_as(C.POINTER(C.c_double)) for b in bufs]
    ev[0].record()
    if L.rf_set_state(h, *ptrs, C.c_double(t_state)) != 0:
        raise RuntimeError(_lib.last_error(h))
    sim.adjoint_record(True)
    newton = 0
    for _ in range(K):
        r = sim.step(dt)
        newton += r["newton_iterations"]
        if r["warning"]:
            raise RuntimeError(f"forward warning {r['warning']}")
    sim.adjoint_record(False)
    fwd_prof = sim.profile(enable=True, reset=True)
    ev[1].record()
    J, grad, gctl = sim.backward()
    ev[2].record()
    bwd_prof = sim.profile(enable=False, reset=True)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    launches = sim.kernel_launches() - launches0
    fwd_ms, bwd_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    dev_ms = max_over_ranks(fwd_ms + bwd_ms, pg, "cuda")
    wall = max_over_ranks(wall, pg, "cuda")
    value = world * n * K / (dev_ms / 1e3)
    check = None
    if rank == 0:
        rng = np.random.default_rng(2024)
        v = rng.standard_normal(n)
        hstep = 1e-4

        def shifted(sign):
            d = copy.deepcopy(deck)
            m = np.exp(sign * hstep * v)
            d.perm_x, d.perm_y, d.perm_z = (np.asarray(a) * m for a in (d.perm_x, d.perm_y, d.perm_z))
            return adjoint_objective(d, dt, K)

        j_fwd = adjoint_objective(deck, dt, K)
        fd = (shifted(1.0) - shifted(-1.0)) / (2 * hstep)
        dd = float(grad @ v)
        check = {"direction": "seeded standard normal over all cells", "step_ln_k": hstep, "adjoint": dd, "fd": fd,
                 "rel_err": abs(dd - fd) / max(abs(fd), 1e-300), "objective": J,
                 "objective_forward_run": j_fwd}
    if rank == 0:
        line = {
            "metric": "FIM cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": dev_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded deck generator)",
            "config": {"workload": desc, "cells": n, "dt_days": dt, "parallelism": f"replicas{world}",
                       "newton_iterations": newton, "parameters": n + len(gctl)},
            "e2e": {"value": world * n * K / wall, "unit": "cell-steps/s", "h2d_bytes_per_step": 4 * 8 * n // K,
                    "d2h_bytes_per_step": 8 * (n + len(gctl)) // K},
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "backward_over_forward": bwd_ms / max(fwd_ms, 1e-9),
            "backward_phase_ms": {k: round(v, 1) for k, v in bwd_prof.items()},
            "gradient_check": check, "clocks": clk, "gpu_launches": int(launches), "roofline": None,
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_setup(args)
    if args.workload == "ensemble":
        return run_ensemble(args, rank, world)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world)
    cpu_job = None
    flags = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload != "2m":
        import multiprocessing as mp

        flags = use_native_oracle()
        pool = mp.get_context("spawn").Pool(1)
        cpu_job = (pool, pool.apply_async(cpu_leg, (args.workload, args.dt, args.warmup, 2, args.cpu_sample_s)))

    import ctypes as C

    import numpy as np
    import torch

    from ressim_b200 import ReservoirSimulator, _abi, _lib

    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}))
        return 1
    torch.cuda.set_device(0)
    # nvidia-smi -i takes the index or UUID that CUDA_VISIBLE_DEVICES names (set per rank above)
    dev_index = (os.environ.get("CUDA_VISIBLE_DEVICES", "") or "0").split(",")[0].strip() or "0"
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", 0))
        pg = dist

    deck, dt_default, desc = make_deck(args.workload)
    dt = args.dt if args.dt is not None else dt_default
    n = deck.n_cells
    sim = ReservoirSimulator.from_deck(deck)
    L = _lib.load()
    h = sim._context()
    sim.set_linear_precision(args.precision)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def l2_flush():
        flush.zero_()
        torch.cuda.synchronize()

    # ---- warm-up (untimed) ----
    for _ in range(args.warmup):
        sim.step(dt)
    l2_flush()

    # ---- device-resident leg ----
    sim.profile(enable=True, reset=True)
    launches0 = sim.kernel_launches()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev_index)
    clocks.start()
    dev_ms = 0.0
    newton = lin = substeps = 0
    reps = []
    gpu_states = []
    for _ in range(args.steps):
        r = sim.step(dt)
        reps.append(r)
        dev_ms += r["device_ms"]
        st = sim.state()  # outside the device-timed region (rf_step's own events)
        gpu_states.append((st["pressure"], st["sat_water"], st["sat_gas"]))
        newton += r["newton_iterations"]
        lin += r["linear_iterations"]
        substeps += r["substeps"]
        l2_flush()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = sim.kernel_launches() - launches0
    prof = sim.profile(enable=False, reset=True)
    dev_ms_max = max_over_ranks(dev_ms, pg, "cuda")
    if pg:
        pg.barrier()
    value = world * n * args.steps / (dev_ms_max / 1e3)

    # ---- mixed form: the plain FP64 path on the same report steps, and the field error ----
    fp64_cmp = None
    if args.precision == "mixed":
        ref = ReservoirSimulator.from_deck(deck)
        for _ in range(args.warmup):
            ref.step(dt)
        ref_ms = 0.0
        ref_newton = 0
        for _ in range(args.steps):
            l2_flush()
            r = ref.step(dt)
            ref_ms += r["device_ms"]
            ref_newton += r["newton_iterations"]
        a, b = sim.state(), ref.state()
        ref.close()
        fp64_cmp = {"fp64_value": n * args.steps / (ref_ms / 1e3), "mixed_over_fp64": (n * args.steps / (dev_ms / 1e3))
                    / (n * args.steps / (ref_ms / 1e3)), "fp64_newton_iterations": ref_newton,
                    "field_error_mixed_vs_fp64": {
                        "pressure_rel": float(np.max(np.abs(a["pressure"] - b["pressure"]) /
                                                     np.maximum(np.abs(b["pressure"]), 1.0))),
                        "sat_water_abs": float(np.max(np.abs(a["sat_water"] - b["sat_water"])))},
                    "profile": "the reference's tolerances on both; the same warm-up and timed report steps"}

    # ---- end-to-end leg: host buffers, copies inside the timed region ----
    # A second simulator of the same deck takes the same warm-up steps (the path is deterministic),
    # so the timed steps here are the same report steps as in the device-resident leg.
    sim2 = ReservoirSimulator.from_deck(deck)
    h = sim2._context()
    sim2.set_linear_precision(args.precision)
    for _ in range(args.warmup):
        sim2.step(dt)
    # per-cell state the step reads and writes: p, sw (two-phase); p, sw, sg, rs (three-phase)
    three = bool(deck.three_phase_mode)
    keys = ("pressure", "sat_water", "sat_gas", "rs") if three else ("pressure", "sat_water")
    st = sim2.state()
    bufs = []
    for key in keys:
        b = torch.empty(n, dtype=torch.float64).pin_memory()
        b.numpy()[:] = st[key]
        bufs.append(b)
    ptrs = [C.cast(b.data_ptr(), C.POINTER(C.c_double)) for b in bufs]
    pp, sp = ptrs[0], ptrs[1]
    gp, rp = (ptrs[2], ptrs[3]) if three else (None, None)
    tt = C.c_double()
    rep = _abi.RfStepReport()
    l2_flush()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rc = L.rf_set_state(h, pp, sp, gp, rp, C.c_double(sim2.time_days))
        if rc != 0:
            raise RuntimeError(f"rf_set_state failed: {_lib.last_error(h)}")
        rc = L.rf_step(h, C.c_double(dt), C.byref(rep))
        if rc < 0:
            raise RuntimeError(f"rf_step failed: {_lib.last_error(h)}")
        sim2.time_days = rep.time_days
        rc = L.rf_get_state(h, pp, sp, None, gp, rp, C.byref(tt))
        if rc != 0:
            raise RuntimeError(f"rf_get_state failed: {_lib.last_error(h)}")
        e2e_s += time.perf_counter() - t0
        l2_flush()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(e2e_s, pg, "cuda")
    e2e_value = world * n * args.steps / e2e_s

    # ---- roofline of the dominant kernel (BiCGStab pressure stage) ----
    peak, peak_kind = measured_hbm_peak()
    iters, launches_b, nnzb = prof["bicgstab_iterations"], prof["bicgstab_launches"], prof["nnzb"]
    kernel_ms = prof["bicgstab_kernel"]
    roof = None
    if launches_b > 0 and kernel_ms > 0:
        bytes_launch = bicgstab_bytes_per_iteration(n, nnzb) * iters / launches_b
        ms_launch = kernel_ms / launches_b
        achieved = bytes_launch / (ms_launch / 1e3) / 1e9
        kname = ("k_bicgstab_level (one thread block, level order)" if prof.get("level_kernels")
                 else "k_bicgstab_dsmem / k_bicgstab_cluster (one thread-block cluster)")
        traffic = (None if prof.get("level_kernels") or args.precision != "fp64"
                   else CLUSTER_DRAM_PER_LAUNCH.get(args.workload))
        roof = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "bytes_per_launch": bytes_launch, "ms_per_launch": ms_launch,
                "iterations_per_launch": iters / launches_b,
                "share_of_step": kernel_ms / max(dev_ms, 1e-9)}
    phases = {k: round(prof[k], 1) for k in _lib.PHASES}

    # ---- CPU baseline (rank 0, N = 1 only) ----
    cpu = None
    field_err = None
    if cpu_job is not None:
        pool, job = cpu_job
        try:
            v, k, el, cnewton, cpu_states = job.get(timeout=900)
            ep = max(float(np.max(np.abs(g[0] - c[0]) / np.maximum(np.abs(c[0]), 1.0)))
                     for g, c in zip(gpu_states, cpu_states))
            es = max(float(np.max(np.abs(g[1] - c[1]))) for g, c in zip(gpu_states, cpu_states))
            eg = max(float(np.max(np.abs(g[2] - c[2]))) for g, c in zip(gpu_states, cpu_states))
            field_err = {"pressure_rel": ep, "sat_water_abs": es, "sat_gas_abs": eg,
                         "report_steps": [args.warmup + i for i in range(min(len(gpu_states), len(cpu_states)))],
                         "against": "FP64 oracle (C++ restatement of the reference), same deck and steps"}
            cpu = {"value": v, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                   "sample": f"report steps {args.warmup}..{args.warmup + k - 1} of the same deck after "
                             f"{args.warmup} untimed ones ({cnewton} Newton iterations, {el:.1f} s), C++ "
                             f"restatement of the reference FIM, 1 thread, {flags}, run beside the GPU legs"}
        except Exception as e:  # noqa: BLE001 - reported in the line
            cpu = {"value": None, "unit": "cell-steps/s", "cores": 1, "kind": "port", "sample": f"failed: {e}"}
        pool.terminate()

    if rank == 0:
        line = {
            "metric": "FIM cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64+f32",
            "data": "synthetic (seeded deck generator)",
            "config": {"workload": desc, "cells": n, "dt_days": dt, "parallelism": f"replicas{world}",
                       "l2": "flushed (256 MB write) between timed report steps",
                       "newton_iterations": newton, "linear_iterations": lin, "substeps": substeps},
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": len(keys) * 8 * n,
                    "d2h_bytes_per_step": len(keys) * 8 * n},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "phase_ms": phases, "precision": args.precision, "field_error_vs_oracle": field_err,
            "mixed_vs_fp64": fp64_cmp,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    sim2.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

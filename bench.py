#!/usr/bin/env python
"""Headline benchmark of the SoftFlow hot path on B200.

Default workload (c3): the 256-channel capsule ensemble (seed 7) advanced in
one context, FP16-shifted population storage with FP32 arithmetic, 5 MDF
sweeps.  The metric is capsule-steps/s (sum over channels of capsules x
steps per second); MLUPS and marker-updates/s are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3|c2|c1|c0]
                  [--precision fp16s|fp32|fp64] [--impl product|reference]

value     device time (CUDA events on the context stream) of K steps with the
          state resident in HBM; max over ranks; whole-job aggregate.
e2e       the same K steps through the public API from host buffers: the
          initial populations are uploaded from pinned host memory inside the
          timed region, and every step's marker positions and velocities land
          in pinned host memory (sfg_get_all_markers_async: copied on a second
          stream while the next step runs; the host takes step s's markers
          before enqueuing step s + 2).
roofline  the lattice kernel (fused collide + stream + bounce-back + lagged
          scalar step), timed live with CUDA events in a profiling pass;
          algorithmic bytes = one read + one write of 9 populations per fluid
          cell (+ the same for the scalar where enabled).
cpu_baseline  the reference engine's own sources (oracle/_ref, Release flags,
          OpenMP over all host cores) on a bounded sample of the workload.

Multi-GPU: the channels are independent, so each rank runs the full
workload on its own GPU with no collective on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default="c3", choices=["c3", "c2", "c2_lattice", "c1", "c0"],
                    help="c2_lattice: configuration 2's fluid alone (the plain stream-collide)")
    ap.add_argument("--precision", default="fp16s", choices=["fp16s", "fp32", "fp64"])
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the per-channel plain form")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (no autotuner trials)")
    ap.add_argument("--mdf", default="auto", choices=["auto", "learned", "plain"],
                    help="forcing form of the timed run (auto: learned on the ensemble)")
    ap.add_argument("--mdf-threshold", type=float, default=1e-4,
                    help="no-slip residual (lu/step) above which a learned channel falls back")
    return ap.parse_args()


# ---------------------------------------------------------------- ranks ----
def dist_setup(args, backend="nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg, local):
    if pg is None:
        return
    import torch
    if pg.get_backend() == "nccl":
        pg.barrier(device_ids=[local])
        torch.cuda.synchronize()
    else:
        pg.barrier()


def allmax(pg, v: float) -> float:
    """Max over ranks (timings are taken as the slowest rank's)."""
    if pg is None:
        return v
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def make_plans(workload, precision, world=1, rank=0):
    """Work of one rank.  The ensemble is sharded: rank r runs channels
    [256 r, 256 (r + 1)) of one seeded sequence, so every rank has a distinct
    256-channel ensemble (weak scaling, no data-path collective).  The
    single-channel workloads run one replica per rank."""
    from softflow_b200 import workloads as W
    if workload == "c3":
        per = 256
        return W.plan_c3(precision, n_channels=per * world)[per * rank: per * (rank + 1)]
    return W.PLANS[workload](precision)


# --------------------------------------------------------------- clocks ----
class ClockSampler:
    """SM clock and clock-event reasons of this rank's GPU while the timed
    region runs.  NVML is polled every 10 ms from a thread (the timed region
    of the default run lasts a fraction of a second); where NVML cannot be
    loaded, nvidia-smi is polled every 200 ms instead.  Reading only: no
    setting of the GPU is changed."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8,
                   "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
        except Exception:
            nv = None
        if nv is not None:
            self.stop_evt = threading.Event()
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                                  None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while True:
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                          mx, int(get_reasons(h))))
                    except Exception:
                        pass
                    if self.stop_evt.wait(0.01):
                        break
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _summary(self, sm, mx, reasons, source):
        if not sm:
            return None
        sm = sorted(sm)
        return {"sm_mhz": sm[len(sm) // 2], "sm_min_mhz": sm[0], "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": source}

    def stop(self):
        if self.thread is not None:
            self.stop_evt.set()
            self.thread.join(timeout=5)
            reasons = set()
            for _, _, bits in self.rows:
                for n, b in self.REASON_BITS.items():
                    if bits & b:
                        reasons.add(n)
            mx = max((r[1] for r in self.rows), default=None)
            return self._summary([r[0] for r in self.rows], mx, reasons, "nvml, 10 ms")
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return self._summary(sm, mx, reasons, "nvidia-smi, 200 ms")


def peaks():
    try:
        with open(PEAKS_FILE) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ------------------------------------------------------------ workloads ----
def bytes_per_cell(precision: str) -> int:
    return {"fp64": 144, "fp32": 72, "fp16s": 36}[precision]


def scalar_bytes_per_cell(precision: str) -> int:
    return 144 if precision == "fp64" else 72


SPREAD_ENTRY_BYTES = 100   # per list entry: force 16, arc length 8, origin 8, weights 64, index 4
SLOT_FINAL_BYTES = 4096    # per force tile, last sweep: final force and force before it, 2 x 2 KB


def spread_geometry(ens, plans):
    """Force tiles (32 x 8), list entries (marker, tile) and touched cells of
    the markers' 4 x 4 stencils, from the marker positions read back."""
    import numpy as np
    slots = entries = touched = 0
    for i, pl in enumerate(plans):
        nx, ny = pl.params.nx, pl.params.ny
        X = np.asarray(ens.capsules(i).positions()).reshape(-1, 2)
        if len(X) == 0:
            continue
        ix = np.floor(X[:, 0]).astype(np.int64)
        iy = np.floor(X[:, 1]).astype(np.int64)
        s = np.arange(-1, 3)
        jx = (ix[:, None, None] + s[None, None, :]) % nx            # [m, 1, 4]
        jy = iy[:, None, None] + s[None, :, None]                   # [m, 4, 1]
        jx, jy = np.broadcast_arrays(jx, jy)
        ok = (jy >= 0) & (jy < ny)
        cell = np.where(ok, jy * nx + jx, -1)
        touched += len(np.unique(cell[ok]))
        tx = (nx + 31) // 32
        tile = np.sort(np.where(ok, (jy // 8) * tx + jx // 32, -1).reshape(len(X), -1), axis=1)
        first = np.ones_like(tile, dtype=bool)
        first[:, 1:] = tile[:, 1:] != tile[:, :-1]
        entries += int(np.sum(first & (tile >= 0)))           # distinct tiles per marker
        slots += len(np.unique(tile[tile >= 0]))
    return slots, entries, touched


def spread_roofline(ens, plans, spread_ms, sweeps, peak, peak_kind):
    """The forcing spread (k_spread_fx on FP32-arithmetic contexts): the
    algorithmic bytes of the step's `sweeps` launches against their phase
    time.  Every launch reads each list entry's marker data; the sweeps
    before the last read (after the first) and write the accumulators at
    the touched cells; the last writes the tiles' final force and the force
    before it at every cell."""
    slots, entries, touched = spread_geometry(ens, plans)
    alg = sweeps * entries * SPREAD_ENTRY_BYTES + touched * 8 * (2 * sweeps - 2) \
        + slots * SLOT_FINAL_BYTES
    ach = alg / (spread_ms / 1e3) / 1e9 if spread_ms > 0 else 0.0
    return {"kernel": "k_spread_fx", "bound": "latency (gathers, shared atomics)",
            "launches_per_step": sweeps, "ms_per_step": spread_ms,
            "force_tiles": slots, "list_entries": entries, "touched_cells": touched,
            "algorithmic_bytes_per_step": alg, "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak, "peak_source": peak_kind,
            "note": "phase time of the profiled pass: the sweeps plus the fallback sweeps "
                    "that return at once; tiles and cells from the final marker positions"}


def lattice_kernel_name(plans, precision):
    """The lattice kernel instantiation a workload runs: the eight-cell
    FP16-shifted kernel when the storage is FP16S, there is no scalar and
    every nx % 8 == 0, otherwise the four-cell kernel (storage, arithmetic,
    scalar fused or not); the template's last argument is the collision
    model."""
    adr = int(any(p.params.scalar.enabled for p in plans))
    coll = "|".join(map(str, sorted({int(p.params.fluid.collision_model) for p in plans})))
    if precision == "fp16s" and not adr and all(p.params.nx % 8 == 0 for p in plans):
        return f"k_lattice_step8h<{coll}>"
    st = {"fp64": "double, double", "fp32": "float, float", "fp16s": "__half, float"}[precision]
    return f"k_lattice_step4<{st}, {adr}, {coll}>"


def measure_form(plans, precision, steps, warmup, local, prof_steps=20):
    """One context holding `plans`: device time of `steps` graph-launched
    steps after `warmup`, then per-phase CUDA-event times of `prof_steps`
    eager steps; throughput figures and the lattice kernel's roofline."""
    from softflow_b200 import workloads as W
    ens = W.build(plans, precision=precision, device=local)
    ctx = ens.context()
    cells, caps, markers, scal = W.totals(plans, ens)
    tuned = ens.autotune(steps_per_trial=5)
    ctx.step(warmup)
    ctx.synchronize()
    ctx.step(steps)
    ctx.synchronize()
    ms = ctx.last_step_ms()
    ctx.set_profiling(True)
    ctx.reset_phase_times()
    ctx.step(prof_steps)
    ctx.synchronize()
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    ens.close()
    sec = ms / 1e3
    lat_ms = phases["lattice"] / prof_steps
    alg = cells * bytes_per_cell(precision) + scal * scalar_bytes_per_cell(precision)
    peak, kind = peaks()
    ach = alg / (lat_ms / 1e3) / 1e9 if lat_ms > 0 else 0.0
    return {"precision": precision, "ms_per_step": ms / steps,
            "capsule_steps_per_s": caps * steps / sec, "mlups": cells * steps / sec / 1e6,
            "marker_updates_per_s": markers * steps / sec,
            "fluid_cells": cells, "capsules": caps, "markers": markers, "launch_shapes": tuned,
            "lattice": {"kernel": lattice_kernel_name(plans, precision), "ms": lat_ms,
                        "algorithmic_bytes": alg, "achieved_gbs": ach, "peak_gbs": peak,
                        "frac": ach / peak, "peak_source": kind},
            "phase_ms_per_step": {k: v / prof_steps for k, v in phases.items() if v > 0}}


def run_c2_forms(args, local):
    """Configuration 2 beside the ensemble: its fluid alone in FP32 (the
    plain stream-collide at 4096 x 1024), and the whole configuration
    (2,000 capsules, the scalar) in the plain form (FP32) and in FP16-shifted
    storage."""
    from softflow_b200 import workloads as W
    steps = max(args.steps, 50)
    out = {"lattice_only_fp32": measure_form(W.plan_c2_lattice("fp32"), "fp32", steps,
                                             args.warmup, local),
           "coupled_fp32": measure_form(W.plan_c2("fp32"), "fp32", steps, args.warmup, local),
           "coupled_fp16s": measure_form(W.plan_c2("fp16s"), "fp16s", steps, args.warmup,
                                         local),
           "steps": steps,
           "config": "4096 x 1024 MRT tau 0.8 fx 1e-5; coupled: 1000 WLC + Helfrich "
                     "(r 6, 48 markers) and 1000 Skalak (r 3, 24 markers) capsules, "
                     "1 forcing sweep, scalar D 0.05"}
    return out


def run_product(args, world, rank, local, pg):
    import numpy as np
    import softflow_b200 as S
    from softflow_b200 import workloads as W
    plans = make_plans(args.workload, args.precision, world, rank)
    learned = args.mdf == "learned" or (args.mdf == "auto" and args.workload == "c3")
    learn_info = None
    net = None
    if learned:
        # the network, trained here on plain runs (untimed, seeded)
        from softflow_b200.learned import training_set, train_network
        t0 = time.perf_counter()
        X, Y = training_set(2_000_000, device=local)
        net, losses = train_network(X, Y, device=local, epochs=8, seed=1)
        learn_info = {"samples": int(X.shape[0]), "adam_steps": int(losses.size),
                      "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                      "setup_s": time.perf_counter() - t0}
        del X, Y
    ens = W.build(plans, precision=args.precision, device=local)
    if learned:
        ens.setLearnedMDF(net, threshold=args.mdf_threshold)
    ctx = ens.context()
    cells, caps, markers, scal = W.totals(plans, ens)
    nch = len(plans)

    # launch shapes chosen by the autotuner on real steps, then the warm-up
    # (graphs are built on the first call); both untimed
    tuned = ens.autotune(steps_per_trial=5) if not args.no_autotune else ens.launchConfig()
    ctx.step(args.warmup)
    ctx.synchronize()
    stats0 = [ens.mdfStats(c) for c in range(nch)] if learned else None

    import torch
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg, local)
    torch.cuda.nvtx.range_push("timed")
    ctx.step(args.steps)
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = ctx.last_step_ms()
    barrier(pg, local)
    clk = clocks.stop()
    ms_max = allmax(pg, ms)
    launches = ctx.launches_per_step()
    if learned:
        st = [ens.mdfStats(c) for c in range(nch)]
        ls = sum(a["learned_steps"] - b["learned_steps"] for a, b in zip(st, stats0))
        fb = sum(a["fallbacks"] - b["fallbacks"] for a, b in zip(st, stats0))
        learn_info.update({"threshold": args.mdf_threshold,
                           "fallback_fraction": fb / ls if ls else None,
                           "gate_residual_median": float(np.median([a["resid_learned"] for a in st])),
                           "gate_residual_max": float(np.max([a["resid_learned"] for a in st]))})

    sec = ms_max / 1e3
    cap_steps = caps * args.steps * world / sec
    mlups = cells * args.steps * world / sec / 1e6
    mk_upd = markers * args.steps * world / sec

    # profiling pass: per-phase CUDA-event times (eager launches)
    prof_steps = max(5, min(args.steps, 50))
    ctx.set_profiling(True)
    ctx.reset_phase_times()
    ctx.step(prof_steps)
    ctx.synchronize()
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    lat_ms = phases["lattice"] / prof_steps
    alg_bytes = cells * bytes_per_cell(args.precision) + scal * scalar_bytes_per_cell(
        args.precision)
    achieved = alg_bytes / (lat_ms / 1e3) / 1e9 if lat_ms > 0 else 0.0
    peak, peak_kind = peaks()
    total_phase = sum(phases.values()) or 1.0
    spread = None
    if args.precision != "fp64" and markers > 0 and phases.get("ibm_spread", 0.0) > 0:
        K = max(p.params.ibm_iterations for p in plans)
        spread = spread_roofline(ens, plans, phases["ibm_spread"] / prof_steps,
                                 3 if (learned and K > 2) else K, peak, peak_kind)
    # the lattice kernel also reads the force tiles' F and G (two floats each
    # per cell) where markers force the fluid: reported beside the
    # populations-only figure
    lattice_force = {}
    if spread is not None and lat_ms > 0:
        ftb = spread["force_tiles"] * SLOT_FINAL_BYTES
        ach_f = (alg_bytes + ftb) / (lat_ms / 1e3) / 1e9
        lattice_force = {"force_tile_bytes_per_launch": ftb,
                         "achieved_with_force_tiles": ach_f,
                         "frac_with_force_tiles": ach_f / peak}

    # e2e: host-resident initial state, per-step marker readback
    e2e = run_e2e(args, plans, ens, pg, local)

    # the same ensemble with the plain forcing sweeps (same steps, same clock)
    batched_plain = None
    if learned:
        ens.close()
        ensp = W.build(plans, precision=args.precision, device=local)
        cp = ensp.context()
        cp.step(args.warmup)
        cp.synchronize()
        cp.step(args.steps)
        cp.synchronize()
        pms = allmax(pg, cp.last_step_ms())
        batched_plain = {"value": caps * args.steps * world / (pms / 1e3),
                         "unit": "capsule-steps/s", "ms_per_step": pms / args.steps,
                         "form": "same ensemble and precision, plain forcing sweeps",
                         "gate_residual_median_plain": float(np.median(
                             [ensp.mdfStats(c)["resid_plain"] for c in range(nch)]))}
        # the method's own difference: the learned and the plain forcing from
        # the same initial state after the same number of steps
        ensl = W.build(plans, precision=args.precision, device=local)
        ensl.setLearnedMDF(net, threshold=args.mdf_threshold)
        ensl.run(args.warmup + args.steps)
        num = den = 0.0
        for c, pl in enumerate(plans):
            rows = slice(1, pl.params.ny - 1)
            ul = np.stack([ensl.field(c).velocity_x()[rows], ensl.field(c).velocity_y()[rows]])
            up = np.stack([ensp.field(c).velocity_x()[rows], ensp.field(c).velocity_y()[rows]])
            num += float(np.sum((ul - up) ** 2))
            den += float(np.sum(up ** 2))
        learn_info["learned_vs_plain_velocity_rel_l2"] = math.sqrt(num / den)
        learn_info["learned_vs_plain_steps"] = args.warmup + args.steps
        learn_info["gate_residual_median_plain"] = batched_plain["gate_residual_median_plain"]
        ensl.close()
        ensp.close()
        ens = None

    # plain per-channel form (each channel its own context, run one after the other)
    plain = None
    if args.workload == "c3" and not args.no_plain:
        plain = run_plain(args, plans, local)
    c2_forms = None
    if args.workload == "c3" and not args.no_plain and world == 1:
        c2_forms = run_c2_forms(args, local)

    metric, value = ("capsule-steps/s", cap_steps) if caps else ("MLUPS", mlups)
    out = {
        "metric": metric,
        "value": value,
        "unit": metric,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp16s": "fp16-storage/fp32", "fp32": "fp32", "fp64": "fp64"}[args.precision],
        "data": "synthetic (seeded placement; no datasets)",
        "config": {"workload": args.workload, "channels": nch, "fluid_cells": cells,
                   "capsules": caps, "markers": markers, "precision": args.precision,
                   "mdf_sweeps": max(p.params.ibm_iterations for p in plans),
                   "mdf": ("learned: network seed for sweeps 1..K-2, last plain sweep, "
                           f"plain fallback above {args.mdf_threshold:g} lu/step")
                          if learned else "plain",
                   "l2": "state larger than L2 (no flush needed)" if alg_bytes > 126e6
                         else "state fits L2 (L2-resident workload)",
                   "launch_shapes": tuned,
                   "parallelism": (f"channel shards x{world} (256 distinct channels per rank)"
                                   if args.workload == "c3" else f"replicas x{world}")},
        "mlups": mlups,
        "marker_updates_per_s": mk_upd,
        "gpu_launches": launches * args.steps,
        "phase_ms_per_step": {k: v / prof_steps for k, v in phases.items()},
        "roofline": {"kernel": lattice_kernel_name(plans, args.precision), "bound": "hbm",
                     "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "share_of_step": phases["lattice"] / total_phase,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     **lattice_force,
                     # DRAM bytes need a profiler; the bench does not run one
                     "traffic": None},
        "spread_roofline": spread,
        "e2e": e2e,
        "clocks": clk,
    }
    if learn_info is not None:
        out["learned_mdf"] = learn_info
    if batched_plain is not None:
        out["batched_plain"] = batched_plain
    if c2_forms is not None:
        out["c2"] = c2_forms
    if plain is not None:
        out["plain"] = plain
        out["batched_vs_plain"] = cap_steps / world / plain["value"] if plain["value"] else None
    if ens is not None:
        ens.close()
    return out


def run_e2e(args, plans, ens, pg, local):
    """K steps from host-resident state through the public API."""
    import numpy as np
    import torch
    from softflow_b200 import _lib as L
    import ctypes as C
    ctx = ens.context()
    lib = ctx._lib
    # pinned host copy of the current state: every channel's [9][ny][nx]
    # populations back to back (the layout sfg_set_all_populations takes)
    flat = [ens.field(i).distributions().ravel() for i in range(len(plans))]
    pops = torch.empty(sum(f.size for f in flat), dtype=torch.float64, pin_memory=True)
    off = 0
    for f in flat:
        pops.numpy()[off:off + f.size] = f
        off += f.size
    del flat
    M = sum(r.rest.num_nodes for c in ens._chans for r in c.caps)
    pos_h = torch.empty(2 * max(M, 1), dtype=torch.float64, pin_memory=True)
    vel_h = torch.empty(2 * max(M, 1), dtype=torch.float64, pin_memory=True)
    lib.sfg_get_all_markers(ctx._h, L.dptr(pos_h.numpy()), L.dptr(vel_h.numpy()))
    h2d = pops.numel() * 8
    d2h_step = 2 * 8 * 2 * M
    # two pinned landing buffers: step s's markers are copied to the host while
    # step s + 1 runs; the host takes step s's markers before enqueuing s + 2
    pos_b = [pos_h, torch.empty_like(pos_h).pin_memory()]
    vel_b = [vel_h, torch.empty_like(vel_h).pin_memory()]
    barrier(pg, local)
    t0 = time.perf_counter()
    L.check(lib.sfg_set_all_populations(ctx._h, L.dptr(pops.numpy())))
    ctx.synchronize()
    t_up = time.perf_counter()
    for s in range(args.steps):
        L.check(lib.sfg_step(ctx._h, 1))
        if s >= 1:
            L.check(lib.sfg_wait_markers(ctx._h, (s - 1) % 2))   # step s - 1 on the host
        L.check(lib.sfg_get_all_markers_async(ctx._h, s % 2, L.dptr(pos_b[s % 2].numpy()),
                                              L.dptr(vel_b[s % 2].numpy())))
    L.check(lib.sfg_wait_markers(ctx._h, (args.steps - 1) % 2))
    ctx.synchronize()
    t1 = time.perf_counter()
    sec = allmax(pg, t1 - t0)
    up = allmax(pg, t_up - t0)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    caps = sum(len(c.caps) for c in ens._chans)
    from softflow_b200 import workloads as W
    units, unit = (caps, "capsule-steps/s") if caps else (W.totals(plans)[0] / 1e6, "MLUPS")
    return {"value": units * args.steps * world / sec, "unit": unit,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h_step,
            "upload_ms": 1e3 * up, "upload_bytes": h2d,
            "per_step_value": units * args.steps * world / (sec - up),
            "per_step_ms": 1e3 * (sec - up) / args.steps,
            "note": "value: the whole timed region, i.e. the one-off upload of the initial "
                    "state from pinned host memory (sfg_set_all_populations, FP64 reference "
                    "layout) followed by the steps; per_step_value: the steps alone, each "
                    "landing its marker positions and velocities in pinned host memory "
                    "(copied on a second stream while the next step runs)"}


def run_plain(args, plans, local, max_channels=256, steps=None):
    """The plain GPU form: every channel in its own context, stepped one after
    the other (no batching), FP32 storage."""
    from softflow_b200 import workloads as W
    steps = steps or max(10, min(args.steps, 40))
    total_caps_steps = 0
    total_ms = 0.0
    for pl in plans[:max_channels]:
        pl.params.precision = "fp32"
        ens = W.build([pl], precision="fp32", device=local)
        ctx = ens.context()
        ctx.step(3)
        ctx.synchronize()
        ctx.step(steps)
        ctx.synchronize()
        total_ms += ctx.last_step_ms()
        total_caps_steps += len(ens._chans[0].caps) * steps
        ens.close()
    return {"value": total_caps_steps / (total_ms / 1e3), "unit": "capsule-steps/s",
            "form": "one context per channel, FP32, stepped sequentially",
            "steps_per_channel": steps}


# ------------------------------------------------------------ CPU side ----
def cpu_kind():
    import oracle as O
    return ("reference", "ref") if os.path.exists(O.REF_FAST_LIB) else ("port", "sfo")


def cpu_sample(workload, precision):
    """The CPU side's channels: the whole workload (for the ensemble, all 256
    channels, the same set the GPU runs)."""
    from softflow_b200 import workloads as W
    plans = W.PLANS[workload](precision)
    what = f"all {len(plans)} channels" if workload == "c3" else "full workload"
    return plans, what


def host_threads() -> int:
    """Threads this process may run at once: its CPU affinity, capped by a
    cgroup CPU quota when one is set (cgroup v2 cpu.max or v1 cfs quota)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    for quota, period in (("/sys/fs/cgroup/cpu.max", None),
                          ("/sys/fs/cgroup/cpu/cpu.cfs_quota_us",
                           "/sys/fs/cgroup/cpu/cpu.cfs_period_us")):
        try:
            if period is None:
                q, p = open(quota).read().split()[:2]
            else:
                q, p = open(quota).read().strip(), open(period).read().strip()
            if q not in ("max", "-1") and int(q) > 0:
                n = min(n, max(1, int(q) // int(p)))
            break
        except Exception:
            continue
    return max(1, n)


def best_threads(sims, impl):
    """The reference build's fastest OpenMP thread count on this host: one
    step of the first 32 channels (each in one call, one after the other) at
    1, 2, 4, ... threads up to host_threads(), plus that count; the channels
    are warmed up by it."""
    top = host_threads() if impl == "ref" else 1
    cands = sorted({1 << k for k in range(top.bit_length()) if (1 << k) <= top} | {top})
    sample = sims[:32]
    time_cpu(sample, 1, cands[-1])
    best, best_t = cands[-1], None
    for t in cands:
        dt = time_cpu(sample, 1, t)
        if best_t is None or dt < best_t:
            best, best_t = t, dt
    return best, cands


def time_cpu(sims, steps, threads):
    """Steps every simulation `steps` steps in one call each, one after the
    other (the sum of per-channel runs), with `threads` OpenMP threads;
    returns seconds."""
    for s in sims:
        s.set_threads(threads)
    t0 = time.perf_counter()
    for s in sims:
        s.step(steps)
    return time.perf_counter() - t0


def run_cpu_baseline(workload, precision, budget_s=15.0):
    """The reference's own sources (oracle/_ref, Release flags) on the GPU
    host's cores: all threads on every channel of the workload for a bounded
    number of steps, and one thread on the same channels for fewer."""
    from oracle.plans import sims_from_plans
    kind, impl = cpu_kind()
    plans, what = cpu_sample(workload, precision)
    sims = sims_from_plans(plans, impl, 1)
    caps = sum(s.num_capsules for s in sims)
    threads, tried = best_threads(sims, impl)
    dt1 = max(time_cpu(sims, 1, threads), 1e-6)          # warm-up step, cost estimate
    n = max(1, min(200, int(budget_s / dt1)))
    sec = time_cpu(sims, n, threads)
    out = {"value": caps * n / sec, "unit": "capsule-steps/s", "cores": threads, "kind": kind,
           "threads_tried": tried, "host_threads": host_threads(),
           "sample": f"{what}, {n} steps per channel in one call each, after 1 warm-up step"}
    if threads > 1:
        n1 = max(1, min(n, int(budget_s / (dt1 * threads))))
        sec1 = time_cpu(sims, n1, 1)
        out["one_thread"] = {"value": caps * n1 / sec1, "unit": "capsule-steps/s", "cores": 1,
                             "sample": f"{what}, {n1} steps per channel in one call each"}
    return out


def run_reference_arm(args):
    """The reference's own CPU implementation (oracle/_ref, Release flags,
    all host threads) on the same workload, channels and metric as the
    product arm: every channel stepped `warmup` then `steps` steps in one
    call each, one channel after the other."""
    from oracle.plans import sims_from_plans
    kind, impl = cpu_kind()
    plans, what = cpu_sample(args.workload, args.precision)
    sims = sims_from_plans(plans, impl, 1)
    caps = sum(s.num_capsules for s in sims)
    threads, tried = best_threads(sims, impl)
    time_cpu(sims, args.warmup, threads)
    sec = time_cpu(sims, args.steps, threads)
    v = caps * args.steps / sec
    sample = f"{what}, {args.steps} steps per channel in one call each"
    return {
        "impl": "reference", "metric": "capsule-steps/s", "value": v, "unit": "capsule-steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": "synthetic (seeded placement; no datasets)",
        "config": {"workload": args.workload, "channels": len(plans), "capsules": caps,
                   "sample": sample},
        "cpu_baseline": {"value": v, "unit": "capsule-steps/s", "cores": threads, "kind": kind,
                         "threads_tried": tried, "host_threads": host_threads(),
                         "sample": sample},
        "e2e": {"value": v, "unit": "capsule-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        print(json.dumps(run_reference_arm(args)), flush=True)
        return 0
    world, rank, local, pg = dist_setup(args)
    out = run_product(args, world, rank, local, pg)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = run_cpu_baseline(args.workload, args.precision)
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "error": str(e)}
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Throughput of cellweave's per-step hot path on B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload campaign|cord|spheroid]

Workload (default ``campaign``): the batched campaign of 64 independent
histories of uneven sizes (16 each at 128^2, 256^2, 512^2, 1024^2; cells at
30% fill, target 49; oxygen and a secreted signal solved to residual 1e-8 by
FP32 SOR with FP64 defect correction, which puts every field within 1e-6 of
its FP64 solution; 8-species RK4 network; Moore-contact CPM).  A step is one lattice step (MCS) of every history: field solves,
means, RK4, fates, Monte Carlo sweep.  Data are synthetic (seeded).

The JSON line reports histories*MCS/s of the batch (``value``), of the same
histories stepped one at a time (``plain``), end to end through the C ABI
with host buffers (``e2e``), the roofline of the dominant kernel (the FP32
SOR sweep), and the reference's algorithm timed on the host cores
(``cpu_baseline``, the CPU oracle on a bounded sample).

Under torchrun every rank runs its own campaign (seeds offset by rank): weak
scaling, no collective on the data path; ranks meet only for the barriers
and the max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "histories·MCS/s batched vs plain on 1 B200 at SOR resid≤1e-6; SOR HBM GB/s"
UNIT = "histories·MCS/s"
# FP32 inner sweep, one pass through HBM: correction read 4 + write 4, right-hand side 4, inverse diagonal 4
SOR_BYTES_PER_SITE_PASS = 16
# DRAM bytes per site of one k_sor32_wide<8> launch on the campaign's oxygen
# field, from ncu (dram__bytes_read.sum + dram__bytes_write.sum: 267.5 MB +
# 65.5 MB over 22,282,240 sites), a launch that reads and writes the
# correction (neither the first nor the last of a solve)
SOR_TRAFFIC_PER_SITE = 14.95


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["campaign", "cord", "spheroid"], default="campaign")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-fit", action="store_true")
    p.add_argument("--fit-iters", type=int, default=10)
    p.add_argument("--no-shapes", action="store_true")
    p.add_argument("--tolerance", type=float, default=None,
                   help="the field solves' residual stop (default: the workload's)")
    p.add_argument("--inner-sweeps", type=int, default=None,
                   help="FP32 sweeps per FP64 correction (default: the library's, 64)")
    p.add_argument("--error-tolerance", type=float, default=None,
                   help="also stop a solve only once its estimated error is below this times the field's largest "
                        "value (default: the workload's)")
    p.add_argument("--profile-step", action="store_true",
                   help="bracket one extra step with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    return p.parse_args()


def workload(name, rank=0):
    """The workload's configuration for one rank: every rank its own
    campaign, the same shapes, seeds offset by the rank (disjoint histories)."""
    from cellweave_b200 import synthetic
    cfg = (synthetic.campaign() if name == "campaign" else synthetic.tumour_cord() if name == "cord" else
           synthetic.spheroid_3d())
    cfg["seeds"] = [s + 100_000 * rank for s in cfg["seeds"]]
    return cfg


def configured(args, rank=0):
    """The workload with the solve options given on the command line, the
    same for every arm."""
    cfg = workload(args.workload, rank)
    if args.tolerance is not None:
        cfg["tolerance"] = args.tolerance
    if args.error_tolerance is not None:
        cfg["error_tolerance"] = args.error_tolerance
    if args.inner_sweeps is not None:
        cfg["inner_sweeps"] = args.inner_sweeps
    return cfg


def max_over_ranks(x, dist, device):
    """The largest x over the ranks (every rank calls it, in the same order)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, histories, steps, ms):
    """Whole-job histories*MCS/s: every rank's histories over the slowest rank's time."""
    return world * histories * steps / (ms / 1e3)


def config_key(name, cfg):
    if name == "campaign":
        stop = f"residual {cfg['tolerance']:g}"
        if cfg.get("error_tolerance"):
            stop += f" and estimated error {cfg['error_tolerance']:g}"
        return {"workload": "batched campaign: 64 histories, 16 each at 128^2/256^2/512^2/1024^2, 30% fill at "
                            f"target 49, Moore contact, 2 fields to {stop} (FP32 SOR + FP64 defect "
                            "correction; each field within 1e-6 of its FP64 solution), 8-species RK4 x8 per MCS", "histories": len(cfg["dims"]),
                "sites": int(sum(w * h * d for w, h, d in cfg["dims"])), "cells": int(sum(cfg["ncells"])),
                "l2": "inputs larger than L2 (the lattices and fields of one step exceed 126 MB)",
                "parallelism": "histories batched in one launch per kernel; ranks own disjoint campaigns",
                "subsweeps": 1}
    if name == "cord":
        return {"workload": "tumour cord 2048^2, ~40k cells of target 64, 3 types, vessel column, 2 fields to "
                            "residual 1e-8, 16-species RK4", "histories": 1,
                "l2": "inputs larger than L2", "parallelism": "one history"}
    return {"workload": "spheroid 256^3, a ball of radius 40 of 5^3 cells (target 125), 26-neighbour contact, "
                        "surface constraint, oxygen to residual 1e-9, 12-species RK4", "histories": 1,
            "l2": "inputs larger than L2", "parallelism": "one history"}


# ------------------------------------------------------------------ GPU clocks
class Clocks:
    """nvidia-smi sampled every 100 ms while the timed region runs; start()
    returns once the sampler has written its first row (up to 3 s), so that
    the samples cover the timed region rather than nvidia-smi's start."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows if len(r) > 8 for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ the CPU reference path
def _cpu_worker(args):
    """One history of the workload on the CPU oracle: `warm` untimed steps,
    then `steps` timed ones; returns (history index, seconds per MCS)."""
    k, cfg, steps, warm = args
    os.environ["OMP_NUM_THREADS"] = "1"
    from oracle import cpu_sim
    h = cpu_sim.CpuHistory(cfg, k)
    for _ in range(warm):
        h.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        h.step()
    return k, (time.perf_counter() - t0) / steps


def lpt_makespan(costs, workers):
    """Makespan of the longest-first list schedule of `costs` over `workers`
    (the order a work-stealing pool fed the longest histories first reaches)."""
    import heapq
    loads = [0.0] * max(1, workers)
    heapq.heapify(loads)
    for c in sorted(costs, reverse=True):
        heapq.heappush(loads, heapq.heappop(loads) + c)
    return max(loads)


CPU_SAMPLE = {"per_size": 4, "warm": 1, "steps": 2}


def cpu_sample(cfg, cores):
    """The reference's campaign on the host cores (src/campaign.rs:196-205:
    every history its own run, rayon spreading the runs over the cores),
    measured on a bounded sample and scheduled over the whole campaign.

    Sample: CPU_SAMPLE["per_size"] histories of every lattice size, each run
    by the oracle (sequential Metropolis, FP64 SOR, RK4: the reference's
    algorithms) in its own process, all of them at once on `cores` processes
    fed largest first, `warm` untimed MCS then `steps` timed ones.  Every
    history of the campaign costs its size's mean seconds per MCS; the
    campaign's MCS takes the makespan of those costs scheduled longest first
    over `cores` workers, so the rate is histories / makespan.  Both CPU arms
    use this one method and sample."""
    sizes = sorted({tuple(d) for d in cfg["dims"]}, key=lambda d: -d[0] * d[1] * d[2])
    picked = []
    for s in sizes:
        picked += [k for k, d in enumerate(cfg["dims"]) if tuple(d) == s][:CPU_SAMPLE["per_size"]]
    procs = max(1, min(cores, len(picked)))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(k, cfg, CPU_SAMPLE["steps"], CPU_SAMPLE["warm"]) for k in picked], chunksize=1)
    wall = time.perf_counter() - t0
    per = {}
    for k, sec in res:
        per.setdefault(tuple(cfg["dims"][k]), []).append(sec)
    mean = {d: sum(v) / len(v) for d, v in per.items()}
    costs = [mean[tuple(d)] for d in cfg["dims"]]
    span = lpt_makespan(costs, cores)
    detail = {"method": "per-size seconds per MCS from the sample; the campaign's histories scheduled longest "
                        "first over the cores; rate = histories / makespan",
              "sampled_histories": len(picked), "per_size": CPU_SAMPLE["per_size"], "warm": CPU_SAMPLE["warm"],
              "timed_mcs": CPU_SAMPLE["steps"], "processes": procs, "wall_s": round(wall, 2),
              "seconds_per_mcs": {f"{d[0]}x{d[1]}x{d[2]}": round(v, 4) for d, v in mean.items()},
              "makespan_s": round(span, 4), "serial_s": round(sum(costs), 3)}
    sample = (f"{len(picked)} of the {len(cfg['dims'])} histories ({CPU_SAMPLE['per_size']} per size) on the oracle, "
              f"{CPU_SAMPLE['steps']} timed MCS each after {CPU_SAMPLE['warm']} untimed; all {len(cfg['dims'])} "
              f"histories' MCS scheduled longest first over {cores} cores")
    return len(cfg["dims"]) / span, detail, sample


# ------------------------------------------------------------------ our path
def network_for(S, seed, refvol):
    import cellweave_b200 as cw
    from cellweave_b200 import synthetic
    d = tempfile.mkdtemp()
    path = os.path.join(d, f"synthetic-{S}.toml")
    with open(path, "w") as fh:
        fh.write(synthetic.network_toml(S, seed))
    return cw.Network.load(path, refvol)


def event_ms(L, a, b):
    ms = C.c_float()
    L.cw_event_elapsed(a, b, C.byref(ms))
    return ms.value


def run_ours(args, rank, world, dist):
    import numpy as np

    import cellweave_b200 as cw
    from cellweave_b200 import _lib
    L = _lib.lib()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    _lib.check(L.cw_set_device(local))
    cfg = configured(args, rank)
    S = cfg.pop("S")
    net = network_for(S, S, cfg["target_volume"])
    nh = len(cfg["dims"])
    sim = cw.Simulation(net, **cfg)
    sim.step(max(args.warmup, 3) if args.warmup >= 3 else args.warmup)

    def barrier():
        L.cw_synchronize()
        if dist is not None:
            dist.barrier()

    # ---- timed region: K batched steps, device time by events
    barrier()
    clocks = Clocks(local)
    clocks.start()
    l0 = L.cw_launch_count()
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 0)
    sim.step(args.steps)
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 1)
    L.cw_synchronize()
    ms = event_ms(L, 0, 1)
    launches = int(L.cw_launch_count() - l0)
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    value = job_rate(world, nh, args.steps, ms)
    stats = sim.stats()
    gsteps, gmiss, gbudget = sim.graph_info()
    graphs = {"steps_replayed": int(gsteps), "budget_misses": int(gmiss), "outer_budgets": [int(b) for b in gbudget]}
    if args.profile_step:
        _lib.check(L.cw_profiler_start())
        sim.step(1)
        _lib.check(L.cw_profiler_stop())

    # ---- end to end through the C ABI: host grids in, step, grids and stats out
    lat = sim.lattice_handle()
    total = int(sum(w * h * d for (w, h, d) in cfg["dims"]))
    try:
        import torch
        grids = torch.empty(total, dtype=torch.int32, pin_memory=True).numpy()
    except Exception:
        grids = np.empty(total, np.int32)
    _lib.check(L.cw_lattice_download_all(lat, _lib.ptr(grids)))
    st_host = np.empty((nh, 4))
    e2e_steps = max(2, min(args.steps, 5))
    barrier()
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 2)
    for _ in range(e2e_steps):
        _lib.check(L.cw_lattice_upload_all(lat, _lib.ptr(grids)))
        sim.step(1)
        _lib.check(L.cw_lattice_download_all(lat, _lib.ptr(grids)))
        _lib.check(L.cw_sim_stats(sim._h, _lib.ptr(st_host)))
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 3)
    e2e_ms = event_ms(L, 2, 3) / e2e_steps
    bytes_grid = int(grids.nbytes)
    e2e_ms = max_over_ranks(e2e_ms, dist, f"cuda:{local}")
    e2e = {"value": job_rate(world, nh, 1, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": bytes_grid,
           "d2h_bytes_per_step": bytes_grid + st_host.nbytes, "steps": e2e_steps,
           "path": "cw_lattice_upload_all (pinned host grids, checked on the device) + cw_sim_step + "
                   "cw_lattice_download_all + cw_sim_stats"}

    # ---- each field against its FP64 solution (the north star's 1e-6 relative)
    ferr = {"oxygen": field_error(L, sim, 0, cfg["o2_dcoef"], 0.0)}
    if cfg.get("nfields", 1) > 1:
        ferr["signal"] = field_error(L, sim, 1, cfg["signal_dcoef"], cfg["signal_decay"])

    # ---- roofline of the dominant kernel: the FP32 SOR sweep on this batch's oxygen field
    f = sim.field_handle(0)
    tuned = sim.tuning()
    depth, window, sweeps = tuned["depth"], tuned["window"], 32
    sites = int(sum(w * h * d for w, h, d in cfg["dims"]))

    def launch_ms(d):
        kms, kl = C.c_float(), C.c_int64()
        _lib.check(L.cw_field_time_inner(f, sweeps, d, window, 1.9, C.byref(kms), C.byref(kl)))  # warm
        _lib.check(L.cw_field_time_inner(f, sweeps, d, window, 1.9, C.byref(kms), C.byref(kl)))
        return kms.value / kl.value

    per_launch_ms = launch_ms(depth)
    # depth 2: one sweep per launch, so a launch moves exactly one sweep's
    # 16 B/site: the unblocked kernel's fraction of the HBM roofline
    one_sweep_ms = launch_ms(2)
    # one launch is one round trip of correction, right-hand side and inverse
    # diagonal through HBM (16 B/site) for `depth` half-sweeps kept on chip
    alg_bytes_per_launch = sites * SOR_BYTES_PER_SITE_PASS
    achieved = alg_bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    sweep_rate = sites * (depth / 2) / (per_launch_ms / 1e3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    shape = {cw.WINDOW_AUTO: "128x64", cw.WINDOW_TALL: "128x128"}.get(window)
    kname = (f"k_sor32_wide<{depth}> (FP32 red-black SOR, {shape} TMA-fed windows, {depth} half-sweeps per launch "
             f"on chip)" if shape else
             f"k_sor32_tb<{depth}> (FP32 red-black SOR, 64x64 windows, {depth} half-sweeps per launch on chip)")
    one_sweep_gbs = alg_bytes_per_launch / (one_sweep_ms / 1e3) / 1e9
    roofline = {"kernel": kname,
                "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 3),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650",
                "traffic": (int(SOR_TRAFFIC_PER_SITE * sites) if SOR_TRAFFIC_PER_SITE and window == cw.WINDOW_AUTO
                            and depth == 8 else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_sor32_wide<8> launch "
                                  "on this workload, per site, times the sites",
                "alg_bytes_per_launch": int(alg_bytes_per_launch),
                "launch_ms": round(per_launch_ms, 4), "site_sweeps_per_s": sweep_rate,
                "alg_bytes": "16 B per site per launch: the correction and both coefficients read once and the "
                             "correction written once; the launch's half-sweeps stay on chip",
                "per_sweep_equivalent_gbs": round(alg_bytes_per_launch * depth / 2 / (per_launch_ms / 1e3) / 1e9, 1),
                "one_sweep_per_launch": {"launch_ms": round(one_sweep_ms, 4), "achieved": round(one_sweep_gbs, 1),
                                         "frac": round(one_sweep_gbs / peak, 3),
                                         "what": "depth 2: one sweep per launch, 16 B/site moved per sweep"}}

    # ---- the plain path: each history stepped alone (rank 0 at N=1)
    plain = plain_graphs = None
    kinetics4 = None
    if not args.no_plain and world == 1:
        del sim
        # the same batch with four sub-sweeps a step: the update-order kinetics
        # that put driven cells (resorption, growth) inside the reference's band
        s4 = cw.Simulation(net, **dict(cfg, subsweeps=4))
        s4.step(max(args.warmup, 3))
        L.cw_synchronize()
        L.cw_event_record_on(L.cw_sim_get_stream(s4._h), 4)
        n4 = min(args.steps, 10)
        s4.step(n4)
        L.cw_event_record_on(L.cw_sim_get_stream(s4._h), 5)
        L.cw_synchronize()
        kinetics4 = {"value": job_rate(1, nh, n4, event_ms(L, 4, 5)), "unit": UNIT, "subsweeps": 4,
                     "how": "the same batch, every colour swept four times a step with each pixel attempting in "
                            "each with probability 1/4 (Binomial(4, 1/4) attempts a step, near the Poisson(1) of "
                            "random pixels)"}
        del s4

        def one_at_a_time(graphs):
            total_ms, units = 0.0, 0
            for k in range(nh):
                one = {kk: (vv[k:k + 1] if kk in ("dims", "ncells", "seeds") else vv) for kk, vv in cfg.items()}
                s1 = cw.Simulation(net, **one, use_graphs=graphs)
                # warm up through the autotuner's trials (seven candidates, one history)
                while s1.tuning()["tuning"]:
                    s1.step(1)
                s1.step(2)
                n = args.steps if args.steps <= 5 else 5
                L.cw_synchronize()
                L.cw_event_record_on(L.cw_sim_get_stream(s1._h), 4)
                s1.step(n)
                L.cw_event_record_on(L.cw_sim_get_stream(s1._h), 5)
                L.cw_synchronize()
                total_ms += event_ms(L, 4, 5)
                units += n
                del s1
            return units / (total_ms / 1e3)

        plain = {"value": one_at_a_time(False), "unit": UNIT,
                 "how": "the same 64 histories, each its own Simulation stepped alone: one history per launch, "
                        "launched kernel by kernel (the path without the batching form)"}
        plain_graphs = {"value": one_at_a_time(True), "unit": UNIT,
                        "how": "as plain, each history's tuned step replayed from CUDA graphs"}
    shapes = None
    if not args.no_shapes and world == 1:
        from cellweave_b200 import synthetic
        shapes = {"cord2048": shape_record(L, synthetic.tumour_cord(), 10, 4, peak),
                  # nine warm-up steps: the autotuner tries its seven factors on a lone history one step each
                  "spheroid256": shape_record(L, synthetic.spheroid_3d(), 6, 9, peak)}
    fit = None
    if not args.no_fit and world == 1:
        fit = run_fit(args, L)
    return dict(value=value, ms=ms / args.steps, launches=launches, clocks=clk, e2e=e2e, roofline=roofline, fit=fit,
                shapes=shapes, field_error=ferr,
                graphs=graphs, plain_graphs=plain_graphs, kinetics4=kinetics4,
                plain=plain, stats=stats, nh=nh, cfg=cfg, tuned=tuned)


def field_error(L, sim, which, dcoef, decay):
    """Largest |field - FP64 solution| / largest |FP64 solution| over the
    histories of a simulation's field: the FP64 solution is the library's
    FP64 relax (the reference's SOR, bit-exact with it) of the problem the
    field last solved, from the field's values to residual 1e-12."""
    import numpy as np

    import cellweave_b200 as cw
    from cellweave_b200 import _lib
    fh = sim.field_handle(which)
    twin = cw.ScalarField(sim.dims, dcoef, decay, 0.0)
    vals = []
    for k, (w, h, d) in enumerate(sim.dims):
        n = w * h * d
        for arr in (cw.VALUES, cw.UPTAKE, cw.PRODUCTION, cw.LIN_SINK):
            out = np.empty(n)
            _lib.check(L.cw_field_download(fh, k, arr, _lib.ptr(out)))
            if arr == cw.VALUES:
                vals.append(out)
            twin.upload(arr, out, k)
        held = np.empty(n, np.uint8)
        _lib.check(L.cw_field_download_held(fh, k, _lib.ptr(held)))
        twin.set_held(held, k)
    twin.relax(1e-12, 20_000_000, stop=cw.STOP_RESIDUAL, precision=cw.FP64)
    worst = 0.0
    for k in range(len(sim.dims)):
        ref = twin.values(k)
        worst = max(worst, float(np.abs(vals[k] - ref).max() / max(np.abs(ref).max(), 1e-300)))
    return worst


def sor_launch_ms(L, f, depth, window, sweeps=32):
    """Device time of one FP32 sweep launch (depth half-sweeps) on a field's
    current residual, the kernel the solves run, after one warm pass."""
    from cellweave_b200 import _lib
    kms, kl = C.c_float(), C.c_int64()
    _lib.check(L.cw_field_time_inner(f, sweeps, depth, window, 1.9, C.byref(kms), C.byref(kl)))
    _lib.check(L.cw_field_time_inner(f, sweeps, depth, window, 1.9, C.byref(kms), C.byref(kl)))
    return kms.value / kl.value


def shape_record(L, cfg, steps, warm, peak):
    """One of the other benchmark shapes (the 2048^2 cord, the 256^3
    spheroid), stepped alone: ms per step and histories*MCS/s by CUDA events,
    the FP32 sweep's roofline on its oxygen field, one Monte Carlo step of
    its lattice alone, the solves' residual and each field's error."""
    import cellweave_b200 as cw
    from cellweave_b200 import _lib
    cfg = dict(cfg)
    S = cfg.pop("S")
    net = network_for(S, S, cfg["target_volume"])
    t0 = time.perf_counter()
    sim = cw.Simulation(net, **cfg)
    setup_s = time.perf_counter() - t0
    sim.step(warm)
    L.cw_synchronize()
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 8)
    sim.step(steps)
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 9)
    L.cw_synchronize()
    ms = event_ms(L, 8, 9) / steps
    stats = sim.stats()
    rec = {"ms_per_step": round(ms, 3), "value": round(len(cfg["dims"]) * 1e3 / ms, 2), "unit": UNIT,
           "steps": steps, "warmup": warm, "setup_s": round(setup_s, 1), "living_cells": float(stats[:, 0].sum()),
           "residual_max": float(stats[:, 3].max()), "tolerance": cfg["tolerance"]}
    errs = {"oxygen": field_error(L, sim, 0, cfg["o2_dcoef"], 0.0)}
    if cfg.get("nfields", 1) > 1:
        errs["signal"] = field_error(L, sim, 1, cfg["signal_dcoef"], cfg["signal_decay"])
    rec["field_error"] = errs
    # the FP32 sweep on the oxygen field: 16 B per site per launch
    tuned = sim.tuning()
    sites = int(sum(w * h * d for w, h, d in cfg["dims"]))
    volume = any(d > 1 for _, _, d in cfg["dims"])
    depth = 2 if volume else tuned["depth"]
    lm = sor_launch_ms(L, sim.field_handle(0), depth, tuned["window"])
    # a volume's launch is one sweep (two half-sweeps) of tiles marched along
    # z (k_sor32_vol); a plane's, `depth` half-sweeps on chip: 16 B per site a launch
    alg = sites * SOR_BYTES_PER_SITE_PASS
    gbs = alg / (lm / 1e3) / 1e9
    rec["sor"] = {"kernel": ("k_sor32_vol<2, %d> (64x%d tiles marched along z, one sweep per launch)" %
                             ((16, 16) if tuned["window"] == 1 else (32, 32))) if volume else
                  f"k_sor32_wide<{depth}> ({depth} half-sweeps per launch on chip)",
                  "launch_ms": round(lm, 4), "alg_bytes_per_launch": int(alg), "achieved_gbs": round(gbs, 1),
                  "frac": round(gbs / peak, 3)}
    # one Monte Carlo step of the lattice alone (the passes of every colour)
    lat = sim.lattice_handle()
    L.cw_synchronize()
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 8)
    _lib.check(L.cw_lattice_mcs(lat, 1))
    L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 9)
    L.cw_synchronize()
    rec["cpm_mcs_ms"] = round(event_ms(L, 8, 9), 3)
    del sim
    return rec


def run_fit(args, L):
    """The differentiated fit at the cord's scale: the 2048^2 cord stepped to
    MCS 500 and frozen; 2000 RK4 steps checkpointed every 100; parameters D,
    k (three types) and 32 network rates; the target from D = 1.3, k = 0.008.
    Gradient-descent iterations (forward + adjoint + a line-search forward)
    are timed one by one with CUDA events."""
    import numpy as np

    import cellweave_b200 as cw
    cfg = workload("cord")
    S = cfg.pop("S")
    net = network_for(S, S, cfg["target_volume"])
    sim = cw.Simulation(net, **cfg)
    sim.step(500)
    lat = sim.lattice()
    w = cfg["dims"][0][0]
    fit = cw.Fit(lat, net, dcoef=1.0, uptake=(0.01, 0.005, 0.0), vessel_x=w // 2, steps=2000, checkpoint_every=100,
                 dt=0.01, nbins=64, bin_width=w / 128.0, tolerance=1e-8, adjoint_tolerance=1e-10,
                 precision=cw.FP32_DC, network_params=32)
    start = fit.params.copy()
    p = start.copy()
    p[0], p[1:4] = 1.3, 0.008
    fit.params = p
    _, h, g = fit.forward()
    fit.set_target(h, g)
    p = start.copy()
    fit.params = p
    times, losses = [], []
    for _ in range(args.fit_iters):
        L.cw_synchronize()
        L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 6)
        loss, grad = fit.gradient()
        d = -grad * p * p  # steepest descent in log p (a parameter at zero stays there)
        rel = np.abs(d / np.where(p != 0, p, 1.0)).max()
        q = np.maximum(p + 0.05 / (rel + 1e-300) * d, 0.0)
        q[0] = max(q[0], 1e-3)
        fit.params = q
        lq = fit.forward()[0]
        L.cw_event_record_on(L.cw_sim_get_stream(sim._h), 7)
        times.append(event_ms(L, 6, 7) / 1e3)
        losses.append(loss)
        if lq < loss:
            p = q
        fit.params = p
    del fit, lat, sim
    return {"seconds_per_iteration": float(np.median(times)), "iterations": len(times),
            "loss_first": losses[0], "loss_last": losses[-1], "parameters": int(len(start)),
            "workload": "2048^2 cord frozen at MCS 500, 2000 RK4 steps (checkpoints every 100), "
                        "FP32 defect-correction forward and adjoint solves, 1 + 3 + 32 parameters; "
                        "an iteration = forward + adjoint + one line-search forward"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded)"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        cfg = configured(args)
        cores = os.cpu_count() or 1
        v, detail, sample = cpu_sample(cfg, cores)
        line = dict(base, impl="reference", value=v, ms_per_step=1e3 * len(cfg["dims"]) / v,
                    dtype="f64", config=config_key(args.workload, cfg),
                    cpu_baseline={"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                                  "detail": detail},
                    e2e={"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return 0

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the CPU leg first, before any GPU context exists in this process
        cfg = configured(args)
        cores = os.cpu_count() or 1
        v, detail, sample = cpu_sample(cfg, cores)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample, "detail": detail}
    r = run_ours(args, rank, world, dist)
    if rank == 0:
        line = dict(base, value=r["value"], ms_per_step=r["ms"], dtype="f32+f64",
                    config=config_key(args.workload, r["cfg"]), clocks=r["clocks"], e2e=r["e2e"],
                    gpu_launches=r["launches"], roofline=r["roofline"], cpu_baseline=cpu,
                    plain=r["plain"], plain_with_graphs=r["plain_graphs"],
                    batched_over_plain=(r["value"] / r["plain"]["value"]) if r["plain"] else None,
                    fit=r["fit"], shapes=r["shapes"], field_error=r["field_error"], cuda_graphs=r["graphs"],
                    subsweeps4=r["kinetics4"],
                    sor_gbs=r["roofline"]["achieved"], sor_site_sweeps_per_s=r["roofline"]["site_sweeps_per_s"],
                    living_cells=float(r["stats"][:, 0].sum()), last_residual_max=float(r["stats"][:, 3].max()),
                    autotuned={"omega_o2": sorted(set(float(v) for v in r["tuned"]["omega_o2"])),
                               "omega_signal": sorted(set(float(v) for v in r["tuned"]["omega_signal"])),
                               "depth": r["tuned"]["depth"]})
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

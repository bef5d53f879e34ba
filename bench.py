#!/usr/bin/env python3
"""Benchmark: 24^3 x 64 Iwasaki (beta = 2.13, c1 = -0.331) pure-gauge HMC,
force-gradient integrator with 8 steps per unit trajectory, on one B200 per
rank.  One "step" is one full trajectory (momentum refresh, molecular
dynamics, both Hamiltonians, Metropolis) through the qlat-compatible API.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is trajectories/s of the mixed form
(FP32 molecular dynamics, FP64 Hamiltonians, FP64 re-unitarisation every 4
steps), summed over ranks (independent chains, one per GPU: the path has no
cross-chain exchange, so multi-GPU runs are replicas).  The plain FP64 form is
timed in the same run, from the same start with the same momenta, and
reported beside it; `delta_h` compares the two forms over the same
trajectories (bench_suite.leg_matched).  Untimed relative to `value`, the line
also carries the other workloads: `c1` (8^4 Wilson leapfrog), `c3` (32^4
Wilson flow), `c4` (flow adjoint at 16^4) and `c5` (256 batched chains), each
timed on the device by itself (bench_suite.py).

`e2e` is the same trajectory through the public API with the configuration in
pinned host memory: every step uploads it (qgb_field_upload_pipelined),
runs the trajectory, reads delta_h and the plaquette back, and downloads the
updated configuration (qgb_field_download_async); all copies are inside the
timed region.

`--impl reference` times the reference Qlattice CPU implementation (built
from source into oracle/_ref by oracle/ref/Makefile) on this host's cores:
whole force-gradient trajectories of the same workload (oracle/_ref/ref_chain),
with the per-pair extrapolation of oracle/_ref/ref_bench as a cross-check.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LATTICE = (24, 24, 24, 64)
BETA, C1 = 2.13, -0.331
N_STEP = 8
SIGMA = 0.3
SEED = "b200-c2-24x64-iwasaki"
METRIC = "24^3x64 Iwasaki HMC traj/s (force-gradient, 8 steps/traj; mixed FP32/FP64)"


def workload_config(lattice, world):
    """The `config` of the bench line, the same for both arms."""
    V = 1
    for v in lattice:
        V *= v
    return {"workload": f"{'x'.join(map(str, lattice))} Iwasaki beta=2.13 c1=-0.331, force-gradient "
                        f"n_step=8 md_time=1, one chain per GPU", "lattice": list(lattice), "sites": V,
            "l2_policy": f"inputs larger than L2 (FP64 links {V * 576 / 1e6:.1f} MB, FP32 "
                         f"{V * 288 / 1e6:.1f} MB per chain; L2 126 MB)",
            "parallelism": f"replicas x{world}"}


def metric_for(lattice):
    """The metric's name for a lattice (the default lattice gives METRIC)."""
    X, Y, Z, T = lattice
    head = f"{X}^3x{T}" if X == Y == Z else f"{X}x{Y}x{Z}x{T}"
    return METRIC.replace("24^3x64", head, 1)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--lattice", type=str, default=",".join(map(str, LATTICE)))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the c1/c3/c4/c5 and matched-delta_h legs")
    ap.add_argument("--ref-trajs", type=int, default=2, help="whole reference trajectories (--impl reference)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# reference arm / CPU baseline (oracle/_ref: the reference's own C++ library)

def reference_arm(args):
    import bench_suite as S
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lattice = tuple(int(v) for v in args.lattice.split(","))
    if S.ref_exe("ref_chain") is None or S.ref_exe("ref_bench") is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref drivers not built "
                          "(the reference sources were not present when build() ran)"}))
        return 0
    threads = os.cpu_count() or 1
    # warm-up: one set_gm_force + gf_evolve pair (first-touch allocations, thread pool)
    S.reference_pairs(lattice, BETA, C1, SIGMA, 1, threads)
    # timed: whole trajectories, each run from its own start (every step is one trajectory)
    n = max(1, args.ref_trajs)
    traj_s, rows, nthreads, wall = S.reference_trajectories(lattice, BETA, C1, N_STEP, SIGMA, SEED, n, threads)
    # cross-check: the per-pair extrapolation (32 force + evolve pairs and the ends)
    _, pair_traj_s, _ = S.reference_pairs(lattice, BETA, C1, SIGMA, 2, threads)
    value = 1.0 / traj_s
    sample = (f"{n} whole force-gradient trajectories of {'x'.join(map(str, lattice))} (momenta, 32 set_gm_force, "
              f"33 gf_evolve, 2 x H, unitarize, Metropolis; hmc.pyx:169-216 through the reference library), "
              f"{wall:.0f} s of CPU work")
    print(json.dumps({
        "impl": "reference", "metric": metric_for(lattice), "value": value, "unit": "traj/s", "n_gpus": 0,
        "steps": n, "warmup": 1, "ms_per_step": traj_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded hot start set_rand(sigma=0.3)",
        "config": workload_config(lattice, 1),
        "cpu_baseline": {"value": value, "unit": "traj/s", "cores": nthreads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "detail": {"seconds_per_trajectory": [r["seconds"] for r in rows],
                   "delta_h": [r["delta_h"] for r in rows],
                   "per_pair_extrapolation_traj_per_s": 1.0 / pair_traj_s,
                   "steps_note": "the reference arm times --ref-trajs whole trajectories; --steps is not used"},
    }))
    return 0


# ---------------------------------------------------------------------------
# our arm

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.splitlines():
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(lattice):
    """Bounded sample of the reference CPU code on this host (rank 0, N = 1):
    2 set_gm_force + gf_evolve pairs and the trajectory ends, extrapolated to
    a trajectory (32 pairs + ends); --impl reference times whole trajectories."""
    import bench_suite as S
    threads = os.cpu_count() or 1
    res = S.reference_pairs(lattice, BETA, C1, SIGMA, 2, threads)
    if res is None:
        return {"value": None, "unit": "traj/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_bench not built"}
    r, traj_s, wall = res
    return {"value": 1.0 / traj_s, "unit": "traj/s", "cores": r["threads"], "kind": "reference",
            "sample": f"2 x (set_gm_force + gf_evolve) + trajectory ends on {'x'.join(map(str, lattice))}, "
                      f"extrapolated to 32 pairs + ends per trajectory ({wall:.1f} s of CPU work)"}


def flags_str(fl):
    return "".join("A" if f else "r" for f in fl)


def max_over_ranks(ms: float, dist, device) -> float:
    """The slowest rank's time: every rank passes its own CUDA-event time and
    gets the maximum back (all ranks must call it, in the same order)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, units_per_rank: int, ms: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank in at most ms."""
    return world * units_per_rank / (ms / 1e3)


def our_arm(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from qlat_b200 import build as B
    B.build()
    import qlat_b200 as q
    q.set_device(torch.cuda.current_device())
    # one non-default stream for torch and the library: the legacy default
    # stream cannot be captured, so trajectories replay as CUDA graphs only here
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    q.set_stream(stream.cuda_stream)

    lattice = tuple(int(v) for v in args.lattice.split(","))
    V = 1
    for v in lattice:
        V *= v
    geo = q.Geometry(lattice)
    ga = q.GaugeAction(BETA, C1)
    rs = q.RngState(SEED).split(f"rank-{rank}")
    gf = q.GaugeField(geo)
    gf.set_rand(rs.split("gf-init"), SIGMA, 1)
    gf0 = q.GaugeField(geo)
    gm = q.GaugeMomentum(geo)
    # autotune the force-kernel launch shape for both precisions (untimed)
    tuned = {"fp64": q.autotune_force(gf, C1, 5)}
    g32 = gf.copy(precision=q.F32)
    tuned["fp32"] = q.autotune_force(g32, C1, 5)
    del g32
    # the FP32 FMA rate of this GPU (chains of scalar FFMA), the compute
    # roofline of the force kernel (untimed)
    fma_peak = ctypes.c_double()
    q._lib.call("qgb_fma_rate", 0, 3, ctypes.byref(fma_peak))

    def trajectory(g, traj, precision):
        """run_hmc_pure_gauge (hmc.pyx:190-216) on the chain state g."""
        nonlocal gf0
        r = rs.split(f"{traj}")
        gf0 @= g
        gm.set_rand(r.split("set_rand_gauge_momentum"), 1.0)
        dh = q.run_hmc_evolve_pure_gauge(gm, gf0, ga, r, N_STEP, 1.0, precision=precision, reunit_interval=4)
        flag, _ = q.metropolis_accept(dh, traj, r.split("metropolis_accept"))
        if flag:
            g @= gf0
        return dh, flag

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(g, n, precision, first_traj, prof=False):
        dhs, flags = [], []
        barrier()
        torch.cuda.synchronize()
        if prof:
            q.prof_reset()
            q.prof_enable(True)
        l0 = q.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # an NVTX range per form, so a profiler can select the timed launches (ncu --nvtx-include timed_mixed/)
        torch.cuda.nvtx.range_push(f"timed_{precision}")
        e0.record(stream)
        for i in range(n):
            dh, fl = trajectory(g, first_traj + i, precision)
            dhs.append(dh)
            flags.append(fl)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if prof:
            q.prof_enable(False)
        launches = q.launch_count() - l0
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
        return ms, dhs, flags, launches

    # warm-up: W trajectories of each form (the chain evolves; all later runs start from its end)
    traj = 0
    for _ in range(max(args.warmup, 3)):
        traj += 1
        trajectory(gf, traj, "mixed")
    for _ in range(max(args.warmup, 3)):
        traj += 1
        trajectory(gf, traj, "fp64")
    start = gf.copy()
    first = traj + 1

    # timed: both forms from the same start, trajectories first..first+K-1 (same momenta)
    g_mixed = start.copy()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms_mixed, dh_mixed, fl_mixed, launches = timed(g_mixed, args.steps, "mixed", first, prof=True)
    clk = clocks.stop()
    prof = {k: q.prof_get(k) for k in ("force_update_evolve", "force_evolve", "corners", "evolve", "reduce", "rng",
                                          "convert", "unitarize")}
    g_fp64 = start.copy()
    ms_fp64, dh_fp64, fl_fp64, _ = timed(g_fp64, args.steps, "fp64", first)
    del g_mixed, g_fp64

    # the two forms over the same trajectories: chains from the same start with the same momenta, and the
    # mixed trajectory from every state of the FP64 chain (untimed)
    matched = None
    if not args.no_extra:
        import bench_suite as S
        matched = S.leg_matched(q, start, ga, rs, first, max(20, args.steps), N_STEP)

    # end to end through the public API: host gauge configuration in pinned
    # memory uploaded every step, trajectory, delta_h + plaquette read back,
    # the updated configuration downloaded.  The uploads go through
    # qgb_field_upload_pipelined: each step commits its configuration
    # (prefetched by the step before; the first is copied when it is
    # committed) and starts the next step's host-to-device copy, which then
    # runs on a copy engine under the trajectory; the downloads go through
    # qgb_field_download_async (converted into a staging slot, then copied to
    # the host on the other copy engine under the next step).  Every copy is
    # inside the timed region: the end waits for the last download.
    e2e = None
    if not args.no_e2e:
        host_in = torch.empty((V, 4, 3, 3), dtype=torch.complex128, pin_memory=True)
        host_in.numpy()[...] = start.to_numpy()
        host_out = [torch.empty((V, 4, 3, 3), dtype=torch.complex128, pin_memory=True) for _ in range(2)]
        n_e2e = max(2, args.steps)  # the same number of trajectories as the device-resident measurement
        g_e2e = q.GaugeField(geo)
        # allocate the staging slots outside the timed region (no prefetch left pending)
        g_e2e.upload_host_pipelined(host_in.data_ptr(), host_in.data_ptr())
        g_e2e.upload_host_pipelined(host_in.data_ptr(), None)
        for h in host_out:
            g_e2e.download_host_async(h.data_ptr())
        q.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plaqs = []
        for i in range(n_e2e):
            g_e2e.upload_host_pipelined(host_in.data_ptr(), host_in.data_ptr() if i + 1 < n_e2e else None)
            trajectory(g_e2e, first + i, "mixed")
            plaqs.append(q.gf_avg_plaq(g_e2e))
            g_e2e.download_host_async(host_out[i % 2].data_ptr())
        q.download_join()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
        ok = bool(np.array_equal(host_out[(n_e2e - 1) % 2].numpy(), g_e2e.to_numpy()))
        e2e = {"value": job_throughput(world, n_e2e, ms_e2e), "unit": "traj/s", "steps": n_e2e,
               "h2d_bytes_per_step": V * 4 * 9 * 16, "d2h_bytes_per_step": V * 4 * 9 * 16 + 8 * 2 + 8 * 6,
               "download_matches_device": ok,
               "copies": "pinned host; per step one full FP64 configuration up (prefetched under the previous "
                         "trajectory, copy stream, two staging slots; the first one is not overlapped) and the "
                         "updated configuration down (staging slot, download stream, overlapping the next step), "
                         "plus delta_h and the plaquette"}
        del g_e2e

    extra = {}
    if not args.no_extra and rank == 0:
        import bench_suite as S
        for name, fn in (("c1", S.leg_c1), ("c3", S.leg_c3), ("c4", S.leg_c4), ("c5", S.leg_c5)):
            extra[name] = fn(q)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    value = job_throughput(world, args.steps, ms_mixed)
    fp64_value = job_throughput(world, args.steps, ms_fp64)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    # dominant kernel: the force-gradient step's fused force + momentum update +
    # link update (FP32, Iwasaki): reads U' (288 B/site), P and U (288 B/site
    # each), writes P and U (288 B/site each); with the corner field (site map
    # 5) it also reads the 16 two-link products per site (1152 B/site), which
    # the corner pass writes from U' (reads 288, writes 1152 B/site)
    fp32_map = q.force_variants()[tuned["fp32"][0]]["site_map"]
    t_fu, n_fu = prof["force_update_evolve"]
    bytes_fu = (1440.0 + (1152.0 if fp32_map == 5 else 0.0)) * V
    achieved = bytes_fu / (t_fu / n_fu / 1e3) / 1e9 if n_fu else None
    t_co, n_co = prof["corners"]
    corners = None
    if n_co:
        a_co = 1440.0 * V / (t_co / n_co / 1e3) / 1e9
        corners = {"kernel": "k_corners (the 16 two-link products per site of U', FP32)", "bound": "hbm",
                   "mean_launch_ms": t_co / n_co, "algorithmic_bytes_per_launch": 1440.0 * V, "achieved": a_co,
                   "peak": hbm, "unit": "GB/s", "frac": a_co / hbm}
    # flops of the staple sum + force counted as 67 full SU(3) products per link
    # at 198 flop each (the FP32 kernel carries link chains as two rows and
    # does fewer)
    flops_site = 4 * (6 * 11 + 1) * 198.0
    tflops = flops_site * V / (t_fu / n_fu / 1e3) / 1e12 if n_fu else None
    traffic = None
    tf_path = os.path.join(ROOT, "profiles", "force_update_evolve_traffic.json")
    if os.path.exists(tf_path):
        try:
            traffic = json.load(open(tf_path)).get("bytes_per_launch_full_size")
        except Exception:
            traffic = None
    out = {
        "metric": metric_for(lattice), "value": value, "unit": "traj/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (MD) + f64 (H, unitarize)",
        "data": "synthetic: seeded hot start set_rand(RngState('b200-c2-24x64-iwasaki').split('gf-init'), 0.3)",
        "config": workload_config(lattice, world),
        "fp64_traj_per_s": fp64_value, "mixed_over_fp64": value / fp64_value,
        "link_updates_per_s": value * 4 * V * N_STEP,
        "delta_h": {"timed_mixed": {"mean": statistics.fmean(dh_mixed), "accepts": flags_str(fl_mixed)},
                    "timed_fp64": {"mean": statistics.fmean(dh_fp64), "accepts": flags_str(fl_fp64)},
                    "timed_max_abs_diff": max(abs(a - b) for a, b in zip(dh_mixed, dh_fp64)),
                    "same_trajectories": matched},
        "roofline": {"kernel": "force_update_evolve (FP32 Iwasaki force fused with P += dt F and U = exp(eps P) U)",
                     "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_launch": bytes_fu, "mean_launch_ms": t_fu / n_fu if n_fu else None,
                     "fp32_tflops_achieved": tflops, "flops_per_site": flops_site,
                     "note": "compute-bound on CUDA cores (FP32); HBM fraction is reported as the metric asks",
                     "compute": {"achieved": tflops, "peak": fma_peak.value, "unit": "TFLOP/s",
                                 "frac": (tflops / fma_peak.value) if tflops and fma_peak.value else None,
                                 "peak_source": "FP32 FFMA chains measured in this run (qgb_fma_rate)"},
                     "corner_pass": corners},
        "kernel_ms_per_traj": {k: v[0] / args.steps for k, v in prof.items()},
        "force_variant": {k: {"variant": v[0], "ms": v[1], **q.force_variants()[v[0]]} for k, v in tuned.items()},
        "clocks": clk, "gpu_launches": launches,
        **extra,
    }
    if e2e:
        out["e2e"] = e2e
    if not args.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline(lattice)
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())

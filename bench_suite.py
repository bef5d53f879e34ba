#!/usr/bin/env python3
"""Measurement legs that bench.py adds to its JSON line, and small-case
drivers for ncu captures.

Each leg times its workload on the device (CUDA events on the library's
stream, after warm-up) and returns a dict:

    leg_matched(q, ...)   the mixed and FP64 forms over the same trajectories:
                          both chains from one start with the same momenta
                          (each form's own Metropolis), and the mixed
                          trajectory re-run from every state of the FP64 chain
    leg_c1(q)             8^4 Wilson beta = 5.5 leapfrog, 6 steps, hot start at
                          scale 1 (trajectories/s, both forms)
    leg_c3(q)             32^4 Wilson flow, RK3 eps = 0.05 x 80 steps, t^2 E and
                          the clover charge every 4 steps; FP32 against FP64
    leg_c4(q)             16^4, backward through 40 Wilson-flow steps with
                          checkpoints every 8 (forward + backward time)
    leg_c5(q)             256 Wilson chains (64 each of 4^4, 6^4, 8^4, 12^4) in
                          one batch, leapfrog with 10 steps: link updates/s and
                          the per-chain plaquette of the mixed form against FP64
    reference_trajectories(...)
                          whole force-gradient trajectories of the reference
                          library (oracle/_ref/ref_chain) on this host's cores

Command line (one JSON line each; the profile-* commands run one small case
of one kernel family, for ncu -k captures):

    python bench_suite.py c1|c3|c4|c5
    python bench_suite.py functions hmc|flow [--reps 20]
    python bench_suite.py slabs [--lattice 24,24,24,64] [--precision mixed|fp64] [--halo 4|2]
    python bench_suite.py profile-force [--lattice 24,24,24,48] [--variants 10,14] [--c1 -0.331]
    python bench_suite.py profile-flow [--lattice 32,32,32,32] [--steps 4]
    python bench_suite.py profile-hmc [--lattice 24,24,24,48] [--trajs 1] [--fp32-variant V]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _lattice(s):
    return tuple(int(v) for v in s.split(","))


class DeviceTimer:
    """CUDA events around a region (milliseconds), on torch's current stream,
    which the caller has made the library's stream (q.set_stream)."""

    def __init__(self, q):
        import torch
        self.torch = torch
        self.q = q
        self.stream = torch.cuda.current_stream()

    def __enter__(self):
        self.q.synchronize()
        self.e0 = self.torch.cuda.Event(enable_timing=True)
        self.e1 = self.torch.cuda.Event(enable_timing=True)
        self.e0.record(self.stream)
        return self

    def __exit__(self, *exc):
        self.e1.record(self.stream)
        self.e1.synchronize()
        self.q.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


def _flags(fl):
    return "".join("A" if f else "r" for f in fl)


def _mean_sem(xs):
    m = statistics.fmean(xs)
    s = statistics.stdev(xs) / len(xs) ** 0.5 if len(xs) > 1 else None
    return m, s


# ---------------------------------------------------------------------------
# C2: the mixed and FP64 forms over the same trajectories

def leg_matched(q, gf_start, ga, rs, first_traj, n_traj, n_step, reunit_interval=4):
    """Both forms as chains of n_traj trajectories from gf_start, trajectory t
    drawing its momenta from rs.split(f"{t}") (run_hmc_pure_gauge,
    hmc.pyx:190-216) and deciding with its own Metropolis step; then, at every
    state of the FP64 chain, the mixed trajectory from that state with the
    same momenta (matched delta_h).  Untimed."""
    out = {"trajectories": n_traj, "first_traj": first_traj}
    chains = {}
    for prec in ("mixed", "fp64"):
        g = gf_start.copy()
        dhs, fl = [], []
        for t in range(first_traj, first_traj + n_traj):
            f, dh = q.run_hmc_pure_gauge(g, ga, t, rs, n_step=n_step, precision=prec,
                                         reunit_interval=reunit_interval)
            dhs.append(dh)
            fl.append(f)
        chains[prec] = (dhs, fl, q.gf_avg_plaq(g))
        m, s = _mean_sem(dhs)
        mexp, sexp = _mean_sem([2.718281828459045 ** (-d) for d in dhs])
        out[f"{prec}_chain"] = {"delta_h_mean": m, "delta_h_sem": s, "exp_minus_delta_h_mean": mexp,
                                "exp_minus_delta_h_sem": sexp, "accepts": _flags(fl),
                                "accept_rate": sum(fl) / len(fl), "plaq_end": chains[prec][2]}
    # matched: the mixed trajectory from each state of the FP64 chain
    g = gf_start.copy()
    diffs, fl_m, fl_64 = [], [], []
    for t in range(first_traj, first_traj + n_traj):
        r = rs.split(f"{t}")
        gm = q.GaugeMomentum(g.geo)
        gm.set_rand(r.split("set_rand_gauge_momentum"), 1.0)
        g64, g32 = g.copy(), g.copy()
        dh64 = q.run_hmc_evolve_pure_gauge(gm.copy(), g64, ga, r, n_step, 1.0, precision="fp64")
        dhmx = q.run_hmc_evolve_pure_gauge(gm.copy(), g32, ga, r, n_step, 1.0, precision="mixed",
                                           reunit_interval=reunit_interval)
        f64, _ = q.metropolis_accept(dh64, t, r.split("metropolis_accept"))
        fmx, _ = q.metropolis_accept(dhmx, t, r.split("metropolis_accept"))
        diffs.append(abs(dhmx - dh64))
        fl_64.append(f64)
        fl_m.append(fmx)
        if f64:
            g @= g64
    out["matched"] = {"max_abs_delta_h_diff": max(diffs), "mean_abs_delta_h_diff": statistics.fmean(diffs),
                      "decisions_fp64": _flags(fl_64), "decisions_mixed_at_fp64_states": _flags(fl_m),
                      "decisions_agree": sum(a == b for a, b in zip(fl_64, fl_m)),
                      "replay_equals_fp64_chain": _flags(fl_64) == out["fp64_chain"]["accepts"]}
    return out


# ---------------------------------------------------------------------------
# C1

def leg_c1(q, n_traj=10):
    """8^4 Wilson beta = 5.5 leapfrog, 6 steps per unit trajectory, hot start
    at scale 1 (RngState('b200-c1-8x4-wilson').split('gf-init')), through
    run_hmc_pure_gauge; device time per trajectory.  The n_traj trajectories
    run three times from the same start with the same random streams: untimed
    (the library records its trajectory graphs), timed with graph replay (the
    default), and timed with the kernels launched one by one."""
    ts = (8, 8, 8, 8)
    ga = q.GaugeAction(5.5, 0.0)
    out = {"lattice": list(ts), "beta": 5.5, "integrator": "leapfrog", "n_step": 6, "trajectories": n_traj}
    for prec in ("fp64", "mixed"):
        rs = q.RngState("b200-c1-8x4-wilson")
        gf = q.GaugeField(q.Geometry(ts))
        gf.set_rand(rs.split("gf-init"), 1.0, 1)
        start = gf.copy()

        def chain():
            nonlocal gf
            gf @= start
            fl = []
            with DeviceTimer(q) as tm:
                for t in range(1, n_traj + 1):
                    f, _ = q.run_hmc_pure_gauge(gf, ga, t, rs.split("hmc"), n_step=6, integrator="leapfrog",
                                                precision=prec)
                    fl.append(f)
            return tm.ms, fl

        chain()
        ms, fl = chain()
        plaq = q.gf_avg_plaq(gf)
        q.set_trajectory_graphs(False)
        ms_direct, fl_direct = chain()
        q.set_trajectory_graphs(True)
        assert fl_direct == fl
        out[prec] = {"traj_per_s": n_traj / (ms / 1e3), "ms_per_traj": ms / n_traj, "accepts": _flags(fl),
                     "plaq_end": plaq, "graph_replay": True,
                     "direct_launches": {"ms_per_traj": ms_direct / n_traj, "plaq_end": q.gf_avg_plaq(gf)}}
    return out


# ---------------------------------------------------------------------------
# C3

def leg_c3(q, lattice=(32, 32, 32, 32), steps=80, every=4, eps=0.05, sigma=0.5):
    """Wilson flow of the hot start set_rand(RngState('b200-c3-32x32-flow')
    .split('gf-init'), sigma, 1): RK3 steps of eps, t^2 E(t) (clover energy
    density) and the clover charge Q every `every` steps, in FP64 and with
    FP32 links (FP64 reductions)."""
    geo = q.Geometry(lattice)
    gf = q.GaugeField(geo)
    gf.set_rand(q.RngState("b200-c3-32x32-flow").split("gf-init"), sigma, 1)
    out = {"lattice": list(lattice), "eps": eps, "steps": steps, "measure_every": every,
           "hot_start": {"sigma": sigma, "n_step": 1}}
    series = {}
    for name, prec in (("fp64", q.F64), ("fp32", q.F32)):
        w = gf.copy(precision=prec)
        q.gf_wilson_flow_step(w, eps, c1=0.0)
        del w
        g = gf.copy(precision=prec)
        t2e, topo = [], []
        with DeviceTimer(q) as tm:
            for i in range(steps):
                q.gf_wilson_flow_step(g, eps, c1=0.0)
                if (i + 1) % every == 0:
                    t = (i + 1) * eps
                    t2e.append(t * t * q.gf_energy_density(g))
                    topo.append(q.gf_topology_clf(g))
        series[name] = (t2e, topo)
        out[name] = {"ms_total": tm.ms, "ms_per_step_incl_measurements": tm.ms / steps,
                     "t2E_final": t2e[-1], "Q_final": topo[-1]}
        g2 = gf.copy(precision=prec)
        with DeviceTimer(q) as tm:
            for i in range(steps):
                q.gf_wilson_flow_step(g2, eps, c1=0.0)
        out[name]["ms_per_step"] = tm.ms / steps
    a, b = series["fp32"], series["fp64"]
    out["fp32_vs_fp64"] = {"max_rel_t2E": max(abs(x - y) / abs(y) for x, y in zip(a[0], b[0]) if y != 0),
                           "max_abs_Q": max(abs(x - y) for x, y in zip(a[1], b[1]))}
    out["fp32_over_fp64_speed"] = out["fp64"]["ms_per_step"] / out["fp32"]["ms_per_step"]
    return out


# ---------------------------------------------------------------------------
# C4

def leg_c4(q, lattice=(16, 16, 16, 16), steps=40, every=8, eps=0.05, beta=5.8, sigma=0.4):
    """Loss = Wilson gauge action (beta) of the field flowed by `steps` RK3
    steps of eps from set_rand(RngState('b200-c4-adjoint').split('gf-init'),
    sigma, 1); gradient by the hand-written adjoint with checkpoints every
    `every` steps.  Device time of forward + backward and of forward only."""
    gf = q.GaugeField(q.Geometry(lattice))
    gf.set_rand(q.RngState("b200-c4-adjoint").split("gf-init"), sigma, 1)
    q.gf_flow_action_grad(gf, eps, steps, beta, checkpoint_every=every)
    q.gf_flow_action(gf, eps, steps, beta)
    with DeviceTimer(q) as tm:
        q.gf_flow_action_grad(gf, eps, steps, beta, checkpoint_every=every)
    fb = tm.ms
    with DeviceTimer(q) as tm:
        q.gf_flow_action(gf, eps, steps, beta)
    return {"lattice": list(lattice), "eps": eps, "steps": steps, "checkpoint_every": every, "beta_loss": beta,
            "ms_forward_and_backward": fb, "ms_forward_only": tm.ms, "backward_over_forward": fb / tm.ms}


# ---------------------------------------------------------------------------
# C5

def leg_c5(q, per_size=64, n_step=10, n_traj=10, warmup=5):
    """256 independent Wilson chains, 64 each of 4^4, 6^4, 8^4, 12^4, betas
    evenly spaced in [5.6, 6.2], hot starts at scale 1, leapfrog with n_step
    steps of total length 1; every phase one launch over all chains, each
    trajectory one CUDA graph.  The warm-up trajectories are always accepted."""
    import numpy as np
    sizes = [(L, L, L, L) for L in (4, 6, 8, 12) for _ in range(per_size)]
    n = len(sizes)
    betas = list(np.linspace(5.6, 6.2, n))
    rs = [q.RngState("b200-c5-batch").split(f"chain-{c}") for c in range(n)]
    sites = int(sum(int(np.prod(s)) for s in sizes))
    out = {"chains": n, "sites": sites, "n_step": n_step, "trajectories": n_traj}
    plaqs = {}
    for prec in ("mixed", "fp64"):
        b = q.ChainBatch(sizes, betas)
        b.set_rand([r.split("gf-init") for r in rs], 1.0, 1)
        tuned = b.autotune(prec)  # the batched force's launch shape (untimed)
        for t in range(1, warmup + 1):
            b.run_hmc(t, rs, n_step, precision=prec, is_always_accept=True)
        acc = 0
        with DeviceTimer(q) as tm:
            for t in range(warmup + 1, warmup + 1 + n_traj):
                flags, _ = b.run_hmc(t, rs, n_step, precision=prec)
                acc += sum(flags)
        link_updates = 4 * sites * n_step * n_traj
        out[prec] = {"ms_per_traj": tm.ms / n_traj, "link_updates_per_s": link_updates / (tm.ms / 1e3),
                     "accept_rate": acc / (n * n_traj), "force_variant": tuned[0], "force_ms": tuned[1]}
        # the same proposals as one CUDA-graph replay and as direct launches: what a
        # single persistent launch could at most save is the difference
        direct = {}
        for use_graph in (True, False):
            m = [r.split("graph-check").split("set_rand_gauge_momentum") for r in rs]
            b.trajectory(m, n_step, precision=prec, use_graph=use_graph)
            l0 = q.launch_count()
            with DeviceTimer(q) as tm:
                for _ in range(n_traj):
                    b.trajectory(m, n_step, precision=prec, use_graph=use_graph)
            direct["graph" if use_graph else "direct"] = {"ms_per_proposal": tm.ms / n_traj,
                                                          "kernels_per_proposal": (q.launch_count() - l0) / n_traj}
        out[prec]["proposal_graph_vs_direct"] = direct
        plaqs[prec] = b.plaq()
        del b
    d = np.abs(plaqs["mixed"] - plaqs["fp64"])
    out["plaq_mixed_vs_fp64"] = {"max_abs": float(d.max()), "mean_abs": float(d.mean())}
    return out


# ---------------------------------------------------------------------------
# the reference library on this host's cores

def ref_exe(name):
    p = os.path.join(ROOT, "oracle", "_ref", name)
    return p if os.path.exists(p) else None


def reference_trajectories(lattice, beta, c1, n_step, sigma, seed, n_traj, threads):
    """Whole trajectories of the reference library (oracle/_ref/ref_chain:
    run_hmc_pure_gauge, hmc.pyx:169-216, through the reference's own
    set_gm_force / gf_evolve / gm_hamilton_node / gf_hamilton_node /
    unitarize), force-gradient, from the hot start set_rand(sigma).
    Returns (seconds per trajectory, rows, threads, wall seconds)."""
    exe = ref_exe("ref_chain")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), q_verbose="-1")
    t0 = time.time()
    out = subprocess.run([exe, *map(str, lattice), repr(beta), repr(c1), "fg", str(n_step), "1.0", seed,
                          f"hot:{sigma!r}:1", str(n_traj), str(n_traj)], capture_output=True, text=True, env=env,
                         check=True).stdout
    wall = time.time() - t0
    rows = [json.loads(ln) for ln in out.splitlines() if ln.startswith("{\"")]
    head, trajs = rows[0], rows[1:]
    return statistics.fmean(r["seconds"] for r in trajs), trajs, head["threads"], wall


def reference_pairs(lattice, beta, c1, sigma, samples, threads):
    """The per-pair sample of the reference library (oracle/_ref/ref_bench):
    the trajectory ends once and `samples` set_gm_force + gf_evolve pairs; a
    force-gradient trajectory with 8 steps is 32 such pairs plus the ends."""
    exe = ref_exe("ref_bench")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), q_verbose="-1")
    t0 = time.time()
    out = subprocess.run([exe, *map(str, lattice), str(beta), str(c1), str(sigma), str(samples)],
                         capture_output=True, text=True, env=env, check=True).stdout
    wall = time.time() - t0
    r = json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])
    return r, 32 * r["t_force_evolve"] + r["t_ends"], wall


# ---------------------------------------------------------------------------
# single API functions, as a user calls them

def functions(q, which, reps=20, lattice=None):
    """Seconds per call of single API functions (launch, kernels and, for the
    scalar results, the read-back; a synchronisation after every call) on the
    hot start set_rand(RngState(name).split('gf-init'), sigma, 1).  hmc: 24^3 x 64
    Iwasaki set_gm_force, gf_evolve, the Hamiltonians, the momentum draw,
    unitarize, gf_avg_plaq (the autotuner first); flow: 32^4 RK3 Wilson flow
    step, energy density, clover and 5-loop charges."""
    hmc = which == "hmc"
    ts = lattice or ((24, 24, 24, 64) if hmc else (32, 32, 32, 32))
    rs = q.RngState("b200-c2-24x64-iwasaki" if hmc else "b200-c3-32x32-flow")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 0.3 if hmc else 0.5, 1)
    out = {"set": which, "lattice": list(ts), "reps": reps}

    def per_call(fn):
        for _ in range(2):
            fn()
        q.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
            q.synchronize()
        return (time.perf_counter() - t0) / reps

    if hmc:
        ga = q.GaugeAction(2.13, -0.331)
        q.autotune_force(gf, ga.c1())
        gm = q.GaugeMomentum(gf.geo)
        gm.set_rand(rs.split("1").split("set_rand_gauge_momentum"), 1.0)
        force = q.GaugeMomentum(gf.geo)
        out["set_gm_force"] = per_call(lambda: q.set_gm_force(force, gf, ga))
        out["gf_evolve"] = per_call(lambda: q.gf_evolve(gf, gm, 1e-3))
        out["gm_hamilton_node"] = per_call(lambda: q.gm_hamilton_node(gm))
        out["gf_hamilton_node"] = per_call(lambda: q.gf_hamilton_node(gf, ga))
        out["set_rand_gauge_momentum"] = per_call(
            lambda: gm.set_rand(rs.split("2").split("set_rand_gauge_momentum"), 1.0))
        out["unitarize"] = per_call(lambda: q.unitarize(gf))
        out["gf_avg_plaq"] = per_call(lambda: q.gf_avg_plaq(gf))
    else:
        out["gf_wilson_flow_step"] = per_call(lambda: q.gf_wilson_flow_step(gf, 0.05, c1=0.0))
        out["gf_energy_density"] = per_call(lambda: q.gf_energy_density(gf))
        out["clf_topology_sum"] = per_call(lambda: q.gf_topology_clf(gf))
        out["topology_charge_5"] = per_call(lambda: q.topology_charge_5(gf))
    return out


# ---------------------------------------------------------------------------
# one chain held as a time slab (the multi-GPU decomposition) on one GPU

def slabs(q, args):
    """Iwasaki (beta 2.13, c1 -0.331) force-gradient trajectories of n_step steps,
    always accepted, from one hot start: the plain single-GPU form and the same
    chain held as a one-rank time slab, whose halo is its own periodic copy
    refreshed through pack / unpack before every force evaluation.  The slab
    form computes the extra halo slices and stops the stream at every
    refresh, which is what a multi-rank run adds besides the network."""
    import ctypes

    import torch
    ts = _lattice(args.lattice)
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("b200-slabs-bench")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    for prec in (q.F64, q.F32):
        q.autotune_force(gf.copy(precision=prec), ga.c1())
    sl = q.TimeSlabs(ts, halo=args.halo)
    out = {"lattice": list(ts), "precision": args.precision, "n_step": args.n_step, "halo": sl.halo,
           "local_time_extent": sl.nt + 2 * sl.halo}

    def run(form):
        if form == "plain":
            g = gf.copy()
            step = lambda t: q.run_hmc_pure_gauge(g, ga, t, rs, n_step=args.n_step, is_always_accept=True,
                                                  precision=args.precision)
        else:
            g = sl.gauge_field()
            sl.set_rand(g, rs.split("gf-init"), 0.3, 1)
            step = lambda t: q.run_hmc_pure_gauge_slabs(sl, g, ga, t, rs, n_step=args.n_step,
                                                        is_always_accept=True, precision=args.precision)
        dhs, ms = [], []
        for t in range(1, args.warmup + 1):
            step(t)
        torch.cuda.synchronize()
        for t in range(args.warmup + 1, args.warmup + 1 + args.trajs):
            t0 = time.perf_counter()
            dhs.append(step(t)[1])
            torch.cuda.synchronize()
            ms.append(round((time.perf_counter() - t0) * 1e3, 2))
        out[form + "_ms_per_traj"] = ms
        return 1e3 * len(ms) / sum(ms), dhs

    for form in args.order.split(","):
        out[form + "_traj_per_s"], dh = run(form)
        if form == "plain":
            dh_plain = dh
        else:
            dh_slab = dh
    out["slab_over_plain"] = out["slab_traj_per_s"] / out["plain_traj_per_s"]
    out["max_delta_h_difference"] = max(abs(a - b) for a, b in zip(dh_plain, dh_slab))
    g32 = sl.gauge_field().copy(precision=q.F32 if args.precision == "mixed" else q.F64)
    for _ in range(3):
        sl.exchange(g32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(20):
        sl.exchange(g32)
    torch.cuda.synchronize()
    n = ctypes.c_int64()
    q._lib.call("qgb_field_tslice_bytes", g32.handle, sl.halo, ctypes.byref(n))
    out["exchange_ms"] = (time.perf_counter() - t0) / 20 * 1e3
    out["exchange_bytes_each_way"] = 2 * n.value
    out["exchanges_per_traj"] = 2 * args.n_step * (2 if args.halo < 4 else 1) + 2
    return out



def domains(q, args):
    """The same chain as `slabs`, held as one rank's domain with the directions
    of --cut cut (halo of --halo sites on either side, each refreshed from the
    rank's own opposite face before every force evaluation) against the plain
    single-GPU form.  The domain's force runs on the owned sites only, so what
    it adds is the exchanges (four faces per cut direction and force
    evaluation, stopping the stream each time) and the element-wise kernels'
    sweep over the halo -- what a decomposed run adds besides the network."""
    import torch
    ts = _lattice(args.lattice)
    cut = tuple(bool(int(c)) for c in args.cut.split(","))
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("b200-domains-bench")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    for prec in (q.F64, q.F32):
        q.autotune_force(gf.copy(precision=prec), ga.c1())
    dom = q.Domains(ts, (1, 1, 1, 1), halo=args.halo, cut=cut)
    local = 1
    for v in dom.dims:
        local *= v
    out = {"lattice": list(ts), "precision": args.precision, "n_step": args.n_step, "halo": args.halo,
           "cut": list(cut), "local_extents": list(dom.dims), "local_over_owned_sites": local / dom.total_volume}
    dhs = {}
    for form in ("plain", "domain"):
        if form == "plain":
            g = gf.copy()
            step = lambda t: q.run_hmc_pure_gauge(g, ga, t, rs, n_step=args.n_step, is_always_accept=True,
                                                  precision=args.precision)
        else:
            g = dom.gauge_field()
            dom.set_rand(g, rs.split("gf-init"), 0.3, 1)
            step = lambda t: q.run_hmc_pure_gauge_domains(dom, g, ga, t, rs, n_step=args.n_step,
                                                          is_always_accept=True, precision=args.precision)
        for t in range(1, args.warmup + 1):
            step(t)
        torch.cuda.synchronize()
        ms, dh = [], []
        for t in range(args.warmup + 1, args.warmup + 1 + args.trajs):
            t0 = time.perf_counter()
            dh.append(step(t)[1])
            torch.cuda.synchronize()
            ms.append(round((time.perf_counter() - t0) * 1e3, 2))
        out[form + "_ms_per_traj"] = ms
        out[form + "_traj_per_s"] = 1e3 * len(ms) / sum(ms)
        dhs[form] = dh
    out["domain_over_plain"] = out["domain_traj_per_s"] / out["plain_traj_per_s"]
    out["max_delta_h_difference"] = max(abs(a - b) for a, b in zip(dhs["plain"], dhs["domain"]))
    g32 = dom.gauge_field().copy(precision=q.F32 if args.precision == "mixed" else q.F64)
    for _ in range(3):
        dom.exchange(g32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(20):
        dom.exchange(g32)
    torch.cuda.synchronize()
    out["exchange_ms"] = (time.perf_counter() - t0) / 20 * 1e3
    out["exchanges_per_traj"] = 4 * args.n_step + 2
    return out


# ---------------------------------------------------------------------------
# small cases for ncu

def profile_force(args):
    """One set_gm_force per listed variant on a seeded hot start (FP32 links),
    for `ncu -k regex:k_force`."""
    import qlat_b200 as q
    ts = _lattice(args.lattice)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("kernel-bench").split("gf-init"), 0.3, 1)
    g = gf.copy(precision=q.F32) if args.precision == "fp32" else gf
    P = q.F32 if args.precision == "fp32" else q.F64
    F = q.GaugeMomentum(gf.geo, precision=P)
    ga = q.GaugeAction(2.13, args.c1)
    variants = [int(v) for v in args.variants.split(",")]
    for v in variants:
        q.force_set_variant(P, args.c1 != 0.0, v)
        q.set_gm_force(F, g, ga)
    q.synchronize()
    return {"lattice": list(ts), "variants": variants, "c1": args.c1, "precision": args.precision}


def profile_flow(args):
    """`steps` RK3 flow steps plus one energy density and clover charge, FP64
    then FP32, for `ncu -k` captures of the flow-stage and clover kernels."""
    import qlat_b200 as q
    ts = _lattice(args.lattice)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("b200-c3-32x32-flow").split("gf-init"), 0.5, 1)
    out = {"lattice": list(ts), "steps": args.steps}
    for name, prec in (("fp64", q.F64), ("fp32", q.F32)):
        g = gf.copy(precision=prec)
        for _ in range(args.steps):
            q.gf_wilson_flow_step(g, 0.05, c1=0.0)
        out[name] = {"E": q.gf_energy_density(g), "Q": q.gf_topology_clf(g)}
    return out


def profile_hmc(args):
    """`trajs` Iwasaki force-gradient trajectories (8 steps) in each form, for
    captures of the trajectory's kernels at a size that fits a capture."""
    import qlat_b200 as q
    ts = _lattice(args.lattice)
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("b200-c2-24x64-iwasaki")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    if args.fp32_variant >= 0:
        q.force_set_variant(q.F32, True, args.fp32_variant)
    out = {"lattice": list(ts), "fp32_variant": q.force_get_variant(q.F32, True)}
    for prec in ("mixed", "fp64"):
        dh = [q.run_hmc_pure_gauge(gf, ga, t, rs, n_step=8, precision=prec, reunit_interval=4)[1]
              for t in range(1, args.trajs + 1)]
        out[prec] = dh
    return out


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("c1", "c3", "c4", "c5"):
        sub.add_parser(name)
    sl = sub.add_parser("slabs")
    sl.add_argument("--lattice", default="24,24,24,64")
    sl.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    sl.add_argument("--n-step", type=int, default=8)
    sl.add_argument("--trajs", type=int, default=5)
    sl.add_argument("--warmup", type=int, default=2)
    sl.add_argument("--order", default="plain,slab")
    sl.add_argument("--halo", type=int, default=4)
    dm = sub.add_parser("domains")
    dm.add_argument("--lattice", default="24,24,24,64")
    dm.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    dm.add_argument("--n-step", type=int, default=8)
    dm.add_argument("--trajs", type=int, default=5)
    dm.add_argument("--warmup", type=int, default=2)
    dm.add_argument("--halo", type=int, default=2)
    dm.add_argument("--cut", default="1,1,1,1", help="per direction: 1 = cut (halo exchanged with itself)")
    fn = sub.add_parser("functions")
    fn.add_argument("set", choices=["hmc", "flow"])
    fn.add_argument("--reps", type=int, default=20)
    a = sub.add_parser("profile-force")
    a.add_argument("--lattice", default="24,24,24,48")
    a.add_argument("--variants", default="10")
    a.add_argument("--c1", type=float, default=-0.331)
    a.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    b = sub.add_parser("profile-flow")
    b.add_argument("--lattice", default="32,32,32,32")
    b.add_argument("--steps", type=int, default=4)
    c = sub.add_parser("profile-hmc")
    c.add_argument("--lattice", default="24,24,24,48")
    c.add_argument("--trajs", type=int, default=1)
    c.add_argument("--fp32-variant", type=int, default=-1, help="FP32 Iwasaki force variant (default: library's)")
    args = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    from qlat_b200 import build as B
    B.build()
    import qlat_b200 as q
    q.set_device(0)
    torch.cuda.set_stream(torch.cuda.Stream())  # not the legacy default stream: trajectories replay as graphs
    q.set_stream(torch.cuda.current_stream().cuda_stream)
    legs = {"c1": leg_c1, "c3": leg_c3, "c4": leg_c4, "c5": leg_c5}
    if args.cmd in legs:
        res = legs[args.cmd](q)
    elif args.cmd == "slabs":
        res = slabs(q, args)
    elif args.cmd == "domains":
        res = domains(q, args)
    elif args.cmd == "functions":
        res = functions(q, args.set, args.reps)
    else:
        res = {"profile-force": profile_force, "profile-flow": profile_flow, "profile-hmc": profile_hmc}[args.cmd](args)
    print(json.dumps(res))


if __name__ == "__main__":
    main()

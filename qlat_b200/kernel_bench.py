"""Kernel-level benchmarks and profiling drivers for the GPU library.

    python -m qlat_b200.kernel_bench force-variants [--lattice 24,24,24,64]
        time every force-kernel launch variant (FP64 / FP32, Wilson / Iwasaki)
    python -m qlat_b200.kernel_bench force-profile --variants 0,7 [--lattice 24,24,24,48] [--c1 -0.331]
        one set_gm_force launch per variant and precision (FP32 then FP64, or --precision fp32), for
        ncu -k regex:k_force
    python -m qlat_b200.kernel_bench fma-peak [--reps 5]
        FMA rate of the device: scalar FP32, packed f32x2 and FP64 chains
    python -m qlat_b200.kernel_bench flow [--lattice 32,32,32,32] [--steps 80] [--every 4]
        gradient flow (RK3, eps = 0.05) with t^2 E(t) and the clover charge Q measured every
        `every` steps, FP64 and FP32 storage; prints timings and the FP32 errors
    python -m qlat_b200.kernel_bench batch [--per-size 64] [--trajs 10]
        256 independent chains of 4^4 ... 12^4 advanced together (CUDA graph per trajectory)
    python -m qlat_b200.kernel_bench flow-adjoint [--lattice 16,16,16,16] [--steps 40] [--every 8]
        backward through the Wilson flow: timing, finite-difference check, flowed-field HMC

    python -m qlat_b200.kernel_bench slabs [--lattice 24,24,24,64] [--precision mixed] [--halo 4]
        one chain as a one-rank time slab (4 halo slices each side and a refresh before every
        force-gradient update, or 2 and a refresh before every force) against the plain single-GPU
        trajectory: traj/s and the exchange time

    python -m qlat_b200.kernel_bench functions hmc|flow [--lattice ...] [--reps 20]
        seconds per call of single API functions (hmc: 24^3x64 Iwasaki set_gm_force, gf_evolve,
        the Hamiltonians, the momentum draw, unitarize, gf_avg_plaq; flow: 32^4 RK3 Wilson flow step,
        energy density, clover and 5-loop charges), each call synchronised

    python -m qlat_b200.kernel_bench c1 [--trajs 10]
        8^4 Wilson (beta 5.5) leapfrog, 6 steps per unit trajectory, hot start at scale 1: the small
        configuration, through run_hmc_pure_gauge, per-trajectory time

Each command prints one JSON line.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import time


def _lattice(s):
    return tuple(int(v) for v in s.split(","))


def force_variants(args):
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    ts = _lattice(args.lattice)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("kernel-bench").split("gf-init"), 0.3, 1)
    g32 = gf.copy(precision=q.F32)
    res = {"lattice": list(ts), "variants": q.force_variants()}
    for name, g in (("fp64", gf), ("fp32", g32)):
        for c1 in (0.0, -0.331):
            res[f"{name} c1={c1} ms"] = [round(q.force_time_variant(g, c1, v, reps=args.reps), 4)
                                         for v in range(len(res["variants"]))]
    print(json.dumps(res))


def force_profile(args):
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    ts = _lattice(args.lattice)
    variants = [int(v) for v in args.variants.split(",")]
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("kernel-bench").split("gf-init"), 0.3, 1)
    g32 = gf.copy(precision=q.F32)
    ga = q.GaugeAction(2.13, args.c1)
    precs = ((q.F32, g32), (q.F64, gf)) if args.precision == "both" else ((q.F32, g32),)
    for prec, g in precs:
        F = q.GaugeMomentum(gf.geo, precision=prec)
        for v in variants:
            q.force_set_variant(prec, args.c1 != 0.0, v)
            q.set_gm_force(F, g, ga)
    q.synchronize()
    print(json.dumps({"lattice": list(ts), "variants": variants, "c1": args.c1,
                      "launches": len(precs) * len(variants)}))


def fma_peak(args):
    import ctypes

    import torch
    from qlat_b200._lib import call
    torch.cuda.set_device(0)
    out = {}
    for name, kind in (("scalar_ffma", 0), ("packed_ffma2", 1), ("fp64_dfma", 2)):
        t = ctypes.c_double()
        call("qgb_fma_rate", kind, int(args.reps), ctypes.byref(t))
        out[name + "_tflops"] = t.value
    print(json.dumps(out))


def flow(args):
    """Gradient flow of a hot start: RK3 steps of eps, t^2 E and clover Q every
    `every` steps, in FP64 and with FP32 links (FP64 reductions)."""
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    ts = _lattice(args.lattice)
    geo = q.Geometry(ts)
    gf = q.GaugeField(geo)
    gf.set_rand(q.RngState("b200-c3-flow").split("gf-init"), args.sigma, args.n_step)
    stream = torch.cuda.current_stream()
    q.set_stream(stream.cuda_stream)
    out = {"lattice": list(ts), "eps": args.eps, "steps": args.steps, "every": args.every,
           "hot_start": {"sigma": args.sigma, "n_step": args.n_step}}
    series = {}
    for name, prec in (("fp64", q.F64), ("fp32", q.F32)):
        g = gf.copy(precision=prec)
        # warm-up: one step on a scratch copy
        w = g.copy()
        q.gf_wilson_flow_step(w, args.eps, c1=args.c1)
        del w
        torch.cuda.synchronize()
        t2e, topo, times = [], [], []
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            q.gf_wilson_flow_step(g, args.eps, c1=args.c1)
            if (i + 1) % args.every == 0:
                t = (i + 1) * args.eps
                t2e.append(t * t * q.gf_energy_density(g))
                topo.append(q.gf_topology_clf(g))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        series[name] = (t2e, topo)
        out[name] = {"ms_total": ms, "ms_per_step": ms / args.steps, "t2E_final": t2e[-1], "Q_final": topo[-1],
                     "plaq_final": g.plaq()}
    d_t2e = max(abs(a - b) for a, b in zip(series["fp32"][0], series["fp64"][0]))
    d_q = max(abs(a - b) for a, b in zip(series["fp32"][1], series["fp64"][1]))
    rel_t2e = max(abs(a - b) / abs(b) for a, b in zip(series["fp32"][0], series["fp64"][0]) if b != 0)
    out["fp32_vs_fp64"] = {"max_abs_t2E": d_t2e, "max_rel_t2E": rel_t2e, "max_abs_Q": d_q}
    out["t2E_fp64"] = series["fp64"][0]
    out["Q_fp64"] = series["fp64"][1]
    out["fp32_over_fp64_speed"] = out["fp64"]["ms_total"] / out["fp32"]["ms_total"]
    print(json.dumps(out))


def batch(args):
    """256 independent Wilson chains: 64 each of 4^4, 6^4, 8^4, 12^4, betas evenly
    spaced in [5.6, 6.2], hot starts at scale 1, leapfrog with 10 steps of total
    length 1, one CUDA graph per trajectory.  Reports aggregate link updates/s
    for the mixed and FP64 forms and the per-chain plaquette difference between
    them after the same trajectories."""
    import numpy as np
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    sizes = [(L, L, L, L) for L in (4, 6, 8, 12) for _ in range(args.per_size)]
    n = len(sizes)
    betas = list(np.linspace(5.6, 6.2, n))
    rs = [q.RngState("b200-c5-batch").split(f"chain-{c}") for c in range(n)]
    out = {"chains": n, "sites": int(sum(np.prod(s) for s in sizes)), "n_step": args.n_step}
    plaqs = {}
    for prec in ("mixed", "fp64"):
        b = q.ChainBatch(sizes, betas)
        b.set_rand([r.split("gf-init") for r in rs], 1.0, 1)
        # warm-up trajectories are always accepted (the reference's scripts do the
        # same for their first trajectories, examples-py/hmc-pure-gauge.py)
        for t in range(1, args.warmup + 1):
            b.run_hmc(t, rs, args.n_step, precision=prec, is_always_accept=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        acc = 0
        for t in range(args.warmup + 1, args.warmup + 1 + args.trajs):
            flags, dh = b.run_hmc(t, rs, args.n_step, precision=prec)
            acc += sum(flags)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        link_updates = 4 * out["sites"] * args.n_step * args.trajs
        out[prec] = {"s_per_traj": dt / args.trajs, "link_updates_per_s": link_updates / dt,
                     "accept_rate": acc / (n * args.trajs)}
        plaqs[prec] = b.plaq()
        del b
    d = np.abs(plaqs["mixed"] - plaqs["fp64"])
    out["plaq_mixed_minus_fp64"] = {"max": float(d.max()), "mean": float(d.mean())}
    out["plaq_fp64_by_size"] = {str(L): float(plaqs["fp64"][i * args.per_size:(i + 1) * args.per_size].mean())
                                for i, L in enumerate((4, 6, 8, 12))}
    print(json.dumps(out))


def flow_adjoint(args):
    """Backward through `steps` Wilson-flow steps of eps on a seeded hot start
    (scale sigma), loss = Wilson gauge action (beta) of the flowed field,
    checkpoints every k steps: timing, the finite-difference check along
    `dirs` random su(3) directions (h = 1e-4, 4-point, FP64), the zero-flow
    identity, and `trajs` flowed-field HMC trajectories (flow time
    eps * hmc_flow_steps) after `hmc_warmup` ordinary Wilson HMC trajectories."""
    import numpy as np
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    ts = _lattice(args.lattice)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("b200-c4-adjoint").split("gf-init"), args.sigma, 1)
    out = {"lattice": list(ts), "eps": args.eps, "steps": args.steps, "checkpoint_every": args.every,
           "beta_loss": args.beta}
    # warm-up of both paths, then wall-clock timing of each (the calls synchronise)
    q.gf_flow_action_grad(gf, args.eps, args.steps, args.beta, checkpoint_every=args.every)
    q.gf_flow_action(gf, args.eps, args.steps, args.beta)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss, grad = q.gf_flow_action_grad(gf, args.eps, args.steps, args.beta, checkpoint_every=args.every)
    torch.cuda.synchronize()
    out["ms_forward_and_backward"] = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    q.gf_flow_action(gf, args.eps, args.steps, args.beta)
    torch.cuda.synchronize()
    out["ms_forward_only"] = 1e3 * (time.perf_counter() - t0)
    G = np.asarray(grad)
    rel = []
    for k in range(args.dirs):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"c4-direction-{k}"), 1.0)
        Xn = np.asarray(X)

        def L(h):
            u = gf.copy()
            q.gf_evolve(u, X, h)
            return q.gf_flow_action(u, args.eps, args.steps, args.beta)

        h = 1e-4
        fd = (8 * (L(h) - L(-h)) - (L(2 * h) - L(-2 * h))) / (12 * h)
        an = float(-0.5 * np.einsum("smij,smji->", G, Xn).real)
        rel.append(abs(fd - an) / abs(fd))
    out["fd_max_rel_err"] = max(rel)
    out["fd_median_rel_err"] = float(np.median(rel))
    _, g0 = q.gf_flow_action_grad(gf, args.eps, 0, args.beta)
    F = q.GaugeMomentum(gf.geo)
    q.set_gm_force(F, gf, q.GaugeAction(args.beta, 0.0))
    out["zero_flow_max_abs_diff_vs_minus2_force"] = float(np.abs(np.asarray(g0) + 2 * np.asarray(F)).max())
    if args.trajs:
        # flowed-field HMC: thermalise with ordinary Wilson HMC, then trajectories
        # whose action is the Wilson action of the field flowed to
        # t = eps * hmc_flow_steps; the energy error of one trajectory at n and 2n
        # steps from the same start checks the dt^2 scaling of the integrator.
        rs = q.RngState("b200-c4-flowed-hmc")
        u = gf.copy()
        ga = q.GaugeAction(args.hmc_beta, 0.0)
        for t in range(1, args.hmc_warmup + 1):
            q.run_hmc_pure_gauge(u, ga, t, rs.split("thermalise"), n_step=args.hmc_steps, integrator="leapfrog",
                                 is_always_accept=t <= args.hmc_warmup // 2)
        dh_n = []
        for n in (args.hmc_steps, 2 * args.hmc_steps):
            _, d = q.run_flowed_hmc_pure_gauge(u.copy(), args.hmc_beta, 0, rs.split("dt-check"), epsilon=args.eps,
                                               flow_steps=args.hmc_flow_steps, n_step=n, checkpoint_every=args.every)
            dh_n.append(d)
        hmc = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t in range(1, args.trajs + 1):
            flag, dh = q.run_flowed_hmc_pure_gauge(u, args.hmc_beta, t, rs, epsilon=args.eps,
                                                   flow_steps=args.hmc_flow_steps, n_step=args.hmc_steps,
                                                   checkpoint_every=args.every)
            hmc.append({"traj": t, "accept": bool(flag), "delta_h": dh, "plaq": u.plaq()})
        torch.cuda.synchronize()
        out["flowed_hmc"] = {"beta": args.hmc_beta, "flow_t": args.eps * args.hmc_flow_steps,
                             "n_step": args.hmc_steps, "thermalisation_trajs": args.hmc_warmup,
                             "delta_h_n_and_2n": dh_n, "delta_h_ratio": dh_n[0] / dh_n[1] if dh_n[1] else None,
                             "accept_rate": sum(h["accept"] for h in hmc) / len(hmc),
                             "s_per_traj": (time.perf_counter() - t0) / args.trajs, "trajectories": hmc}
    print(json.dumps(out))


def slabs(args):
    """Iwasaki (beta 2.13, c1 -0.331) force-gradient trajectories of n_step steps,
    always accepted, from one hot start: the plain single-GPU form and the same
    chain held as a one-rank time slab, whose halo is its own periodic copy
    refreshed through pack / unpack before every force evaluation.  The slab
    form computes the extra halo slices and stops the stream at every
    refresh, which is what a multi-rank run adds besides the network."""
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
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
    print(json.dumps(out))


def functions(args):
    """Per-call time of single API functions, as a user calls them (launch,
    kernels and, for the scalar results, the read-back; a synchronisation
    after every call), on the hot start set_rand(RngState(name).split("gf-init"),
    sigma, 1)."""
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    hmc = args.set == "hmc"
    ts = _lattice(args.lattice or ("24,24,24,64" if hmc else "32,32,32,32"))
    rs = q.RngState("b200-c2-24x64-iwasaki" if hmc else "b200-c3-32x32-flow")
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(rs.split("gf-init"), 0.3 if hmc else 0.5, 1)
    out = {"set": args.set, "lattice": list(ts), "reps": args.reps}

    def per_call(fn):
        for _ in range(2):
            fn()
        q.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.reps):
            fn()
            q.synchronize()
        return (time.perf_counter() - t0) / args.reps

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
    print(json.dumps(out))


def c1(args):
    """The 8^4 Wilson leapfrog chain (10 trajectories, the first always
    accepted) through the qlat-compatible run_hmc_pure_gauge, in FP64 and in
    the mixed form: milliseconds per trajectory and the plaquettes."""
    import torch
    import qlat_b200 as q
    torch.cuda.set_device(0)
    ts = (8, 8, 8, 8)
    ga = q.GaugeAction(5.5, 0.0)
    out = {"lattice": list(ts), "beta": 5.5, "integrator": "leapfrog", "n_step": 6, "trajs": args.trajs}
    for prec in ("fp64", "mixed"):
        rs = q.RngState("b200-c1-8x4-wilson")
        gf = q.GaugeField(q.Geometry(ts))
        gf.set_rand(rs.split("gf-init"), 1.0, 1)
        for t in range(1, 4):  # warm-up chain, discarded
            q.run_hmc_pure_gauge(gf.copy(), ga, t, rs.split("warm"), n_step=6, integrator="leapfrog",
                                 precision=prec)
        q.synchronize()
        t0 = time.perf_counter()
        plaq = []
        for t in range(1, args.trajs + 1):
            q.run_hmc_pure_gauge(gf, ga, t, rs.split("hmc"), n_step=6, integrator="leapfrog", precision=prec,
                                 is_always_accept=t == 1)
            plaq.append(q.gf_avg_plaq(gf))
        q.synchronize()
        out[prec] = {"ms_per_traj": (time.perf_counter() - t0) / args.trajs * 1e3, "plaq": plaq}
        # the same chain as a batch of one (every phase one launch, the trajectory's
        # molecular dynamics one CUDA graph), with run_hmc_pure_gauge's RNG splits
        b = q.ChainBatch([ts], [5.5])
        b.set_rand([rs.split("gf-init")], 1.0, 1)
        for t in range(1, 4):
            b.run_hmc(t, [rs.split("warm")], 6, precision=prec)
        b.set_rand([rs.split("gf-init")], 1.0, 1)  # back to the hot start
        q.synchronize()
        t0 = time.perf_counter()
        bplaq = []
        for t in range(1, args.trajs + 1):
            b.run_hmc(t, [rs.split("hmc")], 6, precision=prec, is_always_accept=t == 1)
            bplaq.append(float(b.plaq()[0]))
        q.synchronize()
        out[prec + "_batch_of_one"] = {"ms_per_traj": (time.perf_counter() - t0) / args.trajs * 1e3,
                                       "max_plaq_difference": max(abs(x - y) for x, y in zip(plaq, bplaq))}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("force-variants")
    a.add_argument("--lattice", default="24,24,24,64")
    a.add_argument("--reps", type=int, default=5)
    b = sub.add_parser("force-profile")
    b.add_argument("--lattice", default="24,24,24,48")
    b.add_argument("--variants", default="0")
    b.add_argument("--c1", type=float, default=-0.331)
    b.add_argument("--precision", default="both", choices=["both", "fp32"])
    c = sub.add_parser("flow")
    c.add_argument("--lattice", default="32,32,32,32")
    c.add_argument("--steps", type=int, default=80)
    c.add_argument("--every", type=int, default=4)
    c.add_argument("--eps", type=float, default=0.05)
    c.add_argument("--c1", type=float, default=0.0)
    c.add_argument("--sigma", type=float, default=0.5)
    c.add_argument("--n-step", type=int, default=1)
    d = sub.add_parser("batch")
    d.add_argument("--per-size", type=int, default=64)
    d.add_argument("--n-step", type=int, default=10)
    d.add_argument("--trajs", type=int, default=10)
    d.add_argument("--warmup", type=int, default=10)
    e = sub.add_parser("flow-adjoint")
    e.add_argument("--lattice", default="16,16,16,16")
    e.add_argument("--eps", type=float, default=0.05)
    e.add_argument("--steps", type=int, default=40)
    e.add_argument("--every", type=int, default=8)
    e.add_argument("--beta", type=float, default=5.8)
    e.add_argument("--sigma", type=float, default=0.4)
    e.add_argument("--dirs", type=int, default=16)
    e.add_argument("--trajs", type=int, default=10)
    e.add_argument("--hmc-beta", type=float, default=5.8)
    e.add_argument("--hmc-steps", type=int, default=20)
    e.add_argument("--hmc-flow-steps", type=int, default=2)
    e.add_argument("--hmc-warmup", type=int, default=10)
    f = sub.add_parser("fma-peak")
    f.add_argument("--reps", type=int, default=5)
    g = sub.add_parser("slabs")
    g.add_argument("--lattice", default="24,24,24,64")
    g.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    g.add_argument("--n-step", type=int, default=8)
    g.add_argument("--trajs", type=int, default=5)
    g.add_argument("--warmup", type=int, default=2)
    g.add_argument("--order", default="plain,slab")
    g.add_argument("--halo", type=int, default=4)
    c1p = sub.add_parser("c1")
    c1p.add_argument("--trajs", type=int, default=10)
    h = sub.add_parser("functions")
    h.add_argument("set", choices=["hmc", "flow"])
    h.add_argument("--lattice", default=None)
    h.add_argument("--reps", type=int, default=20)
    args = ap.parse_args()
    {"force-variants": force_variants, "force-profile": force_profile, "flow": flow, "batch": batch,
     "flow-adjoint": flow_adjoint, "fma-peak": fma_peak, "slabs": slabs, "functions": functions,
     "c1": c1}[args.cmd](args)


if __name__ == "__main__":
    main()

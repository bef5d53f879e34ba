"""Time-slab decomposition of pure-gauge HMC (qlat_b200.slabs).

CPU: the slab geometry and its checks; the halo message pattern of the ring
on 2 and 3 gloo ranks (the library's own _swap, with CPU buffers); a rank that
leaves between steps makes the other rank's exchange fail with an error
instead of waiting for ever.
GPU: a one-rank slab (its halo is its own periodic copy) and two ranks run as
two processes on one GPU, exchanging halos through host memory over gloo (no
kernel waits on another rank), both against the single-GPU trajectory of the
whole lattice, in the FP64 and the mixed FP32/FP64 forms and with halos of 4
slices (one exchange per force-gradient update) and 2 slices (the shifted
field exchanged too): the same links on every owned site, the same delta_h
and the same accept / reject decisions.  A
halo exchange that raises inside the library's trajectory ends the call with
its exception.
"""

import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TS = (4, 4, 4, 16)
BETA, C1 = 2.13, -0.331
N_TRAJ, N_STEP = 3, 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_halo_thinner_than_reach_is_refused():
    """A 1-slice halo cannot carry the rectangle force (reach 2); the check
    runs before any GPU work."""
    sys.path.insert(0, ROOT)
    from qlat_b200.field import GaugeAction
    from qlat_b200.slabs import TimeSlabs
    s = TimeSlabs((4, 4, 4, 8), halo=1)
    with pytest.raises(ValueError):
        s.run_md(None, None, GaugeAction(2.13, -0.331), 4)


def test_slab_geometry():
    sys.path.insert(0, ROOT)
    from qlat_b200.slabs import TimeSlabs
    s = TimeSlabs(TS)
    assert s.world == 1 and s.nt == 16 and tuple(s.geo.total_site) == (4, 4, 4, 24)
    assert s.owned == (4 * 64, 20 * 64) and s.site_offset == -4 * 64
    with pytest.raises(ValueError):
        TimeSlabs((4, 4, 4, 2))  # fewer owned slices than the halo
    with pytest.raises(ValueError):
        TimeSlabs((3, 4, 5, 8))  # X Y Z not a multiple of 32


def _swap_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from qlat_b200.slabs import TimeSlabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = TimeSlabs((4, 4, 4, 12))
        up = torch.full((64,), 10 * rank + 1, dtype=torch.uint8)
        dn = torch.full((64,), 10 * rank + 2, dtype=torch.uint8)
        rbot, rtop = s._swap(up, dn)
        with open(os.path.join(out_dir, f"swap{rank}.json"), "w") as f:
            json.dump({"t0": s.t0, "bot": rbot.unique().tolist(), "top": rtop.unique().tolist()}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_ring_on_gloo_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_swap_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        g = json.load(open(tmp_path / f"swap{r}.json"))
        assert g["t0"] == r * (12 // world)
        assert g["bot"] == [10 * ((r - 1) % world) + 1]  # the lower neighbour's top slices
        assert g["top"] == [10 * ((r + 1) % world) + 2]  # the upper neighbour's bottom slices


# ---- GPU ------------------------------------------------------------------------------------


def _global_run(q, precision="fp64"):
    """The single-GPU reference: hot start and N_TRAJ trajectories of the whole lattice."""
    ga = q.GaugeAction(BETA, C1)
    rs = q.RngState("slabs")
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    rows = []
    for traj in range(1, N_TRAJ + 1):
        flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs.split("hmc"), n_step=N_STEP, is_always_accept=traj < 2,
                                        precision=precision)
        rows.append([bool(flag), dh, q.gf_avg_plaq(gf)])
    return rows, np.asarray(gf)


def _slab_run(q, slabs, precision="fp64"):
    ga = q.GaugeAction(BETA, C1)
    rs = q.RngState("slabs")
    gf = slabs.gauge_field()
    slabs.set_rand(gf, rs.split("gf-init"), 0.3, 1)
    rows = []
    for traj in range(1, N_TRAJ + 1):
        flag, dh = q.run_hmc_pure_gauge_slabs(slabs, gf, ga, traj, rs.split("hmc"), n_step=N_STEP,
                                              is_always_accept=traj < 2, precision=precision)
        slabs.exchange(gf)
        rows.append([bool(flag), dh, slabs.plaq(gf)])
    return rows, slabs.owned_slices(np.asarray(gf))


def _compare(rows, ref_rows, links, ref_links, t0, nt):
    V3 = TS[0] * TS[1] * TS[2]
    for (f, dh, p), (rf, rdh, rp) in zip(rows, ref_rows):
        assert f == rf
        assert abs(dh - rdh) < 1e-9, (dh, rdh)
        assert abs(p - rp) < 1e-12, (p, rp)
    assert np.abs(links - ref_links[t0 * V3:(t0 + nt) * V3]).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,halo", [("fp64", 4), ("mixed", 4), ("fp64", 2), ("mixed", 2)])
def test_one_rank_slab_matches_global(q, precision, halo):
    slabs = q.TimeSlabs(TS, halo=halo)
    rows, links = _slab_run(q, slabs, precision)
    ref_rows, ref_links = _global_run(q, precision)
    _compare(rows, ref_rows, links, ref_links, 0, TS[3])


@pytest.mark.gpu
def test_halo_hook_error_aborts_trajectory(q):
    """An exchange that fails inside the library's trajectory (the third halo
    refresh raises) ends the call with that exception; the library stays
    usable afterwards."""

    class Failing(q.TimeSlabs):
        calls = 0

        def _exchange_handle(self, handle):
            Failing.calls += 1
            if Failing.calls == 3:
                raise ConnectionError("peer gone")
            super()._exchange_handle(handle)

    slabs = Failing(TS)
    ga = q.GaugeAction(BETA, C1)
    gf = slabs.gauge_field()
    slabs.set_rand(gf, q.RngState("hook"), 0.3, 1)  # exchange call 1
    gm = slabs.gauge_momentum()
    slabs.set_rand_momentum(gm, q.RngState("hook-gm"), 1.0)
    with pytest.raises(ConnectionError):
        slabs.run_md(gm, gf, ga, N_STEP)  # calls 2 and 3 are the hook's
    assert Failing.calls == 3
    assert np.isfinite(slabs.plaq(gf))


def _slab_main(rank, world, port, out_dir, precision, halo):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    torch.cuda.set_device(0)  # both ranks share the one GPU; halos go through host memory
    import qlat_b200 as q
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        slabs = q.TimeSlabs(TS, halo=halo)
        rows, links = _slab_run(q, slabs, precision)
        np.save(os.path.join(out_dir, f"links{rank}.npy"), links)
        with open(os.path.join(out_dir, f"rows{rank}.json"), "w") as f:
            json.dump({"t0": slabs.t0, "nt": slabs.nt, "rows": rows}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,halo", [("fp64", 4), ("mixed", 4), ("mixed", 2)])
def test_two_rank_slabs_match_global(q, tmp_path, precision, halo):
    import torch.multiprocessing as mp
    mp.start_processes(_slab_main, args=(2, _free_port(), str(tmp_path), precision, halo), nprocs=2, join=True,
                       start_method="spawn")
    ref_rows, ref_links = _global_run(q, precision)
    for r in range(2):
        g = json.load(open(tmp_path / f"rows{r}.json"))
        _compare(g["rows"], ref_rows, np.load(tmp_path / f"links{r}.npy"), ref_links, g["t0"], g["nt"])


def _leaving_rank_main(rank, world, port, out_dir):
    """Rank 1 leaves right after joining; rank 0's halo exchange must end with
    an error (not wait forever) within the process group's timeout."""
    import datetime
    import time

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from qlat_b200.slabs import TimeSlabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    s = TimeSlabs((4, 4, 4, 12))
    if rank == 1:
        return  # leaves between steps, with nothing in flight
    t = time.time()
    err = None
    try:
        s._swap(torch.zeros(64, dtype=torch.uint8), torch.zeros(64, dtype=torch.uint8))
    except Exception as e:  # the peer is gone
        err = type(e).__name__
    with open(os.path.join(out_dir, "leave.json"), "w") as f:
        json.dump({"error": err, "seconds": time.time() - t}, f)


def test_leaving_rank_is_reported(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_leaving_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    g = json.load(open(tmp_path / "leave.json"))
    assert g["error"] is not None
    assert g["seconds"] < 60

"""Four-dimensional domain decomposition of pure-gauge HMC (qlat_b200.domains).

CPU: the rank grid and domain layout (GeometryNode numbering, x fastest) and
its checks; the whole halo exchange of a 2 x 1 x 1 x 2 grid on four gloo
ranks, with the library's face boxes and message pattern but numpy arrays in
place of GPU fields, filling every halo site -- edges and corners included --
with the value its global site holds; a rank that leaves makes the other's
exchange fail with an error instead of waiting for ever.
GPU: one rank (no cut direction, the owned box is the whole field), and four
ranks on a 2 x 1 x 1 x 2 grid run as four processes on one GPU exchanging
halos through host memory over gloo (no kernel waits on another rank), both
against the single-GPU trajectory of the whole lattice in the FP64 and mixed
forms: the same links on every owned site, the same delta_h and decisions.
The library refuses the whole-lattice entry points on a domain field.
"""

import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TS = (8, 4, 4, 8)
GRID = (2, 1, 1, 2)
BETA, C1 = 2.13, -0.331
N_TRAJ, N_STEP = 3, 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_domain_layout():
    sys.path.insert(0, ROOT)
    from qlat_b200.domains import coordinate_from_index, domain_layout, index_from_coordinate
    assert coordinate_from_index(5, (2, 1, 1, 4)) == (1, 0, 0, 2)
    assert index_from_coordinate((1, 0, 0, 2), (2, 1, 1, 4)) == 5
    d = domain_layout(TS, GRID, 3, halo=2)  # rank 3 = (1, 0, 0, 1)
    assert d["coor"] == (1, 0, 0, 1)
    assert d["owned"] == (4, 4, 4, 4) and d["halo"] == (2, 0, 0, 2) and d["dims"] == (8, 4, 4, 8)
    assert d["origin"] == (4, 0, 0, 4)
    assert d["neighbours"][0] == (2, 2) and d["neighbours"][3] == (1, 1) and d["neighbours"][1] == (3, 3)
    d = domain_layout((8, 8, 8, 12), (2, 2, 1, 3), 7, halo=1)  # (1, 1, 0, 1)
    assert d["origin"] == (4, 4, 0, 4) and d["neighbours"][3] == (3, 11)
    with pytest.raises(ValueError):
        domain_layout((8, 4, 4, 6), (1, 1, 1, 4), 0)  # 6 not divisible by 4
    with pytest.raises(ValueError):
        domain_layout((8, 4, 4, 6), (1, 1, 1, 6), 0, halo=2)  # one owned slice, halo of 2


def _numpy_domains_cls():
    from qlat_b200.domains import Domains

    class NumpyDomains(Domains):
        """The library's exchange (face boxes, order, message pattern) on numpy
        arrays: the handle is an array of shape (T, Z, Y, X) in local
        coordinates."""

        def _pack(self, handle, box, key):
            import torch
            (lo, n) = box
            a = handle[lo[3]:lo[3] + n[3], lo[2]:lo[2] + n[2], lo[1]:lo[1] + n[1], lo[0]:lo[0] + n[0]]
            return torch.from_numpy(np.ascontiguousarray(a))

        def _unpack(self, handle, box, msg):
            (lo, n) = box
            handle[lo[3]:lo[3] + n[3], lo[2]:lo[2] + n[2], lo[1]:lo[1] + n[1], lo[0]:lo[0] + n[0]] = \
                msg.numpy().reshape(n[3], n[2], n[1], n[0])

        def _self_exchange(self, k):
            return False  # the self-exchange, too, through the message path above

    return NumpyDomains


def _fill_and_exchange(d):
    """A local array with its global site index on owned sites and -1 in the
    halo, exchanged; returns (array, the global index every local site should
    hold)."""
    X, Y, Z, T = d.dims
    a = np.full((T, Z, Y, X), -1.0)
    h, n, o, G = d.halo, d.owned, d.origin, d.total_site
    gx = (np.arange(X) - h[0] + o[0]) % G[0]
    gy = (np.arange(Y) - h[1] + o[1]) % G[1]
    gz = (np.arange(Z) - h[2] + o[2]) % G[2]
    gt = (np.arange(T) - h[3] + o[3]) % G[3]
    want = gx[None, None, None, :] + G[0] * (gy[None, None, :, None] + G[1] * (
        gz[None, :, None, None] + G[2] * gt[:, None, None, None]))
    own = (slice(h[3], h[3] + n[3]), slice(h[2], h[2] + n[2]), slice(h[1], h[1] + n[1]), slice(h[0], h[0] + n[0]))
    a[own] = want[own]
    d._exchange_handle(a)
    return a, want


def test_one_rank_with_every_direction_cut_exchanges_with_itself():
    """One rank, all four directions cut: every halo site, edges and corners
    included, ends up with its periodic image's value."""
    sys.path.insert(0, ROOT)
    d = _numpy_domains_cls()((6, 4, 4, 8), (1, 1, 1, 1), halo=2, cut=(1, 1, 1, 1))
    assert d.dims == (10, 8, 8, 12) and d.halo == (2, 2, 2, 2)
    a, want = _fill_and_exchange(d)
    assert (a == want).all()


def _exchange_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d = _numpy_domains_cls()(TS, GRID, halo=2)
        X, Y, Z, T = d.dims
        a = np.full((T, Z, Y, X), -1.0)
        h, n, o = d.halo, d.owned, d.origin
        gx = (np.arange(X) - h[0] + o[0]) % TS[0]
        gy = (np.arange(Y) - h[1] + o[1]) % TS[1]
        gz = (np.arange(Z) - h[2] + o[2]) % TS[2]
        gt = (np.arange(T) - h[3] + o[3]) % TS[3]
        want = gx[None, None, None, :] + TS[0] * (gy[None, None, :, None] + TS[1] * (
            gz[None, :, None, None] + TS[2] * gt[:, None, None, None]))
        own = (slice(h[3], h[3] + n[3]), slice(h[2], h[2] + n[2]), slice(h[1], h[1] + n[1]), slice(h[0], h[0] + n[0]))
        a[own] = want[own]
        d._exchange_handle(a)
        with open(os.path.join(out_dir, f"ex{rank}.json"), "w") as f:
            json.dump({"bad": int((a != want).sum()), "sites": int(a.size)}, f)
    finally:
        dist.destroy_process_group()


def test_four_rank_exchange_fills_every_halo_site(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_exchange_main, args=(4, _free_port(), str(tmp_path)), nprocs=4, join=True,
                       start_method="spawn")
    for r in range(4):
        g = json.load(open(tmp_path / f"ex{r}.json"))
        assert g["bad"] == 0 and g["sites"] == 8 * 4 * 4 * 8


def _leaving_main(rank, world, port, out_dir):
    import datetime
    import time

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    d = _numpy_domains_cls()((8, 4, 4, 4), (2, 1, 1, 1), halo=1)
    if rank == 1:
        return  # leaves between steps, with nothing in flight
    t = time.time()
    err = None
    try:
        d._exchange_handle(np.zeros((4, 4, 4, 6)))
    except Exception as e:  # the peer is gone
        err = type(e).__name__
    with open(os.path.join(out_dir, "leave.json"), "w") as f:
        json.dump({"error": err, "seconds": time.time() - t}, f)


def test_leaving_rank_is_reported(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_leaving_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    g = json.load(open(tmp_path / "leave.json"))
    assert g["error"] is not None
    assert g["seconds"] < 60


# ---- GPU ------------------------------------------------------------------------------------


def _global_run(q, precision):
    ga = q.GaugeAction(BETA, C1)
    rs = q.RngState("domains")
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.3, 1)
    rows = []
    for traj in range(1, N_TRAJ + 1):
        flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs.split("hmc"), n_step=N_STEP, is_always_accept=traj < 2,
                                        precision=precision)
        rows.append([bool(flag), dh, q.gf_avg_plaq(gf)])
    X, Y, Z, T = TS
    return rows, np.asarray(gf).reshape((T, Z, Y, X, 4, 3, 3))


def _domain_run(q, dom, precision):
    ga = q.GaugeAction(BETA, C1)
    rs = q.RngState("domains")
    gf = dom.gauge_field()
    dom.set_rand(gf, rs.split("gf-init"), 0.3, 1)
    rows = []
    for traj in range(1, N_TRAJ + 1):
        flag, dh = q.run_hmc_pure_gauge_domains(dom, gf, ga, traj, rs.split("hmc"), n_step=N_STEP,
                                                is_always_accept=traj < 2, precision=precision)
        dom.exchange(gf)
        rows.append([bool(flag), dh, dom.plaq(gf)])
    return rows, dom.owned_sites(np.asarray(gf))


def _compare(rows, ref_rows, links, ref_links, origin, owned):
    for (f, dh, p), (rf, rdh, rp) in zip(rows, ref_rows):
        assert f == rf
        assert abs(dh - rdh) < 1e-9, (dh, rdh)
        assert abs(p - rp) < 1e-12, (p, rp)
    o, n = origin, owned
    ref = ref_links[o[3]:o[3] + n[3], o[2]:o[2] + n[2], o[1]:o[1] + n[1], o[0]:o[0] + n[0]]
    assert np.abs(links.reshape(ref.shape) - ref).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,cut", [("fp64", None), ("mixed", None), ("fp64", (1, 1, 1, 1)),
                                           ("mixed", (1, 1, 1, 1))])
def test_one_rank_domain_matches_global(q, precision, cut):
    """One rank: nothing cut (the owned box is the whole field), or every
    direction cut with halos of 2 refreshed from the rank's own faces (the
    force on the owned box only, four face exchanges per direction and force
    evaluation, edge halo sites filled through the direction exchanged
    second) -- against the whole-lattice chain."""
    dom = q.Domains(TS, (1, 1, 1, 1), cut=cut)
    rows, links = _domain_run(q, dom, precision)
    ref_rows, ref_links = _global_run(q, precision)
    _compare(rows, ref_rows, links, ref_links, dom.origin, dom.owned)


@pytest.mark.gpu
def test_domain_field_refuses_whole_lattice_calls(q):
    dom = q.Domains(TS, (1, 1, 1, 1))
    gf = dom.gauge_field()
    gm = dom.gauge_momentum()
    with pytest.raises(q.QlatB200Error):
        q.gf_avg_plaq(gf)
    with pytest.raises(q.QlatB200Error):
        q.run_hmc_evolve_pure_gauge(gm, gf, q.GaugeAction(BETA, C1), None, 2)
    with pytest.raises(q.QlatB200Error):
        q.gf_wilson_flow_step(gf, 0.05)
    g2 = q.GaugeField(q.Geometry(TS))
    g2 @= gf  # the copy takes the domain
    with pytest.raises(q.QlatB200Error):
        q.gf_avg_plaq(g2)


def _domain_main(rank, world, port, out_dir, precision):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    torch.cuda.set_device(0)  # every rank shares the one GPU; halos go through host memory
    import qlat_b200 as q
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=180))
    try:
        dom = q.Domains(TS, GRID, halo=2)
        rows, links = _domain_run(q, dom, precision)
        np.save(os.path.join(out_dir, f"links{rank}.npy"), links)
        with open(os.path.join(out_dir, f"rows{rank}.json"), "w") as f:
            json.dump({"origin": dom.origin, "owned": dom.owned, "rows": rows}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_four_rank_domains_match_global(q, tmp_path, precision):
    import torch.multiprocessing as mp
    mp.start_processes(_domain_main, args=(4, _free_port(), str(tmp_path), precision), nprocs=4, join=True,
                       start_method="spawn")
    ref_rows, ref_links = _global_run(q, precision)
    for r in range(4):
        g = json.load(open(tmp_path / f"rows{r}.json"))
        _compare(g["rows"], ref_rows, np.load(tmp_path / f"links{r}.npy"), ref_links, g["origin"], g["owned"])

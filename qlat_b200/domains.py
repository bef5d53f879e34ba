"""Four-dimensional domain decomposition of pure-gauge HMC over ranks.

The reference lays its ranks out on a grid size_node (GeometryNode,
core.h:17-62: coor_node from id_node with x fastest) and gives each rank's
fields an expansion of halo sites on either side (node_site and
expansion_left / expansion_right, core.h:90-110), refreshed from the
neighbouring ranks before each force evaluation (refresh_expanded,
field-expand.h:116-200; hmc.cpp:466-490, which expands by 2 in every
direction for the rectangle action).  Here each rank holds its domain as one
GPU field of extent node_site + 2 halo in every cut direction (a direction
with one rank is not cut and keeps its own periodic wrap), made a domain with
qgb_field_set_domain, so that the library

- evaluates the force on the owned sites only (no work on halo sites),
- sums the _node Hamiltonians over the owned sites,
- draws the owned sites' momenta, and every local site's hot-start links, from
  the random stream of the site's global index (halo momenta are zero: no
  force or sum reads them);

and the molecular dynamics is the library's own kernel sequence
(qgb_run_md_hooked), which calls back into ``exchange`` before every force
evaluation (on the links, and on the force-gradient shift, which is evaluated
on the owned sites too).  The exchange refreshes one cut direction after the
other; each face it sends spans the whole local extent of the other
directions, halos included, so the edge halo sites that a staple reaches
(two directions at once) arrive through the direction exchanged second.
Faces are packed on the device (qgb_field_pack_box) and sent with
torch.distributed point-to-point operations: from device buffers over NCCL,
through host memory over gloo.
"""

from __future__ import annotations

import ctypes

from ._lib import HALO_HOOK, call
from .field import GaugeAction, GaugeField, GaugeMomentum, Geometry, RngState
from .hmc import INTEGRATORS
from .slabs import run_hmc_evolve_slabs, run_hmc_pure_gauge_slabs


def coordinate_from_index(index: int, size):
    """coordinate_from_index (x fastest), as GeometryNode numbers its ranks."""
    c = []
    for s in size:
        c.append(index % s)
        index //= s
    return tuple(c)


def index_from_coordinate(coor, size) -> int:
    idx = 0
    for k in (3, 2, 1, 0):
        idx = idx * size[k] + coor[k] % size[k]
    return idx


def domain_layout(total_site, size_node, rank: int, halo: int = 2, cut=None):
    """The domain of rank ``rank`` on the grid ``size_node``: a dict with the
    local field extents, the global origin of its owned sites, the halo depth
    per direction, the owned extents and the neighbouring ranks (down, up) per
    direction.  A direction is cut (carries a halo) when it has more than one
    rank or when ``cut[k]`` is true; a cut direction with one rank exchanges
    with itself (its halo is its own periodic copy)."""
    total_site = tuple(int(v) for v in total_site)
    size_node = tuple(int(v) for v in size_node)
    if len(total_site) != 4 or len(size_node) != 4 or min(size_node) < 1:
        raise ValueError("domain_layout: total_site and size_node need four positive entries")
    cut = tuple(bool(c) for c in cut) if cut is not None else (False,) * 4
    coor = coordinate_from_index(rank, size_node)
    owned, halos, dims, origin, nbr = [], [], [], [], []
    for k in range(4):
        G, R = total_site[k], size_node[k]
        if G % R:
            raise ValueError(f"domain_layout: extent {G} in direction {k} is not divisible by {R} ranks")
        n = G // R
        h = halo if (R > 1 or cut[k]) else 0
        if h > n:
            raise ValueError(f"domain_layout: {n} owned sites in direction {k}, fewer than the halo depth {h}")
        owned.append(n)
        halos.append(h)
        dims.append(n + 2 * h)
        origin.append(coor[k] * n)
        up = list(coor)
        up[k] += 1
        dn = list(coor)
        dn[k] -= 1
        nbr.append((index_from_coordinate(dn, size_node), index_from_coordinate(up, size_node)))
    return {"coor": coor, "owned": tuple(owned), "halo": tuple(halos), "dims": tuple(dims), "origin": tuple(origin),
            "neighbours": tuple(nbr)}


class Domains:
    """The domain of this rank of ``total_site`` cut over a ``size_node`` grid
    of ranks (the product of size_node must be the group's size)."""

    def __init__(self, total_site, size_node, *, halo: int = 2, cut=None, group=None):
        import torch.distributed as dist
        self._dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.world = self._dist.get_world_size(group) if self._dist else 1
        self.rank = self._dist.get_rank(group) if self._dist else 0
        size_node = tuple(int(v) for v in size_node)
        n = 1
        for v in size_node:
            n *= v
        if n != self.world:
            raise ValueError(f"Domains: a {size_node} grid needs {n} ranks, the group has {self.world}")
        lay = domain_layout(total_site, size_node, self.rank, halo, cut)
        self.total_site = tuple(int(v) for v in total_site)
        self.total_volume = 1
        for v in self.total_site:
            self.total_volume *= v
        self.size_node = size_node
        self.coor = lay["coor"]
        self.owned = lay["owned"]
        self.halo = lay["halo"]
        self.dims = lay["dims"]
        self.origin = lay["origin"]
        self.neighbours = lay["neighbours"]
        self.geo = Geometry(self.dims)
        self.backend = self._dist.get_backend(group) if self._dist else None
        self._bufs = {}

    # ---- fields ---------------------------------------------------------------------------

    def _set_domain(self, handle) -> None:
        i4 = ctypes.c_int32 * 4
        call("qgb_field_set_domain", handle, i4(*self.total_site), i4(*self.origin), i4(*self.halo))

    def gauge_field(self) -> GaugeField:
        f = GaugeField(self.geo)
        self._set_domain(f.handle)
        return f

    def gauge_momentum(self) -> GaugeMomentum:
        f = GaugeMomentum(self.geo)
        self._set_domain(f.handle)
        return f

    def set_rand(self, gf: GaugeField, rng: RngState, sigma: float = 0.5, n_step: int = 1) -> None:
        """GaugeField.set_rand on the domain: every local site, halo included,
        gets the links a single field of the whole lattice gets at its global
        site."""
        gf.set_rand(rng, sigma, n_step)

    def set_rand_momentum(self, gm: GaugeMomentum, rng: RngState, sigma: float = 1.0) -> None:
        gm.set_rand(rng, sigma)

    # ---- communication ----------------------------------------------------------------------

    def _buffer(self, key, nbytes, device):
        import torch
        b = self._bufs.get((key, nbytes, device))
        if b is None:
            b = torch.empty(nbytes, dtype=torch.uint8, device=device)
            self._bufs[(key, nbytes, device)] = b
        return b

    def _host_buffer(self, key, nbytes):
        """A cached pinned host buffer (the gloo path's messages)."""
        import torch
        b = self._bufs.get(("host", key, nbytes))
        if b is None:
            b = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            self._bufs[("host", key, nbytes)] = b
        return b

    def faces(self, k: int):
        """The boxes of direction k's exchange: (the owned layers sent down,
        the owned layers sent up, the lower halo, the upper halo), each as
        (lo, n) over the whole local extent of the other directions."""
        h, n = self.halo[k], self.owned[k]
        ext = list(self.dims)
        ext[k] = h

        def box(start):
            lo = [0, 0, 0, 0]
            lo[k] = start
            return tuple(lo), tuple(ext)
        return box(h), box(n), box(0), box(h + n)

    def exchange(self, f) -> None:
        """Refresh the halo of f from the neighbouring domains (periodic grid)."""
        self._exchange_handle(f.handle)

    def _exchange_handle(self, handle) -> None:
        for k in range(4):
            if self.halo[k] == 0:
                continue
            send_dn, send_up, halo_lo, halo_hi = self.faces(k)
            if self._self_exchange(k):
                self._copy_faces(handle, k)
                continue
            up = self._pack(handle, send_up, ("send_up", k))
            dn = self._pack(handle, send_dn, ("send_dn", k))
            rlo, rhi = self._swap(k, up, dn)
            self._unpack(handle, halo_lo, rlo)
            self._unpack(handle, halo_hi, rhi)

    def _self_exchange(self, k: int) -> bool:
        """Direction k is cut but has one rank: its halo is its own periodic copy."""
        dn, up = self.neighbours[k]
        return self.world == 1 or (dn == self.rank and up == self.rank)

    def _copy_faces(self, handle, k: int) -> None:
        """The self-exchange of direction k, queued on the library stream
        without waiting: each face packed into a device buffer and unpacked
        into the opposite halo, in stream order."""
        i4 = ctypes.c_int32 * 4
        send_dn, send_up, halo_lo, halo_hi = self.faces(k)
        for src, dst, key in ((send_up, halo_lo, "face_up"), (send_dn, halo_hi, "face_dn")):
            nb = ctypes.c_int64()
            call("qgb_field_box_bytes", handle, i4(*src[1]), ctypes.byref(nb))
            buf = self._buffer((key, k), nb.value, "cuda")
            call("qgb_field_pack_box", handle, i4(*src[0]), i4(*src[1]), ctypes.c_void_p(buf.data_ptr()))
            call("qgb_field_unpack_box", handle, i4(*dst[0]), i4(*dst[1]), ctypes.c_void_p(buf.data_ptr()))

    def _pack(self, handle, box, key):
        """The sites of ``box`` of the field as a message: a device buffer over
        NCCL, its host copy over gloo."""
        from . import synchronize
        i4 = ctypes.c_int32 * 4
        (lo, n) = box
        nb = ctypes.c_int64()
        call("qgb_field_box_bytes", handle, i4(*n), ctypes.byref(nb))
        buf = self._buffer(key, nb.value, "cuda")
        call("qgb_field_pack_box", handle, i4(*lo), i4(*n), ctypes.c_void_p(buf.data_ptr()))
        synchronize()
        # one rank exchanges with itself: the message stays on the device
        if self.backend == "nccl" or self.world == 1:
            return buf
        host = self._host_buffer(key, nb.value)
        host.copy_(buf)
        return host

    def _unpack(self, handle, box, msg) -> None:
        import torch
        from . import synchronize
        i4 = ctypes.c_int32 * 4
        (lo, n) = box
        if msg.device.type != "cuda":
            dev = self._buffer(("recv_dev", box), msg.numel(), "cuda")
            dev.copy_(msg)
            msg = dev
        torch.cuda.current_stream().synchronize()
        call("qgb_field_unpack_box", handle, i4(*lo), i4(*n), ctypes.c_void_p(msg.data_ptr()))
        synchronize()

    def _recv_buffer(self, key, like):
        """A cached receive buffer of the shape, type and device of ``like``."""
        import torch
        full = key + (tuple(like.shape), like.dtype, like.device.type)
        b = self._bufs.get(full)
        if b is None:
            b = torch.empty_like(like)
            self._bufs[full] = b
        return b

    def _swap(self, k: int, send_up, send_dn):
        """Send the top owned layers of direction k up and the bottom ones
        down; returns what arrives for the lower halo (the lower neighbour's
        top layers) and for the upper halo (the upper neighbour's bottom
        layers).  With two ranks along k both neighbours are the same rank;
        the tags keep the two messages apart."""
        dn, up = self.neighbours[k]
        if self.world == 1 or (dn == self.rank and up == self.rank):
            return send_up, send_dn
        dist = self._dist
        rlo = self._recv_buffer(("recv_lo", k), send_up)
        rhi = self._recv_buffer(("recv_hi", k), send_dn)
        # posted in the same order on every rank: NCCL pairs the operations
        # between two ranks in order, gloo by tag
        ops = [dist.P2POp(dist.isend, send_up, up, self.group, 2 * k),
               dist.P2POp(dist.isend, send_dn, dn, self.group, 2 * k + 1),
               dist.P2POp(dist.irecv, rlo, dn, self.group, 2 * k),
               dist.P2POp(dist.irecv, rhi, up, self.group, 2 * k + 1)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        return rlo, rhi

    # ---- molecular dynamics and sums ------------------------------------------------------------

    def run_md(self, gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, n_step: int, md_time: float = 1.0, *,
               integrator: str = "force-gradient", reunit_interval: int = 0) -> None:
        """The molecular dynamics of one trajectory on the domain fields (FP64
        or FP32), with a halo exchange before every force evaluation."""
        reach = 2 if ga.c1() != 0.0 else 1
        for k in range(4):
            if 0 < self.halo[k] < reach:
                raise ValueError(f"Domains: a halo of {self.halo[k]} sites is thinner than the force's reach {reach}")
        errors = []

        def hook(handle, user):
            try:
                self._exchange_handle(handle)
                return 0
            except BaseException as e:  # raised again below, after the library call returns
                errors.append(e)
                return 1

        cb = HALO_HOOK(hook)
        try:
            call("qgb_run_md_hooked", gm.handle, gf.handle, ga.beta(), ga.c1(), int(n_step), float(md_time),
                 INTEGRATORS[integrator], int(reunit_interval), 1, cb, None)
        except Exception:
            if errors:
                raise errors[0]
            raise

    def glb_sum(self, x: float) -> float:
        """glb_sum (mpi.h:273-308): FP64 sum over the ranks."""
        if self.world == 1:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self._dist.all_reduce(t, group=self.group)
        return float(t.item())

    def gm_hamilton(self, gm: GaugeMomentum) -> float:
        o = ctypes.c_double()
        call("qgb_gm_hamilton_node", gm.handle, ctypes.byref(o))
        return self.glb_sum(o.value)

    def gf_hamilton(self, gf: GaugeField, ga: GaugeAction) -> float:
        """The gauge action over the whole lattice; the halo must be fresh."""
        o = ctypes.c_double()
        call("qgb_gf_hamilton_node", gf.handle, ga.beta(), ga.c1(), ctypes.byref(o))
        return self.glb_sum(o.value)

    def plaq(self, gf: GaugeField) -> float:
        """gf_avg_plaq over the whole lattice; the halo must be fresh."""
        out = (ctypes.c_double * 2)()
        call("qgb_gf_action_sums_sites", gf.handle, 0, 0, self.geo.total_volume, out)
        return 1.0 + self.glb_sum(out[0]) / (18.0 * self.total_volume)

    def owned_sites(self, a):
        """The owned part of a local field's numpy image (sites, ...), as an
        array over the owned box (t, z, y, x, ...)."""
        X, Y, Z, T = self.dims
        b = a.reshape((T, Z, Y, X) + a.shape[1:])
        h, n = self.halo, self.owned
        return b[h[3]:h[3] + n[3], h[2]:h[2] + n[2], h[1]:h[1] + n[1], h[0]:h[0] + n[0]]


def run_hmc_evolve_domains(dom: Domains, gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, n_step: int,
                           md_time: float = 1.0, **kw) -> float:
    """run_hmc_evolve_pure_gauge (hmc.pyx:169-188) on a domain decomposition:
    the same steps and kernels as on time slabs (run_hmc_evolve_slabs), with
    the exchanges of ``dom``; returns the global delta_h."""
    return run_hmc_evolve_slabs(dom, gm, gf, ga, n_step, md_time, **kw)


def run_hmc_pure_gauge_domains(dom: Domains, gf: GaugeField, ga: GaugeAction, traj: int, rs: RngState, **kw):
    """run_hmc_pure_gauge (hmc.pyx:190-216) on a domain decomposition; every
    rank takes the same Metropolis decision from the global delta_h."""
    return run_hmc_pure_gauge_slabs(dom, gf, ga, traj, rs, **kw)

"""Time-slab domain decomposition of pure-gauge HMC over ranks.

The reference runs its fields on MPI ranks with halo ("expanded") copies of
the neighbouring ranks' sites, refreshed before each force evaluation
(refresh_expanded, field-expand.h; hmc.cpp:466-490), and sums the Hamiltonians
over ranks (glb_sum).  Here the lattice is cut along the time direction: with R
ranks each rank owns T / R time slices and holds them with ``halo`` slices of
its two neighbours on either side, as one ordinary GPU field of time extent
T / R + 2 halo.  The library's kernels run unchanged on that field; the owned
sites are correct as long as the halo slices are fresh copies:

- the Iwasaki force reaches two slices (the Wilson force one), so a
  force-gradient momentum update (the force at U, the shifted
  U' = exp(eps F) U, the force at U') is right on the owned slices when the
  halo is twice the reach deep (4 slices) and was refreshed just before it:
  one exchange per update.  With a halo of just the reach (2 slices, the
  reference's own expansion for the rectangle action) the shifted field is
  exchanged too, before the force at U': two exchanges per update of half the
  slices each, and half the redundant halo work;
- the link updates are site-local and need no exchange;
- the molecular dynamics is the library's own fused kernel sequence
  (qgb_run_md_hooked), which calls back into ``exchange`` before each force
  evaluation: the FP64 form, and the mixed form on FP32 copies of the links
  and momenta (FP32 halos, half the bytes), run the kernels the single-GPU
  trajectories run;
- the Hamiltonians sum over the owned sites only and are then summed over
  ranks in FP64;
- momenta and hot starts use the per-site random streams of the global site
  index, so every owned site draws exactly what a single-GPU run draws.

The halo exchange packs the boundary slices of every component into one
contiguous buffer (qgb_field_pack_tslices) and sends it with torch.distributed
point-to-point operations: over NCCL from device buffers, over gloo through
host memory.  Communication is plumbing; all arithmetic stays in the
library's kernels.
"""

from __future__ import annotations

import ctypes

from ._lib import HALO_HOOK, call
from .field import F32, GaugeAction, GaugeField, GaugeMomentum, Geometry, RngState
from .hmc import INTEGRATORS, metropolis_accept, unitarize


class TimeSlabs:
    """The local slab of a lattice cut into ``world`` time slabs (rank ``rank``).

    ``geo`` is the geometry of the local field (time extent nt + 2 halo);
    ``owned`` the local site range [s0, s1) of the owned slices;
    ``site_offset`` the global index of local site 0 (the owned site s is
    global site s + site_offset)."""

    def __init__(self, total_site, *, halo: int = 4, group=None):
        import torch.distributed as dist
        self._dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.world = self._dist.get_world_size(group) if self._dist else 1
        self.rank = self._dist.get_rank(group) if self._dist else 0
        X, Y, Z, T = (int(v) for v in total_site)
        if T % self.world:
            raise ValueError(f"TimeSlabs: T = {T} is not divisible by {self.world} ranks")
        self.nt = T // self.world
        if self.nt < halo:
            raise ValueError(f"TimeSlabs: {self.nt} owned slices per rank, fewer than the halo depth {halo}")
        self.spatial = X * Y * Z
        if self.spatial % 32:
            raise ValueError("TimeSlabs: X * Y * Z must be a multiple of 32")
        self.halo = halo
        self.total_site = (X, Y, Z, T)
        self.total_volume = X * Y * Z * T
        self.geo = Geometry((X, Y, Z, self.nt + 2 * halo))
        self.t0 = self.rank * self.nt
        self.owned = (halo * self.spatial, (halo + self.nt) * self.spatial)
        self.site_offset = (self.t0 - halo) * self.spatial
        self.backend = self._dist.get_backend(group) if self._dist else None
        self._bufs = {}

    # ---- communication ----------------------------------------------------------------

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

    def exchange(self, f) -> None:
        """Refresh the halo slices of f from the neighbouring ranks (the ring
        of time slabs is periodic)."""
        self._exchange_handle(f.handle)

    def _exchange_handle(self, handle) -> None:
        import torch
        from . import synchronize
        h, nt = self.halo, self.nt
        n = ctypes.c_int64()
        call("qgb_field_tslice_bytes", handle, h, ctypes.byref(n))
        nbytes = n.value
        up_dev = self._buffer("send_up", nbytes, "cuda")
        dn_dev = self._buffer("send_dn", nbytes, "cuda")
        call("qgb_field_pack_tslices", handle, nt, h, ctypes.c_void_p(up_dev.data_ptr()))  # top owned slices
        call("qgb_field_pack_tslices", handle, h, h, ctypes.c_void_p(dn_dev.data_ptr()))   # bottom owned slices
        synchronize()
        if self.world == 1:
            rbot, rtop = up_dev, dn_dev
        else:
            on_host = self.backend != "nccl"
            if on_host:  # gloo: through cached pinned host buffers
                up_h = self._host_buffer("send_up", nbytes)
                dn_h = self._host_buffer("send_dn", nbytes)
                up_h.copy_(up_dev)
                dn_h.copy_(dn_dev)
                rbot_h, rtop_h = self._swap(up_h, dn_h)
                rbot = self._buffer("recv_bot_dev", nbytes, "cuda")
                rtop = self._buffer("recv_top_dev", nbytes, "cuda")
                rbot.copy_(rbot_h)
                rtop.copy_(rtop_h)
            else:
                rbot, rtop = self._swap(up_dev, dn_dev)
            torch.cuda.current_stream().synchronize()
        call("qgb_field_unpack_tslices", handle, 0, h, ctypes.c_void_p(rbot.data_ptr()))
        call("qgb_field_unpack_tslices", handle, nt + h, h, ctypes.c_void_p(rtop.data_ptr()))
        synchronize()

    def _swap(self, send_up, send_dn):
        """Send this rank's packed top slices up the ring and its bottom slices
        down; returns what arrives for the bottom halo (the lower neighbour's
        top slices) and for the top halo (the upper neighbour's bottom slices)."""
        dist = self._dist
        rbot = self._buffer("recv_bot", send_up.numel(), send_up.device.type)
        rtop = self._buffer("recv_top", send_dn.numel(), send_dn.device.type)
        up, dn = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        # posted in the same order on every rank: NCCL pairs the operations
        # between two ranks in order, gloo by tag
        ops = [dist.P2POp(dist.isend, send_up, up, self.group, 0),
               dist.P2POp(dist.isend, send_dn, dn, self.group, 1),
               dist.P2POp(dist.irecv, rbot, dn, self.group, 0),
               dist.P2POp(dist.irecv, rtop, up, self.group, 1)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        return rbot, rtop

    def run_md(self, gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, n_step: int, md_time: float = 1.0, *,
               integrator: str = "force-gradient", reunit_interval: int = 0) -> None:
        """The molecular dynamics of one trajectory on the slab fields (FP64 or
        FP32), with a halo exchange before every force evaluation that needs
        one."""
        reach = 2 if ga.c1() != 0.0 else 1
        if self.halo < reach:
            raise ValueError(f"TimeSlabs: a halo of {self.halo} slices is thinner than the force's reach {reach}")
        shifted = 1 if self.halo < 2 * reach else 0
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
                 INTEGRATORS[integrator], int(reunit_interval), shifted, cb, None)
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

    # ---- fields on the slab -------------------------------------------------------------

    def gauge_field(self) -> GaugeField:
        return GaugeField(self.geo)

    def gauge_momentum(self) -> GaugeMomentum:
        return GaugeMomentum(self.geo)

    def set_rand(self, gf: GaugeField, rng: RngState, sigma: float = 0.5, n_step: int = 1) -> None:
        """GaugeField.set_rand on the slab: the owned sites get the links a
        single-GPU field of the whole lattice gets; then the halo is filled."""
        call("qgb_gf_set_rand_sites", gf.handle, rng.c, float(sigma), int(n_step), self.site_offset)
        self.exchange(gf)

    def set_rand_momentum(self, gm: GaugeMomentum, rng: RngState, sigma: float = 1.0) -> None:
        call("qgb_set_rand_gauge_momentum_sites", gm.handle, float(sigma), rng.c, self.site_offset)

    def gm_hamilton(self, gm: GaugeMomentum) -> float:
        o = ctypes.c_double()
        call("qgb_gm_hamilton_node_sites", gm.handle, self.owned[0], self.owned[1], ctypes.byref(o))
        return self.glb_sum(o.value)

    def gf_hamilton(self, gf: GaugeField, ga: GaugeAction) -> float:
        """The gauge action over the whole lattice; the halo must be fresh."""
        o = ctypes.c_double()
        call("qgb_gf_hamilton_node_sites", gf.handle, ga.beta(), ga.c1(), self.owned[0], self.owned[1],
             ctypes.byref(o))
        return self.glb_sum(o.value)

    def plaq(self, gf: GaugeField) -> float:
        """gf_avg_plaq over the whole lattice; the halo must be fresh."""
        out = (ctypes.c_double * 2)()
        call("qgb_gf_action_sums_sites", gf.handle, 0, self.owned[0], self.owned[1], out)
        return 1.0 + self.glb_sum(out[0]) / (18.0 * self.total_volume)

    def owned_slices(self, a):
        """The owned part of a local field's numpy image (sites, ...)."""
        return a[self.owned[0]:self.owned[1]]


# ---- HMC on the slabs (hmc.pyx:157-216) ----------------------------------------------------


def run_hmc_evolve_slabs(slabs: TimeSlabs, gm: GaugeMomentum, gf: GaugeField, ga: GaugeAction, n_step: int,
                         md_time: float = 1.0, *, integrator: str = "force-gradient", precision: str = "fp64",
                         reunit_interval: int = 4) -> float:
    """run_hmc_evolve_pure_gauge (hmc.pyx:169-188) on time slabs: the same
    Omelyan force-gradient steps with a halo exchange before each momentum
    update, FP64 Hamiltonians over the owned sites summed over ranks; returns
    the global delta_h.  ``precision`` "mixed" runs the molecular dynamics on
    FP32 copies with FP64 re-unitarisation every ``reunit_interval`` steps, as
    run_hmc_evolve_pure_gauge(precision="mixed") does on one GPU."""
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    slabs.exchange(gf)
    energy = slabs.gm_hamilton(gm) + slabs.gf_hamilton(gf, ga)
    if precision == "fp64":
        slabs.run_md(gm, gf, ga, n_step, md_time, integrator=integrator)
    else:
        gf32, gm32 = gf.copy(F32), gm.copy(F32)
        slabs.run_md(gm32, gf32, ga, n_step, md_time, integrator=integrator, reunit_interval=reunit_interval)
        gf @= gf32
        gm @= gm32
    unitarize(gf)
    slabs.exchange(gf)
    return slabs.gm_hamilton(gm) + slabs.gf_hamilton(gf, ga) - energy


def run_hmc_pure_gauge_slabs(slabs: TimeSlabs, gf: GaugeField, ga: GaugeAction, traj: int, rs: RngState, *,
                             n_step: int = 6, md_time: float = 1.0, is_always_accept: bool = False,
                             integrator: str = "force-gradient", precision: str = "fp64", reunit_interval: int = 4):
    """run_hmc_pure_gauge (hmc.pyx:190-216) on time slabs; every rank takes the
    same Metropolis decision from the global delta_h.  Returns (flag, delta_h)."""
    rs = rs.split(f"{traj}")
    gf0 = gf.copy()
    gm = slabs.gauge_momentum()
    slabs.set_rand_momentum(gm, rs.split("set_rand_gauge_momentum"), 1.0)
    delta_h = run_hmc_evolve_slabs(slabs, gm, gf0, ga, n_step, md_time, integrator=integrator,
                                   precision=precision, reunit_interval=reunit_interval)
    flag, _ = metropolis_accept(delta_h, traj, rs.split("metropolis_accept"))
    if flag or is_always_accept:
        gf @= gf0
    return flag, delta_h

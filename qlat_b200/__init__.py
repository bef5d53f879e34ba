"""qlat_b200 -- B200-native pure-gauge SU(3) hot path with Qlattice's API.

``import qlat_b200 as q`` gives the names a Qlattice user calls for
pure-gauge HMC and gradient flow (GaugeField, GaugeMomentum, GaugeAction,
RngState, set_gm_force, gf_evolve, run_hmc_pure_gauge, gf_wilson_flow, ...),
backed by hand-written sm_100a CUDA kernels behind the C ABI declared in
include/qlat_b200.h.  Fields live in GPU memory.  There is no CPU fallback:
the first call loads the built libqlat_b200.so and raises if it is missing
(build it with `python -m qlat_b200.build`).
"""

from ._lib import QlatB200Error, load as _load
from .field import (F32, F64, Coordinate, Field, FieldColorMatrix, FieldRealD, GaugeAction, GaugeField,
                    GaugeMomentum, Geometry, RngState, read_gauge_field_header, set_unit)
from .hmc import (gf_avg_wilson_loop_normalized_tr, gf_avg_plaq, gf_evolve, gf_hamilton, gf_hamilton_node, gf_sum_re_tr_plaq_node_no_comm,
                  gf_sum_re_tr_rect_node_no_comm, glb_sum_double, gm_evolve_fg_pure_gauge, gm_hamilton_node,
                  metropolis_accept, metropolis_accept_cpp, run_hmc_evolve_pure_gauge, run_hmc_pure_gauge,
                  set_gm_force, set_rand_gauge_momentum, unitarize)
from .batch import ChainBatch
from .flowed_hmc import (FlowInfo, FlowStepInfo, gf_flow, gf_flow_and_ln_det_node, gf_flow_inv, gf_hamilton_flowed,
                         set_gm_force_flowed_no_det,
                         gf_hamilton_flowed_node, gm_evolve_fg_flowed, mk_flow_info_step, run_flowed_hmc,
                         run_hmc_evolve_flowed, set_gm_force_flowed)
from .hmc_fa import (MomentumAutoCorr, dot_gauge_momentum, gf_evolve_dual, gf_evolve_fa, gf_evolve_fa_dual,
                     gm_hamilton_node_fa, project_gauge_transform, run_hmc_fa, set_gauge_transform_momentum,
                     set_gm_force_dual, set_rand_gauge_momentum_fa)
from .topo_measure import (gf_energy_derivative_density_field_topo, gf_flow_topo, gf_plaq_action_density,
                           gf_plaq_action_density_field, gf_plaq_field, gf_plaq_flow_force,
                           gf_spatial_plaq_action_density, gf_spatial_plaq_action_density_field, smear_measure_topo)
from .slabs import TimeSlabs, run_hmc_evolve_slabs, run_hmc_pure_gauge_slabs
from .domains import Domains, domain_layout, run_hmc_evolve_domains, run_hmc_pure_gauge_domains
from .flow_adjoint import (FlowedWilsonAction, gf_flow_action, gf_flow_action_grad, gf_wilson_flow_vjp,
                           run_flowed_hmc_pure_gauge, set_anti_hermitian_matrix_from_basis,
                           set_basis_from_anti_hermitian_matrix)
from .wilson_flow import (gf_energy_density_dir_field, topology_charge_5,
                          gf_energy_density, gf_energy_density_field, gf_energy_derivative_density_field,
                          gf_topology, gf_topology_clf, gf_topology_field, gf_topology_field_clf, gf_topology_terms,
                          gf_topology_terms_field, gf_wilson_flow, gf_wilson_flow_force,
                          gf_wilson_flow_step)

__version__ = "0.1.0"


def prof_enable(on: bool = True):
    from ._lib import call
    call("qgb_prof_enable", int(bool(on)))


def prof_reset():
    from ._lib import call
    call("qgb_prof_reset")


def prof_get(name: str):
    """(total_ms, launches) of a kernel class since the last reset."""
    import ctypes
    from ._lib import call
    t = ctypes.c_double()
    n = ctypes.c_int64()
    call("qgb_prof_get", name.encode(), ctypes.byref(t), ctypes.byref(n))
    return t.value, int(n.value)


def rng_ambiguous_count() -> int:
    import ctypes
    from ._lib import call
    n = ctypes.c_int64()
    call("qgb_rng_ambiguous_count", ctypes.byref(n))
    return int(n.value)


def set_trajectory_graphs(enable: bool = True) -> None:
    """Replay trajectories (run_hmc_evolve_pure_gauge, both precisions) as
    CUDA graphs (default) or launch their kernels one by one."""
    from ._lib import call
    call("qgb_set_trajectory_graphs", int(bool(enable)))


def trajectory_graph_count() -> int:
    import ctypes
    from ._lib import call
    n = ctypes.c_int32()
    call("qgb_trajectory_graph_count", ctypes.byref(n))
    return int(n.value)


def launch_count() -> int:
    import ctypes
    from ._lib import call
    n = ctypes.c_int64()
    call("qgb_launch_count", ctypes.byref(n))
    return int(n.value)


def set_stream(stream_ptr: int):
    """Queue all library work on this cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
    import ctypes
    from ._lib import call
    call("qgb_set_stream", ctypes.c_void_p(stream_ptr))


def set_device(device: int):
    from ._lib import call
    call("qgb_set_device", int(device))


def force_variants():
    """The force-kernel launch shapes: list of dicts (block_size, min_blocks,
    threads_per_link, site_map)."""
    import ctypes
    from ._lib import call
    n = ctypes.c_int32()
    call("qgb_force_variant_count", ctypes.byref(n))
    out = []
    for v in range(n.value):
        a = [ctypes.c_int32() for _ in range(4)]
        call("qgb_force_variant_info", v, *[ctypes.byref(x) for x in a])
        out.append(dict(block_size=a[0].value, min_blocks=a[1].value, threads_per_link=a[2].value,
                        site_map=a[3].value))
    return out


def force_set_variant(precision: int, rect: bool, variant: int):
    from ._lib import call
    call("qgb_force_set_variant", int(precision), int(bool(rect)), int(variant))

def force_get_variant(precision: int, rect: bool) -> int:
    import ctypes
    from ._lib import call
    v = ctypes.c_int32()
    call("qgb_force_get_variant", int(precision), int(bool(rect)), ctypes.byref(v))
    return int(v.value)


def autotune_force(gf, c1: float, reps: int = 3):
    """Time every force-kernel variant on gf (its precision) and keep the
    fastest for (precision, c1 != 0).  Returns (variant, ms per launch)."""
    import ctypes
    from ._lib import call
    b = ctypes.c_int32()
    t = ctypes.c_double()
    call("qgb_autotune_force", gf.handle, float(c1), int(reps), ctypes.byref(b), ctypes.byref(t))
    return b.value, t.value


def force_time_variant(gf, c1: float, variant: int, reps: int = 3) -> float:
    import ctypes
    from ._lib import call
    t = ctypes.c_double()
    call("qgb_force_time_variant", gf.handle, float(c1), int(variant), int(reps), ctypes.byref(t))
    return t.value


def synchronize():
    from ._lib import call
    call("qgb_synchronize")


def download_join():
    """Order the library stream after every queued GaugeField.download_host_async."""
    from ._lib import call
    call("qgb_field_download_join")


def release_field_pool() -> int:
    """Free the device storage the library keeps from destroyed fields for
    reuse (torch.cuda.empty_cache for this library's fields); returns the
    bytes freed."""
    import ctypes
    from ._lib import call
    n = ctypes.c_int64()
    call("qgb_field_pool_release", ctypes.byref(n))
    return int(n.value)

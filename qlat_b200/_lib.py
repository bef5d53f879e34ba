"""Loader for libqlat_b200.so (the C ABI of include/qlat_b200.h).

The library is built in-tree (``python -m qlat_b200.build``).  There is no
fallback: if the shared library is missing the import fails with a message
saying how to build it.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqlat_b200.so")

c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_i32_p = ctypes.POINTER(ctypes.c_int32)
c_i64_p = ctypes.POINTER(ctypes.c_int64)
c_u64_p = ctypes.POINTER(ctypes.c_uint64)
c_field = ctypes.c_void_p
c_field_p = ctypes.POINTER(ctypes.c_void_p)
i32x4 = ctypes.c_int32 * 4
# qgb_halo_hook: int (*)(qgb_field* gf, void* user)
HALO_HOOK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)

# name -> (argtypes); every entry point returns int status
SIGNATURES = {
    "qgb_version": [],
    "qgb_set_device": [ctypes.c_int32],
    "qgb_set_stream": [ctypes.c_void_p],
    "qgb_synchronize": [],
    "qgb_field_create": [c_field_p, i32x4, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
    "qgb_field_destroy": [c_field],
    "qgb_field_pool_release": [c_i64_p],
    "qgb_nersc_write_host": [ctypes.c_char_p, c_dbl_p, i32x4, ctypes.c_double, ctypes.c_double, ctypes.c_char_p,
                             ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int64,
                             c_i64_p],
    "qgb_nersc_read_header": [ctypes.c_char_p, i32x4, c_i32_p, c_i32_p, c_dbl_p, c_dbl_p, c_u32_p, c_u32_p],
    "qgb_nersc_read_host": [ctypes.c_char_p, c_dbl_p, i32x4, c_i32_p, c_i64_p],
    "qgb_save_gauge_field": [c_field, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                             ctypes.c_double, ctypes.c_int64, c_i64_p],
    "qgb_load_gauge_field": [c_field, ctypes.c_char_p, c_i32_p, c_i64_p],
    "qgb_flow_info_step": [c_u32_p, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p, c_i32_p],
    "qgb_gf_flow": [c_field, c_field, ctypes.c_void_p, ctypes.c_int32],
    "qgb_gf_flow_inv": [c_field, c_field, ctypes.c_void_p, ctypes.c_int32],
    "qgb_gf_flow_and_ln_det_node": [c_field, c_field, ctypes.c_void_p, ctypes.c_int32, c_dbl_p],
    "qgb_gf_hamilton_flowed_node": [c_field, ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_int32,
                                    c_dbl_p, c_dbl_p],
    "qgb_set_gm_force_flowed": [c_field, c_field, ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_int32,
                                ctypes.c_int32],
    "qgb_set_gm_force_flowed_no_det": [c_field, c_field, c_field, ctypes.c_void_p, ctypes.c_int32],
    "qgb_set_rand_gauge_momentum_fa": [c_field, c_field, c_u32_p],
    "qgb_gm_hamilton_node_fa": [c_field, c_field, c_dbl_p],
    "qgb_gf_evolve_fa": [c_field, c_field, c_field, ctypes.c_double],
    "qgb_gf_evolve_dual": [c_field, c_field, ctypes.c_double],
    "qgb_gf_evolve_fa_dual": [c_field, c_field, c_field, ctypes.c_double],
    "qgb_set_gm_force_dual": [c_field, c_field, c_field],
    "qgb_project_gauge_transform": [c_field, c_field, c_field, c_field, c_dbl_p],
    "qgb_set_gauge_transform_momentum": [c_field, c_field, c_field],
    "qgb_dot_gauge_momentum": [c_field, c_field, c_field],
    "qgb_field_set_u_rand": [c_field, c_u32_p, ctypes.c_double, ctypes.c_double],
    "qgb_field_set_g_rand": [c_field, c_u32_p, ctypes.c_double, ctypes.c_double],
    "qgb_field_fill": [c_field, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64],
    "qgb_field_set_selected": [c_field, c_field, ctypes.c_void_p, ctypes.c_int64],
    "qgb_gf_plaq_field": [c_field, c_field],
    "qgb_gf_energy_density_dir_field": [c_field, c_field],
    "qgb_topology_charge_5": [c_field, c_dbl_p],
    "qgb_gf_avg_wilson_loop_normalized_tr": [c_field, ctypes.c_int32, ctypes.c_int32, c_dbl_p],
    "qgb_gf_plaq_action_density_field": [c_field, c_field, ctypes.c_int32],
    "qgb_set_plaq_flow_z": [c_field, c_field, c_field],
    "qgb_gf_flow_topo": [c_field, ctypes.c_double, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, c_dbl_p],
    "qgb_field_glb_min_max": [c_field, c_dbl_p, c_dbl_p],
    "qgb_field_glb_sum_tslice": [c_field, ctypes.c_int32, c_dbl_p],
    "qgb_field_abs": [c_field],
    "qgb_gm_hamilton_node_sites": [c_field, ctypes.c_int64, ctypes.c_int64, c_dbl_p],
    "qgb_gf_action_sums_sites": [c_field, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, c_dbl_p],
    "qgb_gf_hamilton_node_sites": [c_field, ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_int64,
                                   c_dbl_p],
    "qgb_set_rand_gauge_momentum_sites": [c_field, ctypes.c_double, c_u32_p, ctypes.c_int64],
    "qgb_gf_set_rand_sites": [c_field, c_u32_p, ctypes.c_double, ctypes.c_int32, ctypes.c_int64],
    "qgb_field_tslice_bytes": [c_field, ctypes.c_int32, c_i64_p],
    "qgb_field_pack_tslices": [c_field, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p],
    "qgb_field_unpack_tslices": [c_field, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p],
    "qgb_field_set_domain": [c_field, c_i32_p, c_i32_p, c_i32_p],
    "qgb_field_domain": [c_field, c_i32_p, c_i32_p, c_i32_p, c_i32_p],
    "qgb_field_box_bytes": [c_field, c_i32_p, c_i64_p],
    "qgb_field_pack_box": [c_field, c_i32_p, c_i32_p, ctypes.c_void_p],
    "qgb_field_unpack_box": [c_field, c_i32_p, c_i32_p, ctypes.c_void_p],
    "qgb_field_info": [c_field, i32x4, c_i32_p, c_i32_p, c_i32_p],
    "qgb_field_upload": [c_field, c_dbl_p],
    "qgb_field_download": [c_field, c_dbl_p],
    "qgb_field_upload_device": [c_field, ctypes.c_void_p],
    "qgb_field_upload_pipelined": [c_field, ctypes.c_void_p, ctypes.c_void_p],
    "qgb_field_download_async": [c_field, ctypes.c_void_p],
    "qgb_field_download_join": [],
    "qgb_field_download_device": [c_field, ctypes.c_void_p],
    "qgb_field_copy": [c_field, c_field],
    "qgb_field_set_zero": [c_field],
    "qgb_field_axpby": [c_field, ctypes.c_double, c_field, ctypes.c_double],
    "qgb_field_qnorm": [c_field, c_dbl_p],
    "qgb_rng_seed": [c_u32_p, ctypes.c_char_p],
    "qgb_rng_split": [c_u32_p, c_u32_p, ctypes.c_char_p],
    "qgb_rng_rand_gen": [c_u32_p, c_u64_p],
    "qgb_rng_u_rand_gen": [c_u32_p, ctypes.c_double, ctypes.c_double, c_dbl_p],
    "qgb_rng_g_rand_gen": [c_u32_p, ctypes.c_double, ctypes.c_double, c_dbl_p],
    "qgb_set_unit": [c_field],
    "qgb_gf_set_rand": [c_field, c_u32_p, ctypes.c_double, ctypes.c_int32],
    "qgb_set_rand_gauge_momentum": [c_field, ctypes.c_double, c_u32_p],
    "qgb_gm_hamilton_node": [c_field, c_dbl_p],
    "qgb_gf_hamilton_node": [c_field, ctypes.c_double, ctypes.c_double, c_dbl_p],
    "qgb_gf_sum_re_tr_plaq_node": [c_field, c_dbl_p],
    "qgb_gf_sum_re_tr_rect_node": [c_field, c_dbl_p],
    "qgb_gf_avg_plaq": [c_field, c_dbl_p],
    "qgb_set_gm_force": [c_field, c_field, ctypes.c_double, ctypes.c_double],
    "qgb_gf_evolve": [c_field, c_field, ctypes.c_double],
    "qgb_gm_evolve_fg": [c_field, c_field, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double],
    "qgb_unitarize": [c_field],
    "qgb_metropolis_accept": [ctypes.c_double, ctypes.c_int32, c_u32_p, c_dbl_p, c_i32_p],
    "qgb_run_hmc_evolve": [c_field, c_field, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_double,
                           ctypes.c_int32, c_dbl_p],
    "qgb_run_hmc_evolve_mixed": [c_field, c_field, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                 ctypes.c_double, ctypes.c_int32, ctypes.c_int32, c_dbl_p],
    "qgb_set_trajectory_graphs": [ctypes.c_int32],
    "qgb_trajectory_graph_count": [c_i32_p],
    "qgb_run_md_hooked": [c_field, c_field, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_double,
                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, HALO_HOOK, ctypes.c_void_p],
    "qgb_set_wilson_flow_z": [c_field, c_field, ctypes.c_double],
    "qgb_gf_wilson_flow_step": [c_field, ctypes.c_double, ctypes.c_double],
    "qgb_gf_wilson_flow_step_euler": [c_field, ctypes.c_double, ctypes.c_double],
    "qgb_gf_energy_density_field": [c_field, c_field],
    "qgb_gf_energy_density": [c_field, c_dbl_p],
    "qgb_gf_wilson_flow": [c_field, ctypes.c_double, ctypes.c_int32, ctypes.c_double, c_dbl_p],
    "qgb_gf_wilson_flow_vjp": [c_field, ctypes.c_double, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, c_field,
                               c_field],
    "qgb_gf_flow_action_grad": [c_field, ctypes.c_double, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                ctypes.c_double, ctypes.c_double, c_field, c_dbl_p],
    "qgb_set_anti_hermitian_matrix_from_basis": [c_field, c_field],
    "qgb_set_basis_from_anti_hermitian_matrix": [c_field, c_field],
    "qgb_su3_dexp_adjoint": [c_field, c_field, c_field],
    "qgb_clf_topology_field": [c_field, c_field],
    "qgb_gf_topology_clf": [c_field, c_dbl_p],
    "qgb_clf_topology_field_5_terms": [c_field, c_field],
    "qgb_clf_topology_field_5": [c_field, c_field],
    "qgb_gf_topology_terms": [c_field, c_dbl_p],
    "qgb_gf_topology": [c_field, c_dbl_p],
    "qgb_prof_enable": [ctypes.c_int32],
    "qgb_prof_reset": [],
    "qgb_prof_get": [ctypes.c_char_p, c_dbl_p, c_i64_p],
    "qgb_force_variant_count": [c_i32_p],
    "qgb_force_variant_info": [ctypes.c_int32, c_i32_p, c_i32_p, c_i32_p, c_i32_p],
    "qgb_force_set_variant": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
    "qgb_force_get_variant": [ctypes.c_int32, ctypes.c_int32, c_i32_p],
    "qgb_autotune_force": [c_field, ctypes.c_double, ctypes.c_int32, c_i32_p, c_dbl_p],
    "qgb_force_time_variant": [c_field, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, c_dbl_p],
    "qgb_gf_action_sums_noalloc": [ctypes.c_void_p, i32x4, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p],
    "qgb_batch_create": [c_field_p, ctypes.c_int32, c_i32_p, c_dbl_p, c_dbl_p],
    "qgb_batch_destroy": [c_field],
    "qgb_batch_info": [c_field, c_i32_p, c_i64_p],
    "qgb_batch_set_rand": [c_field, c_u32_p, ctypes.c_double, ctypes.c_int32],
    "qgb_batch_trajectory": [c_field, c_u32_p, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int32, ctypes.c_int32, c_dbl_p],
    "qgb_batch_run_hmc": [c_field, c_u32_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_dbl_p, c_i32_p],
    "qgb_batch_accept": [c_field, c_i32_p],
    "qgb_batch_plaq": [c_field, c_dbl_p],
    "qgb_batch_autotune": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, c_i32_p, c_dbl_p],
    "qgb_batch_set_force_variant": [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32],
    "qgb_batch_download_chain": [c_field, ctypes.c_int32, c_dbl_p],
    "qgb_batch_upload_chain": [c_field, ctypes.c_int32, c_dbl_p],
    "qgb_launch_count": [c_i64_p],
    "qgb_rng_ambiguous_count": [c_i64_p],
}

_lib = None


# exported for the benchmark, not declared in include/qlat_b200.h
INTERNAL = {
    "qgb_fma_rate": [ctypes.c_int32, ctypes.c_int32, c_dbl_p],
}


def load() -> ctypes.CDLL:
    """Load the shared library (building nothing).  Raises RuntimeError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m qlat_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in {**SIGNATURES, **INTERNAL}.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.qgb_last_error.argtypes = []
    lib.qgb_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


class QlatB200Error(RuntimeError):
    """Raised when a C ABI call returns a non-zero status (the reference
    raises RuntimeError from its C++ exceptions through Cython `except +`)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[qgb status {code}] {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != 0:
        raise QlatB200Error(rc, load().qgb_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))

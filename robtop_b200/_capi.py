"""ctypes binding of ``include/rtb200.h`` (the library's C ABI).

The product path always goes through ``librtb200.so``; if the library is
missing or cannot be loaded this module raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librtb200.so")

RT_OK, RT_EINVAL, RT_ECUDA, RT_ENOCONV, RT_ENAN, RT_ETIMEOUT, RT_ENOMEM, RT_ESTATE = range(8)
STATUS_NAMES = {0: "RT_OK", 1: "RT_EINVAL", 2: "RT_ECUDA", 3: "RT_ENOCONV", 4: "RT_ENAN", 5: "RT_ETIMEOUT",
                6: "RT_ENOMEM", 7: "RT_ESTATE"}
MODE_NSCF, MODE_NSFF, MODE_WSCF, MODE_WSFF = range(4)
SMOOTH_GS, SMOOTH_SGS, SMOOTH_JACOBI, SMOOTH_CHEBY = range(4)
FP64, FP32, FP64_FINE = 0, 1, 2
LAYOUT_DENSE, LAYOUT_REF_GS = 0, 1
FIELD_U, FIELD_F, FIELD_R, FIELD_RHO, FIELD_SENS, FIELD_STENCIL, FIELD_VACT, FIELD_EACT, FIELD_VFIX, \
    FIELD_PENALTY = range(10)
WORST_MODPM, WORST_LANCZOS, WORST_BLOCK_LANCZOS = 0, 1, 2


class Params(C.Structure):
    """rt_params (optimization/optimization.h:11-22 plus solver knobs)."""
    _fields_ = [
        ("power_penalty", C.c_float), ("min_rho", C.c_float), ("volume_ratio", C.c_float),
        ("design_step", C.c_float), ("damp_ratio", C.c_float), ("filter_radius", C.c_float),
        ("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double), ("element_length", C.c_double),
        ("mode", C.c_int), ("skip_layer1", C.c_int), ("smoother", C.c_int), ("pre_sweeps", C.c_int),
        ("post_sweeps", C.c_int), ("jacobi_omega", C.c_double), ("precision", C.c_int),
        ("coarsest_elements", C.c_int), ("cycle_gamma", C.c_int), ("coarse_sweeps", C.c_int),
        ("precision_fallback", C.c_int), ("coarse_bf16", C.c_int), ("krylov_fp32", C.c_int),
        ("cycle_gamma_levels", C.c_int),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("inner_iterations", C.c_int), ("vcycles", C.c_int), ("status", C.c_int),
        ("rel_residual", C.c_double), ("value", C.c_double), ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LevelInfo(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ratio", C.c_int),
        ("n_nodes", C.c_longlong), ("n_active_nodes", C.c_longlong), ("n_active_elements", C.c_longlong),
    ]


P = C.c_void_p
I = C.c_int
D = C.c_double
F = C.c_float

# name -> (restype, argtypes); every entry must be exported by the library
SIGNATURES = {
    "rt_ctx_create": (I, [I, P, C.POINTER(P)]),
    "rt_ctx_destroy": (None, [P]),
    "rt_last_error": (C.c_char_p, [P]),
    "rt_ctx_sync": (I, [P]),
    "rt_params_default": (None, [C.POINTER(Params)]),
    "rt_profile_enable": (I, [P, I]),
    "rt_profile_query": (I, [P, I, C.c_char_p, I, C.POINTER(C.c_longlong), C.POINTER(D)]),
    "rt_profile_reset": (I, [P]),
    "rt_launch_count": (C.c_longlong, [P]),
    "rt_hier_create": (I, [P, C.POINTER(Params), I, I, I, P, C.POINTER(P)]),
    "rt_hier_create_from_bits": (I, [P, C.POINTER(Params), I, P, C.POINTER(P)]),
    "rt_hier_destroy": (None, [P]),
    "rt_hier_n_levels": (I, [P]),
    "rt_hier_level_info": (I, [P, I, C.POINTER(LevelInfo)]),
    "rt_hier_set_params": (I, [P, C.POINTER(Params)]),
    "rt_hier_get_params": (I, [P, C.POINTER(Params)]),
    "rt_template_matrix": (I, [P, P]),
    "rt_cube_vertex_bits": (I, [P, I, P, P]),
    "rt_cube_coarsen_bits": (I, [P, I, P, P]),
    "rt_surface_nodes": (I, [P, P]),
    "rt_set_support": (I, [P, P]),
    "rt_set_load_nodes": (I, [P, I, P, P]),
    "rt_init_density": (I, [P, F]),
    "rt_put": (I, [P, I, I, I, P]),
    "rt_get": (I, [P, I, I, I, P]),
    "rt_put_dev": (I, [P, I, I, P]),
    "rt_get_dev": (I, [P, I, I, P]),
    "rt_ref_gs_map": (I, [P, I, P, P, P]),
    "rt_update_stencil": (I, [P]),
    "rt_update_residual": (I, [P, I]),
    "rt_smoother_lmax": (I, [P, I, C.POINTER(D)]),
    "rt_smooth": (I, [P, I, I, I, D]),
    "rt_restrict_residual": (I, [P, I]),
    "rt_prolongate_correction": (I, [P, I]),
    "rt_coarsest_solve": (I, [P]),
    "rt_vcycle": (I, [P, I, I, C.POINTER(D)]),
    "rt_apply_K_dev": (I, [P, P, P]),
    "rt_apply_K": (I, [P, P, P]),
    "rt_compliance": (I, [P, C.POINTER(D)]),
    "rt_relative_residual": (I, [P, C.POINTER(D)]),
    "rt_compliance_noalloc": (I, [P, P, C.c_longlong, P, P]),
    "rt_autotune": (I, [P, I]),
    "rt_tuning_info": (I, [P, I, I, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(D)]),
    "rt_set_tuning": (I, [P, I, I, I, I, I]),
    "rt_bench_fine_kernel": (I, [P, I, I, I, C.POINTER(D)]),
    "rt_bench_level_kernel": (I, [P, I, I, I, I, C.POINTER(D)]),
    "rt_bench_simt_peak": (I, [P, I, I, C.POINTER(D)]),
    "rt_set_level_fused": (I, [P, I, I]),
    "rt_smooth_f32": (I, [P, I, I, I, D]),
    "rt_level_fused_info": (I, [P, I, C.POINTER(I), C.POINTER(D), C.POINTER(D)]),
    "rt_fine_kernel_f32": (I, [P, I, D]),
    "rt_set_shell": (I, [P, P]),
    "rt_voxel_resolution": (I, [I]),
    "rt_voxelize_mesh": (I, [P, P, C.c_long, P, C.c_long, I, P, C.c_long, P, P]),
    "rt_hier_create_from_mesh": (I, [P, C.POINTER(Params), P, C.c_long, P, C.c_long, I, C.POINTER(P)]),
    "rt_bench_voxelize": (I, [P, P, C.c_long, P, C.c_long, I, I, C.POINTER(D)]),
    "rt_level_kernel_info": (I, [P, I, C.POINTER(I), C.POINTER(D), C.POINTER(D)]),
    "rt_set_level_kernel": (I, [P, I, I]),
    "rt_pcg": (I, [P, D, I, C.POINTER(SolveInfo)]),
    "rt_hier_precision_fallbacks": (C.c_longlong, [P]),
    "rt_worst_case": (I, [P, I, I, D, C.c_uint64, C.POINTER(D), C.POINTER(SolveInfo)]),
    "rt_worst_case_block": (I, [P, I, I, D, C.c_uint64, C.POINTER(D), C.POINTER(SolveInfo)]),
    "rt_hier_workspace_create": (I, [P, C.POINTER(P)]),
    "rt_pcg_batch": (I, [C.POINTER(P), I, D, I, C.POINTER(SolveInfo)]),
    "rt_unet_conv3": (I, [P, P, I, I, P, P, I, P, I, I, I, I, I, I, I]),
    "rt_unet_set_conv_variant": (I, [I]),
    "rt_unet_create": (I, [P, I, I, I, C.c_uint64, C.POINTER(P)]),
    "rt_unet_destroy": (None, [P]),
    "rt_unet_n_params": (C.c_longlong, [P]),
    "rt_unet_get_params": (I, [P, P]),
    "rt_unet_set_params": (I, [P, P]),
    "rt_unet_forward": (I, [P, P, P]),
    "rt_unet_gradients": (I, [P, P, P, C.POINTER(D), P]),
    "rt_unet_train_step": (I, [P, I, P, P, F, C.POINTER(D)]),
    "rt_unet_output_scale": (D, [P]),
    "rt_unet_set_output_scale": (I, [P, D]),
    "rt_unet_harvest": (I, [P, P, I, C.c_uint64, P, P]),
    "rt_hier_set_learned": (I, [P, P, D]),
    "rt_hier_learned_stats": (I, [P, C.POINTER(C.c_longlong), C.POINTER(I)]),
    "rt_hier_set_learned_post": (I, [P, I]),
    "rt_force_project": (I, [P, P]),
    "rt_ctx_set_wait_limit": (I, [P, C.c_longlong]),
    "rt_get_force_support": (I, [P, P, P]),
    "rt_set_force_support": (I, [P, P, P]),
    "rt_displacement_project": (I, [P, P]),
    "rt_load_nodes": (I, [P, C.POINTER(I), P]),
    "rt_element_compliance": (I, [P, P, P]),
    "rt_sensitivity": (I, [P, I]),
    "rt_filter_sensitivity": (I, [P, F]),
    "rt_oc_update": (I, [P, F, C.POINTER(F), C.POINTER(I)]),
    "rt_oc_iteration": (I, [P, I, I, D, C.c_uint64, F, C.POINTER(D)]),
    "rt_mma_create": (I, [P, C.c_longlong, P, P, D, D, C.POINTER(P)]),
    "rt_mma_destroy": (I, [P]),
    "rt_mma_update": (I, [P, P, P, D, C.POINTER(I), C.POINTER(D), C.POINTER(D)]),
    "rt_mma_x": (I, [P, C.POINTER(P)]),
    "rt_mma_get_x": (I, [P, P]),
    "rt_mma_set_density": (I, [P, P]),
    "rt_mma_evaluations": (C.c_longlong, [P]),
}

_lib = None


def lib():
    """Load ``librtb200.so`` once (raises if it is absent: no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m robtop_b200.build` (nvcc, sm_100a); "
                "robtop_b200 has no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class RTError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, ctx=None):
    if status != RT_OK:
        msg = lib().rt_last_error(ctx).decode() if ctx else ""
        raise RTError(status, msg)
    return status

"""ctypes binding of ``libcavity_b200.so`` (the C ABI of ``include/cavity.h``).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcavity_b200.so")

CAV_OK = 0
CAV_ERR_ARG = 1
CAV_ERR_TAU = 2
CAV_ERR_DIVERGED = 3
CAV_ERR_MAXU = 4
CAV_ERR_TIMEOUT = 5
CAV_ERR_CUDA = 6
CAV_ERR_STATE = 7
CAV_ERR_NOMEM = 8
CAV_ERR_IO = 9

(CAV_PREC_F64, CAV_PREC_F32, CAV_PREC_F16, CAV_PREC_BF16, CAV_PREC_F16G, CAV_PREC_F16SR,
 CAV_PREC_BF16SR, CAV_PREC_F16GSR) = range(8)
PRECISIONS = {"f64": CAV_PREC_F64, "f32": CAV_PREC_F32, "f16": CAV_PREC_F16, "bf16": CAV_PREC_BF16,
              "f16g": CAV_PREC_F16G, "f16sr": CAV_PREC_F16SR, "bf16sr": CAV_PREC_BF16SR,
              "f16gsr": CAV_PREC_F16GSR}
CAV_INIT_LINEAR, CAV_INIT_ZERO = 0, 1
CAV_STEP_NODE, CAV_STEP_PAIR, CAV_STEP_PAIR_SPLIT = 0, 1, 2
CAV_OCT_LEVEL_NODE, CAV_OCT_LEVEL_FG = 0, 1
(CAV_PHASE_COLLIDE, CAV_PHASE_STREAM, CAV_PHASE_BOUNCE_BACK, CAV_PHASE_THERMAL_BC,
 CAV_PHASE_MACRO, CAV_PHASE_NOSLIP, CAV_PHASE_FUSED_IDENTITY, CAV_PHASE_CHANNEL) = range(8)

_dp = ctypes.POINTER(ctypes.c_double)


class CavParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("ra", ctypes.c_double), ("pr", ctypes.c_double), ("cs", ctypes.c_double),
        ("pr_t", ctypes.c_double), ("utarget", ctypes.c_double),
        ("seed", ctypes.c_uint64), ("jobs", ctypes.c_int32),
        ("alpha_mult", ctypes.c_double), ("nu_start_mult", ctypes.c_double),
        ("has_nu_override", ctypes.c_int32), ("nu_override", ctypes.c_double),
        ("init_mode", ctypes.c_int32), ("noise_amp", ctypes.c_double),
        ("geq_order", ctypes.c_int32),
        ("t_hot_profile", _dp),
        ("t_cold", ctypes.c_double),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
    ]


class CavInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("nu", "alpha", "alpha_phys", "beta_eff", "lz", "lx", "tau", "tau_t")] + [
        ("time_step", ctypes.c_int64), ("spin_up_steps", ctypes.c_int64),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("pitch", ctypes.c_int32),
        ("precision", ctypes.c_int32)]


class CavDiag(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("nusselt_hot", "nusselt_cold", "nusselt_hot_wall_link", "total_mass",
                 "total_f_mass", "max_u", "max_uy", "nu_t_max", "y_plus_hot",
                 "nusselt_volume")] + [("finite", ctypes.c_int32)]


class CavBatchTuning(ctypes.Structure):
    _fields_ = [("rows_per_item", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32), ("kernel", ctypes.c_int32)]


class CavAdjointSpec(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int64), ("window_start", ctypes.c_int64),
                ("checkpoint_every", ctypes.c_int32)]


class CavAdjointResult(ctypes.Structure):
    _fields_ = [("objective", ctypes.c_double), ("grad_cs", ctypes.c_double),
                ("forward_ms", ctypes.c_double), ("reverse_ms", ctypes.c_double),
                ("checkpoints", ctypes.c_int64)]


CAV_OCT_F64, CAV_OCT_F32, CAV_OCT_F32_F16, CAV_OCT_F32_F16G = range(4)
OCT_PRECISIONS = {"f64": CAV_OCT_F64, "f32": CAV_OCT_F32, "f32_f16": CAV_OCT_F32_F16,
                  "f32_f16g": CAV_OCT_F32_F16G}


class CavOctreeParams(ctypes.Structure):
    _fields_ = [
        ("nx0", ctypes.c_int32), ("ny0", ctypes.c_int32), ("bl_width", ctypes.c_int32),
        ("ra", ctypes.c_double), ("pr", ctypes.c_double), ("utarget", ctypes.c_double),
        ("seed", ctypes.c_uint64), ("jobs", ctypes.c_int32), ("odd_exact", ctypes.c_int32),
        ("levels", ctypes.c_int32), ("nu_start_mult", ctypes.c_double),
        ("has_nu_override", ctypes.c_int32), ("nu_override", ctypes.c_double),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
        ("cs", ctypes.c_double), ("pr_t", ctypes.c_double),
    ]


class CavOctreeInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("nu", "alpha", "beta_eff_coarse")] + [
        ("tau_plus", ctypes.c_double * 3)] + [
        (n, ctypes.c_double) for n in ("xi_even", "xi_odd", "xi_thermal", "xi_even_sub",
                                       "xi_odd_sub", "xi_thermal_sub")] + [
        ("time_step", ctypes.c_int64), ("spin_up_steps", ctypes.c_int64),
        ("n_nodes_total", ctypes.c_int64), ("levels", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("nx", ctypes.c_int32 * 5), ("ny", ctypes.c_int32 * 5),
        ("n_ghosts", ctypes.c_int32), ("n_coincident", ctypes.c_int32),
        ("n_ghosts_sub", ctypes.c_int32), ("n_coincident_sub", ctypes.c_int32)]


class CavOctreeDiag(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("nu_hot", "nu_hot_link0", "nu_cold", "nu_hot_fine", "max_u", "mass",
                 "max_rho_dev", "max_rho_dev_ifaces", "finite", "y_plus_fine")]


class CavError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def load(path: str | None = None):
    """Loads the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"CUDA library not built: {p} (run cfd_cavity_b200/build.py)")
    L = ctypes.CDLL(p)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    pp = ctypes.POINTER(CavParams)
    sig = {
        "cav_version": (ctypes.c_char_p, []),
        "cav_default_params": (i32, [pp]),
        "cav_create": (i32, [pp, ctypes.POINTER(vp)]),
        "cav_destroy": (i32, [vp]),
        "cav_last_error": (ctypes.c_char_p, [vp]),
        "cav_init_from_fields": (i32, [vp, _dp, _dp, _dp, _dp]),
        "cav_step": (i32, [vp, i64]),
        "cav_get_fields": (i32, [vp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "cav_set_fields": (i32, [vp, _dp, _dp, _dp, _dp, _dp]),
        "cav_get_populations": (i32, [vp, _dp, _dp]),
        "cav_set_populations": (i32, [vp, _dp, _dp]),
        "cav_get_info": (i32, [vp, ctypes.POINTER(CavInfo)]),
        "cav_set_time_step": (i32, [vp, i64]),
        "cav_diag": (i32, [vp, ctypes.POINTER(CavDiag)]),
        "cav_check_guards": (i32, [vp, ctypes.c_double]),
        "cav_debug_phase": (i32, [vp, i32, i64]),
        "cav_sample": (i32, [vp]),
        "cav_reset_means": (i32, [vp]),
        "cav_get_means": (i32, [vp, _dp, _dp, _dp, _dp, _dp, ctypes.POINTER(i64)]),
        "cav_nusselt_from_mean": (i32, [vp, i32, _dp]),
        "cav_nu_accumulate": (i32, [vp, i32]),
        "cav_nu_accumulated": (i32, [vp, _dp, _dp, ctypes.POINTER(i64)]),
        "cav_sync": (i32, [vp]),
        "cav_get_stream": (i32, [vp, ctypes.POINTER(vp)]),
        "cav_launch_count": (i32, [vp, ctypes.POINTER(i64)]),
        "cav_set_step_kernel": (i32, [vp, i32]),
        "cav_get_step_kernel": (i32, [vp, ctypes.POINTER(i32)]),
        "cav_set_dynamic_sgs": (i32, [vp, i32, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "cav_snapshot_write_fields": (i32, [ctypes.c_char_p, i64, i64, _dp, _dp, _dp, _dp]),
        "cav_snapshot_read_fields": (i32, [ctypes.c_char_p, ctypes.POINTER(i64), ctypes.POINTER(i64), _dp, _dp,
                                           _dp, _dp]),
        "cav_snapshot_write": (i32, [vp, ctypes.c_char_p]),
        "cav_restart_from_snapshot": (i32, [vp, ctypes.c_char_p]),
        "cav_octree_snapshot_write": (i32, [vp, ctypes.c_char_p, ctypes.c_uint64]),
        "cav_octree_restart_from_snapshot": (i32, [vp, ctypes.c_char_p]),
        "cav_dynamic_sgs_stats": (i32, [vp, _dp]),
        "cav_adjoint_run": (i32, [vp, ctypes.POINTER(CavAdjointSpec), _dp,
                                  ctypes.POINTER(CavAdjointResult)]),
        "cav_batch_create": (i32, [pp, i32, ctypes.POINTER(vp)]),
        "cav_batch_destroy": (i32, [vp]),
        "cav_batch_last_error": (ctypes.c_char_p, [vp]),
        "cav_batch_step": (i32, [vp, i64]),
        "cav_batch_get_fields": (i32, [vp, i32, _dp, _dp, _dp, _dp, _dp, _dp]),
        "cav_batch_get_populations": (i32, [vp, i32, _dp, _dp]),
        "cav_batch_diag": (i32, [vp, i32, ctypes.POINTER(CavDiag)]),
        "cav_batch_info": (i32, [vp, ctypes.POINTER(i32), ctypes.POINTER(i64), ctypes.POINTER(i64)]),
        "cav_batch_get_tuning": (i32, [vp, ctypes.POINTER(CavBatchTuning)]),
        "cav_batch_set_tuning": (i32, [vp, ctypes.POINTER(CavBatchTuning)]),
        "cav_batch_autotune": (i32, [vp, i32, ctypes.POINTER(CavBatchTuning)]),
        "cav_batch_sync": (i32, [vp]),
        "cav_batch_debug_stall_copies": (i32, [vp, i32]),
        "cav_batch_get_stream": (i32, [vp, ctypes.POINTER(vp)]),
        "cav_batch_launch_count": (i32, [vp, ctypes.POINTER(i64)]),
        "cav_octree_default_params": (i32, [ctypes.POINTER(CavOctreeParams)]),
        "cav_octree_create": (i32, [ctypes.POINTER(CavOctreeParams), ctypes.POINTER(vp)]),
        "cav_octree_destroy": (i32, [vp]),
        "cav_octree_last_error": (ctypes.c_char_p, [vp]),
        "cav_octree_step": (i32, [vp, i64]),
        "cav_octree_get_info": (i32, [vp, ctypes.POINTER(CavOctreeInfo)]),
        "cav_octree_get_level": (i32, [vp, i32, _dp, _dp, _dp, _dp, _dp, _dp]),
        "cav_octree_set_level": (i32, [vp, i32, _dp, _dp, _dp, _dp, _dp, _dp]),
        "cav_octree_couple": (i32, [vp, i32]),
        "cav_octree_restart_level": (i32, [vp, i32, _dp, _dp, _dp, _dp]),
        "cav_octree_set_time_step": (i32, [vp, i64]),
        "cav_octree_diag": (i32, [vp, ctypes.POINTER(CavOctreeDiag)]),
        "cav_octree_check_guards": (i32, [vp, ctypes.c_double]),
        "cav_octree_sync": (i32, [vp]),
        "cav_octree_get_stream": (i32, [vp, ctypes.POINTER(vp)]),
        "cav_octree_launch_count": (i32, [vp, ctypes.POINTER(i64)]),
        "cav_octree_set_level_kernel": (i32, [vp, i32]),
        "cav_octree_get_level_kernel": (i32, [vp, ctypes.POINTER(i32)]),
        "cav_octree_set_dynamic_sgs": (i32, [vp, i32, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "cav_octree_dynamic_stats": (i32, [vp, _dp]),
        "cav_octree_get_nu_t": (i32, [vp, i32, _dp, _dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int, h=None):
    if rc != CAV_OK:
        msg = load().cav_last_error(h)
        raise CavError(rc, msg.decode() if msg else "")


def check_octree(rc: int, h=None):
    if rc != CAV_OK:
        msg = load().cav_octree_last_error(h)
        raise CavError(rc, msg.decode() if msg else "")


def check_batch(rc: int, b=None):
    if rc != CAV_OK:
        msg = load().cav_batch_last_error(b)
        raise CavError(rc, msg.decode() if msg else "")

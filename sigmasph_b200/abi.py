"""ctypes mirror of include/sph_b200.h and the loader of libsph_b200.so.

The library is built in-tree (sigmasph_b200/_build/libsph_b200.so) by
``sigmasph_b200.build``.  Loading it is mandatory: there is no CPU fallback, and a
missing library raises instead of degrading.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libsph_b200.so")

ABI_VERSION = 4

SPH_OK = 0
STATUS_NAMES = {
    0: "SPH_OK", -1: "SPH_ERR_ARG", -2: "SPH_ERR_CUDA", -3: "SPH_ERR_NOMEM",
    -4: "SPH_ERR_UNSUPPORTED", -5: "SPH_ERR_NOT_BOUND", -6: "SPH_ERR_NEIGHBOUR_CAP",
    -7: "SPH_ERR_TIMEOUT", -8: "SPH_ERR_SCRATCH_CAP",
}
EW_NBR_OVERFLOW = 0x1
EW_HASHED_GRID = 0x2
EW_JC_NO_CONVERGE = 0x4
EW_STS_CAP = 0x8
EW_MLP_TIMEOUT = 0x10
EW_CAND_OVERFLOW = 0x20
EW_NBR_DROPPED = 0x40

# Stage ids of sph_run_stage (include/sph_b200.h).
STAGE_SORT, STAGE_LAM, STAGE_CONTINUITY, STAGE_FORCES, STAGE_DT, STAGE_ADVECT, \
    STAGE_PST, STAGE_BOUNDARY = range(8)

# Reduction indices of sph_reduce.
(RED_KE, RED_KE_OFFGRID, RED_PE, RED_SE, RED_IE, RED_MASS, RED_PX, RED_PY, RED_PZ,
 RED_GROSS_P, RED_ELASTIC, RED_COUNT) = range(12)

_i32, _f32, _f64 = C.c_int32, C.c_float, C.c_double

# (name, ctype) in declaration order of struct SphParams.
PARAM_FIELDS = [
    ("struct_size", _i32), ("is_solid", _i32),
    ("two_d", _i32), ("axisymmetric", _i32), ("plane_strain", _i32),
    ("sym_y", _i32), ("sym_z", _i32), ("walls", _i32),
    ("displacement_positions", _i32), ("compensated_volume", _i32),
    ("support_radius", _f32), ("particle_diameter", _f32), ("V0", _f32),
    ("axi_r_min", _f32), ("domain_size", _f32 * 3), ("padding", _f32),
    ("wall_restitution", _f32),
    ("density0", _f32), ("c0", _f32), ("exponent", _f32), ("stiffness", _f32),
    ("viscosity", _f32), ("CFL", _f32), ("delta_sph", _f32), ("gravity", _f32 * 3),
    ("allow_negative_pressure", _i32), ("track_visc_work", _i32),
    ("l_eig_tol_lam", _f32), ("c_signal", _f32), ("dt_pair_mode", _i32),
    ("pst_enabled", _i32), ("pst_colle", _i32), ("pst_ma_mode", _i32),
    ("pst_clamp_disp", _i32), ("pst_clamp_vel", _i32), ("pst_surface_none", _i32),
    ("pst_normal_eigvec", _i32), ("pst_ale_momentum", _i32),
    ("pst_R", _f32), ("pst_n", _i32), ("pst_max_shift", _f32), ("pst_ma_fixed", _f32),
    ("pst_m_delta", _f32), ("pst_lambda_lo", _f32), ("pst_lambda_hi", _f32),
    ("n_materials", _i32),
    ("mat_rho0", _f32 * 4), ("mat_K", _f32 * 4), ("mat_G", _f32 * 4),
    ("mat_cp", _f32 * 4), ("mat_c0", _f32 * 4), ("mat_delta", _f32 * 4),
    ("plastic_kind", _i32 * 4), ("plastic_sy0", _f32 * 4), ("plastic_H", _f32 * 4),
    ("jc_A", _f32 * 4), ("jc_B", _f32 * 4), ("jc_n", _f32 * 4), ("jc_C", _f32 * 4),
    ("jc_eps0_dot", _f32 * 4),
    ("jc_T0", _f32 * 4), ("jc_Tm", _f32 * 4), ("jc_m", _f32 * 4), ("jc_chi", _f32 * 4),
    ("mat_cv", _f32 * 4), ("mat_stiff", _f32 * 4), ("mat_gamma", _f32 * 4),
    ("mat_T0", _f32 * 4), ("axi_conservative_x", _i32), ("hg_rate", _f32),
    ("kernel_correction", _i32), ("l_eig_tol", _f32), ("hourglass_alpha", _f32),
    ("hourglass_sts", _i32), ("hourglass_sts_cap", _i32),
    ("hourglass_sts_safety", _f32), ("hg_S", _f32), ("hg_W_dx0", _f32),
    ("hg_sts_refresh", _i32), ("ale_history", _i32), ("transport_e", _i32),
    ("ale_diffusion", _f32), ("num_constraints", _i32), ("ramp_time", _f32),
    ("jc_surrogate", _i32), ("jc_surrogate_tol", _f32), ("hg_sts_fixed", _i32),
    ("q_l2", _f32), ("q_cl", _f32), ("av_alpha", _f32), ("av_beta", _f32), ("av_eps", _f32),
    ("hg_sts_rkl", _i32), ("objective_none", _i32), ("axi_image_signed", _i32),
    ("axi_conservative_r", _i32),
    ("delta_pairs_all", _i32), ("c0_mixed", _i32), ("hg_mixed_impedance", _i32),
]


class SphParams(C.Structure):
    _fields_ = PARAM_FIELDS


class SphFieldSet(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("vel", C.c_void_p), ("x0", C.c_void_p),
                ("disp", C.c_void_p), ("shift", C.c_void_p), ("pid", C.c_void_p),
                ("sdev", C.c_void_p), ("bc", C.c_void_p), ("bcdisp", C.c_void_p),
                ("acc", C.c_void_p)]


class SphBuffers(C.Structure):
    _fields_ = [("set", SphFieldSet * 2), ("acc", C.c_void_p), ("lam", C.c_void_p),
                ("lsym", C.c_void_p), ("lgrad", C.c_void_p), ("div", C.c_void_p),
                ("gradv", C.c_void_p), ("aux", C.c_void_p)]


class SphScalars(C.Structure):
    _fields_ = [("dt", _f32), ("max_c_sq", _f32), ("max_accel", _f32), ("max_v", _f32),
                ("off_grid_num", _i32), ("err", _i32), ("sts_stages", _i32),
                ("pad0", _i32), ("off_grid_mass", _f64), ("wall_work", _f64),
                ("visc_work", _f64), ("diff_work", _f64), ("leftover_work", _f64),
                ("plastic_work", _f64), ("hg_work", _f64), ("sim_time", _f64),
                ("load_s", _f32), ("load_sdot", _f32),
                ("constraint_force", (_f64 * 3) * 8),
                ("constraint_disp", (_f64 * 3) * 8)]


class SphError(RuntimeError):
    """A non-zero status from libsph_b200."""

    def __init__(self, status, what=""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        msg = f"{what}: {name}" if what else name
        try:
            detail = lib().sph_strerror(status)
            if detail:
                msg += f" ({detail.decode()})"
        except Exception:  # pragma: no cover - the loader itself failed
            pass
        super().__init__(msg)


class SphMatRow(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("rho0", "K", "G", "cp", "c0", "delta")] + \
               [("plastic_kind", C.c_int32)] + \
               [(k, C.c_float) for k in ("sy0", "H", "jc_A", "jc_B", "jc_n", "jc_C", "jc_eps0_dot",
                                         "jc_T0", "jc_Tm", "jc_m", "jc_chi", "cv", "stiff", "gamma",
                                         "T0")]


class SphInstRow(C.Structure):
    _fields_ = [("c_signal", C.c_float), ("hg_rate", C.c_float), ("ramp_time", C.c_float),
                ("c0", C.c_float), ("visc_coef", C.c_float), ("reserved", C.c_float * 3)]


class SphInstState(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("dt", C.c_float), ("load_s", C.c_float),
                ("load_sdot", C.c_float), ("sts_stages", C.c_int32), ("max_c_sq_bits", C.c_uint32),
                ("max_accel_bits", C.c_uint32), ("constraint_force", (C.c_double * 3) * 2),
                ("constraint_disp", (C.c_double * 3) * 2)]


_LIB = None


def lib():
    """Load libsph_b200.so once.  Raises if it is missing: the hot path has no
    fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libsph_b200.so not found at {LIB_PATH}; build it with "
            "`python -m sigmasph_b200.build` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32
    sig = {
        "sph_abi_version": (C.c_int, []),
        "sph_params_size": (C.c_size_t, []),
        "sph_scalars_size": (C.c_size_t, []),
        "sph_strerror": (C.c_char_p, [C.c_int]),
        "sph_params_layout": (C.c_int, [C.c_char_p, C.c_int]),
        "sph_create": (C.c_int, [C.POINTER(SphParams), i64, C.POINTER(vp)]),
        "sph_destroy": (None, [vp]),
        "sph_bind": (C.c_int, [vp, C.POINTER(SphBuffers), i64]),
        "sph_parity": (C.c_int, [vp]),
        "sph_set_params": (C.c_int, [vp, C.POINTER(SphParams)]),
        "sph_initialize": (C.c_int, [vp, vp]),
        "sph_step": (C.c_int, [vp, C.c_int, vp]),
        "sph_run_stage": (C.c_int, [vp, C.c_int, vp]),
        "sph_set_dt": (C.c_int, [vp, C.c_float, vp]),
        "sph_get_dt": (C.c_int, [vp, C.POINTER(C.c_float), vp]),
        "sph_get_scalars": (C.c_int, [vp, C.POINTER(SphScalars), vp]),
        "sph_constraints": (C.c_int, [vp, vp, vp, C.c_int, vp]),
        "sph_clear_error": (C.c_int, [vp, vp]),
        "sph_reduce": (C.c_int, [vp, C.POINTER(C.c_double), vp]),
        "sph_pairs": (C.c_int, [vp, C.c_int, vp, vp, vp, i64, C.POINTER(i64), vp]),
        "sph_shift_pairs": (C.c_int, [vp, C.c_float, vp, vp, vp, i64, C.POINTER(i64), vp]),
        "sph_list_stats": (C.c_int, [vp, vp, C.c_int, vp]),
        "sph_fma_peak": (C.c_int, [vp, vp]),
        "sph_relax_pass": (C.c_int, [vp, C.c_float, C.POINTER(C.c_float), vp, vp]),
        "sph_relax_move": (C.c_int, [vp, vp]),
        "sph_profile_enable": (C.c_int, [vp, C.c_int]),
        "sph_profile_read": (C.c_int, [vp, C.c_char_p, C.c_int, C.POINTER(C.c_double),
                                       C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
        "sph_mlp_param_count": (C.c_int, []),
        "sph_mlp_packed_bytes": (i64, []),
        "sph_mlp_forward": (C.c_int, [vp, vp, i64, vp, vp]),
        "sph_mlp_grad": (C.c_int, [vp, vp, vp, i64, vp, vp, vp]),
        "sph_mlp_adam": (C.c_int, [vp, vp, vp, vp, i64, C.c_float, vp]),
        "sph_mlp_pack": (C.c_int, [vp, vp, vp]),
        "sph_mlp_infer_tc": (C.c_int, [vp, vp, vp, i64, vp, vp, vp]),
        "sph_jc_surrogate": (C.c_int, [vp, vp, C.c_float, C.c_int, vp]),
        "sph_jc_log": (C.c_int, [vp, vp, i64, vp]),
        "sph_jc_stats": (C.c_int, [vp, C.POINTER(C.c_uint64), C.c_int, vp]),
        "sph_ensemble_set": (C.c_int, [vp, vp, vp, C.c_int, vp, vp]),
        "sph_ensemble_state": (C.c_int, [vp, vp, C.c_int, vp]),
        "sph_set_block": (C.c_int, [vp, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.sph_abi_version() != ABI_VERSION:
        raise RuntimeError(f"libsph_b200 ABI {L.sph_abi_version()} != {ABI_VERSION}; rebuild")
    if L.sph_params_size() != C.sizeof(SphParams):
        raise RuntimeError("SphParams layout mismatch between sph_b200.h and abi.py")
    if L.sph_scalars_size() != C.sizeof(SphScalars):
        raise RuntimeError("SphScalars layout mismatch between sph_b200.h and abi.py")
    _LIB = L
    return L


def check(status, what=""):
    if status != SPH_OK:
        raise SphError(status, what)


def params_layout_from_lib():
    """{field: offset} as the compiled library sees SphParams."""
    L = lib()
    n = L.sph_params_layout(None, 0)
    buf = C.create_string_buffer(n + 1)
    L.sph_params_layout(buf, n + 1)
    out = {}
    for item in buf.value.decode().split(";"):
        if item:
            k, v = item.split("=")
            out[k] = int(v)
    return out


def params_layout_from_ctypes():
    return {name: getattr(SphParams, name).offset for name, _ in PARAM_FIELDS}

"""ctypes binding of libheatflow_b200.so (the C ABI in include/heatflow_b200.h).

The structures below mirror the header field for field.  Loading fails loudly: there is no CPU or PyTorch fallback
for the air substep -- without the sm_100a library and a CUDA device the package refuses to run it.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libheatflow_b200.so")

HF_OK, HF_ERR_ARG, HF_ERR_CUDA, HF_ERR_WORKSPACE, HF_ERR_DEVICE = 0, 1, 2, 3, 4
HF_FLAG_BUOYANCY, HF_FLAG_SOURCE, HF_FLAG_PARTICLES, HF_FLAG_ACTIVE, HF_FLAG_DEFECT_CORRECTION = 1, 2, 4, 8, 16
HF_SCENE_CORRECTED = 16
HF_SCENE_HEAT_MAXITER, HF_SCENE_PRESSURE_MAXITER, HF_SCENE_NONFINITE, HF_SCENE_BARRIER_TIMEOUT = 1, 2, 4, 8
WAIT_LIMIT_NS = 2_000_000_000   # default limit of the CG kernels' bounded waits (hf_set_wait_limit)
CHUNK = 1024
HF_PLAN_STREAMING_CG = 1
HF_PLAN_NO_TMA = 2
HF_PLAN_STREAMING_HEAT = 4
HF_PLAN_SINGLE_REDUCTION_CG = 8
HF_PLAN_LANES_SHIFT = 8
HF_PLAN_RES_TILES_SHIFT = 12

_P = C.c_void_p


class SceneState(C.Structure):
    _fields_ = [("parity", C.c_int32), ("status", C.c_int32), ("substeps", C.c_int64),
                ("heat_iters", C.c_int32), ("pressure_iters", C.c_int32),
                ("heat_rr", C.c_double), ("heat_atol", C.c_double), ("pressure_rr", C.c_double),
                ("pressure_atol", C.c_double), ("pressure_bb", C.c_double), ("heat_bb", C.c_double),
                ("rhs_mean", C.c_double), ("total_heat_iters", C.c_int64), ("total_pressure_iters", C.c_int64),
                ("box", C.c_int32 * 6), ("box_prev", C.c_int32 * 6), ("heat_true_rr", C.c_double),
                ("pressure_true_rr", C.c_double)]


SCENE_DOUBLES = ("h", "rho", "t_amb", "alpha_f_min", "g", "cg_tol", "heat_tol", "kappa_air", "kappa_mat", "rate",
                 "t_cap", "vol", "k_particle", "t_sol", "t_liq", "y_solid", "mu_s", "mu_l", "t_max")
SCENE_PTRS = ("Tw", "kap", "hrhs", "hdiag", "tfix", "alpha", "tsum", "cell_flags", "p", "rhs", "pdiag", "alpha_s",
              "ax", "ay", "az", "qx", "qy", "qz", "kx", "ky", "kz", "mx", "my", "mz", "st_alpha", "st_kx", "st_ky",
              "st_kz", "st_mx", "st_my", "st_mz", "cg_r", "cg_z")


class Scene(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_particles", C.c_int32), ("flags", C.c_uint32), ("cg_max_iter", C.c_int32),
                ("heat_maxiter", C.c_int32), ("reserved_i", C.c_int32 * 3)] + \
               [(f, C.c_double) for f in SCENE_DOUBLES] + \
               [("T", _P * 2), ("u", _P * 2), ("v", _P * 2), ("w", _P * 2)] + \
               [(f, _P) for f in SCENE_PTRS[:31]] + \
               [("cg_r", _P), ("cg_z", _P), ("cg_p", _P * 2), ("cg_Ap", _P),
                ("pos", _P), ("pvel", _P), ("ptemp", _P), ("pmelt", _P), ("pyield", _P), ("pvisc", _P),
                ("hkx", _P), ("hky", _P), ("hkz", _P), ("ayc", _P), ("azc", _P), ("hkzc", _P), ("acc", _P), ("state", _P)]


class Plan(C.Structure):
    _fields_ = [("num_scenes", C.c_int32), ("num_chunks", C.c_int32), ("num_tiles", C.c_int32), ("group_cells", C.c_int32),
                ("tiles_dev", _P), ("scenes_host", _P), ("scenes_dev", _P),
                ("work_dev", _P), ("workspace", _P), ("workspace_bytes", C.c_size_t), ("persistent_blocks", C.c_int32),
                ("options", C.c_int32)]


class HeaterGeometry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("fan", C.c_int32), ("centre", C.c_double * 3), ("facing", C.c_double * 3),
                ("axis", C.c_double * 3), ("up", C.c_double * 3)] + \
               [(f, C.c_double) for f in ("half_length", "shell_in", "shell_out", "cap_half", "cap_radius", "rod_half",
                                          "rod_radius", "rod_front", "rod_dz", "fan_half", "fan_high", "fan_depth",
                                          "trough_half", "trough_radius")] + \
               [("box_lo", C.c_int32 * 3), ("box_hi", C.c_int32 * 3), ("box_trough", C.c_int32), ("sphere", C.c_int32),
                ("t_rod", C.c_double), ("t_amb", C.c_double), ("m_face", C.c_float * 3), ("k_solid", C.c_float),
                ("k_fan", C.c_float), ("sphere_t", C.c_float), ("sphere_lo", C.c_int32), ("sphere_hi", C.c_int32),
                ("sphere_top", C.c_int32), ("pad_", C.c_int32), ("sphere_c", C.c_double), ("sphere_zc", C.c_double),
                ("sphere_rr", C.c_double)]


_lib = None


class HeatflowError(RuntimeError):
    pass


def load():
    """Load libheatflow_b200.so once; raise if it is missing (build it with __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HeatflowError(f"{LIB_PATH} is missing: build the sm_100a library first (python -c 'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB_PATH)
    L.hf_last_error.restype = C.c_char_p
    L.hf_workspace_bytes.restype = C.c_size_t
    L.hf_workspace_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
    L.hf_chunks_for.argtypes = [C.c_int]
    L.hf_tiles_for.argtypes = [C.c_int]
    L.hf_plan_upload.argtypes = [C.POINTER(Plan), _P]
    for name in ("hf_temperature_stage", "hf_heat_solve", "hf_face_stage", "hf_pressure_solve", "hf_substep",
                 "hf_divergence_stage", "hf_pressure_cg"):
        getattr(L, name).argtypes = [C.POINTER(Plan), C.c_double, _P]
    L.hf_obstacle_fields.argtypes = [C.POINTER(Plan), C.c_int, _P]
    L.hf_particle_update.argtypes = [C.POINTER(Plan), _P]
    for name in ("hf_cell_velocity", "hf_divergence_max", "hf_speed_max"):
        getattr(L, name).argtypes = [C.POINTER(Plan), C.c_int, _P, _P]
    L.hf_pack_frame.argtypes = [C.POINTER(Plan), C.c_int, _P, _P, _P, _P, _P]
    L.hf_current_field.argtypes = [C.POINTER(Plan), C.c_int, C.c_int, _P, _P]
    L.hf_scene_statics.argtypes = [C.POINTER(HeaterGeometry), C.c_int, C.c_double] + [_P] * 11 + [_P]
    L.hf_winding_inside.argtypes = [_P, C.c_int, _P, C.c_int, C.c_float, _P, _P, _P]
    L.hf_k_laplacian.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double] + [_P] * 6 + [_P]
    L.hf_k_heat_matvec.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double] + [_P] * 5 + [_P]
    L.hf_k_divide_by.argtypes = [C.c_int, _P, C.c_float, _P, _P]
    L.hf_set_wait_limit.argtypes = [C.c_ulonglong, C.c_int]
    if L.hf_abi_version() != 1:
        raise HeatflowError("libheatflow_b200.so ABI version mismatch")
    _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != HF_OK:
        msg = load().hf_last_error().decode(errors="replace")
        raise HeatflowError(f"{what}: hf status {rc}: {msg}")


def ptr(t) -> int | None:
    """Device address of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()

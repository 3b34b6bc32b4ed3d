"""ctypes binding of libmqct_b200.so (the C ABI declared in include/mqct_b200.h).

The library is built in-tree by mqct_b200/build.py.  Loading fails loudly if
it is missing: there is no CPU fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmqct_b200.so")

MQCT_OK = 0
ERRORS = {-1: "MQCT_E_ARG", -2: "MQCT_E_CUDA", -3: "MQCT_E_NODEV", -4: "MQCT_E_IO",
          -5: "MQCT_E_RANGE", -6: "MQCT_E_DEVICE"}

PREC_FP64, PREC_BF16X3, PREC_F16X3 = 0, 1, 2
PROP_FP64, PROP_FP32 = 0, 1
MODE_STD, MODE_AT, MODE_CS = 0, 1, 2
INTEG_RK4, INTEG_ODEINT, INTEG_AT_ADAPT, INTEG_BK_INT = 0, 1, 2, 3
(ENGINE_AUTO, ENGINE_PER_TRAJECTORY, ENGINE_LOCKSTEP, ENGINE_RESIDENT,
 ENGINE_LOCKSTEP_TAIL) = 0, 1, 2, 3, 4
PES_TABLE, PES_LEGENDRE, PES_SITES1, PES_SITES2 = 0, 1, 2, 3

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
vp = C.c_void_p


class MqctError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Sys(C.Structure):
    _fields_ = [("sys_type", C.c_int32), ("n_channels", C.c_int32), ("j1", vp), ("ka1", vp),
                ("kc1", vp), ("j2", vp), ("ka2", vp), ("kc2", vp), ("vec1", vp), ("vec2", vp),
                ("ldv", C.c_int32), ("n_states", C.c_int32), ("indx_chann", vp), ("j12", vp),
                ("m12", vp), ("parity", vp)]


class Grid(C.Structure):
    _fields_ = [("n_beta", C.c_int32), ("n_gamma", C.c_int32), ("n_alpha", C.c_int32),
                ("n_beta2", C.c_int32), ("n_alpha2", C.c_int32), ("n_gamma2", C.c_int32),
                ("eq_gamma", C.c_int32)]


class Pes(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_terms", C.c_int32), ("params", vp),
                ("n_sites1", C.c_int32), ("n_sites2", C.c_int32), ("sites1", vp),
                ("sites2", vp), ("table", vp)]


class ErrReport(C.Structure):
    _fields_ = [("n_sampled", C.c_int32), ("max_abs_err", C.c_double),
                ("max_rel_err", C.c_double), ("rms_rel_err", C.c_double)]


class Tables(C.Structure):
    _fields_ = [("n_states", C.c_int32), ("j12", vp), ("m12", vp), ("ej", vp), ("P", C.c_int64),
                ("ind_mat", vp), ("nR", C.c_int32), ("R", vp), ("mat", vp), ("y2", vp),
                ("mass_au", C.c_double)]


class TrajInit(C.Structure):
    _fields_ = [("e_coll", C.c_double), ("l_real", C.c_double), ("s_st", C.c_int32),
                ("dt", C.c_double), ("r_start", C.c_double), ("r_fin", C.c_double),
                ("numb_orb_prds", C.c_int32), ("numb_oscl_prds", C.c_int32),
                ("time_lim", C.c_double), ("max_steps", C.c_int64)]


class AtPaths(C.Structure):
    _fields_ = [("rec_off", vp), ("n_rec", vp), ("rec", vp)]


class Integrator(C.Structure):
    _fields_ = [("method", C.c_int32), ("eps", C.c_double), ("hmin", C.c_double)]


# Every symbol declared in include/mqct_b200.h (checked by the ABI test).
EXPORTS = [
    "mqct_last_error", "mqct_version", "mqct_device_count", "mqct_build_matrix",
    "mqct_release_cached_build", "mqct_matrix_plan_set_drain", "mqct_matrix_plan_layout",
    "mqct_matrix_plan_tune", "mqct_matrix_plan_epilogue", "mqct_matrix_plan_set_epilogue",
    "mqct_matrix_plan_create", "mqct_matrix_plan_execute", "mqct_matrix_plan_sync",
    "mqct_matrix_plan_flops", "mqct_matrix_plan_timing", "mqct_matrix_plan_destroy",
    "mqct_spline_y2_noalloc", "mqct_build_matrix_expansion", "mqct_propagate_batch",
    "mqct_propagate_batch_rec", "mqct_propagate_batch_integ", "mqct_prop_plan_set_integrator",
    "mqct_cross_sections_device", "mqct_expansion_plan_create", "mqct_expansion_plan_execute",
    "mqct_expansion_plan_sync", "mqct_expansion_plan_timing", "mqct_expansion_plan_destroy",
    "mqct_surrogate_create", "mqct_surrogate_train", "mqct_surrogate_predict",
    "mqct_surrogate_n_params", "mqct_surrogate_get_params", "mqct_surrogate_loss_grad",
    "mqct_surrogate_destroy", "mqct_matrix_plan_set_surrogate", "mqct_matrix_plan_surrogate_stats",
    "mqct_prop_plan_create", "mqct_prop_plan_run", "mqct_prop_plan_run_device",
    "mqct_prop_plan_sync", "mqct_prop_plan_bytes_per_step", "mqct_prop_plan_timing",
    "mqct_prop_plan_destroy", "mqct_prop_plan_set_coupled_states", "mqct_prop_plan_tune",
    "mqct_prop_plan_shape", "mqct_prop_plan_set_engine", "mqct_prop_plan_engine",
    "mqct_prop_plan_set_cluster", "mqct_prop_plan_cluster", "mqct_prop_plan_handed",
    "mqct_asym_top_level", "mqct_count_states", "mqct_enumerate_states", "mqct_count_pairs",
    "mqct_fill_ind_mat", "mqct_count_states_identical", "mqct_enumerate_states_identical",
    "mqct_count_pairs_identical", "mqct_fill_ind_mat_identical", "mqct_r_grid", "mqct_write_mtrx_uf", "mqct_read_mtrx_uf_header",
    "mqct_read_mtrx_uf", "mqct_write_mtrx_dat", "mqct_read_mtrx_dat_header",
    "mqct_read_mtrx_dat", "mqct_read_expansion_terms", "mqct_write_expansion_terms",
    "mqct_projection_plan_create", "mqct_projection_plan_execute", "mqct_projection_plan_sync",
    "mqct_projection_plan_timing", "mqct_projection_plan_destroy", "mqct_project_terms",
    "mqct_write_opacity", "mqct_write_partial_j", "mqct_write_m_proj",
    "mqct_write_deflection", "mqct_write_diff_cross", "mqct_write_splined_opacity",
    "mqct_write_cross_sections", "mqct_write_cross_sections_footer",
]

_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m mqct_b200.build` "
                          "(the CUDA extension is required; there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.mqct_last_error.restype = C.c_char_p
    L.mqct_version.restype = C.c_int
    L.mqct_device_count.restype = C.c_int
    L.mqct_build_matrix.argtypes = [C.POINTER(Sys), i32p, C.c_int64, f64p, C.c_int32,
                                    C.POINTER(Grid), C.POINTER(Pes), C.c_int32, C.c_double,
                                    C.c_double, C.c_double, f64p, vp, vp, vp]
    L.mqct_matrix_plan_set_drain.argtypes = [vp, C.c_int32]
    L.mqct_matrix_plan_tune.argtypes = [vp, vp, vp, vp]
    L.mqct_matrix_plan_set_epilogue.argtypes = [vp, C.c_int32]
    L.mqct_matrix_plan_epilogue.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_float)]
    L.mqct_matrix_plan_layout.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32)]
    L.mqct_release_cached_build.argtypes = []
    L.mqct_release_cached_build.restype = None
    L.mqct_matrix_plan_create.argtypes = [C.POINTER(Sys), i32p, C.c_int64, f64p, C.c_int32,
                                          C.POINTER(Grid), C.POINTER(Pes), C.c_int32,
                                          C.c_double, C.c_double, C.c_double, C.POINTER(vp)]
    L.mqct_matrix_plan_execute.argtypes = [vp, vp, vp, vp]
    L.mqct_matrix_plan_sync.argtypes = [vp]
    L.mqct_matrix_plan_flops.argtypes = [vp]
    L.mqct_matrix_plan_flops.restype = C.c_double
    L.mqct_matrix_plan_timing.argtypes = [vp, C.POINTER(C.c_float)]
    L.mqct_prop_plan_timing.argtypes = [vp, C.POINTER(C.c_float)]
    L.mqct_matrix_plan_destroy.argtypes = [vp]
    L.mqct_spline_y2_noalloc.argtypes = [vp, C.c_int32, vp, vp, C.c_int64, vp, vp]
    L.mqct_build_matrix_expansion.argtypes = [C.POINTER(Sys), i32p, C.c_int64, f64p, C.c_int32,
                                              C.c_int32, i32p, f64p, C.c_double, C.c_double,
                                              C.c_double, C.c_double, f64p, vp, vp]
    L.mqct_surrogate_create.argtypes = [C.c_int32, C.POINTER(Pes), C.c_int32, C.c_int32,
                                        C.c_uint64, C.c_double, C.c_double, C.POINTER(vp)]
    L.mqct_surrogate_train.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, C.c_double, vp, vp]
    L.mqct_surrogate_predict.argtypes = [vp, vp, C.c_int64, vp]
    L.mqct_surrogate_n_params.argtypes = [vp]
    L.mqct_surrogate_n_params.restype = C.c_int64
    L.mqct_surrogate_get_params.argtypes = [vp, vp]
    L.mqct_surrogate_loss_grad.argtypes = [vp, vp, vp, C.c_int32, vp, vp]
    L.mqct_surrogate_destroy.argtypes = [vp]
    L.mqct_surrogate_destroy.restype = None
    L.mqct_matrix_plan_set_surrogate.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int32]
    L.mqct_matrix_plan_surrogate_stats.argtypes = [vp, vp, vp]
    L.mqct_matrix_plan_destroy.restype = None
    L.mqct_propagate_batch.argtypes = [C.POINTER(Tables), C.POINTER(TrajInit), C.c_int64,
                                       C.c_int32, C.POINTER(AtPaths), C.c_int32, f64p, f64p,
                                       f64p]
    L.mqct_propagate_batch_rec.argtypes = [C.POINTER(Tables), C.POINTER(TrajInit), C.c_int64,
                                           C.c_int32, C.c_int64, f64p, f64p, f64p, f64p,
                                           np.ctypeslib.ndpointer(dtype=np.int64,
                                                                  flags="C_CONTIGUOUS")]
    L.mqct_propagate_batch_integ.argtypes = [C.POINTER(Tables), C.POINTER(TrajInit), C.c_int64,
                                             C.c_int32, C.POINTER(AtPaths), C.c_int32,
                                             C.POINTER(Integrator), f64p, f64p, f64p]
    L.mqct_prop_plan_set_coupled_states.argtypes = [vp, C.c_int32]
    L.mqct_prop_plan_tune.argtypes = [vp, vp, C.c_int64, C.c_int32]
    L.mqct_prop_plan_shape.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_float)]
    L.mqct_prop_plan_set_integrator.argtypes = [vp, C.POINTER(Integrator)]
    L.mqct_prop_plan_set_engine.argtypes = [vp, C.c_int32]
    L.mqct_prop_plan_engine.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.mqct_prop_plan_set_cluster.argtypes = [vp, C.c_int32]
    L.mqct_prop_plan_handed.argtypes = [vp, C.POINTER(C.c_int32)]
    L.mqct_prop_plan_cluster.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.mqct_expansion_plan_create.argtypes = [C.POINTER(Sys), i32p, C.c_int64, f64p, C.c_int32,
                                             C.c_int32, i32p, C.c_double, C.c_double, C.c_double,
                                             C.POINTER(vp)]
    L.mqct_expansion_plan_execute.argtypes = [vp, vp, C.c_double, vp, vp, vp]
    L.mqct_expansion_plan_sync.argtypes = [vp]
    L.mqct_expansion_plan_timing.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.mqct_expansion_plan_destroy.argtypes = [vp]
    L.mqct_expansion_plan_destroy.restype = None
    L.mqct_cross_sections_device.argtypes = [vp, C.c_int64, C.c_int32, i32p, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_double, vp, vp, vp, vp]
    L.mqct_prop_plan_create.argtypes = [C.POINTER(Tables), C.c_int32, C.POINTER(vp)]
    L.mqct_prop_plan_run.argtypes = [vp, C.POINTER(TrajInit), C.c_int64, f64p, f64p, f64p]
    L.mqct_prop_plan_run_device.argtypes = [vp, vp, C.c_int64, vp, vp, vp]
    L.mqct_prop_plan_sync.argtypes = [vp]
    L.mqct_prop_plan_bytes_per_step.argtypes = [vp]
    L.mqct_prop_plan_bytes_per_step.restype = C.c_double
    L.mqct_prop_plan_destroy.argtypes = [vp]
    L.mqct_prop_plan_destroy.restype = None
    L.mqct_asym_top_level.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                      C.c_int32, C.POINTER(C.c_double), f64p]
    L.mqct_count_states.argtypes = [C.c_int32, C.c_int32, i32p, vp]
    L.mqct_enumerate_states.argtypes = [C.c_int32, C.c_int32, i32p, vp, i32p, i32p, i32p]
    L.mqct_count_pairs.argtypes = [C.c_int32, i32p]
    L.mqct_count_pairs.restype = C.c_int64
    L.mqct_fill_ind_mat.argtypes = [C.c_int32, i32p, i32p]
    L.mqct_fill_ind_mat.restype = C.c_int64
    L.mqct_count_states_identical.argtypes = [C.c_int32] + [i32p] * 6
    L.mqct_enumerate_states_identical.argtypes = [C.c_int32] + [i32p] * 10
    L.mqct_count_pairs_identical.argtypes = [C.c_int32, i32p, i32p]
    L.mqct_count_pairs_identical.restype = C.c_int64
    L.mqct_fill_ind_mat_identical.argtypes = [C.c_int32, i32p, i32p, i32p]
    L.mqct_fill_ind_mat_identical.restype = C.c_int64
    L.mqct_r_grid.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_int32, f64p]
    L.mqct_write_mtrx_uf.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, i32p, C.c_int32,
                                     C.c_int64, i32p, C.c_int32, f64p, f64p]
    L.mqct_read_mtrx_uf_header.argtypes = [C.c_char_p] + [C.POINTER(C.c_int32)] * 3 + [
        C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.mqct_read_mtrx_uf.argtypes = [C.c_char_p, C.c_int32, i32p, i32p, f64p, f64p]
    L.mqct_write_mtrx_dat.argtypes = L.mqct_write_mtrx_uf.argtypes
    L.mqct_read_mtrx_dat_header.argtypes = L.mqct_read_mtrx_uf_header.argtypes
    L.mqct_read_mtrx_dat.argtypes = L.mqct_read_mtrx_uf.argtypes
    L.mqct_read_expansion_terms.argtypes = [C.c_char_p, C.c_int32, C.c_int32, f64p, f64p]
    L.mqct_write_expansion_terms.argtypes = [C.c_char_p, C.c_int32, C.c_int32, i32p, C.c_int32,
                                             f64p, f64p]
    L.mqct_projection_plan_create.argtypes = [C.c_int32, C.c_int32, i32p, C.POINTER(Grid),
                                              C.c_int32, C.POINTER(vp)]
    L.mqct_projection_plan_execute.argtypes = [vp, vp, C.c_int32, vp, vp]
    L.mqct_projection_plan_sync.argtypes = [vp]
    L.mqct_projection_plan_timing.argtypes = [vp] + [C.POINTER(C.c_float)] * 3
    L.mqct_projection_plan_destroy.argtypes = [vp]
    L.mqct_projection_plan_destroy.restype = None
    L.mqct_write_opacity.argtypes = [C.c_char_p, C.c_char_p] + [C.c_int32] * 4 + [
        C.c_double, C.c_int32, i32p, C.c_double, C.c_int32, f64p, C.c_int32]
    L.mqct_write_partial_j.argtypes = [C.c_char_p] + [C.c_int32] * 4 + [
        C.c_double, C.c_int32, i32p, C.c_int32, f64p]
    L.mqct_write_m_proj.argtypes = [C.c_char_p] + [C.c_int32] * 5 + [f64p]
    L.mqct_write_deflection.argtypes = [C.c_char_p] + [C.c_int32] * 4 + [
        C.c_double, C.c_int32, i32p, C.c_double] + [f64p] * 5 + [i32p, i32p]
    L.mqct_write_diff_cross.argtypes = [C.c_char_p] + [C.c_int32] * 5 + [f64p, f64p]
    L.mqct_write_splined_opacity.argtypes = [C.c_char_p, C.c_int32, i32p, C.c_double, f64p,
                                             C.c_int32, f64p]
    L.mqct_write_cross_sections.argtypes = [C.c_char_p, C.c_double, C.c_int32, C.c_int32, vp,
                                            f64p, f64p, C.c_double, C.c_int32, C.c_double]
    L.mqct_write_cross_sections_footer.argtypes = [C.c_char_p, C.c_int32]
    L.mqct_project_terms.argtypes = [C.c_int32, C.c_int32, i32p, C.POINTER(Grid), C.c_int32,
                                     C.c_int32, f64p, f64p, vp]
    _lib = L
    return L


def check(rc):
    if rc < 0:
        raise MqctError(rc, lib().mqct_last_error().decode(errors="replace"))
    return rc


def ptr(a):
    return None if a is None else a.ctypes.data_as(vp)

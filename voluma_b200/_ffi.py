"""ctypes binding of include/voluma_b200.h (the library's C ABI)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvoluma_b200.so")

STATUS = {0: "OK", 1: "BAD_ARG", 2: "CUDA", 3: "OOM", 4: "SINGULAR", 5: "NONFINITE", 6: "TIMEOUT",
          7: "UNSUPPORTED", 8: "NO_DEVICE"}

# every entry point include/voluma_b200.h declares
EXPORTS = ["vlm_ctx_create", "vlm_ctx_destroy", "vlm_last_error", "vlm_ctx_stream", "vlm_mesh_register",
           "vlm_mesh_release", "vlm_amul", "vlm_ldu_solve", "vlm_ldu_solve_device", "vlm_gamg_apply",
           "vlm_gamg_levels", "vlm_gamg_level", "vlm_gamg_colours", "vlm_laplacian", "vlm_grad", "vlm_exact_sum",
           "vlm_topology_build", "vlm_topology_levels", "vlm_topology_level", "vlm_topology_destroy",
           "vlm_topology_box", "vlm_barrier_check", "vlm_mesh_set_tail", "vlm_mesh_get_tail",
           "vlm_mesh_set_fusion", "vlm_mesh_get_fusion", "vlm_mesh_get_stream", "vlm_mesh_time_sweeps", "vlm_mesh_sweep_time",
           "vlm_mesh_register_ex", "vlm_mesh_register_batch_ex",
           "vlm_ctx_device_name",
           "vlm_mesh_stats", "vlm_profile_kernel", "vlm_div", "vlm_pressure_solve", "vlm_pressure_solve_device",
           "vlm_mesh_register_batch", "vlm_mesh_systems", "vlm_pressure_solve_batch", "vlm_exact_sum_noalloc", "vlm_precond_apply", "vlm_flow_create", "vlm_flow_set_state",
           "vlm_flow_step", "vlm_flow_run_steady", "vlm_flow_get_state", "vlm_flow_destroy", "vlm_flow_launches",
           "vlm_flow_request_bytes", "vlm_server_create", "vlm_server_clock", "vlm_server_submit",
           "vlm_server_collect", "vlm_server_result_fields", "vlm_server_destroy", "vlm_flow_set_model",
           "vlm_flow_get_model_state", "vlm_flow_write_restart", "vlm_flow_read_restart", "vlm_box_create",
           "vlm_box_desc", "vlm_box_patch_sides", "vlm_box_destroy", "vlm_flow_set_boundary_values"]


class MeshDesc(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_internal_faces", C.c_int32), ("n_faces", C.c_int32),
                ("owner", C.c_void_p), ("neighbour", C.c_void_p), ("magSf", C.c_void_p), ("ndc", C.c_void_p),
                ("V", C.c_void_p), ("Sf", C.c_void_p), ("d", C.c_void_p), ("w", C.c_void_p),
                ("corrVecs", C.c_void_p), ("two_d", C.c_int32), ("empty_dir", C.c_int32), ("n_patches", C.c_int32),
                ("patch_start", C.c_void_p), ("patch_size", C.c_void_p), ("C", C.c_void_p), ("Cf", C.c_void_p),
                ("skewVecs", C.c_void_p)]


class BoxSpec(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int32 * 3),
                ("two_d", C.c_int32), ("beta", C.c_double * 3), ("points", C.c_void_p)]


class SolverCtrl(C.Structure):
    _fields_ = [("solver", C.c_char * 32), ("preconditioner", C.c_char * 32), ("tolerance", C.c_double),
                ("relTol", C.c_double), ("maxIter", C.c_int32), ("minIter", C.c_int32), ("nSweeps", C.c_int32),
                ("smoother", C.c_char * 16), ("precision", C.c_char * 16), ("reproducible", C.c_int32),
                ("mergeLevels", C.c_int32), ("innerRelTol", C.c_double)]


class SolverPerf(C.Structure):
    _fields_ = [("initialResidual", C.c_double), ("finalResidual", C.c_double), ("residualSum", C.c_double),
                ("normFactor", C.c_double), ("iterations", C.c_int32), ("converged", C.c_int32),
                ("outerIterations", C.c_int32), ("status", C.c_int32), ("solver", C.c_char * 32)]


class FlowCtrl(C.Structure):
    _fields_ = [("nu", C.c_double), ("steady", C.c_int32), ("div_scheme", C.c_int32), ("ddt_scheme", C.c_int32),
                ("n_outer", C.c_int32), ("n_corr", C.c_int32), ("n_non_orth_corr", C.c_int32),
                ("momentum_predictor", C.c_int32), ("alpha_u", C.c_double), ("alpha_p", C.c_double),
                ("p_ref_cell", C.c_int32), ("p_ref_value", C.c_double), ("U", SolverCtrl), ("p", SolverCtrl),
                ("p_final", SolverCtrl), ("div_coeff", C.c_double), ("grad_scheme", C.c_int32),
                ("grad_p_scheme", C.c_int32), ("u_robin", C.c_void_p), ("p_robin", C.c_void_p),
                ("u_advective", C.c_void_p)]


class StepInfo(C.Structure):
    _fields_ = [("UInitialResidual", C.c_double), ("pInitialResidual", C.c_double),
                ("continuityError", C.c_double), ("iterations", C.c_int32), ("launches", C.c_int32)]


class FlowModel(C.Structure):
    _fields_ = [("les", C.c_int32), ("Cs", C.c_double), ("van_driest", C.c_int32), ("Aplus", C.c_double),
                ("Cdelta", C.c_double), ("kappa", C.c_double), ("delta_coeff", C.c_double),
                ("nut_max_ratio", C.c_double), ("depth", C.c_double), ("wall_patch", C.c_void_p),
                ("forcing", C.c_int32), ("force", C.c_double * 3), ("Ubar", C.c_double * 3),
                ("relaxation", C.c_double), ("grad_p", C.c_double)]


class FlowRequest(C.Structure):
    _fields_ = [("mesh", C.c_void_p), ("ctrl", C.c_void_p), ("u_type", C.c_void_p), ("u_value", C.c_void_p),
                ("p_type", C.c_void_p), ("p_value", C.c_void_p), ("U0", C.c_void_p), ("p0", C.c_void_p),
                ("n_steps", C.c_int32), ("dt", C.c_double), ("max_iter", C.c_int32), ("residual_tol", C.c_double),
                ("arrival", C.c_double), ("device_bytes", C.c_int64), ("mesh_flags", C.c_int32)]


class FlowResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("iterations", C.c_int32), ("arrival", C.c_double),
                ("admitted", C.c_double), ("finished", C.c_double), ("UInitialResidual", C.c_double),
                ("pInitialResidual", C.c_double), ("continuityError", C.c_double), ("device_bytes", C.c_int64),
                ("launches", C.c_int64)]


_lib = None


def load():
    """Loads the native library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"voluma_b200 native library missing: {LIB_PATH} (run python -m voluma_b200.build)")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    i32 = C.c_int32
    L.vlm_last_error.restype = C.c_char_p
    L.vlm_last_error.argtypes = [P]
    L.vlm_ctx_create.argtypes = [C.c_int, C.POINTER(P)]
    L.vlm_ctx_destroy.argtypes = [P]
    L.vlm_ctx_stream.restype = P
    L.vlm_ctx_stream.argtypes = [P]
    L.vlm_mesh_register.argtypes = [P, C.POINTER(MeshDesc), i32, C.POINTER(P)]
    L.vlm_mesh_register_ex.argtypes = [P, C.POINTER(MeshDesc), i32, i32, C.POINTER(P)]
    L.vlm_mesh_register_batch_ex.argtypes = [P, i32, P, i32, i32, C.POINTER(P)]
    L.vlm_mesh_release.argtypes = [P]
    L.vlm_amul.argtypes = [P, P, P, P, P, P, P]
    L.vlm_ldu_solve.argtypes = [P, P, P, P, P, P, P, C.POINTER(SolverCtrl), C.POINTER(SolverPerf)]
    L.vlm_ldu_solve_device.argtypes = [P, P, P, P, P, P, P, C.POINTER(SolverCtrl), C.POINTER(SolverPerf)]
    L.vlm_gamg_apply.argtypes = [P, P, P, P, P, P, P, C.POINTER(SolverCtrl)]
    L.vlm_precond_apply.argtypes = [P, P, P, P, P, P, P, C.POINTER(SolverCtrl)]
    L.vlm_flow_create.argtypes = [P, P, C.POINTER(FlowCtrl), P, P, P, P, C.POINTER(P)]
    L.vlm_flow_set_state.argtypes = [P, P, P]
    L.vlm_flow_set_boundary_values.argtypes = [P, P, P]
    L.vlm_flow_step.argtypes = [P, C.c_double, C.POINTER(StepInfo)]
    L.vlm_flow_run_steady.argtypes = [P, C.c_int32, C.c_double, C.POINTER(C.c_int32), C.POINTER(StepInfo)]
    L.vlm_flow_get_state.argtypes = [P, P, P, P]
    L.vlm_flow_destroy.argtypes = [P]
    L.vlm_flow_set_model.argtypes = [P, C.POINTER(FlowModel)]
    L.vlm_flow_get_model_state.argtypes = [P, P, P]
    L.vlm_flow_write_restart.argtypes = [P, C.c_char_p]
    L.vlm_flow_read_restart.argtypes = [P, C.c_char_p, C.POINTER(C.c_int32)]
    L.vlm_flow_launches.restype = C.c_int64
    L.vlm_flow_launches.argtypes = [P]
    L.vlm_flow_request_bytes.restype = C.c_int64
    L.vlm_flow_request_bytes.argtypes = [C.c_int32, C.c_int32]
    L.vlm_server_create.argtypes = [C.c_int32, C.c_int64, C.c_int32, C.POINTER(P)]
    L.vlm_server_clock.restype = C.c_double
    L.vlm_server_clock.argtypes = [P]
    L.vlm_server_submit.argtypes = [P, C.POINTER(FlowRequest), C.POINTER(C.c_int64)]
    L.vlm_server_collect.argtypes = [P, C.POINTER(FlowResult), C.c_int32, C.POINTER(C.c_int32), C.c_double]
    L.vlm_server_result_fields.argtypes = [P, C.c_int64, P, P, P]
    L.vlm_server_destroy.argtypes = [P]
    L.vlm_gamg_levels.argtypes = [P, C.POINTER(i32)]
    L.vlm_gamg_level.argtypes = [P, i32, P, P, P, P]
    L.vlm_gamg_colours.argtypes = [P, i32, C.POINTER(i32)]
    L.vlm_laplacian.argtypes = [P, P, P, P, P, P, i32, i32, P, P, P, P, P, P, P]
    L.vlm_grad.argtypes = [P, P, P, P, P, i32, P]
    L.vlm_exact_sum.argtypes = [P, P, C.c_int64, C.POINTER(C.c_double)]
    L.vlm_topology_build.argtypes = [i32, i32, P, P, P, P, i32, C.POINTER(P)]
    L.vlm_topology_levels.argtypes = [P, C.POINTER(i32)]
    L.vlm_topology_level.argtypes = [P, i32, P, P, P, P, P, P, P, P]
    L.vlm_topology_destroy.argtypes = [P]
    L.vlm_topology_box.argtypes = [P, P]
    L.vlm_barrier_check.argtypes = [P, i32, C.c_int64, i32, i32, P, C.POINTER(i32)]
    L.vlm_div.argtypes = [P, P, P, P]
    L.vlm_pressure_solve.argtypes = [P, P, P, P, P, P, P, i32, C.c_double, i32, i32, C.POINTER(SolverCtrl),
                                     C.POINTER(SolverCtrl), P, P]
    L.vlm_pressure_solve_device.argtypes = L.vlm_pressure_solve.argtypes
    L.vlm_mesh_register_batch.argtypes = [P, i32, P, i32, C.POINTER(P)]
    L.vlm_exact_sum_noalloc.argtypes = [P, C.c_int64, P, P]
    L.vlm_mesh_systems.argtypes = [P, P, P, P, P]
    L.vlm_pressure_solve_batch.argtypes = [P, P, P, P, P, P, P, P, C.c_double, i32, i32, C.POINTER(SolverCtrl),
                                           C.POINTER(SolverCtrl), P, P, i32]
    L.vlm_mesh_stats.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.vlm_mesh_set_tail.argtypes = [P, i32, C.c_int64, C.c_int64]
    L.vlm_mesh_set_fusion.argtypes = [P, C.c_int64, C.c_int64, C.c_int64]
    L.vlm_mesh_time_sweeps.argtypes = [P, i32]
    L.vlm_mesh_sweep_time.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.vlm_mesh_get_fusion.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.vlm_mesh_get_stream.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.vlm_ctx_device_name.argtypes = [P, C.c_char_p, i32]
    L.vlm_mesh_get_tail.argtypes = [P, C.POINTER(i32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.vlm_box_create.argtypes = [P, C.POINTER(BoxSpec), C.POINTER(P)]
    L.vlm_box_desc.argtypes = [P, C.POINTER(MeshDesc)]
    L.vlm_box_patch_sides.argtypes = [P, P]
    L.vlm_box_destroy.argtypes = [P]
    L.vlm_profile_kernel.argtypes = [P, P, C.c_char_p, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    for name in EXPORTS:
        keep = ("vlm_last_error", "vlm_ctx_stream", "vlm_flow_request_bytes", "vlm_server_clock", "vlm_flow_launches")
        getattr(L, name).restype = getattr(L, name).restype if name in keep else C.c_int
    _lib = L
    return L


class VlmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status
        self.name = STATUS.get(status, str(status))


def check(rc, ctx=None):
    if rc != 0:
        msg = load().vlm_last_error(ctx).decode(errors="replace")
        raise VlmError(rc, msg)

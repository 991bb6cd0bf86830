"""ctypes binding of libvistio_b200.so (the C ABI in include/vistio_cuda.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvistio_b200.so")

OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_MESH", 2: "INVALID_MATERIAL", 3: "INVALID_CONFIG", 4: "IO", 5: "SERIALIZATION",
    6: "GPU", 7: "SOLVER_DIVERGENCE", 8: "INVARIANT", 9: "TIMEOUT", 10: "OOM", 11: "NOT_SPD", 12: "CAPACITY",
}


class MeshDesc(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32), ("pos_x", C.POINTER(C.c_float)),
                ("pos_y", C.POINTER(C.c_float)), ("pos_z", C.POINTER(C.c_float)),
                ("indices", C.POINTER(C.c_uint32))]


class SolverConfigC(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("al_max_iterations", C.c_uint32), ("tolerance", C.c_double),
                ("gravity", C.c_float * 3), ("damping", C.c_float), ("stretch_weight", C.c_float),
                ("bending_weight", C.c_float), ("rayleigh_mass_damping", C.c_float), ("barrier_d_hat", C.c_float),
                ("barrier_kappa", C.c_float), ("al_mu_initial", C.c_float), ("al_mu_growth", C.c_float),
                ("al_tolerance", C.c_float), ("friction_coefficient", C.c_float), ("contact_damping", C.c_float),
                ("compliant_d_hat_scale", C.c_float), ("contact_damping_max", C.c_float),
                ("contact_velocity_threshold", C.c_float), ("compliant_contact", C.c_int32),
                ("adaptive_contact_damping", C.c_int32), ("refinement_sweeps", C.c_uint32),
                ("host_factorization", C.c_uint32), ("reserved0", C.c_uint32)]


class MaterialDesc(C.Structure):
    _fields_ = [("density", C.c_float), ("stretch_stiffness_warp", C.c_float),
                ("stretch_stiffness_weft", C.c_float), ("shear_stiffness", C.c_float),
                ("bending_stiffness_warp", C.c_float), ("bending_stiffness_weft", C.c_float),
                ("thickness", C.c_float), ("friction", C.c_float), ("damping", C.c_float)]


class ModelDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("warp_stiffness", C.c_float), ("weft_stiffness", C.c_float)]


class SetupDesc(C.Structure):
    _fields_ = [("model", C.c_int32), ("bending", C.c_int32), ("stiffness", C.c_float),
                ("bend_stiffness", C.c_float), ("density_gsm", C.c_float), ("warp_stiffness", C.c_float),
                ("weft_stiffness", C.c_float), ("bend_warp", C.c_float), ("bend_weft", C.c_float),
                ("matrix_dt", C.c_float)]


class ContactDesc(C.Structure):
    _fields_ = [("has_ground", C.c_int32), ("ground_height", C.c_float), ("has_sphere", C.c_int32),
                ("sphere_center", C.c_float * 3), ("sphere_radius", C.c_float), ("self_collision", C.c_int32),
                ("kappa", C.c_float), ("thickness", C.c_float), ("has_cylinder", C.c_int32),
                ("cylinder_center_x", C.c_float), ("cylinder_center_z", C.c_float), ("cylinder_top_y", C.c_float),
                ("cylinder_radius", C.c_float), ("has_box", C.c_int32), ("box_min", C.c_float * 3),
                ("box_max", C.c_float * 3)]


class StepResultC(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("converged", C.c_int32), ("final_residual", C.c_double),
                ("wall_time", C.c_double), ("al_iterations", C.c_uint32), ("active_contacts", C.c_uint32),
                ("last_alpha", C.c_float), ("status", C.c_int32)]


class ContactResultC(C.Structure):
    _fields_ = [("resolved_count", C.c_uint32), ("max_residual_penetration", C.c_float),
                ("total_force_magnitude", C.c_float)]


class ColliderResultsC(C.Structure):
    _fields_ = [("ground", ContactResultC), ("sphere", ContactResultC), ("cylinder", ContactResultC),
                ("box", ContactResultC)]


# Every entry point include/vistio_cuda.h declares, with its ctypes signature.
class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("max_cohort", C.c_uint32),
                ("setup_threads", C.c_uint32), ("steps_per_slice", C.c_uint32), ("cache_bytes", C.c_uint64),
                ("gpu_factorization", C.c_uint32), ("sweep_mode", C.c_uint32), ("admit_wait_ms", C.c_uint32)]


class RequestC(C.Structure):
    _fields_ = [("mesh", MeshDesc), ("pinned", C.POINTER(C.c_uint8)), ("config", SolverConfigC),
                ("setup", SetupDesc), ("has_contact", C.c_int32), ("contact", ContactDesc), ("dt", C.c_float),
                ("steps", C.c_uint32)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("vertex_count", C.c_uint32), ("cohort", C.c_uint32),
                ("cache_hit", C.c_int32), ("submit_s", C.c_double), ("ready_s", C.c_double),
                ("start_s", C.c_double), ("done_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "failed", "cohorts_started", "cohorts_active",
                                          "max_cohorts_active", "bytes_in_use", "max_bytes_in_use", "cache_hits",
                                          "cache_misses", "instance_steps")] + \
               [(n, C.c_double) for n in ("p50_latency_s", "p99_latency_s", "mean_latency_s", "throughput")]


_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
SIGNATURES = {
    "vistio_ctx_create": (C.c_int, [C.c_int32, C.POINTER(_vp)]),
    "vistio_ctx_destroy": (C.c_int, [_vp]),
    "vistio_status_string": (C.c_char_p, [C.c_int]),
    "vistio_last_error": (C.c_char_p, [_vp]),
    "vistio_sync": (C.c_int, [_vp]),
    "vistio_solver_init": (C.c_int, [_vp, C.POINTER(MeshDesc), C.POINTER(SolverConfigC), C.POINTER(C.c_uint8),
                                     C.POINTER(_vp)]),
    "vistio_solver_init_with_material": (C.c_int, [_vp, C.POINTER(MeshDesc), C.POINTER(SolverConfigC),
                                                   C.POINTER(MaterialDesc), C.POINTER(ModelDesc), C.c_int32,
                                                   C.POINTER(C.c_uint8), C.POINTER(_vp)]),
    "vistio_solver_init_explicit": (C.c_int, [_vp, C.POINTER(MeshDesc), C.POINTER(SolverConfigC),
                                              C.POINTER(SetupDesc), C.POINTER(C.c_uint8), C.POINTER(_vp)]),
    "vistio_solver_destroy": (C.c_int, [_vp]),
    "vistio_solver_name": (C.c_char_p, [_vp]),
    "vistio_solver_info": (C.c_int, [_vp, _u32p, _u32p, _u32p, _u64p, _u64p, _u32p, _u32p]),
    "vistio_solver_lumped_masses": (C.c_int, [_vp, _fp]),
    "vistio_solver_set_ground": (C.c_int, [_vp, C.c_int32, C.c_float]),
    "vistio_solver_set_state": (C.c_int, [_vp, _fp, _fp, _fp, _fp, _fp, _fp]),
    "vistio_solver_get_state": (C.c_int, [_vp, _fp, _fp, _fp, _fp, _fp, _fp]),
    "vistio_solver_contact_force": (C.c_int, [_vp, _fp]),
    "vistio_step": (C.c_int, [_vp, C.c_float, C.POINTER(StepResultC)]),
    "vistio_step_with_ipc": (C.c_int, [_vp, C.c_float, C.POINTER(ContactDesc), C.POINTER(StepResultC)]),
    "vistio_resolve_contacts": (C.c_int, [_vp, C.POINTER(ContactDesc), C.POINTER(ColliderResultsC)]),
    "vistio_batch_resolve_contacts": (C.c_int, [_vp, C.POINTER(ContactDesc), C.POINTER(ColliderResultsC)]),
    "vistio_batch_create": (C.c_int, [_vp, C.POINTER(_vp), C.c_uint32, C.POINTER(_vp)]),
    "vistio_batch_destroy": (C.c_int, [_vp]),
    "vistio_batch_step": (C.c_int, [_vp, C.c_float, C.c_uint32, C.POINTER(ContactDesc)]),
    "vistio_batch_set_state": (C.c_int, [_vp, C.c_uint32, _fp, _fp, _fp, _fp, _fp, _fp]),
    "vistio_batch_get_state": (C.c_int, [_vp, C.c_uint32, _fp, _fp, _fp, _fp, _fp, _fp]),
    "vistio_batch_upload_positions": (C.c_int, [_vp, _fp]),
    "vistio_batch_download_positions": (C.c_int, [_vp, _fp]),
    "vistio_batch_info": (C.c_int, [_vp, _u32p, _u64p, _u64p, _u64p, _u64p, _u64p]),
    "vistio_batch_launches_per_step": (C.c_int, [_vp, _u32p]),
    "vistio_batch_factor_stats": (C.c_int, [_vp, _u32p, _fp]),
    "vistio_batch_stream": (_vp, [_vp]),
    "vistio_batch_launch_phase": (C.c_int, [_vp, C.c_int32]),
    "vistio_batch_phase_bytes": (C.c_int, [_vp, C.c_int32, _u64p]),
    "vistio_diag_wait_timeout": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_tune": (C.c_int, [_vp, _u32p, _fp]),
    "vistio_batch_tune_local": (C.c_int, [_vp, _u32p, _u32p, _fp]),
    "vistio_batch_set_local_shape": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "vistio_batch_set_self_ccd_dedup": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_set_group_limit": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_get_group_limit": (C.c_int, [_vp, _u32p]),
    "vistio_batch_set_warp_limit": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_set_sweep_mode": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_get_sweep_mode": (C.c_int, [_vp, _u32p, _u32p]),
    "vistio_batch_set_sweep_blocks": (C.c_int, [_vp, C.c_uint32]),
    "vistio_batch_get_sweep_blocks": (C.c_int, [_vp, _u32p, _fp]),
    "vistio_solver_clone": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "vistio_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(_vp)]),
    "vistio_server_destroy": (C.c_int, [_vp]),
    "vistio_server_last_error": (C.c_char_p, [_vp]),
    "vistio_server_submit": (C.c_int, [_vp, C.POINTER(RequestC), _u64p]),
    "vistio_server_tick": (C.c_int, [_vp, _u32p]),
    "vistio_server_drain": (C.c_int, [_vp, C.c_double]),
    "vistio_server_query": (C.c_int, [_vp, C.c_uint64, C.POINTER(RequestInfo)]),
    "vistio_server_result": (C.c_int, [_vp, C.c_uint64, _fp, _fp, _fp, _fp, _fp, _fp]),
    "vistio_server_release": (C.c_int, [_vp, C.c_uint64]),
    "vistio_server_get_stats": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "vistio_solver_device_bytes": (C.c_int, [_vp, C.c_int32, _u64p]),
    "vistio_sparse_factorize": (C.c_int, [_vp, C.c_uint32, _u32p, _u32p, _fp, C.POINTER(_vp)]),
    "vistio_symbolic_cache_info": (C.c_int, [C.POINTER(C.c_uint64)] * 4),
    "vistio_symbolic_cache_set_limit": (C.c_int, [C.c_uint64]),
    "vistio_sparse_solve": (C.c_int, [_vp, _fp, _fp]),
    "vistio_sparse_destroy": (C.c_int, [_vp]),
    "vistio_broadphase_pairs": (C.c_int, [_vp, C.c_uint32, _fp, _fp, _fp, C.c_uint32, _u32p, C.c_float, _u32p,
                                          C.c_uint64, _u64p]),
    "vistio_barrier_grad": (C.c_int, [_vp, C.c_uint32, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                                       C.POINTER(C.c_double)]),
    "vistio_ccd_hits": (C.c_int, [_vp, C.c_uint32, _fp, _fp, C.c_uint32, _u32p, C.c_uint64, _u32p, _u32p,
                                  C.c_uint64, _u64p, _fp]),
    "vistio_broadphase_pairs_noalloc": (C.c_int, [_vp, C.c_uint32, _fp, _fp, _fp, C.c_uint32, _u32p, C.c_float,
                                                  _u32p, C.c_uint64, _u64p]),
}

_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m vistio_b200.build` (nvcc, sm_100a). "
                "There is no CPU fallback.")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class VistioError(RuntimeError):
    """A non-OK vistio_status (mirrors the reference's VistioError)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def check(status: int, ctx=None):
    if status != OK:
        msg = lib().vistio_last_error(ctx)
        raise VistioError(status, msg.decode() if msg else "")

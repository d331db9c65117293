"""ctypes binding of libpowergrid_b200.so (the C ABI in include/powergrid_b200.h).

There is no CPU fallback: if the CUDA library is missing or no sm_100a GPU
is present, every operator constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PG_LIBRARY=checks loads the PG_CHECKS build (device-side index checks,
# reported by pg_checks_read) instead of the product library.
LIB_PATH = os.path.join(HERE, "lib", "libpowergrid_b200_checks.so" if os.environ.get("PG_LIBRARY") == "checks"
                        else "libpowergrid_b200.so")

P = C.c_void_p
U64 = C.c_uint64
F32 = C.c_float

STATUS = {0: "PG_OK", 1: "PG_INVALID_ARG", 2: "PG_OUT_OF_MEMORY", 3: "PG_CUDA_ERROR", 4: "PG_TIMEOUT",
          5: "PG_CANCELLED", 6: "PG_NOT_INITIALIZED", 7: "PG_CUFFT_ERROR", 8: "PG_REJECTED", 9: "PG_NOT_READY"}
PG_OK, PG_NOT_READY = 0, 9


class PGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Penalty(C.Structure):
    _fields_ = [("kind", C.c_int), ("nx", U64), ("ny", U64), ("nz", U64), ("beta", F32), ("delta", F32),
                ("dims2penalize", U64)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", U64), ("max_inflight", C.c_uint32), ("reserved", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("nx", U64), ("ny", U64), ("nz", U64), ("n_slices", U64), ("nc", U64), ("n_samples", U64),
                ("L", U64), ("niter", U64), ("beta", F32), ("kx", P), ("ky", P), ("kz", P), ("t", P),
                ("field_map", P), ("sense_map", P), ("data", P), ("image_out", P)]


class RequestStats(C.Structure):
    _fields_ = [("t_submit_ms", C.c_double), ("t_start_ms", C.c_double), ("t_done_ms", C.c_double),
                ("iters_done", U64), ("bytes_resident", U64), ("status", C.c_int), ("setup_ms", C.c_double),
                ("solve_ms", C.c_double), ("jobs", U64), ("error", C.c_char * 160)]


class Acquisition(C.Structure):
    _fields_ = [("kspace_encode_step_1", C.c_uint32), ("kspace_encode_step_2", C.c_uint32), ("slice", C.c_uint32),
                ("repetition", C.c_uint32), ("average", C.c_uint32), ("contrast", C.c_uint32), ("phase", C.c_uint32),
                ("number_of_samples", C.c_uint32), ("active_channels", C.c_uint32),
                ("trajectory_dimensions", C.c_uint32), ("data", P), ("traj", P)]


class EncodingLimits(C.Structure):
    _fields_ = [("shots", C.c_uint32), ("partitions", C.c_uint32), ("slices", C.c_uint32),
                ("repetitions", C.c_uint32), ("averages", C.c_uint32), ("contrasts", C.c_uint32),
                ("phases", C.c_uint32)]


class AcqRequest(C.Structure):
    _fields_ = [("nx", U64), ("ny", U64), ("nz", U64), ("L", U64), ("niter", U64), ("beta", F32),
                ("field_map", P), ("sense_map", P), ("image_out", P)]


_lib = None

# Every symbol the header declares, with its ctypes signature.
SIGNATURES = {
    "pg_init": (C.c_int, [C.c_int]),
    "pg_shutdown": (C.c_int, []),
    "pg_status_string": (C.c_char_p, [C.c_int]),
    "pg_last_error": (C.c_char_p, []),
    "pg_kernel_launch_count": (U64, []),
    "pg_gnufft_create": (C.c_int, [C.POINTER(P), U64, F32, U64, U64, U64, P, P, P]),
    "pg_gdft_create": (C.c_int, [C.POINTER(P), U64, U64, P, P, P, P, P, P, P, P]),
    "pg_gdftr2_create": (C.c_int, [C.POINTER(P), U64, U64, P, P, P, P, P, P, P, P, U64, U64, U64]),
    "pg_timeseg_create": (C.c_int, [C.POINTER(P), P, P, P, U64, U64, U64, U64, U64]),
    "pg_sense_create": (C.c_int, [C.POINTER(P), P, P, U64, U64, U64]),
    "pg_pcsense_timeseg_create": (C.c_int, [C.POINTER(P), P, P, P, U64, U64, U64, U64, U64, P, U64, U64, P, P, P,
                                            U64]),
    "pg_pcsense_create": (C.c_int, [C.POINTER(P), P, P, P, U64, U64, U64, U64, U64, P, P, P, P, U64]),
    "pg_lowrank_create": (C.c_int, [C.POINTER(P), U64, U64, U64, U64, P, P]),
    "pg_gnufft_grid_length": (C.c_int, [P, C.POINTER(U64)]),
    "pg_gnufft_forward_spatial_interp": (C.c_int, [P, P, P]),
    "pg_gnufft_adjoint_spatial_interp": (C.c_int, [P, P, P]),
    "pg_gnufft_forward_spatial_interp_device": (C.c_int, [P, P, P, P]),
    "pg_gnufft_adjoint_spatial_interp_device": (C.c_int, [P, P, P, P]),
    "pg_density_compensation": (C.c_int, [P, P, P, U64, U64, U64, P]),
    "pg_grid_coil_images": (C.c_int, [P, P, P, U64, P]),
    "pg_sum_of_squares_image": (C.c_int, [P, U64, U64, P]),
    "pg_op_destroy": (C.c_int, [P]),
    "pg_op_shape": (C.c_int, [P, C.POINTER(U64), C.POINTER(U64)]),
    "pg_op_forward": (C.c_int, [P, P, P]),
    "pg_op_adjoint": (C.c_int, [P, P, P]),
    "pg_op_forward_device": (C.c_int, [P, P, P, P]),
    "pg_op_adjoint_device": (C.c_int, [P, P, P, P]),
    "pg_gdft_forward_noalloc": (C.c_int, [U64, U64, P, P, P, P, P, P, P, P, P, P, P]),
    "pg_pcg_solve": (C.c_int, [P, P, P, P, C.POINTER(Penalty), U64, P, C.POINTER(U64)]),
    "pg_pcg_solve_device": (C.c_int, [P, P, P, P, C.POINTER(Penalty), U64, P, P, P]),
    "pg_recon_solve": (C.c_int, [P, C.POINTER(Penalty), P, U64, P]),
    "pg_pcg_state_size": (C.c_int, [P, C.POINTER(U64)]),
    "pg_pcg_state_save": (C.c_int, [P, P, U64]),
    "pg_pcg_state_load": (C.c_int, [P, C.POINTER(Penalty), P, U64]),
    "pg_pcg_resume": (C.c_int, [P, P, P, C.POINTER(Penalty), U64, P, C.POINTER(U64)]),
    "pg_pcg_resume_device": (C.c_int, [P, P, P, C.POINTER(Penalty), U64, P, P, P]),
    "pg_penalty_gradient_device": (C.c_int, [C.POINTER(Penalty), P, P, P]),
    "pg_penalty_denom_device": (C.c_int, [C.POINTER(Penalty), P, P, C.POINTER(C.c_double)]),
    "pg_pcg_solve_lowrank": (C.c_int, [P, P, P, P, C.POINTER(Penalty), U64, U64, P, U64, P, C.POINTER(U64)]),
    "pg_pcg_solve_lowrank_device": (C.c_int, [P, P, P, P, C.POINTER(Penalty), U64, U64, P, U64, P, C.POINTER(U64),
                                              P]),
    "pg_lowrank_penalty_gradient_device": (C.c_int, [C.POINTER(Penalty), U64, U64, P, P, P, P]),
    "pg_lowrank_penalty_denom_device": (C.c_int, [C.POINTER(Penalty), U64, U64, P, P, P, C.POINTER(C.c_double)]),
    "pg_acq_index_create": (C.c_int, [C.POINTER(P), C.POINTER(Acquisition), U64, C.POINTER(EncodingLimits)]),
    "pg_acq_index_destroy": (C.c_int, [P]),
    "pg_acq_index_lookup": (C.c_int, [P] + [C.c_uint32] * 7 + [C.POINTER(C.c_int64)]),
    "pg_acq_index_limits": (C.c_int, [P, C.POINTER(EncodingLimits)]),
    "pg_acq_gather_size": (C.c_int, [P] + [C.c_uint32] * 5 + [C.POINTER(U64)] * 3),
    "pg_acq_gather": (C.c_int, [P] + [C.c_uint32] * 5 + [P] * 5),
    "pg_acq_gather_device": (C.c_int, [P] + [C.c_uint32] * 5 + [P] * 6),
    "pg_write_nifti_real": (C.c_int, [C.c_char_p, P, U64, U64, U64, U64, U64]),
    "pg_write_nifti_mag_phs": (C.c_int, [C.c_char_p, P, U64, U64, U64, U64, U64]),
    "pg_server_create": (C.c_int, [C.POINTER(P), C.POINTER(ServerConfig)]),
    "pg_server_destroy": (C.c_int, [P]),
    "pg_submit": (C.c_int, [P, C.POINTER(Request), C.POINTER(U64)]),
    "pg_submit_acquisitions": (C.c_int, [P, P, C.POINTER(AcqRequest), C.POINTER(U64)]),
    "pg_poll": (C.c_int, [P, U64, C.POINTER(RequestStats)]),
    "pg_wait": (C.c_int, [P, U64, C.POINTER(RequestStats)]),
    "pg_cancel": (C.c_int, [P, U64]),
    "pg_request_footprint": (U64, [C.POINTER(Request)]),
    "pg_checks_read": (C.c_int, [C.POINTER(U64), C.POINTER(C.c_int)]),
    "pg_debug_fail_allocation_after": (None, [U64]),
    "pg_util_kb_lut": (U64, [F32, P, U64, C.POINTER(F32)]),
    "pg_profile_enable": (C.c_int, [C.c_int]),
    "pg_profile_stage_ms": (C.c_int, [C.c_char_p, C.POINTER(F32)]),
    "pg_profile_only": (C.c_int, [C.c_char_p]),
    "pg_util_gnufft_binning": (C.c_int, [P, P, P, C.POINTER(U64)]),
}


def load() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"powergrid_b200: CUDA library missing at {LIB_PATH}; run __graft_entry__.build()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != PG_OK:
        raise PGError(status, load().pg_last_error().decode(errors="replace"))


def launches() -> int:
    return int(load().pg_kernel_launch_count())

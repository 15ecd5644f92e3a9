"""ctypes declarations of include/zinq_qd.h (the library's C-ABI).

Every struct mirrors the header field by field; `load()` opens the in-tree
libzinq_qd.so and fails loudly when it has not been built (there is no CPU
fallback for the propagator).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzinq_qd.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "zinq_qd.h")

ZQD_OK = 0
STATUS = {
    0: "ZQD_OK", -1: "ZQD_ERR_INVALID_INPUT", -2: "ZQD_ERR_OUT_OF_MEMORY", -3: "ZQD_ERR_DEVICE_OOM",
    -4: "ZQD_ERR_PLAN_FAILED", -5: "ZQD_ERR_EIGEN_FAILED", -6: "ZQD_ERR_EXPRESSION", -7: "ZQD_ERR_UNSUPPORTED",
    -8: "ZQD_ERR_DEVICE", -9: "ZQD_ERR_TIMEOUT", -10: "ZQD_ERR_CANCELLED", -11: "ZQD_ERR_NOT_FOUND",
    -12: "ZQD_ERR_NO_DEVICE", -13: "ZQD_ERR_NUMERIC",
}

POT = {"harmonic": 0, "time_linear": 1, "tully_1": 2, "tully_2": 3, "tully_3": 4, "custom": 5, "lvc": 6, "file": 7}
WRITE = {"acf": 1 << 0, "kinetic_energy": 1 << 1, "momentum": 1 << 2, "norm": 1 << 3, "population": 1 << 4,
         "position": 1 << 5, "potential_energy": 1 << 6, "total_energy": 1 << 7, "wavefunction": 1 << 8}
SERIES = {"position": 0, "momentum": 1, "population": 2, "potential_energy": 3, "kinetic_energy": 4,
          "total_energy": 5, "norm": 6, "acf": 7}
PRECISION = {"fp64": 0, "fp32": 1, "auto": 2}
FFT_PLAN = {"estimate": 0, "measure": 1, "patient": 2, "exhaustive": 3}

DP = C.POINTER(C.c_double)


class ZqdPotential(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("harmonic_k", DP), ("harmonic_ndim", C.c_uint32),
        ("p", C.c_double * 5),
        ("custom_matrix", C.POINTER(C.c_char_p)), ("custom_nstate", C.c_uint32), ("custom_ndim", C.c_uint32),
        ("custom_time_dependent", C.c_int),
        ("lvc_frequencies", DP), ("lvc_nmode", C.c_uint32),
        ("lvc_excitation_energies", DP), ("lvc_nstate", C.c_uint32),
        ("lvc_kappa", DP), ("lvc_lambda", DP),
        ("file_table", DP), ("file_nrow", C.c_uint32), ("file_ncol", C.c_uint32), ("file_ndim", C.c_uint32),
    ]


class ZqdOptions(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("ndim", C.c_uint32), ("npoint", C.c_uint32), ("grid_bounds", DP),
        ("ic_position", DP), ("ic_momentum", DP), ("ic_gamma", DP), ("ic_state", C.c_uint32), ("ic_adiabatic", C.c_int),
        ("potential", ZqdPotential),
        ("time_step", C.c_double), ("iterations", C.c_uint32), ("mass", DP), ("write_mask", C.c_uint32),
        ("adiabatic", C.c_int), ("log_interval", C.c_uint32),
        ("has_absorbing_potential", C.c_int), ("cap_track_population", C.c_int), ("cap_bounds", DP),
        ("cap_exponent", C.c_double), ("cap_has_stop_norm", C.c_int), ("cap_stop_norm", C.c_double),
        ("fft_plan", C.c_int),
        ("imaginary_nstate", C.c_uint32),
        ("has_spectrum", C.c_int), ("spectrum_padding", C.c_uint32), ("spectrum_threshold", C.c_double),
        ("precision", C.c_int), ("log", C.c_int), ("ic_wavefunction", DP),
    ]


class ZqdObservables(C.Structure):
    _fields_ = [
        ("ndim", C.c_uint32), ("nstate", C.c_uint32),
        ("pos", C.c_double * 3), ("mom", C.c_double * 3), ("pop", C.c_double * 4),
        ("epot", C.c_double), ("ekin", C.c_double), ("norm", C.c_double),
        ("acf_re", C.c_double), ("acf_im", C.c_double),
    ]


WRITE_PATH_FIELDS = ("acf", "position", "momentum", "population", "potential_energy", "kinetic_energy", "norm",
                     "total_energy", "spectrum_acf", "spectrum", "wavefunction")


class ZqdWritePaths(C.Structure):
    _fields_ = [(n, C.c_char_p) for n in WRITE_PATH_FIELDS]


class ZqdObsRows(C.Structure):
    _fields_ = [("solve", C.c_uint32), ("first_row", C.c_uint32), ("nrows", C.c_uint32), ("width", C.c_uint32),
                ("rows", DP), ("solve_finished", C.c_int)]


class ZqdServerConfig(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("workers", C.c_uint32), ("max_batch", C.c_uint32),
                ("device_budget_bytes", C.c_uint64), ("stream_steps", C.c_uint32), ("stream_rows", C.c_int),
                ("max_events", C.c_uint32), ("persistent_lines", C.c_int), ("service_ctas", C.c_uint32),
                ("service_idle_us", C.c_double), ("fetch_wavefunction", C.c_int)]


class ZqdServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "failed", "cancelled", "queued",
                                          "grouped_launches", "grouped_jobs", "joined_jobs", "device_budget_bytes",
                                          "device_bytes_in_use", "peak_device_bytes", "pending_events",
                                          "dropped_events", "service_jobs", "service_launches")]


EVENT = {0: "rows", 1: "done", 2: "failed", 3: "cancelled"}


class ZqdOnchip(C.Structure):
    _fields_ = [("smem_bytes_per_cycle_per_sm", C.c_double), ("smem_gbs_per_sm", C.c_double),
                ("syncthreads_cycles", C.c_double), ("cluster_barrier_cycles", C.c_double),
                ("sm_clock_mhz", C.c_double), ("sms", C.c_uint32)]


class ZqdTuneEntry(C.Structure):
    _fields_ = [("ndim", C.c_uint32), ("npoint", C.c_uint32), ("nstate", C.c_uint32), ("precision", C.c_int),
                ("cluster_ctas", C.c_uint32), ("radix_log2", C.c_uint32), ("rows_per_cta", C.c_uint32),
                ("tile_lines", C.c_uint32), ("us_per_step", C.c_double), ("default_us_per_step", C.c_double),
                ("candidates", C.c_uint32), ("tma_row_block", C.c_int32), ("tma_tile_lines", C.c_int32)]


class ZqdNdShape(C.Structure):
    _fields_ = [("tma_row_block", C.c_uint32), ("tma_row_ctas", C.c_uint32), ("tma_row_threads", C.c_uint32),
                ("tma_tile_lines", C.c_uint32), ("tma_tile_ctas", C.c_uint32), ("tma_tile_threads", C.c_uint32),
                ("rows_per_cta", C.c_uint32), ("tile_lines", C.c_uint32)]


class ZqdEvent(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("kind", C.c_int), ("status", C.c_int), ("solve", C.c_uint32),
                ("first_row", C.c_uint32), ("nrows", C.c_uint32), ("width", C.c_uint32), ("solve_finished", C.c_int),
                ("rows", DP)]


# (name, restype, argtypes) for every entry point of zinq_qd.h
VP = C.c_void_p
SIGNATURES = [
    ("zqd_status_string", C.c_char_p, [C.c_int]),
    ("zqd_last_error", C.c_char_p, []),
    ("zqd_options_init", None, [C.POINTER(ZqdOptions)]),
    ("zqd_potential_init", None, [C.POINTER(ZqdPotential), C.c_int]),
    ("zqd_result_nsolve", C.c_uint32, [VP]),
    ("zqd_result_final", C.c_int, [VP, C.c_uint32, C.POINTER(ZqdObservables)]),
    ("zqd_result_series", C.c_int, [VP, C.c_uint32, C.c_int, C.POINTER(DP), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t)]),
    ("zqd_result_wavefunction", C.c_int, [VP, C.c_uint32, DP, C.c_size_t]),
    ("zqd_result_spectrum", C.c_int, [VP, C.c_uint32, C.POINTER(DP), C.POINTER(C.c_size_t), C.POINTER(DP),
                                      C.POINTER(C.c_size_t)]),
    ("zqd_result_device_ms", C.c_double, [VP]),
    ("zqd_result_precision", C.c_int, [VP]),
    ("zqd_result_export", C.c_int, [VP, C.c_uint32, C.POINTER(ZqdWritePaths)]),
    ("zqd_result_wavefunction_series", C.c_int, [VP, C.c_uint32, DP, C.c_size_t, C.POINTER(C.c_size_t),
                                                 C.POINTER(C.c_size_t)]),
    ("zqd_result_destroy", None, [VP]),
    ("zqd_run", C.c_int, [C.POINTER(ZqdOptions), C.POINTER(VP)]),
    ("zqd_job_create", C.c_int, [C.POINTER(ZqdOptions), C.POINTER(VP)]),
    ("zqd_job_run", C.c_int, [VP]),
    ("zqd_job_result", C.c_int, [VP, C.POINTER(VP)]),
    ("zqd_job_info", C.c_int, [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                               C.POINTER(C.c_uint32), C.POINTER(C.c_size_t)]),
    ("zqd_job_nd_shape", C.c_int, [VP, C.POINTER(ZqdNdShape)]),
    ("zqd_job_device_ms", C.c_double, [VP]),
    ("zqd_job_destroy", None, [VP]),
    ("zqd_job_step", C.c_int, [VP, C.c_uint32]),
    ("zqd_job_progress", C.c_int, [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int)]),
    ("zqd_job_observables", C.c_int, [VP, C.POINTER(ZqdObsRows)]),
    ("zqd_run_batch", C.c_int, [C.POINTER(C.POINTER(ZqdOptions)), C.c_uint32, C.POINTER(VP)]),
    ("zqd_batch_create", C.c_int, [C.POINTER(C.POINTER(ZqdOptions)), C.c_uint32, C.POINTER(VP)]),
    ("zqd_batch_run", C.c_int, [VP]),
    ("zqd_batch_result", C.c_int, [VP, C.c_uint32, C.POINTER(VP)]),
    ("zqd_batch_device_ms", C.c_double, [VP]),
    ("zqd_batch_launches", C.c_uint32, [VP]),
    ("zqd_batch_destroy", None, [VP]),
    ("zqd_result_transfer_bytes", C.c_int, [VP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("zqd_fft_plan_create", C.c_int, [C.c_uint32, C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(VP)]),
    ("zqd_fft_execute", C.c_int, [VP, VP, VP]),
    ("zqd_fft_destroy", None, [VP]),
    ("zqd_fft_execute_noalloc", C.c_int, [C.c_uint32, C.POINTER(C.c_int), C.c_int, C.c_int, VP, VP]),
    ("zqd_expr_compile", C.c_int, [C.c_char_p, C.c_size_t, C.c_size_t, C.POINTER(VP)]),
    ("zqd_expr_eval_points", C.c_int, [VP, DP, C.c_size_t, C.c_double, DP]),
    ("zqd_expr_destroy", None, [VP]),
    ("zqd_eigh_batch", C.c_int, [C.c_uint32, C.c_size_t, DP, DP, DP]),
    ("zqd_potential_plot", C.c_int, [C.POINTER(ZqdOptions), C.c_double, DP, C.c_size_t, C.c_char_p]),
    ("zqd_server_config_init", None, [C.POINTER(ZqdServerConfig)]),
    ("zqd_server_create", C.c_int, [C.POINTER(ZqdServerConfig), C.POINTER(VP)]),
    ("zqd_server_submit", C.c_int, [VP, C.POINTER(ZqdOptions), C.POINTER(C.c_uint64)]),
    ("zqd_server_wait", C.c_int, [VP, C.c_uint64, C.POINTER(VP), C.POINTER(C.c_double)]),
    ("zqd_server_wait_timeout", C.c_int, [VP, C.c_uint64, C.c_uint32, C.POINTER(VP), C.POINTER(C.c_double)]),
    ("zqd_server_cancel", C.c_int, [VP, C.c_uint64]),
    ("zqd_server_poll", C.c_int, [VP, C.POINTER(ZqdEvent), C.c_uint32, C.POINTER(C.c_uint32)]),
    ("zqd_server_stats_get", C.c_int, [VP, C.POINTER(ZqdServerStats)]),
    ("zqd_server_destroy", None, [VP]),
    ("zqd_testing_fail_device_allocations", None, [C.c_uint64, C.c_uint64]),
    ("zqd_testing_tma_withhold_load", C.c_int, [C.c_uint32, C.c_double]),
    ("zqd_testing_service_idle", C.c_int, [C.c_int, C.c_uint32, C.c_uint32, C.c_double, C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_double)]),
    ("zqd_autotune", C.c_int, [C.POINTER(ZqdTuneEntry)]),
    ("zqd_tune_save", C.c_int, [C.c_char_p]),
    ("zqd_tune_load", C.c_int, [C.c_char_p]),
    ("zqd_tune_clear", None, []),
    ("zqd_tune_size", C.c_uint32, []),
    ("zqd_measure_onchip", C.c_int, [C.POINTER(ZqdOnchip)]),
    ("zqd_device_count", C.c_int, []),
    ("zqd_set_device", C.c_int, [C.c_int]),
]

_lib = None


class ZqdError(RuntimeError):
    """A non-zero zqd_status; .status holds the code, the message the library's detail."""

    def __init__(self, status, detail):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m zinq_b200.build` (needs nvcc)")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(rc):
    if rc != ZQD_OK:
        raise ZqdError(rc, load().zqd_last_error().decode())
    return rc

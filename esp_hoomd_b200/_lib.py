"""ctypes binding of the C ABI declared in include/esp_b200.h.

The library is built in-tree (``python -m esp_hoomd_b200.build``) and loaded
from next to this file. There is no fallback: if the library is missing the
import of the compute classes raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libesp_b200.so")

ESP_LONG_RANGE = 1
ESP_SHORT_RANGE = 2
ESP_ALL = 3

ERRORS = {-1: "ESP_ERR_INVALID", -2: "ESP_ERR_CUDA", -3: "ESP_ERR_ALLOC", -4: "ESP_ERR_UNSUPPORTED",
          -5: "ESP_ERR_OVERFLOW"}

# every symbol include/esp_b200.h declares
EXPORTS = [
    "esp_params_default", "esp_last_error", "esp_create", "esp_set_params", "esp_set_box", "esp_invalidate",
    "esp_compute", "esp_get_info", "esp_destroy", "esp_batch_create", "esp_batch_compute", "esp_batch_get_info",
    "esp_batch_total_particles", "esp_batch_destroy", "esp_pswf_eval_pairs", "esp_batch_build_nlist",
    "esp_batch_nve_step1", "esp_batch_nve_step2", "esp_spread", "esp_get_sort", "esp_get_potential",
    "esp_batch_md_run", "esp_batch_md_run_f64", "esp_batch_set_timing", "esp_batch_stage_times", "esp_spread_noalloc",
    "esp_server_create", "esp_server_submit", "esp_server_start", "esp_server_status", "esp_server_wait_all",
    "esp_server_get_stats", "esp_server_destroy", "esp_set_exclusions", "esp_batch_set_exclusions",
    "esp_compute_f64", "esp_batch_compute_f64", "esp_batch_autotune", "esp_batch_lj", "esp_batch_lj_f64",
    "esp_batch_nve_step1_f64", "esp_batch_nve_step2_f64", "esp_batch_build_pairlist", "esp_batch_pairlist_check",
    "esp_compute_hoomd", "esp_batch_set_rigid_water", "esp_batch_device_errors", "esp_batch_nlist_check",
]

ESP_FP32 = 0
ESP_FP64 = 1

STAGES = ["bin", "sort", "spread", "fft", "interp", "pair", "nlist", "nve"]


class EspParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("order", ctypes.c_int),
                ("kappa", ctypes.c_double), ("rcut", ctypes.c_double), ("alpha", ctypes.c_double),
                ("n_table", ctypes.c_int), ("target_error", ctypes.c_double), ("window_c", ctypes.c_double),
                ("window_degree", ctypes.c_int), ("tile", ctypes.c_int), ("threads_per_particle", ctypes.c_int),
                ("precision", ctypes.c_int), ("fft_mode", ctypes.c_int), ("interp_mode", ctypes.c_int)]


class EspInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("order", ctypes.c_int),
                ("tile", ctypes.c_int), ("window_degree", ctypes.c_int), ("c_split", ctypes.c_double),
                ("c_window", ctypes.c_double), ("rcut", ctypes.c_double), ("lambda0", ctypes.c_double),
                ("m2", ctypes.c_double), ("split_fit_err", ctypes.c_double), ("window_fit_err", ctypes.c_double),
                ("device_bytes", ctypes.c_longlong)]


class EspServerConfig(ctypes.Structure):
    _fields_ = [("params", EspParams), ("hbm_budget", ctypes.c_longlong), ("max_systems", ctypes.c_int),
                ("max_particles", ctypes.c_int)]


class EspRequest(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("rcut", ctypes.c_double), ("skin", ctypes.c_double), ("nlist_cap", ctypes.c_int),
                ("nsteps", ctypes.c_int), ("dt", ctypes.c_double), ("arrival", ctypes.c_double),
                ("pos4", ctypes.c_void_p), ("vel4", ctypes.c_void_p), ("charge", ctypes.c_void_p),
                ("out_pos4", ctypes.c_void_p), ("out_vel4", ctypes.c_void_p), ("out_force4", ctypes.c_void_p),
                ("out_energy", ctypes.c_void_p), ("rigid_doh", ctypes.c_double), ("rigid_dhh", ctypes.c_double)]


class EspRequestStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("t_arrival", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("footprint", ctypes.c_longlong)]


class EspServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("rounds", ctypes.c_longlong), ("particle_steps", ctypes.c_longlong),
                ("influence_builds", ctypes.c_longlong), ("influence_hits", ctypes.c_longlong),
                ("max_active", ctypes.c_int), ("peak_bytes", ctypes.c_longlong), ("arena_bytes", ctypes.c_longlong)]


_lib = None


class EspError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = get_lib().esp_last_error().decode(errors="replace")
        super().__init__("%s failed (%s): %s" % (where, ERRORS.get(code, code), msg))
        self.code = code


def get_lib() -> ctypes.CDLL:
    """Load the library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libesp_b200.so not built: run `python -m esp_hoomd_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        lib.esp_last_error.restype = ctypes.c_char_p
        lib.esp_last_error.argtypes = []
        lib.esp_params_default.argtypes = [ctypes.POINTER(EspParams)]
        lib.esp_create.argtypes = [ctypes.POINTER(EspParams), D, D, D, I, ctypes.POINTER(P)]
        lib.esp_set_params.argtypes = [P, ctypes.POINTER(EspParams)]
        lib.esp_set_box.argtypes = [P, D, D, D]
        lib.esp_invalidate.argtypes = [P]
        lib.esp_compute.argtypes = [P, P, P, P, I, P, P, P, P, P, P, I]
        lib.esp_get_info.argtypes = [P, ctypes.POINTER(EspInfo)]
        lib.esp_destroy.argtypes = [P]
        lib.esp_batch_create.argtypes = [ctypes.POINTER(EspParams), I, P, P, P, ctypes.POINTER(P)]
        lib.esp_batch_compute.argtypes = [P, P, P, P, P, P, P, P, P, P, I]
        lib.esp_batch_get_info.argtypes = [P, I, ctypes.POINTER(EspInfo)]
        lib.esp_batch_total_particles.argtypes = [P]
        lib.esp_batch_destroy.argtypes = [P]
        lib.esp_pswf_eval_pairs.argtypes = [P, I, P, P, D, I, P, P, P, P, P, P, P]
        lib.esp_batch_build_nlist.argtypes = [P, P, P, D, I, P, P, P]
        lib.esp_batch_nve_step1.argtypes = [P, P, P, P, P, D]
        lib.esp_batch_nve_step2.argtypes = [P, P, P, P, P, D]
        lib.esp_spread.argtypes = [P, P, P, P, I, P]
        lib.esp_get_sort.argtypes = [P, P, P, P]
        lib.esp_get_potential.argtypes = [P, P, P]
        lib.esp_batch_md_run.argtypes = [P, P, P, P, P, P, P, P, P, P, P, I, D, I]
        lib.esp_batch_md_run_f64.argtypes = [P, P, P, P, P, P, P, P, P, P, P, I, D, D, D, D, I]
        lib.esp_batch_set_timing.argtypes = [P, I]
        lib.esp_batch_stage_times.argtypes = [P, P, P]
        lib.esp_server_create.argtypes = [ctypes.POINTER(EspServerConfig), ctypes.POINTER(P)]
        lib.esp_server_submit.argtypes = [P, ctypes.POINTER(EspRequest), ctypes.POINTER(ctypes.c_longlong)]
        lib.esp_server_start.argtypes = [P]
        lib.esp_server_status.argtypes = [P, ctypes.c_longlong, ctypes.POINTER(EspRequestStatus)]
        lib.esp_server_wait_all.argtypes = [P, D]
        lib.esp_server_get_stats.argtypes = [P, ctypes.POINTER(EspServerStats)]
        lib.esp_server_destroy.argtypes = [P]
        lib.esp_set_exclusions.argtypes = [P, P, P, I]
        lib.esp_batch_set_exclusions.argtypes = [P, P, P, I]
        lib.esp_compute_f64.argtypes = [P, P, P, P, I, P, P, P, P, P, P, I]
        lib.esp_batch_compute_f64.argtypes = [P, P, P, P, P, P, P, P, P, P, I]
        lib.esp_batch_lj.argtypes = [P, P, P, P, P, P, D, D, D, P, P]
        lib.esp_batch_lj_f64.argtypes = [P, P, P, P, P, P, D, D, D, P, P]
        lib.esp_batch_nve_step1_f64.argtypes = [P, P, P, P, P, D]
        lib.esp_batch_nve_step2_f64.argtypes = [P, P, P, P, P, D]
        lib.esp_batch_set_rigid_water.argtypes = [P, P, P, D, D]
        lib.esp_batch_autotune.argtypes = [P, P, P, P, P, P, P, I, I, ctypes.POINTER(EspParams), P, I]
        lib.esp_spread_noalloc.argtypes = [P, ctypes.POINTER(EspParams), D, D, D, P, P, I, P]
        lib.esp_batch_build_pairlist.argtypes = [P, P, P, D, I]
        lib.esp_batch_device_errors.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        lib.esp_compute_hoomd.argtypes = [P, P, P, P, I, P, P, P, P, P, I, P, I]
        lib.esp_batch_pairlist_check.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        lib.esp_batch_nlist_check.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        for name in EXPORTS:
            if name != "esp_last_error":
                getattr(lib, name).restype = ctypes.c_int
        _lib = lib
    return _lib


def check(code: int, where: str) -> None:
    if code != 0:
        raise EspError(code, where)

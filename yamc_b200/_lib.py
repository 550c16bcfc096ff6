"""ctypes binding of libyamc_b200.so (the C ABI of include/yamc.h).

The library is built in-tree (``yamc_b200/libyamc_b200.so``, see build.py).
There is no CPU implementation of the engine: if the library cannot be loaded,
or no CUDA device is present, calls raise instead of falling back.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the engine library; YAMC_LIBRARY names another build of it (the bounds-checked
# libyamc_b200_checked.so, for instance)
LIB_PATH = os.environ.get("YAMC_LIBRARY") or os.path.join(HERE, "libyamc_b200.so")

YAMC_OK = 0
YAMC_ELIMITS = -2
YAMC_EPARAMETER = -3
YAMC_EWRONG_FUNCTION = -5
YAMC_ERNG_EXHAUSTED = -12
YAMC_ENAN = -13
YAMC_EBOUNDS = -15
YAMC_KSPACE_AUTO = 0
YAMC_KSPACE_REGISTERS = 1
YAMC_KSPACE_STREAMED = 2
YAMC_FP64 = 0
YAMC_MIXED = 1


class YamcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "sr", "sk", "alphaL", "temp", "external_permutivity", "BoxLength", "density",
        "dr_a", "d_angle_degree", "xlambda_c", "xlambda_f", "pressure",
        "pressure_step_multiplier", "max_volume_scaling",
        "n_store_traj_interval", "n_store_energy_interval")] + [
        ("max_cycle", ctypes.c_int32), ("random_seed", ctypes.c_int32),
        ("input_nbytes_xyz", ctypes.c_int32), ("input_nbytes_ang", ctypes.c_int32),
        ("output_nbytes_xyz", ctypes.c_int32), ("output_nbytes_ang", ctypes.c_int32)] + [
        (n, ctypes.c_double) for n in (
        "alpha", "rmax", "rmax2", "kT_kcal_mol", "dbjr_a", "dbjr", "xclb",
        "alpha_over_sqrt_pi", "two_alpha_over_sqrt_pi", "kext", "minus_two_kext",
        "dr", "d_angle", "log_max_volume_scaling", "pressure_angstr_kT")] + [
        ("kmax", ctypes.c_int32), ("precision", ctypes.c_int32)]


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class YamcSystem(ctypes.Structure):
    _fields_ = [("natom", ctypes.c_int32), ("nmol", ctypes.c_int32),
                ("x", _dp), ("y", _dp), ("z", _dp), ("charge", _dp), ("sigma", _dp), ("epsilon", _dp),
                ("hard_core_angstr", _dp), ("mass", _dp), ("first_atom", _ip), ("last_atom", _ip),
                ("n_species", ctypes.c_int32), ("mol_numbers", _ip), ("move_weights", _dp)]


class MoveRecord(ctypes.Structure):
    _fields_ = [("imol", ctypes.c_int32), ("flags", ctypes.c_int32), ("cursor", ctypes.c_int64),
                ("du_real", ctypes.c_double), ("du_k_coul", ctypes.c_double),
                ("du_k_lj", ctypes.c_double), ("du_ext", ctypes.c_double)]


MOVE_RECORD_DTYPE = np.dtype([("imol", np.int32), ("flags", np.int32), ("cursor", np.int64),
                              ("du_real", np.float64), ("du_k_coul", np.float64),
                              ("du_k_lj", np.float64), ("du_ext", np.float64)])
assert MOVE_RECORD_DTYPE.itemsize == ctypes.sizeof(MoveRecord)

class VolumeRecord(ctypes.Structure):
    _fields_ = [("cycle", ctypes.c_int64), ("flags", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("cursor", ctypes.c_int64), ("box_old", ctypes.c_double), ("box_new", ctypes.c_double),
                ("du", ctypes.c_double), ("arg", ctypes.c_double)]


VOLUME_RECORD_DTYPE = np.dtype([("cycle", np.int64), ("flags", np.int32), ("pad", np.int32), ("cursor", np.int64),
                                ("box_old", np.float64), ("box_new", np.float64), ("du", np.float64),
                                ("arg", np.float64)])
assert VOLUME_RECORD_DTYPE.itemsize == ctypes.sizeof(VolumeRecord)

# every entry point declared in include/yamc.h, with (restype, argtypes)
_VP = ctypes.c_void_p
_PPP = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES = {
    "yamc_params_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(YamcParams)]),
    "yamc_params_init": (ctypes.c_int, [ctypes.POINTER(YamcParams), ctypes.c_int32]),
    "yamc_params_recalc": (ctypes.c_int, [ctypes.POINTER(YamcParams), ctypes.c_double]),
    "yamc_inputs_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _PPP]),
    "yamc_inputs_get": (ctypes.c_int, [_VP, ctypes.POINTER(YamcSystem), ctypes.POINTER(YamcParams)]),
    "yamc_inputs_free": (ctypes.c_int, [_VP]),
    "yamc_create": (ctypes.c_int, [ctypes.POINTER(YamcSystem), ctypes.POINTER(YamcParams), ctypes.c_int32, _PPP]),
    "yamc_destroy": (ctypes.c_int, [_VP]),
    "yamc_energies": (ctypes.c_int, [_VP, _dp]),
    "yamc_full_sums": (ctypes.c_int, [_VP, _dp]),
    "yamc_get_positions": (ctypes.c_int, [_VP, _dp, _dp, _dp]),
    "yamc_sizes": (ctypes.c_int, [_VP, _ip]),
    "yamc_set_positions": (ctypes.c_int, [_VP, _dp, _dp, _dp, _dp]),
    "yamc_forces": (ctypes.c_int, [_VP, _dp, _dp, _dp, _dp, _dp]),
    "yamc_move_old": (ctypes.c_int, [_VP, ctypes.c_int32, _dp, _dp]),
    "yamc_move_eval": (ctypes.c_int, [_VP, ctypes.c_int32, _dp, _dp, _dp, _dp, _ip, _dp, _dp]),
    "yamc_move_commit": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "yamc_run_chain": (ctypes.c_int, [_VP, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int32, _ip]),
    "yamc_run_chain_device": (ctypes.c_int, [_VP, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int32, _ip]),
    "yamc_run_mc": (ctypes.c_int, [_VP, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int64,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_int32, _ip]),
    "yamc_volume_eval": (ctypes.c_int, [_VP, ctypes.c_double, _dp, _ip]),
    "yamc_volume_commit": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "yamc_get_params": (ctypes.c_int, [_VP, ctypes.POINTER(YamcParams)]),
    "yamc_set_xchange_weights": (ctypes.c_int, [_VP, _dp]),
    "yamc_rdf_create": (ctypes.c_int, [ctypes.c_int32, _ip, ctypes.c_int32, _ip, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, _PPP]),
    "yamc_rdf_destroy": (ctypes.c_int, [_VP]),
    "yamc_rdf_nbin": (ctypes.c_int, [_VP, _ip]),
    "yamc_rdf_add_frame": (ctypes.c_int, [_VP, _dp, _dp, _dp, ctypes.c_double]),
    "yamc_rdf_add_ctx": (ctypes.c_int, [_VP, _VP]),
    "yamc_rdf_result": (ctypes.c_int, [_VP, _dp, _dp, _ip]),
    "yamc_xchange_eval": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32, _dp, _ip]),
    "yamc_xchange_commit": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "yamc_set_refresh": (ctypes.c_int, [_VP, ctypes.c_int64]),
    "yamc_refresh_count": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "yamc_set_launch": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32]),
    "yamc_set_kspace_layout": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "yamc_get_launch": (ctypes.c_int, [_VP, _ip]),
    "yamc_last_kernel_ms": (ctypes.c_int, [_VP, _dp]),
    "yamc_phase_cycles": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]),
    "yamc_checked_build": (ctypes.c_int, [_ip]),
    "yamc_bounds_check_selftest": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, _dp, _ip]),
    "yamc_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(YamcSystem), ctypes.POINTER(YamcParams),
                                         ctypes.c_int32, _PPP]),
    "yamc_batch_destroy": (ctypes.c_int, [_VP]),
    "yamc_batch_replica": (ctypes.c_int, [_VP, ctypes.c_int32, _PPP]),
    "yamc_batch_run_device": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_int64, _VP, _VP, _VP]),
    "yamc_batch_run": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_int64, _VP, _VP, _VP]),
    "yamc_batch_tune": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_int64, _dp]),  # pointer arrays as void*
    "yamc_batch_set_launch": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32]),
    "yamc_batch_set_kspace_layout": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "yamc_batch_get_launch": (ctypes.c_int, [_VP, _ip]),
    "yamc_batch_groups": (ctypes.c_int, [_VP, _ip]),
    "yamc_batch_group_launch": (ctypes.c_int, [_VP, ctypes.c_int32, _ip]),
    "yamc_batch_last_kernel_ms": (ctypes.c_int, [_VP, _dp]),
    "yamc_batch_last_launches": (ctypes.c_int, [_VP, _ip]),
    "yamc_realspace_sums_static": (ctypes.c_int, [ctypes.POINTER(YamcParams), ctypes.c_int32] + [_VP] * 7 +
                                   [ctypes.c_int32] + [_VP] * 8),
    "yamc_fma_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _dp]),
    "yamc_state_size": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "yamc_save_state": (ctypes.c_int, [_VP, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]),
    "yamc_load_state": (ctypes.c_int, [_VP, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "yamc_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "yamc_last_error_detail": (ctypes.c_char_p, []),
}

_lib = None


class YamcError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = _lib
        msg = lib.yamc_error_string(status).decode() if lib else str(status)
        detail = lib.yamc_last_error_detail().decode() if lib else ""
        super().__init__(f"{where}: {msg} ({status}){': ' + detail if detail else ''}")
        self.status = status


def load(path: str = LIB_PATH):
    """Load the library (building it first if it is missing or stale)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            from . import build as _build
            _build.build()
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, where: str) -> int:
    if status != YAMC_OK:
        raise YamcError(status, where)
    return status


def declared_symbols(header: str = os.path.join(HERE, "..", "include", "yamc.h")):
    """Names of the functions declared in the public header."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yamc_[a-z_0-9]+)\s*\(", text)))

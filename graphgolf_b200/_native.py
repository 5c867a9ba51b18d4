"""Loading of the package's native libraries (ctypes, no torch types).

The CUDA library is the only compute path: if it is missing or cannot be
loaded, every entry point raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "_lib"

_lock = threading.Lock()
_libs: dict[str, C.CDLL] = {}


class NativeLibraryMissing(RuntimeError):
    """A native library of graphgolf_b200 is not built or cannot be loaded."""


class ggb_result(C.Structure):
    """Mirror of ``ggb_result`` in include/graphgolf_b200.h."""

    _fields_ = [
        ("connected", C.c_int),
        ("diameter", C.c_int),
        ("aspl", C.c_double),
        ("total", C.c_longlong),
        ("levels", C.c_longlong),
        ("windows", C.c_int),
        ("window_bits", C.c_int),
        ("dense_levels", C.c_longlong),
    ]


class ggb_partial(C.Structure):
    """Mirror of ``ggb_partial`` in include/graphgolf_b200.h."""

    _fields_ = [
        ("diam", C.c_int),
        ("disconnected", C.c_int),
        ("sum", C.c_longlong),
        ("levels", C.c_longlong),
        ("windows", C.c_int),
        ("window_bits", C.c_int),
        ("dense_levels", C.c_longlong),
    ]


class ggb_sa_stats(C.Structure):
    """Mirror of ``ggb_sa_stats`` in include/graphgolf_b200.h."""

    _fields_ = [
        ("step", C.c_longlong),
        ("accepts", C.c_longlong),
        ("multi_accepts", C.c_longlong),
        ("moved_swaps", C.c_longlong),
        ("evals", C.c_longlong),
        ("pred_accepts", C.c_longlong),
        ("unevaluated", C.c_longlong),
        ("cur_diam", C.c_int),
        ("best_diam", C.c_int),
        ("cur_total", C.c_longlong),
        ("best_total", C.c_longlong),
        ("cur_aspl", C.c_double),
        ("best_aspl", C.c_double),
        ("temp", C.c_double),
        ("done", C.c_int),
        ("delta", C.c_int),
    ]


_I = C.c_int
_LL = C.c_longlong
_P = C.c_void_p
_IP = C.POINTER(C.c_int)

CORE_SIGNATURES = {
    "ggb_init": (_I, [_I, _I, _I]),
    "ggb_finalize": (None, []),
    "ggb_last_error": (C.c_char_p, []),
    "ggb_version": (C.c_char_p, []),
    "ggb_device_count": (_I, []),
    "ggb_set_tuning": (_I, [_I, _I]),
    "ggb_set_ball": (_I, [_I]),
    "ggb_set_barrier_test": (_I, [_LL, _I]),
    "ggb_eval_general": (_I, [_I, _I, _I, _I, _P, _I, C.POINTER(ggb_result)]),
    "ggb_eval_grid": (_I, [_I, _I, _I, _P, _I, _P, C.POINTER(ggb_result)]),
    "ggb_eval_general_nonregular": (_I, [_I, _I, _I, _I, _P, _P, _I, C.POINTER(ggb_result)]),
    "ggb_eval_grid_nonregular": (_I, [_I, _I, _P, _I, _P, _I, _P, C.POINTER(ggb_result)]),
    "ggb_eval_general_device": (_I, [_I, _I, _I, _I, _P, _I, _P, C.POINTER(ggb_result)]),
    "ggb_launch_general_device": (_I, [_I, _I, _I, _I, _P, _I, _P]),
    "ggb_collect": (_I, [_P, C.POINTER(ggb_result)]),
    "ggb_launch_general_partial_device": (_I, [_I, _I, _I, _I, _P, _I, _I, _I, _P]),
    "ggb_collect_partial": (_I, [_P, C.POINTER(ggb_partial)]),
    "ggb_kernel_launches": (_LL, []),
    "ggb_h2d_bytes": (_LL, []),
    "ggb_trace_enable": (_I, [_I]),
    "ggb_set_timing": (_I, [_I]),
    "ggb_kernel_times": (_I, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ggb_probe_l2_gather": (_I, [_I, _I, _I, _I, C.POINTER(C.c_double)]),
    "ggb_probe_l2_stream": (_I, [_I, _I, C.POINTER(C.c_double)]),
    "ggb_trace_read": (_I, [_P, _I]),
    "ggb_eval_general_partial": (_I, [_I, _I, _I, _I, _P, _I, _I, _I, C.POINTER(ggb_partial)]),
    "ggb_finish_general": (_I, [_I, C.POINTER(ggb_partial), C.POINTER(ggb_result)]),
    "ggb_finish_grid": (_I, [_I, C.POINTER(ggb_partial), C.POINTER(ggb_result)]),
    "ggb_eval_general_noalloc": (_I, [_I, _I, _I, _I, _P, _I, _P, C.POINTER(ggb_result)]),
    "ggb_noalloc_scratch_bytes": (_LL, []),
    "ggb_noalloc_last_error": (C.c_char_p, []),
    "ggb_batch_create": (_I, [_I, _P, _P, _P, _P, C.POINTER(_P)]),
    "ggb_batch_destroy": (None, [_P]),
    "ggb_batch_set_plan": (_I, [_P, _I, _I]),
    "ggb_batch_get_plan": (_I, [_P, _IP, _IP, _IP]),
    "ggb_batch_autotune": (_I, [_P, _I, _IP, _IP, C.POINTER(C.c_double)]),
    "ggb_batch_adj_device": (_I, [_P, _I, C.POINTER(_P)]),
    "ggb_batch_upload": (_I, [_P, _P, _P]),
    "ggb_batch_launch": (_I, [_P, _P]),
    "ggb_batch_collect": (_I, [_P, _P, _P]),
    "ggb_batch_eval": (_I, [_P, _P, _P]),
    "ggb_batch_kernel_ms": (_I, [_P, C.POINTER(C.c_double)]),
    "ggb_mlp_create": (_I, [_I, C.c_ulonglong, C.POINTER(_P)]),
    "ggb_mlp_destroy": (None, [_P]),
    "ggb_mlp_param_count": (_I, []),
    "ggb_mlp_set_params": (_I, [_P, _P]),
    "ggb_mlp_get_params": (_I, [_P, _P]),
    "ggb_mlp_set_adam": (_I, [_P, C.c_float, C.c_float, C.c_float, C.c_float]),
    "ggb_mlp_forward_host": (_I, [_P, _P, _I, _P]),
    "ggb_mlp_time_forward": (_I, [_P, _P, _I, _I, C.POINTER(C.c_double)]),
    "ggb_mlp_grads_host": (_I, [_P, _P, _P, _I, _P, _P]),
    "ggb_mlp_train_host": (_I, [_P, _P, _P, _I, _I, _P]),
    "ggb_sa_create": (_I, [_I, _I, _P, _I, _I, _I, C.c_ulonglong, C.POINTER(_P)]),
    "ggb_sa_create_symmetric": (_I, [_I, _I, _I, _P, _I, _I, C.c_ulonglong, C.POINTER(_P)]),
    "ggb_sa_set_grid": (_I, [_P, _I, _I]),
    "ggb_sa_destroy": (None, [_P]),
    "ggb_sa_set_schedule": (_I, [_P, C.c_double, C.c_double, _I]),
    "ggb_sa_set_target": (_I, [_P, _I, _LL]),
    "ggb_sa_set_predicted": (_I, [_P, _I, _I]),
    "ggb_sa_autotune": (_I, [_P, _I, _IP, _IP, C.POINTER(C.c_double)]),
    "ggb_sa_run": (_I, [_P, _LL, C.POINTER(ggb_sa_stats)]),
    "ggb_sa_edges": (_I, [_P, _I, _P]),
    "ggb_sa_profile": (_I, [_P, _P]),
    "ggb_sa_base_plan": (_I, [_P, _IP, _IP]),
    "ggb_sa_checkpoint_bytes": (_LL, [_P]),
    "ggb_sa_save": (_I, [_P, _P, _LL]),
    "ggb_sa_restore": (_I, [_P, _P, _LL]),
    "ggb_sa_checkpoint_info": (_I, [_P, _LL, _IP, _IP, _IP, _IP]),
    "ggb_sa_checkpoint_edges": (_I, [_P, _LL, _I, _P]),
    "ggb_sa_last_step": (_I, [_P, _P, _P]),
    "ggb_sa_check_delta": (_I, [_P, _IP, _IP, _IP, _IP]),
}

HOST_SIGNATURES = {
    "ggbh_random_regular": (_I, [_I, _I, C.c_uint64, _P]),
    "ggbh_symmetric_regular": (_I, [_I, _I, _I, C.c_uint64, _P]),
    "ggbh_grid_regular": (_I, [_I, _I, _I, _I, _LL, C.c_uint64, _P]),
    "ggbh_create_adj": (_I, [_I, _I, _I, _P, _P]),
    "ggbh_rotate_hash": (_I, [_I, _I, _I, _I, _P]),
    "ggbh_count_lines": (_LL, [C.c_char_p]),
    "ggbh_read_general": (_LL, [C.c_char_p, _P, _LL]),
    "ggbh_write_general": (_I, [C.c_char_p, _LL, _P]),
    "ggbh_read_grid": (_LL, [C.c_char_p, _P, _LL, _IP, _IP]),
    "ggbh_write_grid": (_I, [C.c_char_p, _LL, _P, _I]),
    "ggbh_verify": (_I, [_I, _LL, _I, _P, _I, _I]),
}

LIB_FILES = {
    "core": "libgraphgolf_b200.so",
    "general": "libgg_general.so",
    "grid": "libgg_grid.so",
    "general_nr": "libgg_general_nr.so",
    "grid_nr": "libgg_grid_nr.so",
    "host": "libggb_host.so",
}


def _bind(lib: C.CDLL, sigs: dict) -> None:
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def load(which: str = "core") -> C.CDLL:
    """Returns the loaded library ``which`` (core/general/grid/host)."""
    with _lock:
        if which in _libs:
            return _libs[which]
        path = LIB_DIR / LIB_FILES[which]
        if not path.exists():
            raise NativeLibraryMissing(
                f"{path} is not built; run `python -m graphgolf_b200.build` (needs nvcc for sm_100a)")
        try:
            lib = C.CDLL(str(path), mode=C.RTLD_GLOBAL if which == "core" else C.RTLD_LOCAL)
        except OSError as e:
            raise NativeLibraryMissing(f"cannot load {path}: {e}") from e
        if which == "core":
            _bind(lib, CORE_SIGNATURES)
        elif which == "host":
            _bind(lib, HOST_SIGNATURES)
        _libs[which] = lib
        return lib


def last_error() -> str:
    return load("core").ggb_last_error().decode(errors="replace")

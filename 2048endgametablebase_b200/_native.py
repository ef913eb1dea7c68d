"""ctypes binding of libegtb_gpu.so (the C ABI declared in include/egtb_gpu.h).

The shared library is built in-tree by build_lib.py into _lib/. Loading fails
loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# EGTB_LIB_PATH: load another build of the library (a build kept beside this one)
LIB_PATH = os.environ.get("EGTB_LIB_PATH") or os.path.join(HERE, "_lib", "libegtb_gpu.so")

EGTB_OK = 0
ERR_NAMES = {
    -1: "EGTB_ERR_ARG",
    -2: "EGTB_ERR_CUDA",
    -3: "EGTB_ERR_NOMEM",
    -4: "EGTB_ERR_IO",
    -5: "EGTB_ERR_CAPACITY",
    -6: "EGTB_ERR_TIMEOUT",
    -7: "EGTB_ERR_UNSUPPORTED",
}
MAX_MASKS = 32
MAX_PATH = 4096

DTYPE_CODES = {"uint32": 0, "uint64": 1, "float32": 2, "float64": 3, "1-float32": 4, "1-float64": 5}


class NativeError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class PatternSpecC(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 64),
        ("pattern_masks", ctypes.c_uint64 * MAX_MASKS),
        ("n_masks", ctypes.c_int32),
        ("success_shifts", ctypes.c_uint8 * 16),
        ("n_shifts", ctypes.c_int32),
        ("symm_mode", ctypes.c_int32),
    ]


class RunOptionsC(ctypes.Structure):
    _fields_ = [
        ("target", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("docheck_step", ctypes.c_int32),
        ("pathname", ctypes.c_char * MAX_PATH),
        ("is_free", ctypes.c_int32),
        ("is_variant", ctypes.c_int32),
        ("spawn_rate4", ctypes.c_double),
        ("success_rate_dtype", ctypes.c_int32),
        ("deletion_threshold", ctypes.c_double),
        ("compress", ctypes.c_int32),
        ("compress_temp_files", ctypes.c_int32),
        ("optimal_branch_only", ctypes.c_int32),
        ("chunked_solve", ctypes.c_int32),
        ("num_threads", ctypes.c_int32),
        ("direct_io", ctypes.c_int32),
        ("direct_io_queue_depth", ctypes.c_int32),
        ("direct_io_chunk_mib", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("write_files", ctypes.c_int32),
    ]


class BuildStatsC(ctypes.Structure):
    _fields_ = [
        ("raw_boards", ctypes.c_uint64),
        ("book_entries", ctypes.c_uint64),
        ("max_layer", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("lookups", ctypes.c_uint64),
        ("layers", ctypes.c_int32),
        ("retries", ctypes.c_int32),
        ("forward_ms", ctypes.c_double),
        ("backward_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class KernelTimeC(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


class BatchParamsC(ctypes.Structure):
    _fields_ = [
        ("expand_chunk", ctypes.c_int32),
        ("expand_blocks_per_sm", ctypes.c_int32),
        ("digit_nibbles", ctypes.c_int32),
        ("index_load", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class BatchStatsC(ctypes.Structure):
    _fields_ = [
        ("raw_boards", ctypes.c_uint64),
        ("book_entries", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("lookups", ctypes.c_uint64),
        ("tables", ctypes.c_int32),
        ("max_steps", ctypes.c_int32),
        ("retries", ctypes.c_int32),
        ("graphs_used", ctypes.c_int32),
        ("forward_ms", ctypes.c_double),
        ("sort_ms", ctypes.c_double),
        ("backward_ms", ctypes.c_double),
        ("pack_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("graph_launches", ctypes.c_uint64),
        ("params", BatchParamsC),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "params"}
        d["params"] = self.params.as_dict()
        return d


class AdParamC(ctypes.Structure):
    """egtb_ad_param (AdvancedMaskParam)."""
    _fields_ = [
        ("pos_fixed_32k_mask", ctypes.c_uint64),
        ("small_tile_sum_limit", ctypes.c_uint32),
        ("target", ctypes.c_uint32),
        ("num_free_32k", ctypes.c_uint32),
        ("num_fixed_32k", ctypes.c_uint32),
    ]


class AdTileCountC(ctypes.Structure):
    """egtb_ad_tile_count (TileCountResult / TileCount4Result)."""
    _fields_ = [
        ("pos_bitmap", ctypes.c_uint64),
        ("total_sum", ctypes.c_uint32),
        ("count_32k", ctypes.c_int32),
        ("pos_rank", ctypes.c_uint32),
        ("merged_tile_found", ctypes.c_uint32),
        ("merged_tile", ctypes.c_uint32),
        ("is_success", ctypes.c_uint32),
    ]


# every entry point of include/egtb_gpu.h with its ctypes signature
_P = ctypes.c_void_p
_SIGS = {
    "egtb_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "egtb_version": (ctypes.c_char_p, []),
    "egtb_device_count": (ctypes.c_int, []),
    "egtb_set_stream": (ctypes.c_int, [ctypes.c_int, _P]),
    "egtb_profile": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "egtb_profile_read": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(KernelTimeC), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int)]),
    "egtb_set_spin_limit": (ctypes.c_int, [ctypes.c_uint32]),
    "egtb_release": (ctypes.c_int, [ctypes.c_int32]),
    "egtb_get_build_progress": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "egtb_reset_build_progress": (ctypes.c_int, [ctypes.c_uint32]),
    "egtb_build": (ctypes.c_int, [_P, ctypes.c_size_t, ctypes.POINTER(PatternSpecC), ctypes.POINTER(RunOptionsC),
                                  ctypes.POINTER(BuildStatsC)]),
    "egtb_generate": (ctypes.c_int, [_P, ctypes.c_size_t, ctypes.POINTER(PatternSpecC), ctypes.POINTER(RunOptionsC),
                                     ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(BuildStatsC)]),
    "egtb_solve": (ctypes.c_int, [_P, ctypes.c_size_t, _P, ctypes.c_size_t, ctypes.POINTER(PatternSpecC),
                                  ctypes.POINTER(RunOptionsC), ctypes.POINTER(BuildStatsC)]),
    "egtb_sort_unique_u64": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P, _P, _P]),
    "egtb_sort_unique_u64_noalloc": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P, _P, _P]),
    "egtb_book_layer_copy": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, _P, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_uint64)]),
    "egtb_move_all_dir": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P]),
    "egtb_move_all_dir_variant": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P]),
    "egtb_canonical": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, ctypes.c_int32, _P]),
    "egtb_apply_sym": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, ctypes.c_int32, _P]),
    "egtb_ad_move_all_dir": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P, _P]),
    "egtb_ad_mask_board": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, ctypes.c_int32, _P]),
    "egtb_ad_tile_stats": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, ctypes.POINTER(AdParamC), ctypes.c_int32,
                                          _P]),
    "egtb_ad_validate": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P, ctypes.POINTER(AdParamC), _P]),
    "egtb_ad_unmask": (ctypes.c_int, [ctypes.c_int, _P, ctypes.c_size_t, _P, ctypes.POINTER(AdParamC), _P, _P,
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]),
    "egtb_ad_row_tables": (ctypes.c_int, [_P, _P]),
    "egtb_ad_tiles_combinations": (ctypes.c_int, [_P, _P]),
    "egtb_book_open": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(PatternSpecC),
                                      ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(_P)]),
    "egtb_book_close": (ctypes.c_int, [_P]),
    "egtb_book_set_variant": (ctypes.c_int, [_P, ctypes.c_int32]),
    "egtb_book_load_all": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "egtb_book_lookup": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.c_int32, _P, _P, _P]),
    "egtb_book_lookup_device": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.c_int32, _P, _P, _P]),
    "egtb_find_classic_value": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int32,
                                               ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_int32)]),
    "egtb_build_batch": (ctypes.c_int, [ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P]),
    "egtb_batch_autotune": (ctypes.c_int, [ctypes.c_int32, _P, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "egtb_batch_book_copy": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "egtb_serve_start": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32,
                                        ctypes.POINTER(_P)]),
    "egtb_serve_submit": (ctypes.c_int, [_P, ctypes.c_int32, _P, ctypes.c_uint64, _P, _P,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "egtb_serve_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "egtb_serve_register": (ctypes.c_int, [_P, _P, ctypes.c_uint64]),
    "egtb_serve_unregister": (ctypes.c_int, [_P, _P]),
    "egtb_serve_stats": (ctypes.c_int, [_P] + [ctypes.POINTER(ctypes.c_uint64)] * 4),
    "egtb_serve_replay": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, ctypes.c_uint64, _P, _P, _P,
                                         ctypes.POINTER(ctypes.c_double)]),
    "egtb_serve_stop": (ctypes.c_int, [_P]),
}

_lib = None


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libegtb_gpu.so is not built ({LIB_PATH}); run __graft_entry__.build() or "
                "python 2048endgametablebase_b200/build_lib.py"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib().egtb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != EGTB_OK:
        raise NativeError(rc, f"{ERR_NAMES.get(rc, rc)}: {last_error()}")


def profile(device: int, enable: bool) -> None:
    check(lib().egtb_profile(int(device), int(bool(enable))))


def profile_read(device: int) -> dict[str, tuple[int, float]]:
    arr = (KernelTimeC * 16)()
    n = ctypes.c_int(0)
    check(lib().egtb_profile_read(int(device), arr, 16, ctypes.byref(n)))
    return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(n.value)}


def release(device: int = 0) -> None:
    """Free the buffers the library keeps on a device between builds (egtb_release)."""
    check(lib().egtb_release(int(device)))


def set_stream(device: int, stream_ptr: int | None) -> None:
    check(lib().egtb_set_stream(int(device), ctypes.c_void_p(stream_ptr or None)))


def device_count() -> int:
    return int(lib().egtb_device_count())

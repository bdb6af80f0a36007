"""ctypes bindings of libgicops_b200.so (the C ABI of include/gicops_b200.h).

The library is loaded from the package tree (gicops_b200/_lib); there is no
fallback: a missing or stale library raises.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libgicops_b200.so")

HIST_BINS = 802
MAX_HEAP = 31
MAX_LENGTHS = 64
MAX_PEAKS = 1024
NOALLOC_MAX_WINDOWS = 1 << 19

SUCCESS = 0
STATUS_NAMES = {
    0: "SUCCESS", -3001: "ERR_INVLD_MEMORY", -3002: "ERR_INVLD_PARAM", -3003: "ERR_INVLD_INDEX",
    -3004: "ERR_INVLD_SIZE", -3007: "ERR_BAD_MEM_ALLOC", -3008: "ERR_INVLD_PTR", -3010: "ERR_INVLD_MOD",
    -3012: "ERR_NOT_ENOUGH_DATA", -3050: "ERR_CUDA", -3051: "ERR_DEVICE_GUARD",
}

FLAG_WIDE_SCORECARD = 1
FLAG_PLAIN = 2
STATUS_LEARNED_TAIL = 16
STATUS_PEAK_LIMIT = 32

TAIL_WINDOW = 128
TAIL_IN = 132
TAIL_HIDDEN = 256
TAIL_OUT = 2
TAIL_NPARAM = TAIL_HIDDEN * TAIL_IN + TAIL_HIDDEN + TAIL_HIDDEN * TAIL_HIDDEN + TAIL_HIDDEN + TAIL_OUT * TAIL_HIDDEN \
    + TAIL_OUT
TAIL_MAX_KEEP = 512
TAIL_SAMPLE_DTYPE = np.dtype([("query", "<u4"), ("keep", "<u4"), ("seed", "<u8")])

CELL_DTYPE = np.dtype([("hyperscore", "<f4"), ("psid", "<i4"), ("idxoffset", "<u2"),
                       ("sharedions", "<u2"), ("totalions", "<u2"), ("pad", "<u2")])
RESULT_DTYPE = np.dtype([
    ("cpsms", "<i4"), ("status", "<i4"), ("top", CELL_DTYPE), ("maxhyp", "<i4"),
    ("mu", "<i4"), ("beta", "<i4"), ("stt1", "<i4"), ("end1", "<i4"), ("pad", "<i4"),
    ("slope", "<f8"), ("icpt", "<f8"), ("e_x", "<f8"), ("e_fp64", "<f8"),
])
PEP_ENTRY_DTYPE = np.dtype([("mass", "<f4"), ("seqid", "<u4"), ("sites", "<u8"), ("modnum", "<u4"), ("pad", "<u4")])


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("launches", C.c_uint64), ("total_ms", C.c_double)]


def kernel_times() -> dict:
    """{kernel name: (launches, total ms)} recorded since profiling was enabled."""
    arr = (KernelTime * 64)()
    n = lib().gx_profile_read(arr, 64)
    return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(min(n, 64))}


class GxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class LengthDesc(C.Structure):
    _fields_ = [("peplen", C.c_uint32), ("npep", C.c_uint32), ("speclen", C.c_uint32), ("pad", C.c_uint32),
                ("mass", C.c_void_p), ("bA", C.c_void_p), ("iA", C.c_void_p)]


class Ms2Raw(C.Structure):
    _fields_ = [("nspec", C.c_uint32), ("nvalues", C.c_uint32), ("seg", C.c_void_p), ("size", C.c_void_p),
                ("mz", C.c_void_p), ("intn", C.c_void_p), ("prec", C.c_void_p), ("charge", C.c_void_p),
                ("rtime", C.c_void_p)]


class Mod(C.Structure):
    _fields_ = [("residues", C.c_char * 4), ("mass", C.c_double), ("max_per_pep", C.c_uint32)]


class BuildParams(C.Structure):
    _fields_ = [("maxz", C.c_uint32), ("scale", C.c_uint32), ("min_mass", C.c_uint32), ("max_mass", C.c_uint32),
                ("nmods", C.c_uint32), ("mods_per_pep", C.c_uint32), ("mods", C.POINTER(Mod)),
                ("threads", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("dM", C.c_double), ("dF", C.c_uint32), ("scale", C.c_uint32), ("max_mass", C.c_double),
                ("min_shp", C.c_uint32), ("min_cpsm", C.c_uint32), ("topmatches", C.c_uint32),
                ("flags", C.c_uint32), ("expect_max", C.c_double)]


class Queries(C.Structure):
    _fields_ = [("nspec", C.c_uint32), ("npeaks", C.c_uint32), ("idx", C.c_void_p), ("moz", C.c_void_p),
                ("intn", C.c_void_p), ("prec", C.c_void_p), ("charge", C.c_void_p), ("dM", C.c_void_p)]


class StreamStats(C.Structure):
    _fields_ = [("chunks", C.c_uint32), ("pad", C.c_uint32), ("total_ms", C.c_double), ("upload_ms", C.c_double),
                ("search_ms", C.c_double), ("download_ms", C.c_double)]


class Tiles(C.Structure):
    _fields_ = [("chunks_per_lane", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("tile", C.c_uint32),
                ("sorted", C.c_uint32), ("pipeline", C.c_uint32)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


TUNE_MAX = 32


class TuneResult(C.Structure):
    _fields_ = [("best", Tiles), ("ncand", C.c_uint32), ("cached", C.c_uint32), ("cand", Tiles * TUNE_MAX),
                ("ms", C.c_float * TUNE_MAX)]


class TailAdam(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("w_slope", C.c_float), ("w_lgs", C.c_float)]


_lib = None

# (name, restype, argtypes) of every exported entry point
_SIGS = [
    ("gx_index_upload", C.c_int32, [C.POINTER(LengthDesc), C.c_int32, C.c_uint32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("gx_index_free", C.c_int32, [C.c_void_p]),
    ("gx_index_bytes", C.c_uint64, [C.c_void_p]),
    ("gx_index_save", C.c_int32, [C.c_void_p, C.c_char_p]),
    ("gx_index_load", C.c_int32, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    ("gx_build_length", C.c_int32, [C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(BuildParams),
                                    C.POINTER(C.c_void_p)]),
    ("gx_host_length_desc", C.c_int32, [C.c_void_p, C.POINTER(LengthDesc)]),
    ("gx_host_length_entries", C.c_void_p, [C.c_void_p]),
    ("gx_host_length_seqs", C.c_void_p, [C.c_void_p, C.POINTER(C.c_uint32)]),
    ("gx_host_length_free", None, [C.c_void_p]),
    ("gx_build_length_entries", C.c_int32, [C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(BuildParams),
                                            C.POINTER(C.c_void_p)]),
    ("gx_index_build", C.c_int32, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(BuildParams), C.c_int32,
                                   C.POINTER(C.c_void_p)]),
    ("gx_index_read_length", C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gx_merge_shards_device", C.c_int32, [C.c_uint32, C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.POINTER(Params), C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    ("gx_ms2_read", C.c_int32, [C.c_char_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("gx_ms2_desc", C.c_int32, [C.c_void_p, C.POINTER(Ms2Raw)]),
    ("gx_ms2_free", None, [C.c_void_p]),
    ("gx_pickpeaks_device", C.c_int32, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                        C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gx_workspace_create", C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("gx_workspace_free", C.c_int32, [C.c_void_p]),
    ("gx_workspace_set_graph", C.c_int32, [C.c_void_p, C.c_int32]),
    ("gx_workspace_get_tiles", C.c_int32, [C.c_void_p, C.POINTER(Tiles)]),
    ("gx_workspace_set_tiles", C.c_int32, [C.c_void_p, C.POINTER(Tiles)]),
    ("gx_autotune", C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(Queries), C.POINTER(Params), C.c_uint32,
                                C.c_uint32, C.POINTER(TuneResult), C.c_void_p]),
    ("gx_search_host", C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(Queries), C.POINTER(Params), C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    ("gx_search_device", C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(Queries), C.POINTER(Params), C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gx_search_device_noalloc", C.c_int32, [C.c_void_p, C.POINTER(Queries), C.POINTER(Params), C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gx_streamer_create", C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("gx_streamer_free", C.c_int32, [C.c_void_p]),
    ("gx_streamer_workspace", C.c_void_p, [C.c_void_p]),
    ("gx_search_stream", C.c_int32, [C.c_void_p, C.POINTER(Queries), C.POINTER(Params), C.c_void_p,
                                     C.POINTER(StreamStats)]),
    ("gx_traffic_host", C.c_int32, [C.POINTER(LengthDesc), C.c_int32, C.POINTER(Queries), C.POINTER(Params),
                                    C.c_void_p, C.c_void_p, C.c_int32]),
    ("gx_heap_capacity", C.c_int32, [C.c_uint32]),
    ("gx_lgfact", None, [C.c_void_p]),
    ("gx_profile_enable", C.c_int32, [C.c_int32]),
    ("gx_profile_read", C.c_int32, [C.c_void_p, C.c_int32]),
    ("gx_tail_model_create", C.c_int32, [C.c_int32, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("gx_tail_model_free", C.c_int32, [C.c_void_p]),
    ("gx_tail_model_set", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("gx_tail_model_get", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    ("gx_tail_features", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                     C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    ("gx_tail_fit_rows", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("gx_tail_grad", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    ("gx_tail_train_step", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(TailAdam),
                                       C.c_void_p, C.c_void_p]),
    ("gx_tail_predict", C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("gx_tail_apply", C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                  C.c_uint32, C.c_double, C.c_void_p]),
    ("gx_tail_check", C.c_int32, [C.c_void_p]),
    ("gx_tail_set_wait_limit", C.c_int32, [C.c_uint64]),
    ("gx_tail_set_loss", C.c_int32, [C.c_void_p, C.c_float]),
    ("gx_workspace_set_tail", C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32]),
    ("gx_tail_gemm", C.c_int32, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_int32,
                                 C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p]),
    ("gx_last_error", C.c_char_p, []),
    ("gx_launch_count", C.c_uint64, []),
]

EXPORTED = [n for n, _, _ in _SIGS]


def lib():
    """The loaded library (built on demand if the sources are newer)."""
    global _lib
    if _lib is None:
        from . import build as _build
        if not _build.up_to_date():
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libgicops_b200.so not found at {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        assert C.sizeof(Params) == 48 and RESULT_DTYPE.itemsize == 80 and CELL_DTYPE.itemsize == 16
        assert TAIL_SAMPLE_DTYPE.itemsize == 16 and C.sizeof(TailAdam) == 24
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != SUCCESS:
        msg = lib().gx_last_error()
        raise GxError(code, msg.decode() if msg else "")


def ptr(a) -> int | None:
    return None if a is None else a.ctypes.data

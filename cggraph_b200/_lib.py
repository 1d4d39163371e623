"""ctypes binding of libcgb200.so (include/cgb200.h, include/cgb200_gen.h).

The library is the only compute path: importing this module does not build
anything, and every call fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcgb200.so")

VALUE_MAX = 999999999

# cgb_status
OK, EINVAL, EFORMAT, EIO, ENOMEM, ECUDA, ETIMEOUT, EOVERFLOW, EUNSUPPORTED = range(9)
STATUS_NAMES = ["CGB_OK", "CGB_EINVAL", "CGB_EFORMAT", "CGB_EIO", "CGB_ENOMEM", "CGB_ECUDA", "CGB_ETIMEOUT",
                "CGB_EOVERFLOW", "CGB_EUNSUPPORTED"]

# cgb_schedule / cgb_variant / flags / kernel classes
SCHED_HEURISTIC, SCHED_LEARNED, SCHED_FIXED = 0, 1, 2
VAR_AUTO, VAR_TWC, VAR_PULL, VAR_PUSH, VAR_DENSE = 0, 1, 2, 3, 4
FLAG_KERNEL_TIMING, FLAG_TRACE, FLAG_BATCH_SEQUENTIAL, FLAG_CC_WEAK = 0x1, 0x2, 0x4, 0x8
K_PUSH, K_PULL, K_PR, K_HOOK, K_COMPRESS, K_FRONTIER, K_INIT, K_OTHER = range(8)
KERNEL_CLASS_NAMES = ["push", "pull", "pagerank", "hook", "compress", "frontier", "init", "other"]

# Exported symbols, exactly as declared in include/*.h.
EXPORTS = [
    "cgb_graph_create", "cgb_graph_load_files", "cgb_graph_create_from_edges", "cgb_graph_load_edge_file", "cgb_graph_reorder", "cgb_graph_partition", "cgb_graph_destroy", "cgb_graph_set_stream", "cgb_graph_set_weights", "cgb_graph_info", "cgb_graph_device_csr",
    "cgb_graph_result_device", "cgb_graph_result_download", "cgb_run", "cgb_run_batch", "cgb_run_stats_get", "cgb_trace_get",
    "cgb_last_error_string", "cgb_status_string", "cgb_abi_version", "cgb_gen_rmat", "cgb_gen_grid", "cgb_gen_chunglu",
    "cgb_graph_download", "cgb_bfs_noalloc", "cgb_policy_load", "cgb_policy_collect", "cgb_policy_train",
    "cgb_policy_forward", "cgb_policy_loss_grad", "cgb_batch_create", "cgb_batch_destroy", "cgb_batch_run",
    "cgb_batch_info", "cgb_batch_stats", "cgb_server_create", "cgb_server_submit", "cgb_server_start",
    "cgb_server_wait", "cgb_server_poll", "cgb_server_stats", "cgb_server_destroy", "cgb_tuning_get",
    "cgb_tuning_set", "cgb_autotune", "cgb_memory_trim", "cgb_memory_info", "cgb_memory_reserve",
    "cgb_check_barrier_timeout",
]
POLICY_FEATURES, POLICY_OUTPUTS, POLICY_PARAMS = 24, 14, 6670


class Options(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("schedule", ctypes.c_int32),
        ("variant", ctypes.c_int32),
        ("sssp_delta", ctypes.c_uint32),
        ("bfs_alpha", ctypes.c_double),
        ("bfs_beta", ctypes.c_double),
        ("max_iterations", ctypes.c_uint64),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 7),
    ]


class RunStats(ctypes.Structure):
    _fields_ = [
        ("ms", ctypes.c_double),
        ("iterations", ctypes.c_uint64),
        ("traversed_edges", ctypes.c_uint64),
        ("reached", ctypes.c_uint64),
        ("alg_bytes", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double * 8),
        ("kernel_launches", ctypes.c_uint64 * 8),
        ("pushes_td", ctypes.c_uint64),
        ("pulls_bu", ctypes.c_uint64),
        ("sssp_delta", ctypes.c_uint32),
        ("cc_path", ctypes.c_int32),
        ("launches", ctypes.c_uint64),
    ]


class IterTrace(ctypes.Structure):
    _fields_ = [
        ("iteration", ctypes.c_uint32),
        ("algorithm", ctypes.c_uint32),
        ("frontier_vertices", ctypes.c_uint64),
        ("frontier_edges", ctypes.c_uint64),
        ("unvisited_vertices", ctypes.c_uint64),
        ("unvisited_edges", ctypes.c_uint64),
        ("max_frontier_degree", ctypes.c_uint32),
        ("variant", ctypes.c_int32),
        ("delta", ctypes.c_uint32),
        ("ms", ctypes.c_float),
    ]


class CgbError(RuntimeError):
    def __init__(self, status: int, message: str):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {message}")
        self.status = status
        self.message = message


_lib = None

class PartitionInfo(ctypes.Structure):
    """cgb_partition_info (include/cgb200.h)."""
    _fields_ = [
        ("segment_num", ctypes.c_uint32),
        ("bucket_start", ctypes.c_uint32 * 5),
        ("can_hold_all", ctypes.c_int32),
        ("reached_bucket", ctypes.c_uint32),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("push_big_deg", ctypes.c_uint32),
        ("push_chunk", ctypes.c_uint32),
        ("push_ctas_per_sm", ctypes.c_uint32),
        ("persist_enter", ctypes.c_uint32),
        ("persist_deg", ctypes.c_uint32),
        ("ms_edges", ctypes.c_uint32),
        ("pr_unroll", ctypes.c_uint32),
        ("pr_ctas_per_sm", ctypes.c_uint32),
        ("persist_ctas", ctypes.c_uint32),
        ("sssp_pull_alpha", ctypes.c_uint32),
        ("cluster_enter", ctypes.c_uint32),
        ("sssp_dense_alpha", ctypes.c_uint32),
        ("push_block", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 2),
    ]


TUNE_BATCH, TUNE_KEEP_DEFAULT, TUNE_CC_WEAK = 0x1, 0x2, 0x4
TUNING_FIELDS = ("push_big_deg", "push_chunk", "push_ctas_per_sm", "persist_enter", "persist_deg", "ms_edges",
                 "pr_unroll", "pr_ctas_per_sm", "persist_ctas", "sssp_pull_alpha",
                 "cluster_enter", "sssp_dense_alpha", "push_block")


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("bfs_slots", ctypes.c_uint32),
        ("sssp_slots", ctypes.c_uint32),
        ("sssp_delta", ctypes.c_uint32),
        ("memory_budget", ctypes.c_uint64),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 5),
    ]


SERVER_NO_BFS, SERVER_NO_SSSP, SERVER_HOST_TICKS, SERVER_BATCH_ONLY, SERVER_ADMIT_ANY_SLOT = 0x1, 0x2, 0x4, 0x8, 0x10


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64),
        ("algorithm", ctypes.c_int32),
        ("root", ctypes.c_uint32),
        ("arrival_us", ctypes.c_double),
        ("admit_us", ctypes.c_double),
        ("done_us", ctypes.c_double),
        ("traversed_edges", ctypes.c_uint64),
        ("reached", ctypes.c_uint32),
        ("depth", ctypes.c_uint32),
        ("status", ctypes.c_int32),
        ("slot", ctypes.c_uint32),
    ]


_P = ctypes.c_void_p
_u32p = ctypes.POINTER(ctypes.c_uint32)


def lib() -> ctypes.CDLL:
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"cgb200 CUDA library missing at {LIB_PATH}; build it with "
                               "`python -m cggraph_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        i = ctypes.c_int
        u32 = ctypes.c_uint32
        L.cgb_graph_create.argtypes = [_P, _P, _P, u32, u32, u32, i, ctypes.POINTER(_P)]
        L.cgb_graph_load_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, u32, u32, i,
                                           ctypes.POINTER(_P)]
        L.cgb_graph_destroy.argtypes = [_P]
        L.cgb_graph_create_from_edges.argtypes = [_P, ctypes.c_uint64, u32, i, ctypes.POINTER(_P)]
        L.cgb_graph_load_edge_file.argtypes = [ctypes.c_char_p, u32, i, ctypes.POINTER(_P)]
        L.cgb_graph_reorder.argtypes = [_P, i, _P, _u32p, ctypes.POINTER(_P)]
        L.cgb_graph_partition.argtypes = [_P, i, ctypes.c_uint32, _P, _P, _P, _P, _P, ctypes.POINTER(PartitionInfo)]
        L.cgb_graph_set_stream.argtypes = [_P, _P]
        L.cgb_graph_set_weights.argtypes = [_P, _P]
        L.cgb_graph_info.argtypes = [_P, _u32p, _u32p, ctypes.POINTER(ctypes.c_int32)]
        L.cgb_graph_device_csr.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P)]
        L.cgb_graph_result_device.argtypes = [_P, ctypes.POINTER(_P)]
        L.cgb_graph_result_download.argtypes = [_P, _P]
        L.cgb_run.argtypes = [_P, i, u32, ctypes.POINTER(Options), _P, _P, ctypes.POINTER(ctypes.c_double)]
        L.cgb_run_batch.argtypes = [_P, i, _P, u32, ctypes.POINTER(Options), _P, ctypes.POINTER(ctypes.c_double)]
        L.cgb_run_stats_get.argtypes = [_P, ctypes.POINTER(RunStats)]
        L.cgb_trace_get.argtypes = [_P, ctypes.POINTER(IterTrace), u32, _u32p]
        L.cgb_last_error_string.restype = ctypes.c_char_p
        L.cgb_status_string.restype = ctypes.c_char_p
        L.cgb_status_string.argtypes = [i]
        L.cgb_abi_version.restype = i
        L.cgb_gen_rmat.argtypes = [u32, u32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   i, i, u32, i, ctypes.POINTER(_P)]
        L.cgb_gen_grid.argtypes = [u32, u32, ctypes.c_uint64, u32, i, ctypes.POINTER(_P)]
        L.cgb_gen_chunglu.argtypes = [u32, ctypes.c_uint64, u32, ctypes.c_uint64, i, u32, i, ctypes.POINTER(_P)]
        L.cgb_graph_download.argtypes = [_P, _P, _P, _P]
        L.cgb_bfs_noalloc.argtypes = [_P, _P, u32, u32, u32, _P, _P]
        L.cgb_policy_load.argtypes = [_P]
        L.cgb_policy_collect.argtypes = [_P, i, u32, ctypes.POINTER(Options), _P, _P, _P, u32, _u32p]
        L.cgb_policy_train.argtypes = [_P, _P, _P, u32, u32, u32, ctypes.c_float, ctypes.c_uint64, _P, _P,
                                       ctypes.POINTER(ctypes.c_float)]
        L.cgb_policy_forward.argtypes = [_P, _P, u32, _P]
        L.cgb_policy_loss_grad.argtypes = [_P, _P, _P, _P, u32, ctypes.POINTER(ctypes.c_float), _P]
        L.cgb_batch_create.argtypes = [u32, _P, _P, _P, _P, _P, i, ctypes.POINTER(_P)]
        L.cgb_batch_destroy.argtypes = [_P]
        L.cgb_batch_run.argtypes = [_P, i, _P, _P, ctypes.POINTER(ctypes.c_double)]
        L.cgb_batch_info.argtypes = [_P, _u32p, _u32p, ctypes.POINTER(ctypes.c_int32)]
        L.cgb_batch_stats.argtypes = [_P, ctypes.POINTER(RunStats)]
        L.cgb_server_create.argtypes = [_P, ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]
        L.cgb_server_submit.argtypes = [_P, i, u32, ctypes.c_double, _P, ctypes.POINTER(ctypes.c_uint64)]
        L.cgb_server_start.argtypes = [_P]
        L.cgb_server_wait.argtypes = [_P, ctypes.c_double, _u32p]
        L.cgb_server_poll.argtypes = [_P, ctypes.POINTER(RequestInfo), u32, _u32p]
        L.cgb_server_stats.argtypes = [_P, ctypes.POINTER(ctypes.c_uint64), _u32p, _u32p,
                                       ctypes.POINTER(ctypes.c_double)]
        L.cgb_server_destroy.argtypes = [_P]
        L.cgb_memory_trim.argtypes = [i]
        L.cgb_memory_info.argtypes = [i, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.cgb_memory_reserve.argtypes = [i, ctypes.c_uint64]
        L.cgb_tuning_get.argtypes = [_P, i, ctypes.POINTER(Tuning)]
        L.cgb_tuning_set.argtypes = [_P, i, ctypes.POINTER(Tuning)]
        L.cgb_autotune.argtypes = [_P, i, _P, u32, u32, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
        for name in EXPORTS:
            f = getattr(L, name)
            if name not in ("cgb_last_error_string", "cgb_status_string", "cgb_abi_version"):
                f.restype = ctypes.c_int
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        msg = lib().cgb_last_error_string()
        raise CgbError(status, msg.decode() if msg else "")

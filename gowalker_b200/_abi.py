"""ctypes binding of libgowalker.so (include/gowalker.h).

The library is built in-tree (gowalker_b200/libgowalker.so).  Loading fails
loudly when it is missing: there is no CPU fallback for the walk path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgowalker.so")

GW_OK = 0
GW_NODE2VEC, GW_SOPR, GW_SOSR = 0, 1, 2
GW_INIT_PER_VERTEX, GW_INIT_SINGLE_SOURCE, GW_INIT_RANDOM = 0, 1, 2
GW_POLICY_PLAIN, GW_POLICY_LEARNED, GW_POLICY_SA = 0, 1, 2
GW_PATHS_NONE, GW_PATHS_FULL = 0, 1
GW_EDGES_SYMMETRIC, GW_EDGES_SORT, GW_EDGES_DEDUP = 1, 2, 4
GW_SPLIT_REFERENCE, GW_SPLIT_EQUAL_EDGES = 0, 1
GW_LAUNCH_PERSISTENT, GW_LAUNCH_PER_HOP = 0, 1
GW_LEARNED_EVICT, GW_LEARNED_ZERO_SWITCH = 1, 2
GW_LEARNED_AUTO = 0

# Every symbol include/gowalker.h declares.
EXPORTS = (
    "gw_version", "gw_status_string", "gw_config_default", "gw_create", "gw_destroy", "gw_last_error",
    "gw_set_config", "gw_stream", "gw_set_graph_meta", "gw_host_block", "gw_device_graph", "gw_cache_reset",
    "gw_host_weights", "gw_device_weights",
    "gw_init_walkers", "gw_init_walker_range", "gw_run", "gw_num_walkers", "gw_get_paths", "gw_path_lengths", "gw_path_hashes", "gw_checksum",
    "gw_bucket_counts", "gw_rmat_csr", "gw_web_csr", "gw_edges_csr", "gw_split_blocks", "gw_sa_choose_blocks",
    "gw_plain_choose_block", "gw_device_free", "gw_memcpy", "gw_walk_noalloc", "gw_philox_rate",
    "gw_mlp_forward", "gw_mlp_grad", "gw_mlp_train", "gw_host_alloc", "gw_host_free",
)
GW_MLP_INPUTS = 16
GW_MLP_PARAMS = 5313
GW_MLP_GRAD_WS_FLOATS = 32 * (GW_MLP_PARAMS + 1)


class GwConfig(ctypes.Structure):
    _fields_ = [
        ("cache_size", ctypes.c_uint64),
        ("blocksize", ctypes.c_uint64),
        ("algorithm", ctypes.c_uint32),
        ("p", ctypes.c_float),
        ("q", ctypes.c_float),
        ("alpha", ctypes.c_float),
        ("maxhops", ctypes.c_uint32),
        ("walkpersource", ctypes.c_uint32),
        ("numwalks", ctypes.c_uint32),
        ("blockpergrid", ctypes.c_uint32),
        ("threadperblock", ctypes.c_uint32),
        ("zero_threshold", ctypes.c_uint32),
        ("zero_copy", ctypes.c_uint32),
        ("init_mode", ctypes.c_uint32),
        ("term_prob", ctypes.c_float),
        ("seed", ctypes.c_uint64),
        ("record_paths", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("strict_blocks", ctypes.c_uint32),
        ("prefetch", ctypes.c_uint32),
        ("compress_blocks", ctypes.c_uint32),
        ("learned_sync", ctypes.c_uint32),
        ("launch_mode", ctypes.c_uint32),
        ("learned_mode", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 2),
    ]


class GwStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_uint64),
        ("trials", ctypes.c_uint64),
        ("walkers", ctypes.c_uint64),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("block_loads", ctypes.c_uint64),
        ("zero_copy_steps", ctypes.c_uint64),
        ("iterations", ctypes.c_uint32),
        ("launches", ctypes.c_uint32),
        ("kernel_ms", ctypes.c_float),
        ("total_ms", ctypes.c_float),
        ("learned_iterations", ctypes.c_uint32),
        ("policy_reverted", ctypes.c_uint32),
        ("train_loss", ctypes.c_float),
        ("pred_error", ctypes.c_float),
        ("kernel_variant", ctypes.c_uint32),
        ("persist_error", ctypes.c_float),
        ("bucket_ms", ctypes.c_float),
        ("walker_chunk", ctypes.c_uint32),
        ("coop_small_steps", ctypes.c_uint64),
        ("coop_small_attempts", ctypes.c_uint64),
        ("coop_large_steps", ctypes.c_uint64),
        ("coop_large_attempts", ctypes.c_uint64),
        ("learned_parts", ctypes.c_uint32),
        ("copy_ms", ctypes.c_float),
        ("zero_copy_sectors", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if not n.startswith("reserved")}


_LIB = None


def load():
    """Load libgowalker.so and declare its signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "gowalker_b200/libgowalker.so is not built; run `make -C gowalker_b200/csrc` "
            "(or __graft_entry__.build()).  The walk engine has no CPU fallback.")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    u32p = ctypes.POINTER(ctypes.c_uint32)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    sig = {
        "gw_version": ([], i32),
        "gw_status_string": ([i32], ctypes.c_char_p),
        "gw_config_default": ([ctypes.POINTER(GwConfig)], i32),
        "gw_create": ([ctypes.POINTER(GwConfig), ctypes.POINTER(vp)], i32),
        "gw_destroy": ([vp], i32),
        "gw_last_error": ([vp, ctypes.c_char_p, ctypes.c_size_t], i32),
        "gw_set_config": ([vp, ctypes.POINTER(GwConfig)], i32),
        "gw_stream": ([vp, ctypes.POINTER(vp)], i32),
        "gw_set_graph_meta": ([vp, u32, u64, u32, u32p, u64p], i32),
        "gw_host_block": ([vp, u32, vp, vp], i32),
        "gw_device_graph": ([vp, vp, vp], i32),
        "gw_cache_reset": ([vp], i32),
        "gw_host_weights": ([vp, u32, vp], i32),
        "gw_device_weights": ([vp, vp], i32),
        "gw_init_walkers": ([vp, u32, u32, u64], i32),
        "gw_init_walker_range": ([vp, u32, u32, u64, u64, u64], i32),
        "gw_run": ([vp, u32, ctypes.POINTER(GwStats)], i32),
        "gw_num_walkers": ([vp, u64p], i32),
        "gw_get_paths": ([vp, u64, u64, vp, vp], i32),
        "gw_path_hashes": ([vp, u64, u64, vp], i32),
        "gw_path_lengths": ([vp, u64, u64, vp], i32),
        "gw_checksum": ([vp, u64p, u64p], i32),
        "gw_bucket_counts": ([vp, vp], i32),
        "gw_rmat_csr": ([u32, u32, u64, u32p, u64, i32, u64, ctypes.POINTER(vp), ctypes.POINTER(vp), u64p], i32),
        "gw_web_csr": ([u32, u32, u32p, ctypes.c_double, ctypes.c_double, u32, u32, u32, u64, u64,
                        ctypes.POINTER(vp), ctypes.POINTER(vp), u64p], i32),
        "gw_edges_csr": ([vp, vp, u64, u32, u32, ctypes.POINTER(vp), ctypes.POINTER(vp), u64p, u32p], i32),
        "gw_split_blocks": ([vp, u32, u32, u64, vp, vp, u32, u32p], i32),
        "gw_sa_choose_blocks": ([vp, u32, vp, u32, u32, u64, u32, vp], i32),
        "gw_plain_choose_block": ([vp, u32, vp, u32, u32, u32, vp], i32),
        "gw_device_free": ([vp], i32),
        "gw_philox_rate": ([i32, u32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)], i32),
        "gw_memcpy": ([vp, vp, u64], i32),
        "gw_walk_noalloc": ([ctypes.POINTER(GwConfig), vp, vp, u32, u64, u64, vp, vp, vp, vp,
                             ctypes.POINTER(GwStats)], i32),
        "gw_host_alloc": ([u64, ctypes.POINTER(vp)], i32),
        "gw_host_free": ([vp], i32),
        "gw_mlp_forward": ([vp, vp, u32, vp], i32),
        "gw_mlp_grad": ([vp, vp, vp, u32, vp, vp, vp], i32),
        "gw_mlp_train": ([vp, vp, vp, u32, u32, ctypes.c_float, u64, vp, ctypes.POINTER(ctypes.c_float)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


class GwError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (load().gw_status_string(status).decode(), status, message))
        self.status = status

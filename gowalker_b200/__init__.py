"""gowalker_b200 -- a B200-native second-order random-walk engine with the
interface of GOWalker's walk path (Node2vec / SOPR / SOSR).

The engine itself is libgowalker.so (C ABI in include/gowalker.h, kernels in
gowalker_b200/csrc).  This package is its Python binding; importing it loads
the library and fails loudly when it has not been built.
"""
from ._abi import (GW_LAUNCH_PER_HOP, GW_LAUNCH_PERSISTENT, GW_LEARNED_AUTO, GW_LEARNED_EVICT, GW_LEARNED_ZERO_SWITCH, GW_EDGES_DEDUP, GW_EDGES_SORT, GW_EDGES_SYMMETRIC, GW_SPLIT_EQUAL_EDGES, GW_SPLIT_REFERENCE,
                   GW_INIT_PER_VERTEX, GW_INIT_RANDOM, GW_INIT_SINGLE_SOURCE, GW_NODE2VEC, GW_PATHS_FULL,
                   GW_PATHS_NONE, GW_POLICY_LEARNED, GW_POLICY_PLAIN, GW_POLICY_SA, GW_SOPR, GW_SOSR, GwConfig, GwError,
                   GwStats, LIB_PATH, load)
from .engine import (DeviceGraph, WalkEngine, default_config, plain_choose_block, sa_choose_blocks,
                     split_blocks_device)

__all__ = [
    "GW_NODE2VEC", "GW_SOPR", "GW_SOSR", "GW_INIT_PER_VERTEX", "GW_INIT_SINGLE_SOURCE", "GW_INIT_RANDOM",
    "GW_POLICY_PLAIN", "GW_POLICY_LEARNED", "GW_POLICY_SA", "sa_choose_blocks", "plain_choose_block", "GW_PATHS_NONE", "GW_PATHS_FULL", "GwConfig", "GwStats",
    "GwError", "WalkEngine", "DeviceGraph", "default_config", "load", "LIB_PATH", "split_blocks_device",
    "GW_EDGES_SYMMETRIC", "GW_EDGES_SORT", "GW_EDGES_DEDUP", "GW_SPLIT_REFERENCE", "GW_SPLIT_EQUAL_EDGES",
    "GW_LAUNCH_PERSISTENT", "GW_LAUNCH_PER_HOP", "GW_LEARNED_EVICT", "GW_LEARNED_ZERO_SWITCH", "GW_LEARNED_AUTO",
]

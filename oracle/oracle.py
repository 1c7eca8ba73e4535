"""CPU oracle for the GOWalker walk step -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
module, and only as the checker or the timed CPU baseline.  The product
(gowalker_b200) never imports it.

Contents:
  * ctypes wrappers over liboracle.so (gw_oracle.c): Philox4x32-10, the
    counter-based R-MAT sampler and the Node2vec / SOPR / SOSR whole-walk
    restatement of engine/engine.hpp:158-404;
  * a numpy CSR builder (drop self loops, optional symmetrisation, dedup,
    sorted adjacency) for the synthetic R-MAT graphs, the edge-list converter
    restatement (convert_edges) and a line-by-line one of the reference's
    streaming converter (convert_stream) that pins it;
  * writers for the reference's on-disk format: ``<base>.beg`` (u64, V+1),
    ``<base>.csr`` (u32, E), ``<base>.meta`` (packed u32 nvertices, u64 nedges,
    u32 min_vert; preprocess/graph_converter.hpp finalize()), and the block
    files ``sowalker_<MB>/<name>_<MB>MB.{vert,edge}.blocks``
    (util/util.hpp:148-165, preprocess/split.hpp:74-84);
  * a restatement of the reference's block splitter
    (preprocess/split.hpp:15-87) and the equal-edge-mass splitter;
  * a loader for oracle/_ref/libref_step*.so, the harness that runs the
    reference's own sidewalkupdate.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

ALG_NODE2VEC, ALG_SOPR, ALG_SOSR = 0, 1, 2
INIT_PER_VERTEX, INIT_SINGLE_SOURCE, INIT_RANDOM = 0, 1, 2
KEY_HOP_ATTEMPT, KEY_TRIAL = 0, 1

RMAT_ABC = (0.57, 0.19, 0.19)


class Cfg(ctypes.Structure):
    _fields_ = [
        ("algo", ctypes.c_uint32),
        ("maxhops", ctypes.c_uint32),
        ("p", ctypes.c_float),
        ("q", ctypes.c_float),
        ("alpha", ctypes.c_float),
        ("term_prob", ctypes.c_float),
        ("seed", ctypes.c_uint64),
        ("keying", ctypes.c_uint32),
        ("init_mode", ctypes.c_uint32),
        ("wps", ctypes.c_uint32),
        ("numwalks", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_uint64),
        ("trials", ctypes.c_uint64),
        ("probes", ctypes.c_uint64),
        ("search_sectors", ctypes.c_uint64),
        ("off_sectors", ctypes.c_uint64),
        ("dead_ends", ctypes.c_uint64),
        ("terminated", ctypes.c_uint64),
        ("acc_sectors", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class SchedStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("iterations", "loads", "steps", "parks", "rescues", "finished",
                                               "zc_steps")]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


_LIB = None


def build_oracle(with_ref: bool = False) -> None:
    """Compile liboracle.so (and the reference harness when asked)."""
    target = "all" if with_ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        L = ctypes.CDLL(path)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.oracle_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.oracle_rmat_edges.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, u32p,
                                        ctypes.c_uint64, u32p, u32p, ctypes.c_int]
        L.oracle_web_degrees.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_uint32,
                                         ctypes.c_uint64, u64p]
        L.oracle_web_edges.argtypes = [ctypes.c_uint32, ctypes.c_uint32, u32p, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint64, u64p, u32p, u32p]
        L.oracle_walk.argtypes = [u64p, u32p, ctypes.c_uint32, ctypes.POINTER(Cfg), ctypes.c_uint32,
                                  ctypes.c_uint32, u32p, u32p, u64p, u32p, ctypes.POINTER(Stats),
                                  ctypes.c_int]
        L.oracle_walk.restype = ctypes.c_int
        f32p = ctypes.POINTER(ctypes.c_float)
        L.oracle_walk_ids.argtypes = [u64p, u32p, ctypes.c_uint32, ctypes.POINTER(Cfg), u32p, ctypes.c_uint32,
                                      u32p, u32p, u64p, ctypes.POINTER(Stats), ctypes.c_int]
        L.oracle_walk_ids.restype = ctypes.c_int
        L.oracle_walk_reqs.argtypes = [u64p, u32p, ctypes.c_uint32, ctypes.POINTER(Cfg), u32p, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint16), u32p,
                                       ctypes.c_int]
        L.oracle_walk_reqs.restype = ctypes.c_int
        L.oracle_sched_replay.argtypes = [ctypes.POINTER(ctypes.c_uint16), u32p, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                          ctypes.c_uint64, ctypes.POINTER(SchedStats)]
        L.oracle_sched_replay.restype = ctypes.c_int64
        L.oracle_sched_study.argtypes = [ctypes.POINTER(ctypes.c_uint16), u32p, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_uint64, u64p, u64p, u64p]
        L.oracle_sched_study.restype = ctypes.c_int64
        L.oracle_walk_weighted.argtypes = [u64p, u32p, f32p, u32p, ctypes.c_uint32, ctypes.POINTER(Cfg),
                                           ctypes.c_uint32, ctypes.c_uint32, u32p, u32p, u64p, u32p,
                                           ctypes.POINTER(Stats), ctypes.c_int]
        L.oracle_walk_weighted.restype = ctypes.c_int
        L.oracle_build_alias.argtypes = [u64p, f32p, ctypes.c_uint32, f32p, u32p]
        L.oracle_build_alias.restype = ctypes.c_int
        L.oracle_walk_traced.argtypes = [u64p, u32p, ctypes.POINTER(Cfg), ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u32p,
                                         u32p, ctypes.c_uint64, u64p, u32p]
        L.oracle_walk_traced.restype = ctypes.c_uint32
        L.oracle_walker_source.argtypes = [ctypes.POINTER(Cfg), ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_walker_source.restype = ctypes.c_uint32
        L.oracle_hash_init.argtypes = [ctypes.c_uint32]
        L.oracle_hash_init.restype = ctypes.c_uint64
        _LIB = L
    return _LIB


def _p(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# ------------------------------------------------------------------ Philox

def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c, ctypes.c_uint32), _p(k, ctypes.c_uint32), _p(out, ctypes.c_uint32))
    return out


# ------------------------------------------------------------------ graphs

def rmat_thresholds(a: float, b: float, c: float) -> np.ndarray:
    """Cumulative quadrant thresholds a, a+b, a+b+c scaled to 2^32, as u32."""
    t = [int(a * 4294967296.0), int((a + b) * 4294967296.0), int((a + b + c) * 4294967296.0)]
    return np.array([min(x, 0xFFFFFFFF) for x in t], dtype=np.uint32)


def rmat_edges(scale: int, first: int, count: int, seed: int = 1, abc=RMAT_ABC, nthreads: int = 0):
    thr = rmat_thresholds(*abc)
    src = np.empty(count, dtype=np.uint32)
    dst = np.empty(count, dtype=np.uint32)
    lib().oracle_rmat_edges(scale, first, count, _p(thr, ctypes.c_uint32), seed,
                            _p(src, ctypes.c_uint32), _p(dst, ctypes.c_uint32), nthreads)
    return src, dst


def web_degrees(nverts: int, dmin: float = 6.0, tail: float = 1.1, max_degree: int = 65536, seed: int = 1):
    """Out-degree draws of the web-shaped graph (gw_oracle.c oracle_web_degrees)."""
    deg = np.empty(nverts, dtype=np.uint64)
    lib().oracle_web_degrees(nverts, dmin, tail, max_degree, seed, _p(deg, ctypes.c_uint64))
    return deg


def web_graph(scale: int, nverts: int, dmin: float = 6.0, tail: float = 1.1, max_degree: int = 65536,
              local_permille: int = 800, window: int = 65536, seed: int = 1, abc=RMAT_ABC):
    """The web-shaped graph's CSR before thinning (gw_web_csr restated):
    power-law degrees, each vertex's edges drawn in place, dropped ones
    removed, repeats removed, adjacency sorted."""
    deg = web_degrees(nverts, dmin, tail, max_degree, seed)
    estart = np.zeros(nverts + 1, dtype=np.uint64)
    estart[1:] = np.cumsum(deg)
    m = int(estart[-1])
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    thr = rmat_thresholds(*abc)
    lib().oracle_web_edges(scale, nverts, _p(thr, ctypes.c_uint32), local_permille, window, seed,
                           _p(estart, ctypes.c_uint64), _p(src, ctypes.c_uint32), _p(dst, ctypes.c_uint32))
    keep = dst != 0xFFFFFFFF
    return build_csr(nverts, src[keep], dst[keep], symmetric=False)


def thin_sorted(beg: np.ndarray, csr: np.ndarray, target: int):
    """Keep `target` of the U sorted unique edges: edge i goes when
    floor((i+1)k/U) > floor(ik/U), k = U - target (the device's k_thin)."""
    U = len(csr)
    k = U - target
    if U >= (1 << 20):
        raise ValueError("thin_sorted is for small cases")
    keep = np.array([(ii + 1) * k // U == ii * k // U for ii in range(U)], dtype=bool)
    src = np.repeat(np.arange(len(beg) - 1, dtype=np.int64), np.diff(beg.astype(np.int64)))[keep]
    nb = np.zeros(len(beg), dtype=np.uint64)
    nb[1:] = np.cumsum(np.bincount(src, minlength=len(beg) - 1)).astype(np.uint64)
    return nb, csr[keep]


def build_csr(nverts: int, src: np.ndarray, dst: np.ndarray, symmetric: bool = True):
    """CSR with u64 offsets and sorted, duplicate-free u32 adjacency; self loops
    dropped (preprocess/graph_converter.hpp:362-363)."""
    src = src.astype(np.uint64)
    dst = dst.astype(np.uint64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    if symmetric:
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    keys = np.unique((src << np.uint64(32)) | dst)
    s = (keys >> np.uint64(32)).astype(np.int64)
    csr = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    beg = np.zeros(nverts + 1, dtype=np.uint64)
    beg[1:] = np.cumsum(np.bincount(s, minlength=nverts)).astype(np.uint64)
    return beg, csr


def convert_edges(src, dst, nverts: int = 0, symmetric: bool = False, sort: bool = False, dedup: bool = False):
    """Edge list -> (beg, csr, nverts): the reference's converter
    (graph_converter::convert, preprocess/graph_converter.hpp:286-449) with
    its optional neighbour sort (sort_vertex_neighbors,
    preprocess/precompute.hpp:42-133), generalised to lists that are not
    source-sorted.  Self loops are dropped (graph_converter.hpp:362-363).
    Without ``sort`` a vertex keeps its edges in input order (a stable sort
    by source); ``symmetric`` puts (dst, src) right after each edge; ``dedup``
    keeps one copy of each (src, dst) and implies ``sort``.  nverts 0 means
    the largest kept id + 1.  Raises ValueError on an id >= nverts (or
    2^32-1, when nverts is 0)."""
    src = np.asarray(src, dtype=np.uint64)
    dst = np.asarray(dst, dtype=np.uint64)
    lim = nverts if nverts else 0xFFFFFFFF
    if len(src) and (int(src.max()) >= lim or int(dst.max()) >= lim):
        raise ValueError("vertex id out of range")
    keep = src != dst
    src, dst = src[keep], dst[keep]
    if symmetric:
        src, dst = np.stack([src, dst], 1).reshape(-1), np.stack([dst, src], 1).reshape(-1)
    if not nverts:
        nverts = int(max(src.max(), dst.max())) + 1 if len(src) else 0
    keys = (src << np.uint64(32)) | dst
    if dedup:
        keys = np.unique(keys)
    elif sort:
        keys = np.sort(keys, kind="stable")
    else:
        keys = keys[np.argsort(keys >> np.uint64(32), kind="stable")]
    s = (keys >> np.uint64(32)).astype(np.int64)
    beg = np.zeros(nverts + 1, dtype=np.uint64)
    beg[1:] = np.cumsum(np.bincount(s, minlength=nverts)).astype(np.uint64)
    return beg, (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32), nverts


def convert_stream(edges, sort: bool = False):
    """Line-by-line restatement of the converter's streaming loop for a
    source-sorted list (graph_converter.hpp:167-216 convert, 220-226
    dealfirstline, 257-263 finalize), pure Python for small inputs: pins
    convert_edges.  Returns (beg, csr, nverts) with nverts = max_vert + 1."""
    beg, csr = [0], []
    adj, curr, max_vert, first = [], 0, 0, True
    for frm, to in edges:
        if first:
            if frm != 0:
                beg.extend([0] * frm)  # sync_zeros(from)
                curr = frm
            first = False
        if frm == to:
            continue
        max_vert = max(max_vert, frm, to)
        if frm == curr:
            adj.append(to)
        elif frm < curr:
            raise ValueError("edge list is not source-sorted")
        else:
            csr.extend(adj)
            beg.append(len(csr))
            beg.extend([len(csr)] * (frm - curr - 1))
            curr, adj = frm, [to]
    csr.extend(adj)
    beg.append(len(csr))
    if max_vert > curr:
        beg.extend([len(csr)] * (max_vert - curr))
    if sort:
        for v in range(len(beg) - 1):
            csr[beg[v]:beg[v + 1]] = sorted(csr[beg[v]:beg[v + 1]])
    return np.array(beg, dtype=np.uint64), np.array(csr, dtype=np.uint32), len(beg) - 1


def rmat_graph(scale: int, edgefactor: int = 16, seed: int = 1, abc=RMAT_ABC, symmetric: bool = True):
    """Synthetic R-MAT graph: (edgefactor << scale) counter-based samples."""
    n = edgefactor << scale
    src, dst = rmat_edges(scale, 0, n, seed, abc)
    return build_csr(1 << scale, src, dst, symmetric)


def check_csr(beg: np.ndarray, csr: np.ndarray) -> None:
    assert beg.dtype == np.uint64 and csr.dtype == np.uint32
    assert int(beg[0]) == 0 and int(beg[-1]) == len(csr)
    assert np.all(np.diff(beg.astype(np.int64)) >= 0)


# ------------------------------------------------------------------ walks

def make_cfg(algo=ALG_NODE2VEC, maxhops=80, p=2.0, q=0.5, alpha=0.2, term_prob=0.0, seed=42,
             keying=KEY_HOP_ATTEMPT, init_mode=INIT_PER_VERTEX, wps=1, numwalks=0) -> Cfg:
    return Cfg(algo, maxhops, p, q, alpha, term_prob, seed, keying, init_mode, wps, numwalks)


def build_alias(beg, w):
    """Walker's alias tables of every vertex's out-edge weights
    (gw_oracle.c oracle_build_alias): (prob float32, alias u32 local index)."""
    beg = np.ascontiguousarray(beg, dtype=np.uint64)
    w = np.ascontiguousarray(w, dtype=np.float32)
    prob = np.zeros(len(w), dtype=np.float32)
    alias = np.zeros(len(w), dtype=np.uint32)
    rc = lib().oracle_build_alias(_p(beg, ctypes.c_uint64), _p(w, ctypes.c_float), len(beg) - 1,
                                  _p(prob, ctypes.c_float), _p(alias, ctypes.c_uint32))
    if rc != 0:
        raise ValueError("edge weights must be positive finite numbers")
    return prob, alias


def walk(beg, csr, cfg: Cfg, wid_begin: int, count: int, paths: bool = True, finals: bool = False,
         nthreads: int = 0, alias=None):
    """Walk walkers [wid_begin, wid_begin+count).  Returns a dict with
    paths (count x maxhops+1, zero padded), lens, hashes, finals, stats.
    alias = (prob, alias) from build_alias: weighted Node2vec."""
    nverts = len(beg) - 1
    stride = cfg.maxhops + 1
    P = np.zeros((count, stride), dtype=np.uint32) if paths else None
    L = np.zeros(count, dtype=np.uint32)
    H = np.zeros(count, dtype=np.uint64)
    F = np.zeros((count, 3), dtype=np.uint32) if finals else None
    st = Stats()
    if alias is not None:
        rc = lib().oracle_walk_weighted(_p(beg, ctypes.c_uint64), _p(csr, ctypes.c_uint32),
                                        _p(alias[0], ctypes.c_float), _p(alias[1], ctypes.c_uint32), nverts,
                                        ctypes.byref(cfg), wid_begin, count, _p(P, ctypes.c_uint32),
                                        _p(L, ctypes.c_uint32), _p(H, ctypes.c_uint64), _p(F, ctypes.c_uint32),
                                        ctypes.byref(st), nthreads)
    else:
        rc = lib().oracle_walk(_p(beg, ctypes.c_uint64), _p(csr, ctypes.c_uint32), nverts, ctypes.byref(cfg),
                               wid_begin, count, _p(P, ctypes.c_uint32), _p(L, ctypes.c_uint32),
                               _p(H, ctypes.c_uint64), _p(F, ctypes.c_uint32), ctypes.byref(st), nthreads)
    if rc != 0:
        raise ValueError("oracle_walk rejected the configuration")
    return {"paths": P, "lens": L, "hashes": H, "finals": F, "stats": st.as_dict()}


def walk_ids(beg, csr, cfg: Cfg, ids, paths: bool = False, nthreads: int = 0):
    """Walk the listed walkers (u32 ids, any order): row i is walker ids[i].
    Returns a dict with paths (or None), lens, hashes, stats."""
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    n = ids.size
    P = np.zeros((n, cfg.maxhops + 1), dtype=np.uint32) if paths else None
    L = np.zeros(n, dtype=np.uint32)
    H = np.zeros(n, dtype=np.uint64)
    st = Stats()
    rc = lib().oracle_walk_ids(_p(beg, ctypes.c_uint64), _p(csr, ctypes.c_uint32), len(beg) - 1, ctypes.byref(cfg),
                               _p(ids, ctypes.c_uint32), n, _p(P, ctypes.c_uint32), _p(L, ctypes.c_uint32),
                               _p(H, ctypes.c_uint64), ctypes.byref(st), nthreads)
    if rc != 0:
        raise ValueError("oracle_walk_ids rejected the configuration")
    return {"paths": P, "lens": L, "hashes": H, "stats": st.as_dict()}


def walk_requirements(beg, csr, cfg: Cfg, vstart, wid_begin: int, count: int, nthreads: int = 0):
    """The blocks walkers [wid_begin, wid_begin+count) will need, in order
    (gw_oracle.c oracle_walk_reqs): count x (maxhops+1) u16 entries (block,
    bit 14 terminal, bit 15 needs the previous block under the lazy rule) and
    the entry count of each walker."""
    vstart = np.ascontiguousarray(vstart, dtype=np.uint32)
    stride = cfg.maxhops + 1
    reqs = np.zeros((count, stride), dtype=np.uint16)
    nent = np.zeros(count, dtype=np.uint32)
    rc = lib().oracle_walk_reqs(_p(beg, ctypes.c_uint64), _p(csr, ctypes.c_uint32), len(beg) - 1, ctypes.byref(cfg),
                                _p(vstart, ctypes.c_uint32), len(vstart) - 1, wid_begin, count,
                                reqs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), _p(nent, ctypes.c_uint32),
                                nthreads)
    if rc != 0:
        raise ValueError("oracle_walk_reqs rejected the configuration")
    return reqs, nent


def sched_replay(reqs, nent, nb: int, nslots: int, prefetch: bool = True, lazy: bool = True,
                 zero_threshold: int = 0, log: bool = False, evict_incident: bool = False, zero_tail: bool = False):
    """The out-of-core engine's plain block schedule replayed on the CPU
    (gw_oracle.c oracle_sched_replay).  evict_incident: the victim is the
    cached block with the fewest incident walkers; zero_tail: GOWalker's zero
    mode (the rest through mapped host memory once nothing scores above
    zero_threshold; those steps in stats["zc_steps"]).  Returns (stats dict,
    per-iteration log of (loaded block, replaced position, steps) or None)."""
    reqs = np.ascontiguousarray(reqs, dtype=np.uint16)
    nent = np.ascontiguousarray(nent, dtype=np.uint32)
    cap = 1 << 22 if log else 0
    lg = np.zeros((cap, 3), dtype=np.int32) if log else None
    st = SchedStats()
    it = lib().oracle_sched_replay(reqs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), _p(nent, ctypes.c_uint32),
                                   len(nent), reqs.shape[1], nb, nslots, int(prefetch), int(lazy), zero_threshold,
                                   int(evict_incident), int(zero_tail), lg.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if log else None, cap,
                                   ctypes.byref(st))
    if it < 0:
        raise ValueError("schedule replay failed (bad arguments or no progress)")
    return st.as_dict(), (lg[:it].copy() if log else None)


def sched_study(reqs, nent, nb: int, nslots: int, policy: int = 0, zero_threshold: int = 0, lazy: bool = True):
    """Another block policy on the same walks (gw_oracle.c oracle_sched_study,
    no prefetch): 0 GOWalker's choice, 1 clairvoyant one-iteration yield, 2
    GOWalker's choice with clairvoyant eviction, 3-5 GOWalker's choice
    evicting the fewest incident walkers / the lowest average use / the least
    recently used block; zero_threshold > 0 stops
    loading where the reference's zero rule does.  Returns a dict of
    iterations, loads, steps taken by the block loads, and steps left to the
    mapped-host tail."""
    reqs = np.ascontiguousarray(reqs, dtype=np.uint16)
    nent = np.ascontiguousarray(nent, dtype=np.uint32)
    loads, steps, zc = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    it = lib().oracle_sched_study(reqs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), _p(nent, ctypes.c_uint32),
                                  len(nent), reqs.shape[1], nb, nslots, int(lazy), policy, zero_threshold,
                                  ctypes.byref(loads), ctypes.byref(steps), ctypes.byref(zc))
    if it < 0:
        raise ValueError("schedule study failed (bad arguments or no progress)")
    return {"iterations": int(it), "loads": int(loads.value), "steps": int(steps.value), "zc_steps": int(zc.value)}


def walk_traced(beg, csr, cfg: Cfg, wid: int, prev: int, cur: int, hop: int, cap: int = 1 << 16):
    path = np.zeros(cfg.maxhops + 1, dtype=np.uint32)
    trace = np.zeros((cap, 4), dtype=np.uint32)
    n = ctypes.c_uint64(0)
    final = np.zeros(3, dtype=np.uint32)
    moves = lib().oracle_walk_traced(_p(beg, ctypes.c_uint64), _p(csr, ctypes.c_uint32), ctypes.byref(cfg),
                                     wid, prev, cur, hop, _p(path, ctypes.c_uint32),
                                     _p(trace, ctypes.c_uint32), cap, ctypes.byref(n),
                                     _p(final, ctypes.c_uint32))
    return int(moves), path[:moves], trace[: min(int(n.value), cap)], final


def path_hash(path) -> int:
    """FNV-1a over 32-bit vertex ids (the engine's per-walker path hash)."""
    h = 0xCBF29CE484222325
    for v in path:
        h = ((h ^ int(v)) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


# ------------------------------------------------------------------ files

def block_names(base: str, blocksize_mb: int):
    folder = os.path.join(os.path.dirname(base) or ".", "sowalker_%d" % blocksize_mb)
    name = os.path.basename(base)
    vb = os.path.join(folder, "%s_%dMB.vert.blocks" % (name, blocksize_mb))
    eb = os.path.join(folder, "%s_%dMB.edge.blocks" % (name, blocksize_mb))
    return folder, vb, eb


def write_dataset(base: str, beg: np.ndarray, csr: np.ndarray, min_vert: int = 0) -> None:
    beg.astype(np.uint64).tofile(base + ".beg")
    csr.astype(np.uint32).tofile(base + ".csr")
    meta = np.zeros(16, dtype=np.uint8)
    meta[0:4] = np.frombuffer(np.uint32(len(beg) - 1).tobytes(), np.uint8)
    meta[4:12] = np.frombuffer(np.uint64(len(csr)).tobytes(), np.uint8)
    meta[12:16] = np.frombuffer(np.uint32(min_vert).tobytes(), np.uint8)
    meta.tofile(base + ".meta")


def write_blocks(base: str, blocksize_mb: int, vblocks, eblocks) -> None:
    folder, vb, eb = block_names(base, blocksize_mb)
    os.makedirs(folder, exist_ok=True)
    np.asarray(vblocks, dtype=np.uint32).tofile(vb)
    np.asarray(eblocks, dtype=np.uint64).tofile(eb)


def split_blocks_reference(beg: np.ndarray, block_size: int):
    """Restatement of split_blocks (preprocess/split.hpp:15-87): walk beg[] and
    cut a block when its edges exceed block_size/4 (the cut goes one vertex
    back) or its vertices reach block_size/8."""
    max_nedges = block_size // 4
    max_nverts = block_size // 8
    nv = len(beg)  # the file holds V+1 offsets; the reference calls that nvertices
    vblocks, eblocks = [0], [0]
    cur_pos, rd_edges = 0, 0
    for v in range(nv):
        if int(beg[v]) - rd_edges > max_nedges:
            cur_pos = v - 1
            vblocks.append(cur_pos)
            rd_edges = int(beg[v - 1])
            eblocks.append(rd_edges)
        elif v - cur_pos >= max_nverts:
            cur_pos = v
            vblocks.append(cur_pos)
            rd_edges = int(beg[v])
            eblocks.append(rd_edges)
    vblocks.append(nv - 1)
    eblocks.append(int(beg[nv - 1]))
    return np.array(vblocks, dtype=np.uint32), np.array(eblocks, dtype=np.uint64)


def split_equal_edge_mass(beg: np.ndarray, nblocks: int):
    """Vertex-range blocks of (nearly) equal edge mass: block b ends at the
    first vertex whose offset reaches b*E/nblocks."""
    V = len(beg) - 1
    E = int(beg[-1])
    targets = np.array([k * E // nblocks for k in range(1, nblocks)], dtype=np.uint64)
    cuts = np.searchsorted(beg[:-1], targets, side="left").astype(np.int64)
    cuts = np.maximum.accumulate(np.clip(cuts, 1, max(V - 1, 1)))
    vb = np.concatenate([[0], cuts, [V]]).astype(np.int64)
    vb = np.maximum.accumulate(vb)
    vb = vb.astype(np.uint32)
    eb = beg[vb.astype(np.int64)].astype(np.uint64)
    return vb, eb


# ------------------------------------------------------------------ GOWalker block choice

def max_choose_blocks(counts, cached, nslots: int, zero_threshold: int = 0):
    """Restatement of GOwalker_scheduler_t::max_choose_blocks
    (engine/schedule.hpp:70-138).  counts: nb x nb walkers per (prev block,
    cur block); cached: the scheduler's list of resident blocks in order (its
    `buckets`); nslots: cache slots (graph_cache::ncblock).

    Cache not full (len(cached) < nslots, 108-131): every uncached block i
    scores sum over cached c of counts[i,c] + counts[c,i], plus counts[i,i];
    the best is appended.  Full (83-107): s_j = counts[i,c_j] + counts[c_j,i],
    the score is sum_j s_j - min_j s_j, and i replaces the cached block of the
    first smallest s_j (strict `<` from 0xffffffff, 95-98).  A block is taken
    only if its score is > 0 and > zero_threshold (101, 124).  The reference
    orders scores with std::sort (not stable); among equal best scores this
    takes the lowest block id, which is libstdc++'s order when at most 16
    blocks are uncached (its insertion sort keeps the ascending order in which
    pre_cached is built, 79-84).

    Returns (action, block, position): (0, -1, -1) when nothing qualifies (the
    reference returns false), (1, i, len(cached)) when i is appended,
    (2, i, j) when i replaces cached[j]."""
    c = np.asarray(counts, dtype=np.uint64)
    nb = c.shape[0]
    c = c.reshape(nb, nb)
    cached = [int(x) for x in cached]
    isc = np.zeros(nb, dtype=bool)
    isc[cached] = True
    pre = [i for i in range(nb) if not isc[i]]
    if not pre:
        return (0, -1, -1)
    cl = np.array(cached, dtype=np.int64)
    best_i, best_s, best_pos = -1, -1, -1
    full = len(cached) >= nslots
    for i in pre:
        links = (c[i, cl] + c[cl, i]) if len(cl) else np.zeros(0, dtype=np.uint64)
        if full:
            mn, idx = 0xFFFFFFFF, 0
            for j, v in enumerate(links):
                if int(v) < mn:
                    mn, idx = int(v), j
            score = int(links.sum()) - mn
            pos = idx
        else:
            score = int(links.sum()) + int(c[i, i])
            pos = len(cached)
        if score > best_s:  # first (lowest id) of equal scores
            best_i, best_s, best_pos = i, score, pos
    if best_s > 0 and best_s > zero_threshold:
        return (2 if full else 1, best_i, best_pos)
    return (0, -1, -1)


# ------------------------------------------------------------------ SOWalker annealing block choice

TAG_SA = 0x53414E4E  # 'SANN'


def sa_log_draw(z: int) -> float:
    """ln(z * 2^-32) by the fixed steps the device uses (every operation an
    IEEE double rounded to nearest): z = 2^e * m, m in [sqrt(1/2), sqrt(2)),
    ln = e ln2 + 2 atanh((m-1)/(m+1)), the atanh series to s^23/23 by Horner
    in s^2, ln2 = 45426 * 2^-16 + 1.4286068203094172e-06.  z = 0 gives -inf.
    Bit-identical to the device's version."""
    if z == 0:
        return -math.inf
    e = z.bit_length() - 1
    m = float(z) * math.ldexp(1.0, -e)
    if m >= 1.4142135623730951:
        m = m * 0.5
        e += 1
    s = (m - 1.0) / (m + 1.0)
    s2 = s * s
    inv = [1.0 / (2 * j + 1) for j in range(12)]
    q = inv[11]
    for j in range(10, -1, -1):
        q = inv[j] + s2 * q
    lnm = (2.0 * s) * q
    ex = float(e - 32)
    return (ex * 0.693145751953125 + ex * 1.4286068203094172e-06) + lnm


def sa_choose_blocks(counts, cached, k: int, seed: int, call: int):
    """Restatement of SOwalker_scheduler_t::choose_blocks
    (engine/schedule.hpp:455-593): rank blocks by walkers whose current block
    they are (ties by id), take the first k-1 and the best partner for the
    k-th (schedule.hpp:488-500), then anneal one-for-one swaps (523-583):
    score = walkers inside the set // blocks of the set not resident (0 when
    all are), accept better, or worse-but-positive with probability
    exp((y_tmp - y_can)/T) -- as (y_tmp - y_can)/T > ln(u) for the round's
    uniform u (sa_log_draw) -- in float, T = 100 x 0.998^i while > 0.001, at most
    C(nb, k) rounds.  Round i of call c draws Philox(i, c, 0, 'SANN') under
    seed where the reference calls std::rand."""
    bw = [[int(v) for v in row] for row in np.asarray(counts, dtype=np.uint64)]
    nb = len(bw)
    k = min(k, nb)
    isc = [0] * nb
    for b in cached:
        isc[int(b)] = 1
    pw = [sum(bw[p][c] for p in range(nb)) for c in range(nb)]
    idx = sorted(range(nb), key=lambda b: (-pw[b], b))
    if 0 < k < nb:
        best, bi = 0, None
        for pi in range(k - 1, nb):
            p = idx[pi]
            w = sum(bw[p][idx[ci]] + bw[idx[ci]][p] for ci in range(k - 1))
            if w > best:
                best, bi = w, pi
        if bi is not None:
            idx[k - 1], idx[bi] = idx[bi], idx[k - 1]
    cand = idx[:k]
    if 0 < k < nb:
        f32 = np.float32
        score = sum(bw[p][c] for p in cand for c in cand)
        comm = sum(isc[b] for b in cand)

        def y(sc, cm):
            return f32(sc // (k - cm)) if cm < k else f32(0.0)

        ycan = y(score, comm)
        maxiter = min(math.comb(nb, k), 1 << 20)
        T = f32(100.0)
        key = [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF]
        it = 0
        while it < maxiter and T > f32(0.001):
            r = [int(v) for v in philox([it, call, 0, TAG_SA], key)]
            pos = k + r[0] % (nb - k)
            tp = r[1] % k
            out, inn = cand[tp], idx[pos]
            a = sum(bw[out][x] + bw[x][out] for x in cand)
            b = sum(bw[inn][x] + bw[x][inn] for j, x in enumerate(cand) if j != tp)
            score2 = score - (a - bw[out][out]) + (b + bw[inn][inn])
            comm2 = comm - isc[out] + isc[inn]
            y2 = y(score2, comm2)
            acc = bool(y2 > ycan)
            if not acc and y2 > 0:
                d = f32(f32(y2 - ycan) / T)
                acc = float(d) > sa_log_draw(r[2])
            if acc:
                cand[tp], idx[pos] = inn, out
                score, comm, ycan = score2, comm2, y2
            T = f32(T * f32(0.998))
            it += 1
    return np.array(cand, dtype=np.uint32)


# ------------------------------------------------------------------ reference harness

def ref_lib(unmodified: bool = False):
    """Load the harness built from the reference's own headers."""
    name = "libref_step_unmod.so" if unmodified else "libref_step.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    L.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                           ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.ref_open.restype = ctypes.c_int
    L.ref_set_seed.argtypes = [ctypes.c_uint64]
    L.ref_walk.argtypes = [ctypes.c_uint32] * 6 + [u32p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(ctypes.c_int), u32p]
    L.ref_walk.restype = ctypes.c_int
    L.ref_get_block.argtypes = [ctypes.c_uint32]
    L.ref_get_block.restype = ctypes.c_uint32
    return L


def ref_choose_blocks(base: str, cases):
    """Open the reference harness on the dataset at `base` (its block count is
    the scheduler's nblocks) and run the reference's own
    GOwalker_scheduler_t::max_choose_blocks once per case (counts, cached,
    nslots, zero_threshold).  Returns one (chose, list after) per case.  Run in
    a fresh process ('spawn'): the harness keeps global state."""
    L = ref_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref harness not built")
    u32p = ctypes.POINTER(ctypes.c_uint32)
    L.ref_max_choose_blocks.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u32p, u32p]
    L.ref_max_choose_blocks.restype = ctypes.c_int
    nb = L.ref_open(base.encode(), ALG_NODE2VEC, 0.5, 2.0, 0.2, 80, 1, 1)
    out = []
    for counts, cached, nslots, zt in cases:
        c = np.ascontiguousarray(counts, dtype=np.uint32).reshape(-1)
        assert c.size == nb * nb
        cl = np.ascontiguousarray(cached, dtype=np.uint32)
        lst = np.zeros(nb + 1, dtype=np.uint32)
        n = ctypes.c_uint32(0)
        r = L.ref_max_choose_blocks(_p(c, ctypes.c_uint32), _p(cl, ctypes.c_uint32) if cl.size else None, cl.size,
                                    nslots, zt, _p(lst, ctypes.c_uint32), ctypes.byref(n))
        if r < 0:
            raise RuntimeError("reference harness refused the case")
        out.append((bool(r), lst[: n.value].copy()))
    return out


def ref_walk(L, wid, prev, cur, hop, prev_blk, cur_blk, cap=1 << 16):
    trace = np.zeros((cap, 4), dtype=np.uint32)
    n = ctypes.c_uint64(0)
    pushed = ctypes.c_int(0)
    state = np.zeros(5, dtype=np.uint32)
    run = L.ref_walk(wid, prev, cur, hop, prev_blk, cur_blk, _p(trace, ctypes.c_uint32), cap,
                     ctypes.byref(n), ctypes.byref(pushed), _p(state, ctypes.c_uint32))
    return run, trace[: min(int(n.value), cap)], bool(pushed.value), state


def ref_scenario(base: str, algo: int, p: float, q: float, alpha: float, maxhops: int, blocksize_mb: int,
                 seed: int, starts, unmodified: bool = False, cpu_batch: int = 1):
    """Open the reference harness on the dataset at `base` and run one
    sidewalkupdate per start tuple (wid, prev, cur, hop, prev_blk, cur_blk).
    The harness keeps global state, so call this in a fresh process
    (multiprocessing 'spawn')."""
    L = ref_lib(unmodified)
    if L is None:
        raise FileNotFoundError("oracle/_ref harness not built")
    nb = L.ref_open(base.encode(), algo, p, q, alpha, maxhops, blocksize_mb, cpu_batch)
    L.ref_set_seed(seed)
    return nb, [ref_walk(L, *s) for s in starts]


def ref_single_steps(base: str, algo: int, p: float, q: float, alpha: float, seed: int, starts,
                     unmodified: bool = False):
    """One reference step per start tuple (wid, prev, cur, hop, prev_blk,
    cur_blk) on a dataset whose current block holds every neighbour of cur:
    the reference's cross-block loop (engine/engine.hpp:173-274) then stops
    after one step and re-buckets the walker, whose new vertex is returned
    (-1 when it was not re-bucketed).  Run in a fresh process ('spawn')."""
    L = ref_lib(unmodified)
    if L is None:
        raise FileNotFoundError("oracle/_ref harness not built")
    L.ref_open(base.encode(), algo, p, q, alpha, 1 << 20, 1, 64)
    L.ref_set_seed(seed)
    tr = np.zeros((4, 4), dtype=np.uint32)
    n, pushed = ctypes.c_uint64(0), ctypes.c_int(0)
    state = np.zeros(5, dtype=np.uint32)
    out = np.full(len(starts), -1, dtype=np.int64)
    for i, s in enumerate(starts):
        L.ref_walk(*s, _p(tr, ctypes.c_uint32), 4, ctypes.byref(n), ctypes.byref(pushed), _p(state, ctypes.c_uint32))
        if pushed.value:
            out[i] = int(state[1])
    return out


def harness_graph(beg: np.ndarray, csr: np.ndarray):
    """Graph G' for driving the reference's cross-block loop from a walk's
    first step: vertex V+v is a copy of v's adjacency (nothing points to it),
    so a walker at (prev=V+v, cur=v) takes exactly the step that (prev=v,
    cur=v) takes, while prev and cur sit in different one-vertex blocks."""
    V = len(beg) - 1
    beg2 = np.concatenate([beg, beg[-1] + beg[1:]]).astype(np.uint64)
    csr2 = np.concatenate([csr, csr]).astype(np.uint32)
    vblocks = np.arange(2 * V + 1, dtype=np.uint32)
    eblocks = beg2.copy()
    return beg2, csr2, vblocks, eblocks

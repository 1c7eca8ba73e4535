"""Python face of the walk engine: a thin owner of a gw_handle.

Mirrors the reference's run sequence (apps/Node2vec.cu:154-185): set the
graph (graph_block + graph_driver), create walkers (graph_engine::prologue ->
graph_walk::gpu_createwalk), run (graph_engine::pipe_run), read results.
Every call goes through libgowalker.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import GwConfig, GwError, GwStats


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def default_config(**kw) -> GwConfig:
    L = _abi.load()
    c = GwConfig()
    L.gw_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError("unknown gw_config field %r" % k)
        setattr(c, k, v)
    return c


class WalkEngine:
    """One engine handle on one device."""

    def __init__(self, cfg: GwConfig | None = None, **kw):
        self.L = _abi.load()
        self.cfg = cfg if cfg is not None else default_config(**kw)
        if cfg is not None:
            for k, v in kw.items():
                setattr(self.cfg, k, v)
        h = ctypes.c_void_p()
        st = self.L.gw_create(ctypes.byref(self.cfg), ctypes.byref(h))
        if st != 0:
            raise GwError(st, "gw_create failed")
        self.h = h
        self._keep = []  # host buffers borrowed by the handle

    # -- errors
    def _check(self, st):
        if st != 0:
            buf = ctypes.create_string_buffer(512)
            self.L.gw_last_error(self.h, buf, 512)
            raise GwError(st, buf.value.decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.gw_destroy(self.h)
            self.h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration
    def set_config(self, **kw):
        for k, v in kw.items():
            setattr(self.cfg, k, v)
        self._check(self.L.gw_set_config(self.h, ctypes.byref(self.cfg)))

    def stream_handle(self) -> int:
        """cudaStream_t of the handle's compute stream (as an int)."""
        s = ctypes.c_void_p()
        self._check(self.L.gw_stream(self.h, ctypes.byref(s)))
        return int(s.value or 0)

    # -- graph
    def set_graph_meta(self, nverts, nedges, vblocks, eblocks):
        vb = np.ascontiguousarray(vblocks, dtype=np.uint32)
        eb = np.ascontiguousarray(eblocks, dtype=np.uint64)
        self._check(self.L.gw_set_graph_meta(self.h, int(nverts), int(nedges), len(vb) - 1,
                                             vb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                             eb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        self.vblocks, self.eblocks = vb, eb
        self._keep = []

    def set_host_graph(self, beg, csr, vblocks=None, eblocks=None):
        """Register a host CSR (numpy arrays or pinned torch tensors) split into
        blocks; the arrays are borrowed and must stay alive."""
        nverts = len(beg) - 1
        nedges = int(beg[-1])
        if vblocks is None:
            vblocks = np.array([0, nverts], dtype=np.uint32)
            eblocks = np.array([0, nedges], dtype=np.uint64)
        self.set_graph_meta(nverts, nedges, vblocks, eblocks)
        for b in range(len(self.vblocks) - 1):
            v0, v1 = int(self.vblocks[b]), int(self.vblocks[b + 1])
            e0 = int(self.eblocks[b])
            bv = beg[v0:v1 + 1]
            bc = csr[e0:int(self.eblocks[b + 1])]
            self._keep += [bv, bc]
            self._check(self.L.gw_host_block(self.h, b, _ptr(bv), _ptr(bc)))
        self._keep += [beg, csr]

    def set_host_weights(self, w):
        """Edge weights (float32 per edge, aligned with the CSR) for weighted
        Node2vec, split like the graph's blocks; borrowed like the graph."""
        w = np.ascontiguousarray(w, dtype=np.float32) if not hasattr(w, "data_ptr") else w
        for b in range(len(self.vblocks) - 1):
            e0, e1 = int(self.eblocks[b]), int(self.eblocks[b + 1])
            bw = w[e0:e1]
            self._keep.append(bw)
            self._check(self.L.gw_host_weights(self.h, b, _ptr(bw) if e1 > e0 else ctypes.c_void_p(0)))
        self._keep.append(w)

    def set_device_weights(self, d_w_ptr):
        self._check(self.L.gw_device_weights(self.h, ctypes.c_void_p(d_w_ptr)))

    def set_device_graph(self, nverts, nedges, d_beg_ptr, d_csr_ptr):
        self.set_graph_meta(nverts, nedges, [0, nverts], [0, nedges])
        self._check(self.L.gw_device_graph(self.h, ctypes.c_void_p(d_beg_ptr), ctypes.c_void_p(d_csr_ptr)))

    def cache_reset(self):
        self._check(self.L.gw_cache_reset(self.h))

    # -- walks
    def init_walkers(self, algo=None, walkpersource=None, seed=None, first=0, count=None):
        """The whole walker population, or the shard of walker ids
        [first, first+count) of it (gw_init_walker_range)."""
        algo = self.cfg.algorithm if algo is None else algo
        wps = self.cfg.walkpersource if walkpersource is None else walkpersource
        seed = self.cfg.seed if seed is None else seed
        self.cfg.algorithm, self.cfg.walkpersource, self.cfg.seed = algo, wps, seed
        if first == 0 and count is None:
            self._check(self.L.gw_init_walkers(self.h, algo, wps, seed))
        else:
            self._check(self.L.gw_init_walker_range(self.h, algo, wps, seed, first,
                                                    0xFFFFFFFFFFFFFFFF if count is None else count))

    def run(self, policy=_abi.GW_POLICY_PLAIN) -> dict:
        st = GwStats()
        self._check(self.L.gw_run(self.h, policy, ctypes.byref(st)))
        return st.as_dict()

    def num_walkers(self) -> int:
        n = ctypes.c_uint64()
        self._check(self.L.gw_num_walkers(self.h, ctypes.byref(n)))
        return int(n.value)

    def paths(self, first=0, n=None):
        n = self.num_walkers() - first if n is None else n
        stride = self.cfg.maxhops + 1
        out = np.zeros((n, stride), dtype=np.uint32)
        lens = np.zeros(n, dtype=np.uint32)
        self._check(self.L.gw_get_paths(self.h, first, n, _ptr(out), _ptr(lens)))
        return out, lens

    def hashes(self, first=0, n=None):
        n = self.num_walkers() - first if n is None else n
        out = np.zeros(n, dtype=np.uint64)
        self._check(self.L.gw_path_hashes(self.h, first, n, _ptr(out)))
        return out

    def checksum(self):
        hs, steps = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.L.gw_checksum(self.h, ctypes.byref(hs), ctypes.byref(steps)))
        return int(hs.value), int(steps.value)

    def bucket_counts(self):
        nb = len(self.vblocks) - 1
        out = np.zeros(nb * nb, dtype=np.uint32)
        self._check(self.L.gw_bucket_counts(self.h, _ptr(out)))
        return out.reshape(nb, nb)


class DeviceGraph:
    """CSR built on the device (gw_rmat_csr, or gw_edges_csr through
    ``from_edges``); frees itself."""

    def __init__(self, scale, nverts=None, nsamples=None, edgefactor=16, abc=(0.57, 0.19, 0.19), seed=1,
                 symmetric=True, target_edges=0):
        L = _abi.load()
        self.L = L
        self.beg_ptr = self.csr_ptr = None
        nverts = (1 << scale) if nverts is None else nverts
        nsamples = (edgefactor << scale) if nsamples is None else nsamples
        a, b, c = abc
        thr = [int(a * 4294967296.0), int((a + b) * 4294967296.0), int((a + b + c) * 4294967296.0)]
        thr = (ctypes.c_uint32 * 3)(*[min(t, 0xFFFFFFFF) for t in thr])
        db, dc, ne = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        st = L.gw_rmat_csr(scale, nverts, nsamples, thr, seed, 1 if symmetric else 0, target_edges,
                           ctypes.byref(db), ctypes.byref(dc), ctypes.byref(ne))
        if st != 0:
            raise GwError(st, "gw_rmat_csr failed")
        self.nverts, self.nedges = nverts, int(ne.value)
        self.beg_ptr, self.csr_ptr = db.value, dc.value

    @classmethod
    def web(cls, scale, nverts, dmin=6.0, tail=1.1, max_degree=65536, local_permille=800, window=65536,
            abc=(0.57, 0.19, 0.19), seed=1, target_edges=0):
        """Web-shaped locality-ordered graph built on the device by gw_web_csr:
        power-law out-degrees (P(D >= d) = (d/dmin)^-tail), local edges within
        +-window of the source, the rest to R-MAT-distributed destinations."""
        L = _abi.load()
        self = cls.__new__(cls)
        self.L = L
        self.beg_ptr = self.csr_ptr = None
        a, b, c = abc
        thr = [int(a * 4294967296.0), int((a + b) * 4294967296.0), int((a + b + c) * 4294967296.0)]
        thr = (ctypes.c_uint32 * 3)(*[min(t, 0xFFFFFFFF) for t in thr])
        db, dc, ne = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        st = L.gw_web_csr(scale, nverts, thr, dmin, tail, max_degree, local_permille, window, seed, target_edges,
                          ctypes.byref(db), ctypes.byref(dc), ctypes.byref(ne))
        if st != 0:
            raise GwError(st, "gw_web_csr failed")
        self.nverts, self.nedges = nverts, int(ne.value)
        self.beg_ptr, self.csr_ptr = db.value, dc.value
        return self

    @classmethod
    def from_edges(cls, src, dst, nverts=0, symmetric=False, sort=True, dedup=False):
        """CSR of the edge list (src[i], dst[i]) built on the device by
        gw_edges_csr (the reference converter plus its neighbour sort,
        preprocess/graph_converter.hpp:286-449, preprocess/precompute.hpp:42-133).
        src / dst: u32 numpy arrays (host) or objects with ``data_ptr()``
        (device tensors of 4-byte ints).  nverts 0 takes the largest id + 1."""
        L = _abi.load()
        self = cls.__new__(cls)
        self.L = L
        self.beg_ptr = self.csr_ptr = None
        keep = []

        def ptr(a):
            if hasattr(a, "data_ptr"):
                if a.element_size() != 4 or not a.is_contiguous():
                    raise ValueError("edge arrays must be contiguous 4-byte integers")
                return a.data_ptr(), a.numel()
            a = np.ascontiguousarray(a, dtype=np.uint32)
            keep.append(a)
            return a.ctypes.data, a.size

        ps, n = ptr(src)
        pd, nd = ptr(dst)
        if n != nd:
            raise ValueError("src and dst differ in length")
        flags = ((_abi.GW_EDGES_SYMMETRIC if symmetric else 0) | (_abi.GW_EDGES_SORT if sort else 0) |
                 (_abi.GW_EDGES_DEDUP if dedup else 0))
        db, dc, ne, nv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint32()
        st = L.gw_edges_csr(ctypes.c_void_p(ps), ctypes.c_void_p(pd), n, nverts, flags, ctypes.byref(db),
                            ctypes.byref(dc), ctypes.byref(ne), ctypes.byref(nv))
        if st != 0:
            raise GwError(st, "gw_edges_csr failed")
        self.nverts, self.nedges = int(nv.value), int(ne.value)
        self.beg_ptr, self.csr_ptr = db.value, dc.value
        return self

    def split(self, mode=_abi.GW_SPLIT_REFERENCE, param=1024 << 20, cap=1 << 16):
        """Block split points (vblocks u32, eblocks u64) from the resident offsets."""
        return split_blocks_device(ctypes.c_void_p(self.beg_ptr), self.nverts, mode, param, cap)

    def to_host(self, pinned=False):
        """Copy to host numpy arrays (or pinned torch tensors)."""
        if pinned:
            import torch
            beg = torch.empty(self.nverts + 1, dtype=torch.int64, pin_memory=True)
            csr = torch.empty(max(self.nedges, 1), dtype=torch.int32, pin_memory=True)
            dst_b, dst_c = beg.data_ptr(), csr.data_ptr()
        else:
            beg = np.empty(self.nverts + 1, dtype=np.uint64)
            csr = np.empty(max(self.nedges, 1), dtype=np.uint32)
            dst_b, dst_c = beg.ctypes.data, csr.ctypes.data
        st = self.L.gw_memcpy(ctypes.c_void_p(dst_b), ctypes.c_void_p(self.beg_ptr), (self.nverts + 1) * 8)
        st |= self.L.gw_memcpy(ctypes.c_void_p(dst_c), ctypes.c_void_p(self.csr_ptr), self.nedges * 4)
        if st != 0:
            raise GwError(-2, "device graph copy failed")
        if not pinned:
            csr = csr[: self.nedges]
        return beg, csr

    def free(self):
        if self.beg_ptr:
            self.L.gw_device_free(ctypes.c_void_p(self.beg_ptr))
            self.L.gw_device_free(ctypes.c_void_p(self.csr_ptr))
            self.beg_ptr = self.csr_ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def split_blocks_device(beg, nverts, mode=_abi.GW_SPLIT_REFERENCE, param=1024 << 20, cap=1 << 16):
    """gw_split_blocks: the reference splitter (param = block size in bytes,
    preprocess/split.hpp:15-87) or equal edge mass (param = block count), run
    on the device over offsets in host (numpy) or device memory (a pointer)."""
    L = _abi.load()
    if isinstance(beg, np.ndarray):
        beg = np.ascontiguousarray(beg, dtype=np.uint64)
        p = ctypes.c_void_p(beg.ctypes.data)
    else:
        p = beg
    vb = np.zeros(cap + 1, dtype=np.uint32)
    eb = np.zeros(cap + 1, dtype=np.uint64)
    nb = ctypes.c_uint32()
    st = L.gw_split_blocks(p, nverts, mode, param, ctypes.c_void_p(vb.ctypes.data), ctypes.c_void_p(eb.ctypes.data),
                           cap, ctypes.byref(nb))
    if st != 0:
        raise GwError(st, "gw_split_blocks failed (%d blocks)" % nb.value)
    k = int(nb.value)
    return vb[: k + 1].copy(), eb[: k + 1].copy()


def sa_choose_blocks(counts, cached, k, seed=42, call=0):
    """gw_sa_choose_blocks: SOWalker's annealed block set (engine/schedule.hpp:455-593)
    computed on the device from the nb x nb (prev, cur) walker counts, the
    resident blocks and the slot count k."""
    L = _abi.load()
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    nb = counts.shape[0]
    cached = np.ascontiguousarray(cached, dtype=np.uint32)
    out = np.zeros(max(min(k, nb), 1), dtype=np.uint32)
    st = L.gw_sa_choose_blocks(ctypes.c_void_p(counts.ctypes.data), nb,
                               ctypes.c_void_p(cached.ctypes.data if cached.size else 0), cached.size, k, seed, call,
                               ctypes.c_void_p(out.ctypes.data))
    if st != 0:
        raise GwError(st, "gw_sa_choose_blocks failed")
    return out[: min(k, nb)]


def plain_choose_block(counts, cached, nslots, zero_threshold=0):
    """gw_plain_choose_block: GOWalker's block choice (max_choose_blocks,
    engine/schedule.hpp:70-138) as the device takes it, from the nb x nb
    (prev, cur) walker counts, the scheduler's cached list and the slot count.
    Returns (action, block, position)."""
    L = _abi.load()
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    nb = counts.shape[0]
    cached = np.ascontiguousarray(cached, dtype=np.uint32)
    out = np.zeros(3, dtype=np.int32)
    st = L.gw_plain_choose_block(ctypes.c_void_p(counts.ctypes.data), nb,
                                 ctypes.c_void_p(cached.ctypes.data if cached.size else 0), cached.size, nslots,
                                 zero_threshold, ctypes.c_void_p(out.ctypes.data))
    if st != 0:
        raise GwError(st, "gw_plain_choose_block failed")
    return int(out[0]), int(out[1]), int(out[2])

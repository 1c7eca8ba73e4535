"""GOWalker's on-disk graph format and block splitting.

Files (written and read exactly as the reference does):
  <base>.beg   u64 x (V+1) absolute CSR offsets
  <base>.csr   u32 x E     neighbour ids, sorted per vertex
  <base>.wht   f32 x E     edge weights (weighted datasets only)
  <base>.meta  16 packed bytes: u32 nvertices, u64 nedges, u32 min_vert
               (preprocess/graph_converter.hpp finalize(), util/io.hpp:29-42)
  <dir>/sowalker_<MB>/<name>_<MB>MB.vert.blocks  u32 x (nblocks+1)
  <dir>/sowalker_<MB>/<name>_<MB>MB.edge.blocks  u64 x (nblocks+1)
               (util/util.hpp:148-165, preprocess/split.hpp:74-84)

Splitters:
  split_blocks            the reference rule (preprocess/split.hpp:15-87)
  split_equal_edge_mass   vertex ranges of (nearly) equal edge mass
"""
from __future__ import annotations

import os

import numpy as np


def block_paths(base: str, blocksize_mb: int):
    folder = os.path.join(os.path.dirname(base) or ".", "sowalker_%d" % blocksize_mb)
    name = os.path.basename(base)
    return (folder, os.path.join(folder, "%s_%dMB.vert.blocks" % (name, blocksize_mb)),
            os.path.join(folder, "%s_%dMB.edge.blocks" % (name, blocksize_mb)))


def write_dataset(base: str, beg: np.ndarray, csr: np.ndarray, min_vert: int = 0) -> None:
    np.asarray(beg, dtype=np.uint64).tofile(base + ".beg")
    np.asarray(csr, dtype=np.uint32).tofile(base + ".csr")
    meta = (np.uint32(len(beg) - 1).tobytes() + np.uint64(len(csr)).tobytes() + np.uint32(min_vert).tobytes())
    with open(base + ".meta", "wb") as f:
        f.write(meta)


def write_weights(base: str, w: np.ndarray) -> None:
    """<base>.wht: one float32 (real_t) per edge, aligned with <base>.csr
    (util/util.hpp:136-138)."""
    np.asarray(w, dtype=np.float32).tofile(base + ".wht")


def read_meta(base: str):
    raw = open(base + ".meta", "rb").read(16)
    if len(raw) != 16:
        raise ValueError("%s.meta: expected 16 bytes, found %d" % (base, len(raw)))
    nverts = int(np.frombuffer(raw[0:4], np.uint32)[0])
    nedges = int(np.frombuffer(raw[4:12], np.uint64)[0])
    min_vert = int(np.frombuffer(raw[12:16], np.uint32)[0])
    return nverts, nedges, min_vert


def load_dataset(base: str, mmap: bool = True):
    """beg, csr (memory-mapped by default) with size checks against .meta."""
    nverts, nedges, _ = read_meta(base)
    if mmap:
        beg = np.memmap(base + ".beg", np.uint64, "r")
        csr = np.memmap(base + ".csr", np.uint32, "r") if nedges else np.zeros(0, np.uint32)
    else:
        beg = np.fromfile(base + ".beg", np.uint64)
        csr = np.fromfile(base + ".csr", np.uint32)
    if len(beg) != nverts + 1:
        raise ValueError("%s.beg holds %d offsets, .meta says %d vertices" % (base, len(beg), nverts))
    if len(csr) != nedges:
        raise ValueError("%s.csr holds %d ids, .meta says %d edges" % (base, len(csr), nedges))
    return beg, csr


def write_blocks(base: str, blocksize_mb: int, vblocks, eblocks) -> None:
    folder, vb, eb = block_paths(base, blocksize_mb)
    os.makedirs(folder, exist_ok=True)
    np.asarray(vblocks, dtype=np.uint32).tofile(vb)
    np.asarray(eblocks, dtype=np.uint64).tofile(eb)


def load_blocks(base: str, blocksize_mb: int):
    """vblocks, eblocks from the block files (engine/cache.hpp:150-158), checked
    for monotonicity."""
    _, vb, eb = block_paths(base, blocksize_mb)
    v = np.fromfile(vb, np.uint32)
    e = np.fromfile(eb, np.uint64)
    if len(v) != len(e) or len(v) < 2:
        raise ValueError("block files disagree: %d vertex and %d edge split points" % (len(v), len(e)))
    if np.any(np.diff(v.astype(np.int64)) < 0) or np.any(np.diff(e.astype(np.int64)) < 0):
        raise ValueError("block split points are not monotone")
    return v, e


def split_blocks(beg: np.ndarray, block_size: int):
    """The reference splitter (preprocess/split.hpp:15-87): a block is cut
    when its edges would exceed block_size/4 (the cut goes one vertex back) or
    its vertices reach block_size/8."""
    max_nedges = block_size // 4
    max_nverts = block_size // 8
    nv = len(beg)
    b = np.asarray(beg, dtype=np.int64)
    vblocks, eblocks = [0], [0]
    cur_pos, rd_edges = 0, 0
    for v in range(nv):
        if b[v] - rd_edges > max_nedges:
            cur_pos = v - 1
            vblocks.append(cur_pos)
            rd_edges = int(b[v - 1])
            eblocks.append(rd_edges)
        elif v - cur_pos >= max_nverts:
            cur_pos = v
            vblocks.append(cur_pos)
            rd_edges = int(b[v])
            eblocks.append(rd_edges)
    vblocks.append(nv - 1)
    eblocks.append(int(b[nv - 1]))
    return np.array(vblocks, dtype=np.uint32), np.array(eblocks, dtype=np.uint64)


def split_equal_edge_mass(beg: np.ndarray, nblocks: int):
    """Vertex-range blocks of nearly equal edge mass: block k ends at the first
    vertex whose offset reaches k*E/nblocks (at least one vertex per block)."""
    beg = np.asarray(beg)
    V = len(beg) - 1
    E = int(beg[-1])
    if nblocks < 1 or nblocks > V:
        raise ValueError("need 1 <= nblocks <= nvertices")
    targets = np.array([k * E // nblocks for k in range(1, nblocks)], dtype=np.uint64)
    cuts = np.searchsorted(beg[:-1], targets, side="left").astype(np.int64)
    cuts = np.maximum.accumulate(np.clip(cuts, 1, max(V - 1, 1)))
    vb = np.concatenate([[0], cuts, [V]]).astype(np.int64)
    vb = np.maximum.accumulate(vb).astype(np.uint32)
    eb = beg[vb.astype(np.int64)].astype(np.uint64)
    return vb, eb

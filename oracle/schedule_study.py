"""Block-schedule study on the C3 workload's shape -- TEST INFRASTRUCTURE.

Walks do not depend on the block schedule, so the blocks every walker will
need are fixed by the oracle's walks (gw_oracle.c oracle_walk_reqs); any
block policy can then be replayed on the CPU over the same walks and its
block loads counted exactly (oracle_sched_replay is checked against the
engine's own runs by tests/test_gpu_ooc.py).  This script compares, on a
C3-shaped graph (directed R-MAT (0.57, 0.19, 0.19, 0.05) with C3's vertex,
sample and edge counts scaled by 2^(scale-26), 64 equal-edge-mass blocks,
Node2vec p=0.5 q=2 length 80, one walker per vertex, walk seed 42):

  plain        GOWalker's block choice (engine/schedule.hpp:70-138)
  clairvoyant  the block whose load gives the most steps this iteration,
               computed exactly from the walks (no forecast can do better
               for a one-iteration objective)
  evict-need   GOWalker's choice, evicting the cached block the fewest
               waiting walkers need within their next four blocks (exact)
  evict-incident  GOWalker's choice, evicting the cached block with the
               fewest walkers at or from it now (what the learned policy's
               forecast refines)
  evict-usage  GOWalker's choice, evicting the block with the lowest running
               average of steps taken in it
  evict-lru    GOWalker's choice, evicting the block unused the longest
  zero rule    GOWalker's choice, loads stopped where the reference's zero
               threshold (blocksize/3072 walkers, apps/Node2vec.cu:100-108)
               stops them; the rest would read mapped host memory

    python oracle/schedule_study.py [--scale 17] [--slots 12]
    python oracle/schedule_study.py --shape c5 --scale 19 --blocks 256 --slots 77

`--shape c5` replays the web-shaped C5 graph instead (256 blocks, a cache of
about 30 % of them in C5).
"""
import argparse
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import oracle as O  # noqa: E402


def c3_shaped_graph(scale):
    f = 2.0 ** (scale - 26)
    V, ns, target = int(41_600_000 * f), int(2_600_000_000 * f), int(1_470_000_000 * f)
    src, dst = O.rmat_edges(scale, 0, ns, seed=1)
    keep = (src < V) & (dst < V)
    beg, csr = O.build_csr(V, src[keep], dst[keep], symmetric=False)
    U = len(csr)
    if U > target:  # thin evenly to exactly `target` edges, as the device generator does
        k = U - target
        i = np.arange(U, dtype=np.int64)
        m = ((i + 1) * k // U) == (i * k // U)
        s = np.repeat(np.arange(V, dtype=np.int64), np.diff(beg.astype(np.int64)))[m]
        csr = csr[m]
        beg = np.zeros(V + 1, dtype=np.uint64)
        beg[1:] = np.cumsum(np.bincount(s, minlength=V))
    return beg, csr


def c5_shaped_graph(scale):
    """The C5 (web-shaped) graph's construction at 2^(scale-28) of its size:
    power-law out-degrees (P(D >= d) = (d/6.8)^-1.1, cap 65,536), 80 % of the
    edges within +-65,536 of the source (the window scaled likewise, at
    least 64), the rest to R-MAT destinations."""
    f = 2.0 ** (scale - 28)
    V = int(133_600_000 * f)
    window = max(64, int(65_536 * f))
    return O.web_graph(scale, V, dmin=6.8, tail=1.1, max_degree=65536, local_permille=800, window=window)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", choices=["c3", "c5"], default="c3")
    ap.add_argument("--scale", type=int, default=17)
    ap.add_argument("--blocks", type=int, default=64)
    ap.add_argument("--slots", type=int, default=12)
    ap.add_argument("--no-clairvoyant", action="store_true", help="skip the slow exact-yield policy")
    a = ap.parse_args()
    t0 = time.time()
    beg, csr = c3_shaped_graph(a.scale) if a.shape == "c3" else c5_shaped_graph(a.scale)
    V, E = len(beg) - 1, len(csr)
    vb, eb = O.split_equal_edge_mass(beg, a.blocks)
    cfg = O.make_cfg(algo=0, maxhops=80, p=0.5, q=2.0, seed=42)
    reqs, nent = O.walk_requirements(beg, csr, cfg, vb, 0, V)
    st = O.walk(beg, csr, cfg, 0, min(V, 200_000), paths=False)["stats"]
    zc_bytes = 32.0 * (st["trials"] + st["search_sectors"]) / st["steps"]  # csr sectors a mapped step reads
    blk_bytes = 4.0 * E / a.blocks
    zt = int(blk_bytes * 1.0 / 3072)  # the reference's threshold for a block of this size
    print("%s shape at scale %d: V=%d E=%d, %d blocks, %d slots, %d walkers (%.0fs to build)"
          % (a.shape.upper(), a.scale, V, E, a.blocks, a.slots, V, time.time() - t0))
    base = O.sched_study(reqs, nent, a.blocks, a.slots, policy=0)
    tot = base["steps"]
    rows = [("plain", base)]
    if not a.no_clairvoyant:
        rows.append(("clairvoyant", O.sched_study(reqs, nent, a.blocks, a.slots, policy=1)))
    rows.append(("evict-need", O.sched_study(reqs, nent, a.blocks, a.slots, policy=2)))
    rows.append(("evict-incident", O.sched_study(reqs, nent, a.blocks, a.slots, policy=3)))
    rows.append(("evict-usage", O.sched_study(reqs, nent, a.blocks, a.slots, policy=4)))
    rows.append(("evict-lru", O.sched_study(reqs, nent, a.blocks, a.slots, policy=5)))
    rows.append(("zero rule (%d walkers)" % zt, O.sched_study(reqs, nent, a.blocks, a.slots, zero_threshold=zt)))
    print("| policy | block loads | vs plain | steps by mapped reads | host-link bytes vs plain |")
    print("|---|---|---|---|---|")
    b0 = base["loads"] * blk_bytes
    for name, r in rows:
        b = r["loads"] * blk_bytes + r["zc_steps"] * zc_bytes
        print("| %s | %d | %.3f | %.2f%% | %.3f |" % (name, r["loads"], r["loads"] / base["loads"],
                                                     100.0 * r["zc_steps"] / tot, b / b0))
    print("(block bytes uncompressed %.0f; mapped reads %.0f B per step: candidate and N(prev) sectors)"
          % (blk_bytes, zc_bytes))


if __name__ == "__main__":
    main()

"""Bit-exact parity at the sizes of the benchmark workloads.

  C1  Node2vec p=2 q=0.5 length 80 on R-MAT scale 20 (in-core): every walker's
      path, length and hash against the oracle.
  C2  SOPR alpha 0.2, termination 0.15, length 20, 4 walkers per vertex on
      R-MAT scale 24 (in-core, 67 M walkers): the whole run's sum of path
      hashes and step count against the oracle's (tests/golden/
      config_checksums.json, made by make_config_checksums.py on the CPU),
      hashes of a random sample of 2^20 walkers, and full paths of 1024
      random runs of 1024 walkers.
  C3  out-of-core Node2vec p=0.5 q=2 length 80 on the 41.6 M-vertex,
      1.47 B-edge R-MAT graph, 64 blocks, 1.5 GB cache, compressed blocks and
      prefetch, under the learned and the plain block policy: every walker's
      hash equal to the in-core run's on the same graph, and full paths of
      1024 random runs of 1024 walkers (2^20 walkers) against the oracle.
The graphs come from the device generator; the C1 and C2 graphs are checked
against the oracle's R-MAT restatement by their SHA-256."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "config_checksums.json")))


def digest(beg, csr):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(beg, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(csr, dtype=np.uint32).tobytes())
    return h.hexdigest()


def cfg_of(oracle, w):
    return oracle.make_cfg(algo=w["algo"], maxhops=w["maxhops"], p=w["p"], q=w["q"], alpha=w["alpha"],
                           term_prob=w["term"], seed=w["seed"], wps=w["wps"])


def random_runs(rng, n, runs=1024, width=1024):
    starts = np.sort(rng.choice(n // width, runs, replace=False)) * width
    return [int(s) for s in starts]


def test_c1_every_walker_vs_oracle(gw, oracle):
    w = GOLDEN["c1"]
    dg = gw.DeviceGraph(w["scale"], edgefactor=w["ef"], seed=1, symmetric=True)
    beg, csr = dg.to_host()
    assert digest(beg, csr) == w["graph_sha256"]
    eng = gw.WalkEngine(algorithm=w["algo"], maxhops=w["maxhops"], p=w["p"], q=w["q"], seed=w["seed"],
                        walkpersource=w["wps"], record_paths=1)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(w["algo"], w["wps"], w["seed"])
    st = eng.run()
    P, L = eng.paths()
    H = eng.hashes()
    ref = oracle.walk(beg, csr, cfg_of(oracle, w), 0, w["walkers"], paths=True)
    assert np.array_equal(H, ref["hashes"])
    assert np.array_equal(L, ref["lens"])
    assert np.array_equal(P, ref["paths"])
    assert st["steps"] == ref["stats"]["steps"] == w["steps"] and st["trials"] == w["trials"]
    hs, steps = eng.checksum()
    assert str(hs) == w["path_hash_sum"] and steps == w["steps"]
    eng.close()
    dg.free()


def test_c2_whole_run_checksum_and_samples(gw, oracle):
    w = GOLDEN["c2"]
    dg = gw.DeviceGraph(w["scale"], edgefactor=w["ef"], seed=1, symmetric=True)
    beg, csr = dg.to_host()
    assert digest(beg, csr) == w["graph_sha256"]
    eng = gw.WalkEngine(algorithm=w["algo"], maxhops=w["maxhops"], alpha=w["alpha"], term_prob=w["term"],
                        seed=w["seed"], walkpersource=w["wps"], record_paths=1)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(w["algo"], w["wps"], w["seed"])
    st = eng.run()
    hs, steps = eng.checksum()
    assert str(hs) == w["path_hash_sum"] and steps == w["steps"] == st["steps"]
    assert st["trials"] == w["trials"] and st["walkers"] == w["walkers"]
    H = eng.hashes()
    cfg = cfg_of(oracle, w)
    rng = np.random.default_rng(2024)
    ids = np.sort(rng.choice(w["walkers"], 1 << 20, replace=False)).astype(np.uint32)
    assert np.array_equal(oracle.walk_ids(beg, csr, cfg, ids)["hashes"], H[ids])
    for s in random_runs(rng, w["walkers"]):
        P, L = eng.paths(s, 1024)
        r = oracle.walk(beg, csr, cfg, s, 1024, paths=True)
        assert np.array_equal(P, r["paths"]) and np.array_equal(L, r["lens"]), s
    eng.close()
    dg.free()


def test_c3_out_of_core_learned_and_plain(gw, oracle):
    sys.path.insert(0, ROOT)
    import bench
    from gowalker_b200.preprocess import split_equal_edge_mass
    wl = dict(bench.WORKLOADS["c3"])
    dg = bench.build_graph(gw, wl)
    beg_t, csr_t, beg, csr = bench.host_graph(dg)
    kw = dict(algorithm=0, maxhops=80, p=0.5, q=2.0, seed=42, walkpersource=1)
    inc = gw.WalkEngine(record_paths=0, **kw)
    inc.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    inc.init_walkers(0, 1, 42)
    st_in = inc.run()
    H = inc.hashes()
    inc.close()
    dg.free()
    vb, eb = split_equal_edge_mass(beg, wl["nblocks"])
    cfg = oracle.make_cfg(algo=0, maxhops=80, p=0.5, q=2.0, seed=42, wps=1)
    rng = np.random.default_rng(3)
    runs = random_runs(rng, len(H))
    for policy, paths in ((gw.GW_POLICY_LEARNED, 1), (gw.GW_POLICY_PLAIN, 0)):
        eng = gw.WalkEngine(record_paths=paths, cache_size=wl["cache"], prefetch=1, compress_blocks=1, **kw)
        eng.set_host_graph(beg_t, csr_t[: len(csr)], vb, eb)
        eng.init_walkers(0, 1, 42)
        st = eng.run(policy)
        assert st["block_loads"] > 64 and st["steps"] == st_in["steps"]
        assert np.array_equal(eng.hashes(), H), policy
        if paths:
            for s in runs:
                P, L = eng.paths(s, 1024)
                r = oracle.walk(beg, csr, cfg, s, 1024, paths=True)
                assert np.array_equal(P, r["paths"]) and np.array_equal(L, r["lens"]), s
                assert np.array_equal(H[s:s + 1024], r["hashes"]), s
        eng.close()

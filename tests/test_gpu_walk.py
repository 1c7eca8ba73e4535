"""GPU parity tests: the CUDA walk path (through the C ABI) against the oracle.

Bit-exact: paths, lengths and 64-bit path hashes are integer data, so every
comparison is equality.
"""
import ctypes
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")


def run_engine(gw, beg, csr, algo, maxhops, wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, seed=42, paths=True,
               init_mode=0, numwalks=0, blocks=None, **cfg):
    eng = gw.WalkEngine(algorithm=algo, maxhops=maxhops, p=p, q=q, alpha=alpha, term_prob=term, seed=seed,
                        walkpersource=wps, record_paths=1 if paths else 0, init_mode=init_mode,
                        numwalks=numwalks, cache_size=1 << 34, **cfg)
    vb, eb = (None, None) if blocks is None else blocks
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, wps, seed)
    st = eng.run()
    return eng, st


def oracle_cfg(O, algo, maxhops, wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, seed=42, init_mode=0, numwalks=0):
    return O.make_cfg(algo=algo, maxhops=maxhops, p=p, q=q, alpha=alpha, term_prob=term, seed=seed, wps=wps,
                      init_mode=init_mode, numwalks=numwalks)


def test_device_philox_matches_curand_and_oracle(oracle, tmp_path):
    so = tmp_path / "probe.so"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-shared", "-Xcompiler", "-fPIC",
                    "-I", os.path.join(ROOT, "gowalker_b200", "csrc"), "-o", str(so),
                    os.path.join(ROOT, "tests", "cuda", "philox_curand.cu")], check=True)
    L = ctypes.CDLL(str(so))
    n = 4096
    ours = np.zeros((n, 8), dtype=np.uint32)
    theirs = np.zeros((n, 8), dtype=np.uint32)
    seed, sub0 = 0x0123456789ABCDEF, (1 << 32) - 100
    assert L.probe_philox(ctypes.c_uint64(seed), ctypes.c_uint64(sub0), n, ours.ctypes.data_as(ctypes.c_void_p),
                          theirs.ctypes.data_as(ctypes.c_void_p)) == 0
    assert np.array_equal(ours, theirs)
    key = [seed & 0xFFFFFFFF, seed >> 32]
    for i in range(0, n, 257):
        sub = sub0 + i
        assert np.array_equal(oracle.philox([0, 0, sub & 0xFFFFFFFF, sub >> 32], key), ours[i, :4])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*_s8.npz"))))
def test_golden_fixtures(gw, path):
    z = np.load(path)
    eng, st = run_engine(gw, z["beg"], z["csr"], int(z["algo"]), int(z["maxhops"]), wps=int(z["wps"]),
                         p=float(z["p"]), q=float(z["q"]), alpha=float(z["alpha"]), seed=int(z["seed"]))
    P, L = eng.paths()
    assert np.array_equal(L, z["lens"])
    assert np.array_equal(P, z["paths"])
    assert np.array_equal(eng.hashes(), z["hashes"])
    assert st["steps"] == int(z["steps"])
    eng.close()


SWEEP = [
    # algo, scale, ef, symmetric, maxhops, wps, p, q, alpha, term
    (0, 11, 16, True, 40, 1, 2.0, 0.5, 0.2, 0.0),
    (0, 11, 16, True, 25, 2, 0.25, 4.0, 0.2, 0.0),
    (0, 11, 8, False, 30, 1, 1.0, 1.0, 0.2, 0.0),
    (1, 11, 16, True, 20, 4, 0.5, 2.0, 0.2, 0.15),
    (2, 10, 16, False, 20, 2, 0.5, 2.0, 0.35, 0.15),
    (1, 12, 4, True, 12, 1, 0.5, 2.0, 0.9, 0.0),
]


@pytest.mark.parametrize("case", SWEEP)
def test_sweep_vs_oracle(gw, oracle, case):
    algo, scale, ef, sym, maxhops, wps, p, q, alpha, term = case
    beg, csr = oracle.rmat_graph(scale, ef, seed=5, symmetric=sym)
    V = len(beg) - 1
    eng, st = run_engine(gw, beg, csr, algo, maxhops, wps, p, q, alpha, term, seed=1234)
    cfg = oracle_cfg(oracle, algo, maxhops, wps, p, q, alpha, term, seed=1234)
    ref = oracle.walk(beg, csr, cfg, 0, V * wps, paths=True)
    P, L = eng.paths()
    assert np.array_equal(L, ref["lens"])
    assert np.array_equal(P, ref["paths"])
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["steps"] == ref["stats"]["steps"]
    assert st["trials"] == ref["stats"]["trials"]
    hs, steps = eng.checksum()
    assert hs == int(ref["hashes"].astype(np.uint64).sum(dtype=np.uint64))
    eng.close()


@pytest.mark.parametrize("algo,init_mode", [(1, 1), (2, 1), (0, 2)])
def test_init_modes_vs_oracle(gw, oracle, algo, init_mode):
    beg, csr = oracle.rmat_graph(10, 16, seed=9)
    n = 3000
    eng, st = run_engine(gw, beg, csr, algo, 20, wps=1, term=0.15 if algo else 0.0, seed=77, init_mode=init_mode,
                         numwalks=n)
    cfg = oracle_cfg(oracle, algo, 20, 1, term=0.15 if algo else 0.0, seed=77, init_mode=init_mode, numwalks=n)
    ref = oracle.walk(beg, csr, cfg, 0, n, paths=True)
    P, L = eng.paths()
    assert np.array_equal(P, ref["paths"])
    assert np.array_equal(eng.hashes(), ref["hashes"])
    eng.close()


def test_launch_shape_and_graph_mode_invariance(gw, oracle):
    beg, csr = oracle.rmat_graph(12, 16, seed=2)
    V = len(beg) - 1
    base = None
    for grid in (0, 1, 7, 333):
        eng, _ = run_engine(gw, beg, csr, 0, 30, 1, 2.0, 0.5, paths=False, blockpergrid=grid)
        h = eng.hashes()
        eng.close()
        base = h if base is None else base
        assert np.array_equal(h, base)
    # device-resident graph gives the same walks as host blocks
    dg = gw.DeviceGraph(12, edgefactor=16, seed=2)
    b2, c2 = dg.to_host()
    assert np.array_equal(b2, beg) and np.array_equal(c2, csr)
    eng = gw.WalkEngine(algorithm=0, maxhops=30, p=2.0, q=0.5, seed=42, record_paths=0)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(0, 1, 42)
    eng.run()
    assert np.array_equal(eng.hashes(), base)
    eng.close()
    dg.free()


def test_multiblock_host_graph_incore(gw, oracle):
    """Blocks that all fit the cache are assembled into one resident CSR."""
    beg, csr = oracle.rmat_graph(11, 16, seed=4)
    vb, eb = oracle.split_equal_edge_mass(beg, 5)
    V = len(beg) - 1
    eng, st = run_engine(gw, beg, csr, 0, 20, 1, 2.0, 0.5, blocks=(vb, eb))
    ref = oracle.walk(beg, csr, oracle_cfg(oracle, 0, 20, 1, 2.0, 0.5), 0, V, paths=False)
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["h2d_bytes"] == (V + 1) * 8 + len(csr) * 4
    eng.close()


@pytest.mark.parametrize("sym,cap,target", [(True, None, 0), (False, 3000, 0), (True, None, 50000)])
def test_device_rmat_matches_oracle(gw, oracle, sym, cap, target):
    scale = 12
    V = (1 << scale) if cap is None else cap
    n = 16 << scale
    src, dst = oracle.rmat_edges(scale, 0, n, seed=3)
    keep = (src < V) & (dst < V)
    beg, csr = oracle.build_csr(V, src[keep], dst[keep], symmetric=sym)
    if target:
        keys = (np.repeat(np.arange(V, dtype=np.uint64), np.diff(beg.astype(np.int64))) << np.uint64(32)) | csr
        U, k = len(keys), len(keys) - target
        i = np.arange(U, dtype=np.uint64)
        keep_i = (i * np.uint64(k)) // np.uint64(U) == ((i + np.uint64(1)) * np.uint64(k)) // np.uint64(U)
        keys = keys[keep_i]
        s = (keys >> np.uint64(32)).astype(np.int64)
        csr = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        beg = np.zeros(V + 1, dtype=np.uint64)
        beg[1:] = np.cumsum(np.bincount(s, minlength=V))
    dg = gw.DeviceGraph(scale, nverts=V, nsamples=n, seed=3, symmetric=sym, target_edges=target)
    b2, c2 = dg.to_host()
    dg.free()
    assert np.array_equal(b2, beg)
    assert np.array_equal(c2, csr)


def test_corrupt_graph_is_rejected(gw, oracle):
    beg, csr = oracle.rmat_graph(9, 8, seed=1)
    bad = csr.copy()
    bad[len(bad) // 2] = len(beg) + 5  # neighbour id beyond nverts
    eng = gw.WalkEngine(algorithm=0, maxhops=10, cache_size=1 << 30)
    eng.set_host_graph(beg, bad)
    eng.init_walkers(0, 1, 1)
    with pytest.raises(gw.GwError) as e:
        eng.run()
    assert e.value.status == -7
    # the handle stays usable with a good graph
    eng.set_host_graph(beg, csr)
    eng.init_walkers(0, 1, 1)
    eng.run()
    eng.close()


def test_c1_node2vec_sample_vs_oracle(gw, oracle):
    """Scale-20 R-MAT, Node2vec p=2 q=0.5 length 80 (the in-core C1 workload):
    full GPU run, first 20k walkers and a strided sample checked against the oracle."""
    dg = gw.DeviceGraph(20, edgefactor=16, seed=1)
    beg, csr = dg.to_host()
    V = dg.nverts
    eng = gw.WalkEngine(algorithm=0, maxhops=80, p=2.0, q=0.5, seed=42, record_paths=0)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(0, 1, 42)
    st = eng.run()
    H = eng.hashes()
    cfg = oracle_cfg(oracle, 0, 80, 1, 2.0, 0.5, seed=42)
    ref = oracle.walk(beg, csr, cfg, 0, 20000, paths=False)
    assert np.array_equal(H[:20000], ref["hashes"])
    for w0 in range(20000, V, 97531):
        r = oracle.walk(beg, csr, cfg, w0, 64, paths=False)
        assert np.array_equal(H[w0:w0 + 64], r["hashes"])
    assert st["walkers"] == V
    hs, _ = eng.checksum()
    assert hs == int(H.sum(dtype=np.uint64))
    eng.close()
    dg.free()


def hub_ring_graph(leaves):
    """Vertex 0 joined to every leaf 1..leaves; leaf i also joined to its ring
    neighbours.  A walker stepping leaf -> hub has prev degree 3 next to a hub
    of degree `leaves`: the hard, position-decided cooperative steps, with runs
    of N(prev) at every offset of N(hub)."""
    V = leaves + 1
    i = np.arange(1, V, dtype=np.int64)
    nxt = np.where(i == leaves, 1, i + 1)
    src = np.concatenate([np.zeros(leaves, np.int64), i, i, nxt])
    dst = np.concatenate([i, np.zeros(leaves, np.int64), nxt, i])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    beg = np.zeros(V + 1, dtype=np.uint64)
    beg[1:] = np.cumsum(np.bincount(src, minlength=V))
    return beg, dst.astype(np.uint32)


HUB_CASES = [
    # algo, leaves, p, q, alpha
    (1, 60000, 0.5, 2.0, 0.2),     # SOPR: ~4000 trials per hub step
    (2, 5000, 0.5, 2.0, 0.6),      # SOSR, smaller hub
    (0, 60000, 0.05, 20.0, 0.2),   # Node2vec: only the run of prev accepts often
    (0, 60000, 0.05, 0.5, 0.2),    # Node2vec: not-found bound above the min bound
    (1, 1, 0.5, 2.0, 0.2),         # hub of degree 1
]


@pytest.mark.parametrize("case", HUB_CASES)
def test_hub_steps_vs_oracle(gw, oracle, case):
    algo, leaves, p, q, alpha = case
    beg, csr = hub_ring_graph(leaves)
    n = 3000
    eng, st = run_engine(gw, beg, csr, algo, 9, wps=1, p=p, q=q, alpha=alpha, seed=99, init_mode=2, numwalks=n)
    cfg = oracle_cfg(oracle, algo, 9, 1, p, q, alpha, seed=99, init_mode=2, numwalks=n)
    ref = oracle.walk(beg, csr, cfg, 0, n, paths=True, nthreads=8)
    P, L = eng.paths()
    assert np.array_equal(L, ref["lens"])
    assert np.array_equal(P, ref["paths"])
    assert st["trials"] == ref["stats"]["trials"]
    if leaves > 1000:
        assert st["coop_small_steps"] > 0
    eng.close()


def test_c2_sopr_sample_vs_oracle(gw, oracle):
    """Scale-24 symmetrised R-MAT, SOPR alpha 0.2, termination 0.15, length 20,
    4 walkers per vertex (the in-core C2 workload): full GPU run, a strided
    sample of walkers checked against the oracle."""
    dg = gw.DeviceGraph(24, edgefactor=16, seed=1, symmetric=True)
    beg, csr = dg.to_host()
    V = dg.nverts
    eng = gw.WalkEngine(algorithm=1, maxhops=20, alpha=0.2, term_prob=0.15, seed=42, walkpersource=4,
                        record_paths=0)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(1, 4, 42)
    st = eng.run()
    H = eng.hashes()
    cfg = oracle_cfg(oracle, 1, 20, 4, alpha=0.2, term=0.15, seed=42)
    for w0 in range(0, 4 * V - 512, 4 * V // 40):
        r = oracle.walk(beg, csr, cfg, w0, 512, paths=False, nthreads=8)
        assert np.array_equal(H[w0:w0 + 512], r["hashes"])
    assert st["walkers"] == 4 * V
    assert st["coop_small_steps"] > 0 and st["coop_large_steps"] > 0
    eng.close()
    dg.free()


def _ru32(x):
    """Smallest float32 >= the float64 x."""
    f = np.float32(x)
    return f if float(f) >= x else np.nextafter(f, np.float32(np.inf))


def test_windowed_rand_bounds_match_search(tmp_path):
    """The cooperative step's integer rand bounds (an estimate checked on an
    eight-wide window) equal the exhaustive binary search's."""
    so = tmp_path / "rb.so"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-shared", "-Xcompiler", "-fPIC",
                    "-I", os.path.join(ROOT, "gowalker_b200", "csrc"), "-o", str(so),
                    os.path.join(ROOT, "tests", "cuda", "rand_bounds_check.cu")], check=True)
    L = ctypes.CDLL(str(so))
    rng = np.random.default_rng(7)
    rows = []
    # SOPR thresholds as the kernels form them, from (deg, prev_deg, alpha)
    for _ in range(3000):
        deg = int(rng.integers(1, 1 << int(rng.integers(1, 32))))
        pdeg = int(rng.integers(1, 1 << int(rng.integers(1, 24))))
        alpha = float(rng.choice([0.0, 1.0, float(np.float32(rng.random()))]))
        tp = (1.0 - alpha) / deg
        inv_deg = np.float32(tp)
        s = np.float32(inv_deg + np.float32(np.float32(alpha) / np.float32(pdeg)))
        rows.append((inv_deg, s, _ru32(tp), 0, 0))
    sopr = np.array(rows, dtype=np.float32)
    # Node2vec constants from (p, q), plus raw extremes
    rows = []
    for _ in range(3000):
        p, q = (np.float32(2.0 ** rng.uniform(-20, 20)) for _ in range(2))
        ip, iq = np.float32(1) / p, np.float32(1) / q
        mx = max(ip, max(iq, np.float32(1)))
        mn = min(ip, min(iq, np.float32(1)))
        rows.append((mx, mn, ip, iq, 0))
    for _ in range(1000):
        mx = np.float32(2.0 ** rng.uniform(-140, 100))
        rows.append((mx, np.float32(mx * rng.random()), np.float32(mx * rng.uniform(0, 2)),
                     np.float32(mx * rng.random()), 0))
    n2v = np.array(rows, dtype=np.float32)
    for flag, thr in ((1, sopr), (0, n2v)):
        n = len(thr)
        fast = np.zeros(4 * n, dtype=np.uint32)
        slow = np.zeros(4 * n, dtype=np.uint32)
        assert L.check_bounds(flag, thr.ctypes.data_as(ctypes.c_void_p), n, fast.ctypes.data_as(ctypes.c_void_p),
                              slow.ctypes.data_as(ctypes.c_void_p)) == 0
        assert np.array_equal(fast, slow), np.nonzero(fast != slow)[0][:10]


def test_path_rows_zero_padded_after_longer_walks(gw, oracle):
    """gw_get_paths pads each row past the walk's length with zeros, also when
    the device rows still hold an earlier, longer run's vertices."""
    beg, csr = oracle.rmat_graph(11)
    V = len(beg) - 1
    eng = gw.WalkEngine(algorithm=1, maxhops=20, alpha=0.2, term_prob=0.0, seed=4, walkpersource=1, record_paths=1,
                        cache_size=1 << 34)
    eng.set_host_graph(beg, csr)
    eng.init_walkers(1, 1, 4)
    eng.run()
    eng.set_config(term_prob=0.3)
    eng.init_walkers(1, 1, 4)
    eng.run()
    P, L = eng.paths()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=1, maxhops=20, alpha=0.2, term_prob=0.3, seed=4), 0, V)
    assert (L < 21).any()
    assert np.array_equal(L, ref["lens"]) and np.array_equal(P, ref["paths"])
    eng.close()


@pytest.mark.parametrize("algo,maxhops,term,p,q,wps", [(0, 30, 0.0, 2.0, 0.5, 1), (1, 20, 0.15, 0.5, 2.0, 2),
                                                      (2, 15, 0.15, 0.5, 2.0, 1), (0, 25, 0.0, 0.05, 20.0, 1)])
def test_one_launch_per_hop_same_walks(gw, oracle, algo, maxhops, term, p, q, wps):
    """The plain one-launch-per-hop form (GW_LAUNCH_PER_HOP: a thread per
    walker, one launch per hop, state in memory) walks exactly the walks of
    the persistent work-stealing kernel and of the oracle: paths, lengths,
    hashes, steps and trials."""
    beg, csr = oracle.rmat_graph(13, 16, seed=8)
    runs = {}
    for mode in (0, 1):
        eng, st = run_engine(gw, beg, csr, algo, maxhops, wps=wps, p=p, q=q, term=term, seed=21, launch_mode=mode)
        runs[mode] = (eng.paths(), eng.hashes(), st)
        eng.close()
    (P0, L0), H0, s0 = runs[0]
    (P1, L1), H1, s1 = runs[1]
    assert np.array_equal(P0, P1) and np.array_equal(L0, L1) and np.array_equal(H0, H1)
    assert (s0["steps"], s0["trials"]) == (s1["steps"], s1["trials"])
    assert s1["launches"] == maxhops
    V = len(beg) - 1
    ref = oracle.walk(beg, csr, oracle_cfg(oracle, algo, maxhops, wps, p, q, term=term, seed=21), 0, V * wps,
                      paths=False)
    assert np.array_equal(H1, ref["hashes"])

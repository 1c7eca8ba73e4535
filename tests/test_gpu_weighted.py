"""GPU tests of weighted Node2vec (gw_host_weights / gw_device_weights): the
device's alias tables and walks against the oracle's restatement, bit for
bit; equal weights walk exactly as unweighted; bad inputs fail with a
status."""
import numpy as np
import pytest

from test_gpu_walk import run_engine

pytestmark = pytest.mark.gpu


def weighted_run(gw, beg, csr, w, maxhops=20, p=2.0, q=0.5, seed=11, wps=1, algo=0, **cfg):
    eng = gw.WalkEngine(algorithm=algo, maxhops=maxhops, p=p, q=q, seed=seed, walkpersource=wps, record_paths=1,
                        cache_size=1 << 34, **cfg)
    eng.set_host_graph(beg, csr)
    eng.set_host_weights(w)
    eng.init_walkers(algo, wps, seed)
    st = eng.run()
    return eng, st


@pytest.mark.parametrize("scale,dist", [(12, "uniform"), (14, "lognormal"), (16, "heavy")])
def test_weighted_walks_match_oracle(gw, oracle, scale, dist):
    beg, csr = oracle.rmat_graph(scale)
    rng = np.random.default_rng(scale)
    if dist == "uniform":
        w = rng.uniform(0.5, 2.0, len(csr))
    elif dist == "lognormal":
        w = rng.lognormal(0.0, 1.0, len(csr))
    else:
        w = rng.pareto(1.5, len(csr)) + 1e-3
    w = w.astype(np.float32)
    V = len(beg) - 1
    eng, st = weighted_run(gw, beg, csr, w, maxhops=20)
    cfg = oracle.make_cfg(algo=0, maxhops=20, p=2.0, q=0.5, seed=11, wps=1)
    ref = oracle.walk(beg, csr, cfg, 0, V, paths=True, alias=oracle.build_alias(beg, w))
    P, L = eng.paths()
    assert np.array_equal(L, ref["lens"])
    assert np.array_equal(P, ref["paths"])
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["steps"] == ref["stats"]["steps"] and st["trials"] == ref["stats"]["trials"]
    eng.close()


def test_equal_weights_walk_as_unweighted(gw, oracle):
    beg, csr = oracle.rmat_graph(13)
    e1, s1 = weighted_run(gw, beg, csr, np.full(len(csr), 0.25, np.float32), maxhops=30)
    e2, s2 = run_engine(gw, beg, csr, 0, 30, p=2.0, q=0.5, seed=11)
    assert np.array_equal(e1.hashes(), e2.hashes()) and s1["steps"] == s2["steps"]
    e1.close()
    e2.close()


def test_device_weights_and_termination(gw, oracle):
    """Weights given on the device with a device graph, and the geometric
    termination draw, still match the oracle."""
    import torch
    beg, csr = oracle.rmat_graph(13)
    w = np.random.default_rng(2).uniform(0.1, 10.0, len(csr)).astype(np.float32)
    V = len(beg) - 1
    d_beg = torch.from_numpy(beg.view(np.int64)).cuda()
    d_csr = torch.from_numpy(csr.view(np.int32)).cuda()
    d_w = torch.from_numpy(w).cuda()
    eng = gw.WalkEngine(algorithm=0, maxhops=25, p=0.5, q=2.0, seed=4, walkpersource=2, record_paths=0,
                        term_prob=0.1)
    eng.set_device_graph(V, len(csr), d_beg.data_ptr(), d_csr.data_ptr())
    eng.set_device_weights(d_w.data_ptr())
    eng.init_walkers(0, 2, 4)
    st = eng.run()
    cfg = oracle.make_cfg(algo=0, maxhops=25, p=0.5, q=2.0, term_prob=0.1, seed=4, wps=2)
    ref = oracle.walk(beg, csr, cfg, 0, 2 * V, paths=False, alias=oracle.build_alias(beg, w))
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["steps"] == ref["stats"]["steps"]
    # weights dropped: unweighted again
    eng.set_device_weights(0)
    eng.init_walkers(0, 2, 4)
    eng.run()
    ref_u = oracle.walk(beg, csr, cfg, 0, 2 * V, paths=False)
    assert np.array_equal(eng.hashes(), ref_u["hashes"])
    eng.close()


@pytest.mark.parametrize("bad", [0.0, -1.0, float("nan"), float("inf")])
def test_bad_weight_fails_with_graph_status(gw, oracle, bad):
    beg, csr = oracle.rmat_graph(10)
    w = np.ones(len(csr), np.float32)
    w[len(w) // 2] = bad
    with pytest.raises(gw.GwError) as ei:
        weighted_run(gw, beg, csr, w)
    assert ei.value.status == -7


def test_weighted_needs_node2vec(gw, oracle):
    """Weighted walks are Node2vec walks, in-core and out-of-core; the
    out-of-core zero-copy tail reads unweighted blocks only; a bad weight
    fails an out-of-core run with the graph status too."""
    beg, csr = oracle.rmat_graph(11)
    w = np.ones(len(csr), np.float32)
    with pytest.raises(gw.GwError) as ei:
        weighted_run(gw, beg, csr, w, algo=1)
    assert ei.value.status == -1
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, 8)
    maxe = int(np.diff(eb.astype(np.int64)).max())
    cache = len(beg) * 8 + 3 * ((maxe + 3) & ~3) * 12
    for algo, zc, wv, status in ((1, 0, 1.0, -1), (0, 1, 1.0, -1), (0, 0, -1.0, -7)):
        eng = gw.WalkEngine(algorithm=algo, maxhops=10, seed=1, walkpersource=1, cache_size=cache, zero_copy=zc)
        eng.set_host_graph(beg, csr, vb, eb)
        ww = w.copy()
        ww[len(ww) // 3] = wv
        eng.set_host_weights(ww)
        eng.init_walkers(algo, 1, 1)
        with pytest.raises(gw.GwError) as ei:
            eng.run()
        assert ei.value.status == status, (algo, zc, wv)
        eng.close()


@pytest.mark.parametrize("prefetch,compress,strict,slots", [(0, 0, 0, 3), (1, 1, 0, 4), (1, 0, 1, 5), (0, 1, 0, 2)])
def test_out_of_core_weighted_matches_oracle(gw, oracle, prefetch, compress, strict, slots):
    """Weighted Node2vec out-of-core: every block's alias tables are built on
    the device from its weights once and copied behind its neighbour list
    with each load (the reference copies weights with every block,
    gpu/memory.hpp:134-137); the walks equal the oracle's weighted
    restatement bit for bit whatever the cache size, prefetch, compression or
    residency rule, and the H2D bytes carry the alias tables."""
    from gowalker_b200.preprocess import split_equal_edge_mass
    beg, csr = oracle.rmat_graph(14, 12, seed=6)
    w = np.random.default_rng(7).lognormal(0.0, 1.0, len(csr)).astype(np.float32)
    nb = 12
    vb, eb = split_equal_edge_mass(beg, nb)
    maxe = int(np.diff(eb.astype(np.int64)).max())
    slot = ((maxe + 3) & ~3) * 12  # neighbour ids + alias tables
    stage = 2 * (len(csr) * 4 // nb + (1 << 20)) if compress else 0
    eng = gw.WalkEngine(algorithm=0, maxhops=25, p=0.5, q=2.0, seed=13, walkpersource=1, record_paths=1,
                        cache_size=len(beg) * 8 + slots * slot + stage, prefetch=prefetch, compress_blocks=compress,
                        strict_blocks=strict)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.set_host_weights(w)
    eng.init_walkers(0, 1, 13)
    st = eng.run()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=25, p=0.5, q=2.0, seed=13), 0, len(beg) - 1,
                      paths=True, alias=oracle.build_alias(beg, w))
    P, L = eng.paths()
    assert st["block_loads"] > nb
    assert np.array_equal(L, ref["lens"]) and np.array_equal(P, ref["paths"])
    assert np.array_equal(eng.hashes(), ref["hashes"]) and st["steps"] == ref["stats"]["steps"]
    # every load moves the block's alias tables (8 bytes per edge) with it
    assert st["h2d_bytes"] > st["block_loads"] * 8 * min(np.diff(eb.astype(np.int64)))
    # a second run reuses the tables; new weights rebuild them
    eng.init_walkers(0, 1, 13)
    eng.run()
    assert np.array_equal(eng.hashes(), ref["hashes"])
    w2 = np.ones(len(csr), np.float32)
    eng.set_host_weights(w2)
    eng.init_walkers(0, 1, 13)
    eng.run()
    ref2 = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=25, p=0.5, q=2.0, seed=13), 0, len(beg) - 1,
                       paths=False)
    assert np.array_equal(eng.hashes(), ref2["hashes"])  # equal weights walk as unweighted
    eng.close()

"""GPU tests of the out-of-core path: device block cache, bucketing, block
choice, zero-copy tail.  Walks must be bit-identical to the oracle whatever
the cache size or schedule (counter-based draws)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def graph(oracle, scale=13, ef=8, sym=False, cap=6000, seed=21):
    src, dst = oracle.rmat_edges(scale, 0, ef << scale, seed=seed)
    keep = (src < cap) & (dst < cap)
    return oracle.build_csr(cap, src[keep], dst[keep], symmetric=sym)


def cache_for(beg, eb, slots):
    """Cache bytes for the resident vertex offsets plus `slots` neighbour slots."""
    maxe = int(np.diff(eb.astype(np.int64)).max())
    return len(beg) * 8 + ((max(maxe, 1) + 3) & ~3) * 4 * slots


def run_ooc(gw, beg, csr, nblocks, slots, algo=0, maxhops=20, wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, seed=5,
            zero_copy=0, zero_threshold=0, paths=1, policy=0, learned_mode=0):
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, nblocks)
    cache = cache_for(beg, eb, slots)
    eng = gw.WalkEngine(algorithm=algo, maxhops=maxhops, p=p, q=q, alpha=alpha, term_prob=term, seed=seed,
                        walkpersource=wps, record_paths=paths, cache_size=cache, zero_copy=zero_copy,
                        zero_threshold=zero_threshold, learned_mode=learned_mode)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, wps, seed)
    st = eng.run(policy)
    return eng, st


@pytest.mark.parametrize("algo,term,sym", [(0, 0.0, False), (1, 0.15, False), (0, 0.0, True), (2, 0.15, True)])
def test_ooc_matches_oracle(gw, oracle, algo, term, sym):
    beg, csr = graph(oracle, sym=sym)
    V = len(beg) - 1
    eng, st = run_ooc(gw, beg, csr, 12, 3, algo=algo, term=term, wps=2)
    cfg = oracle.make_cfg(algo=algo, maxhops=20, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=5, wps=2)
    ref = oracle.walk(beg, csr, cfg, 0, 2 * V, paths=True)
    P, L = eng.paths()
    assert np.array_equal(L, ref["lens"])
    assert np.array_equal(P, ref["paths"])
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["steps"] == ref["stats"]["steps"]
    assert st["trials"] == ref["stats"]["trials"]
    assert st["block_loads"] >= 3 and st["h2d_bytes"] > 0 and st["iterations"] >= 3
    assert int(eng.bucket_counts().sum()) == 0  # every walker finished
    eng.close()


def test_schedule_invariance(gw, oracle):
    """Same walks for every cache size, with and without the zero-copy tail."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=True, cap=7000, seed=3)
    base = None
    loads = {}
    for slots, zc, zt in ((2, 0, 0), (4, 0, 0), (7, 0, 0), (3, 1, 400), (10, 0, 0)):
        eng, st = run_ooc(gw, beg, csr, 10, slots, algo=1, term=0.15, wps=1, zero_copy=zc, zero_threshold=zt,
                          paths=0)
        h = eng.hashes()
        loads[(slots, zc)] = (st["block_loads"], st["zero_copy_steps"])
        eng.close()
        base = h if base is None else base
        assert np.array_equal(h, base), (slots, zc)
    assert loads[(3, 1)][1] > 0          # the tail ran through mapped host memory
    assert loads[(2, 0)][0] >= loads[(10, 0)][0]


def test_ooc_learned_policy_same_walks(gw, oracle):
    """The learned policy trains on the first plain iterations, then decides;
    the walks stay those of the plain policy and of the oracle."""
    beg, csr = graph(oracle, scale=14, ef=8, sym=False, cap=12000, seed=8)
    e1, s1 = run_ooc(gw, beg, csr, 16, 4, algo=0, maxhops=30, paths=0, policy=0)
    e2, s2 = run_ooc(gw, beg, csr, 16, 4, algo=0, maxhops=30, paths=0, policy=1,
                     learned_mode=gw.GW_LEARNED_EVICT | gw.GW_LEARNED_ZERO_SWITCH)
    h1, h2 = e1.hashes(), e2.hashes()
    assert np.array_equal(h1, h2)
    V = len(beg) - 1
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=30, p=0.5, q=2.0, seed=5), 0, V, paths=False)
    assert np.array_equal(h2, ref["hashes"])
    assert s1["learned_iterations"] == 0
    if s2["iterations"] > 23:
        assert s2["train_loss"] > 0.0
        assert s2["learned_iterations"] > 0 or s2["policy_reverted"] == 1
    # a second learned run reuses the trained model from its first iteration
    e2.init_walkers(0, 1, 5)
    s3 = e2.run(1)
    assert np.array_equal(e2.hashes(), h1)
    e1.close()
    e2.close()


def test_learned_zero_switch(gw, oracle):
    """The learned zero-copy switch alone.  On a fresh handle no tail has
    been timed, so the learned run takes exactly the plain schedule --
    GOWalker's zero_threshold -- and times its tail; the next learned run
    prices each load against that tail and may switch at another iteration.
    Every run walks the oracle's walks."""
    beg, csr = graph(oracle, scale=15, ef=10, sym=False, cap=20000, seed=12)
    V = len(beg) - 1
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=40, p=0.5, q=2.0, seed=5), 0, V, paths=False)
    e0, s0 = run_ooc(gw, beg, csr, 16, 4, algo=0, maxhops=40, paths=0, policy=0, zero_copy=1, zero_threshold=300)
    e1, s1 = run_ooc(gw, beg, csr, 16, 4, algo=0, maxhops=40, paths=0, policy=1, zero_copy=1, zero_threshold=300,
                     learned_mode=gw.GW_LEARNED_ZERO_SWITCH)
    assert np.array_equal(e0.hashes(), ref["hashes"])
    assert np.array_equal(e1.hashes(), ref["hashes"])
    assert s0["zero_copy_steps"] > 0
    for k in ("iterations", "block_loads", "zero_copy_steps", "h2d_bytes"):
        assert s1[k] == s0[k], k
    assert s1["learned_iterations"] == 0 and s1["learned_parts"] == gw.GW_LEARNED_ZERO_SWITCH
    e1.init_walkers(0, 1, 5)
    s2 = e1.run(gw.GW_POLICY_LEARNED)
    assert np.array_equal(e1.hashes(), ref["hashes"])
    assert s2["steps"] == s0["steps"] and s2["learned_iterations"] <= 1
    if s2["learned_iterations"] == 1:
        assert s2["zero_copy_steps"] > 0
    e0.close()
    e1.close()


def test_learned_parts_chosen_run_by_run(gw, oracle):
    """learned_mode 0 (automatic): after a plain run has timed a tail, the
    first learned run uses both parts (forecast eviction and the priced
    switch), the second the switch alone, the third the faster of the two on
    this workload.  The walks never change."""
    beg, csr = graph(oracle, scale=15, ef=10, sym=False, cap=20000, seed=12)
    V = len(beg) - 1
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=40, p=0.5, q=2.0, seed=5), 0, V, paths=False)
    eng, s0 = run_ooc(gw, beg, csr, 16, 4, algo=0, maxhops=40, paths=0, policy=0, zero_copy=1, zero_threshold=300)
    assert s0["zero_copy_steps"] > 0 and s0["learned_parts"] == 0
    both, sw = gw.GW_LEARNED_EVICT | gw.GW_LEARNED_ZERO_SWITCH, gw.GW_LEARNED_ZERO_SWITCH
    parts, ms = [], {}
    for _ in range(3):
        eng.init_walkers(0, 1, 5)
        st = eng.run(gw.GW_POLICY_LEARNED)
        assert np.array_equal(eng.hashes(), ref["hashes"])
        parts.append(st["learned_parts"])
        ms.setdefault(st["learned_parts"], st["total_ms"])
    eng.close()
    if 0 in parts:  # the judge handed the workload back to the plain rule
        assert parts[:2] == [both, sw] and parts[2] == 0
    else:
        assert parts[:2] == [both, sw] and parts[2] in (both, sw)


def test_ooc_rejects_tiny_cache(gw, oracle):
    beg, csr = graph(oracle)
    with pytest.raises(gw.GwError):
        run_ooc(gw, beg, csr, 8, 1)


def test_zero_copy_leaves_neighbouring_host_data_writable(gw, oracle):
    """The zero-copy tail maps host blocks page by page.  Results copied back
    into host memory that shares a page with a mapped block must still land."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=True, cap=7000, seed=3)
    V = len(beg) - 1
    arena = np.zeros(V + 1 + V, dtype=np.uint64)   # offsets, then the hash output in the same pages
    arena[:V + 1] = beg
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, 10)
    eng = gw.WalkEngine(algorithm=1, maxhops=20, alpha=0.2, term_prob=0.15, seed=5, walkpersource=1,
                        record_paths=0, cache_size=cache_for(beg, eb, 3), zero_copy=1, zero_threshold=400)
    eng.set_host_graph(arena[:V + 1], csr, vb, eb)
    eng.init_walkers(1, 1, 5)
    st = eng.run()
    assert st["zero_copy_steps"] > 0
    out = arena[V + 1:]
    eng._check(eng.L.gw_path_hashes(eng.h, 0, V, out.ctypes.data_as(ctypes.c_void_p)))
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=1, maxhops=20, alpha=0.2, term_prob=0.15, seed=5), 0, V,
                      paths=False)
    assert np.array_equal(out, ref["hashes"])
    eng.close()


@pytest.mark.parametrize("sym", [False, True])
def test_lazy_previous_block_same_walks_fewer_loads(gw, oracle, sym):
    """Node2vec walkers may step with only their current block resident until
    a trial needs N(prev): identical walks and trial counts, fewer loads than
    requiring both blocks."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=sym, cap=7000, seed=3)
    V = len(beg) - 1
    res = {}
    for strict in (1, 0):
        from gowalker_b200.preprocess import split_equal_edge_mass
        vb, eb = split_equal_edge_mass(beg, 16)
        eng = gw.WalkEngine(algorithm=0, maxhops=30, p=0.5, q=2.0, seed=5, walkpersource=1, record_paths=1,
                            cache_size=cache_for(beg, eb, 4), strict_blocks=strict)
        eng.set_host_graph(beg, csr, vb, eb)
        eng.init_walkers(0, 1, 5)
        st = eng.run()
        P, L = eng.paths()
        res[strict] = (P, L, eng.hashes(), st)
        assert int(eng.bucket_counts().sum()) == 0
        eng.close()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=30, p=0.5, q=2.0, seed=5), 0, V, paths=True)
    for strict in (1, 0):
        P, L, H, st = res[strict]
        assert np.array_equal(P, ref["paths"]) and np.array_equal(L, ref["lens"])
        assert np.array_equal(H, ref["hashes"])
        assert st["steps"] == ref["stats"]["steps"] and st["trials"] == ref["stats"]["trials"]
    assert res[0][3]["block_loads"] < res[1][3]["block_loads"]


@pytest.mark.parametrize("algo,policy", [(0, 0), (1, 0), (0, 1)])
def test_prefetch_same_walks(gw, oracle, algo, policy):
    """Block choices taken one iteration ahead, copies overlapped with the
    step kernel in a staging slot: the walks stay those of the oracle."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=algo == 1, cap=7000, seed=3)
    V = len(beg) - 1
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, 12)
    eng = gw.WalkEngine(algorithm=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2, term_prob=0.15 if algo else 0.0,
                        seed=11, walkpersource=1, record_paths=1, cache_size=cache_for(beg, eb, 4), prefetch=1)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, 1, 11)
    st = eng.run(policy)
    P, L = eng.paths()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2,
                                                term_prob=0.15 if algo else 0.0, seed=11), 0, V, paths=True)
    assert np.array_equal(P, ref["paths"]) and np.array_equal(L, ref["lens"])
    assert st["steps"] == ref["stats"]["steps"] and st["trials"] == ref["stats"]["trials"]
    assert st["block_loads"] > 0 and int(eng.bucket_counts().sum()) == 0
    eng.close()


@pytest.mark.parametrize("algo,prefetch", [(0, 0), (0, 1), (1, 0), (2, 1)])
def test_compressed_blocks_same_walks(gw, oracle, algo, prefetch):
    """Blocks copied as compressed neighbour lists and decoded on the device:
    the walks are the oracle's and fewer bytes cross the host link."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=algo != 0, cap=7000, seed=3)
    V = len(beg) - 1
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, 12)
    term = 0.15 if algo else 0.0
    out = {}
    for comp in (0, 1):
        eng = gw.WalkEngine(algorithm=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=11,
                            walkpersource=1, record_paths=1, cache_size=cache_for(beg, eb, 6),
                            prefetch=prefetch, compress_blocks=comp)
        eng.set_host_graph(beg, csr, vb, eb)
        eng.init_walkers(algo, 1, 11)
        st = eng.run()
        P, L = eng.paths()
        out[comp] = (P, L, st)
        assert st["block_loads"] > 0 and int(eng.bucket_counts().sum()) == 0
        eng.close()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2, term_prob=term,
                                                seed=11), 0, V, paths=True)
    for comp in (0, 1):
        P, L, st = out[comp]
        assert np.array_equal(P, ref["paths"]) and np.array_equal(L, ref["lens"])
        assert st["steps"] == ref["stats"]["steps"] and st["trials"] == ref["stats"]["trials"]
    per_load = [out[c][2]["h2d_bytes"] / max(out[c][2]["block_loads"], 1) for c in (0, 1)]
    assert per_load[1] < 0.8 * per_load[0]


def test_compressed_blocks_unsorted_duplicates(gw, oracle):
    """Exact round trip whatever the neighbour order: every adjacency list
    shuffled (negative deltas) with duplicate edges (zero deltas); compressed
    and plain block copies give bit-identical walks."""
    beg, csr = graph(oracle, scale=13, ef=12, sym=False, cap=7000, seed=5)
    rng = np.random.default_rng(3)
    V = len(beg) - 1
    deg = np.diff(beg.astype(np.int64))
    lists = []
    for v in range(V):
        a = csr[int(beg[v]):int(beg[v + 1])].copy()
        if v == 0:  # a hub: decoded in groups of 32 chunks by several warps
            a = np.concatenate([a, np.arange(1, V, dtype=np.uint32)])
        if len(a) and v % 3 == 0:
            a = np.concatenate([a, a[: 1 + len(a) // 4]])  # duplicates
        rng.shuffle(a)
        lists.append(a)
    deg = np.array([len(a) for a in lists])
    beg2 = np.zeros(V + 1, dtype=np.uint64)
    beg2[1:] = np.cumsum(deg)
    csr2 = np.concatenate(lists).astype(np.uint32)
    assert (deg > 32).sum() > 10 and (deg == 0).sum() > 0 and deg.max() > 4 * 1024
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg2, 10)
    hs = {}
    for comp in (0, 1):
        eng = gw.WalkEngine(algorithm=0, maxhops=30, p=0.5, q=2.0, seed=21, walkpersource=2, record_paths=1,
                            cache_size=cache_for(beg2, eb, 5), compress_blocks=comp)
        eng.set_host_graph(beg2, csr2, vb, eb)
        eng.init_walkers(0, 2, 21)
        st = eng.run()
        P, L = eng.paths()
        assert st["block_loads"] > 0
        hs[comp] = (P, L, eng.hashes(), st["steps"], st["trials"])
        eng.close()
    for a, b in zip(hs[0], hs[1]):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("case", ["sopr_single_source", "node2vec_32_blocks"])
def test_trained_predictor_beats_carrying_demand_forward(gw, oracle, case):
    """What the trained network gains over the method without it.  The plain
    rule treats the walkers waiting now as the demand to come; the network,
    retrained every 16 iterations on the last 20, forecasts log1p(mean demand
    over the next 3 iterations) per block.  Both forecasts are scored by the
    engine against the realised demand (mean |error| on the log1p scale):
    here the network's error is lower by 5-14 % (asserted: at least 5 %).  The run trains in step with
    its decisions (learned_sync), so every forecast comes from the weights
    fitted to the latest window; by default a training never delays a
    decision and its weights arrive some iterations later.  (Its block
    choices do not cut block loads on these graphs -- the judge hands the
    choice back to the plain rule -- and the walks stay those of the oracle
    either way.)"""
    from gowalker_b200.preprocess import split_equal_edge_mass
    if case == "sopr_single_source":
        beg, csr = graph(oracle, scale=13, ef=10, sym=True, cap=7000, seed=9)
        nb, slots, algo, maxhops, kw = 16, 4, 1, 40, dict(init_mode=1, numwalks=200000, walkpersource=0)
        wps, bound = 0, 0.95
    else:
        beg, csr = graph(oracle, scale=16, ef=12, sym=True, cap=60000, seed=4)
        nb, slots, algo, maxhops, kw = 32, 8, 0, 80, dict(walkpersource=1)
        wps, bound = 1, 0.95
    vb, eb = split_equal_edge_mass(beg, nb)
    eng = gw.WalkEngine(algorithm=algo, maxhops=maxhops, p=0.5, q=2.0, alpha=0.2, seed=5, record_paths=0,
                        cache_size=cache_for(beg, eb, slots), learned_sync=1, learned_mode=gw.GW_LEARNED_EVICT,
                        **kw)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, wps, 5)
    st = eng.run(gw.GW_POLICY_LEARNED)
    hs = eng.checksum()
    eng.close()
    assert st["pred_error"] > 0 and st["persist_error"] > 0
    assert st["pred_error"] < bound * st["persist_error"], (st["pred_error"], st["persist_error"])
    e0 = gw.WalkEngine(algorithm=algo, maxhops=maxhops, p=0.5, q=2.0, alpha=0.2, seed=5, record_paths=0,
                       cache_size=cache_for(beg, eb, slots), **kw)
    e0.set_host_graph(beg, csr, vb, eb)
    e0.init_walkers(algo, wps, 5)
    e0.run(gw.GW_POLICY_PLAIN)
    assert e0.checksum() == hs
    e0.close()


@pytest.mark.parametrize("algo,prefetch,strict,slots", [(0, 0, 0, 5), (0, 1, 0, 6), (0, 0, 1, 5), (0, 1, 1, 6),
                                                         (1, 1, 0, 6), (1, 0, 0, 4)])
def test_block_schedule_matches_cpu_replay(gw, oracle, algo, prefetch, strict, slots):
    """The engine's whole plain block schedule -- GOWalker's choice each
    iteration (engine/schedule.hpp:70-138), the rescue when nothing
    qualifies, the residency rule, prefetch one iteration ahead -- replayed on
    the CPU from the walkers' block requirements (the oracle's walks), gives
    the same number of iterations and block loads, and the same steps, as the
    GPU run."""
    from gowalker_b200.preprocess import split_equal_edge_mass
    beg, csr = graph(oracle, scale=14, ef=8, cap=12000, seed=31)
    nb = 16
    vb, eb = split_equal_edge_mass(beg, nb)
    term = 0.15 if algo else 0.0
    eng = gw.WalkEngine(algorithm=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=9, walkpersource=1,
                        record_paths=0, cache_size=cache_for(beg, eb, slots), zero_copy=0, zero_threshold=0,
                        prefetch=prefetch, strict_blocks=strict)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, 1, 9)
    st = eng.run(gw.GW_POLICY_PLAIN)
    eng.close()
    cfg = oracle.make_cfg(algo=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=9)
    reqs, nent = oracle.walk_requirements(beg, csr, cfg, vb, 0, len(beg) - 1)
    lazy = algo == 0 and not strict
    rs, _ = oracle.sched_replay(reqs, nent, nb, slots, prefetch=bool(prefetch), lazy=lazy)
    assert (st["iterations"], st["block_loads"], st["steps"]) == (rs["iterations"], rs["loads"], rs["steps"])
    assert rs["loads"] > 2 * nb


@pytest.mark.parametrize("algo,compress", [(0, 0), (0, 1), (1, 0)])
def test_zero_copy_tail_with_prefetch(gw, oracle, algo, compress):
    """GOWalker's zero mode with the block copies prefetched: once no block
    scores above zero_threshold (engine/schedule.hpp:101,124), every
    remaining walker runs to its end reading the absent blocks through mapped
    host memory (engine/engine.hpp:593-634).  Same walks as the oracle, fewer
    block loads than without the tail, and the mapped reads are counted into
    the host-to-device bytes."""
    from gowalker_b200.preprocess import split_equal_edge_mass
    beg, csr = graph(oracle, scale=14, ef=8, cap=12000, seed=33)
    vb, eb = split_equal_edge_mass(beg, 16)
    term = 0.15 if algo else 0.0
    res = {}
    for zc in (0, 1):
        stage = 2 * (len(csr) * 4 // 16 + (1 << 16)) if compress else 0
        eng = gw.WalkEngine(algorithm=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=4,
                            walkpersource=1, record_paths=0, cache_size=cache_for(beg, eb, 6) + stage, prefetch=1,
                            compress_blocks=compress, zero_copy=zc, zero_threshold=60 if zc else 0)
        eng.set_host_graph(beg, csr, vb, eb)
        eng.init_walkers(algo, 1, 4)
        st = eng.run()
        res[zc] = (eng.hashes(), st)
        eng.close()
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, term_prob=term, seed=4),
                      0, len(beg) - 1, paths=False)
    for zc in (0, 1):
        assert np.array_equal(res[zc][0], ref["hashes"]), zc
    s0, s1 = res[0][1], res[1][1]
    assert s1["zero_copy_steps"] > 0 and s0["zero_copy_steps"] == 0
    assert s1["block_loads"] < s0["block_loads"]
    assert s1["steps"] == s0["steps"] == ref["stats"]["steps"]
    # the tail's mapped reads (at least one 32-byte sector per tail step's
    # candidate from an absent block) are in the host-to-device bytes
    assert s1["h2d_bytes"] > 0

"""CPU tests of the oracle: golden fixtures, reference harness, properties."""
import glob
import multiprocessing as mp
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _cfg_from(O, z, **kw):
    return O.make_cfg(algo=int(z["algo"]), maxhops=int(z["maxhops"]), p=float(z["p"]), q=float(z["q"]),
                      alpha=float(z["alpha"]), seed=int(z["seed"]), wps=int(z["wps"]), **kw)


def test_philox_fixture(oracle):
    z = np.load(os.path.join(GOLDEN, "philox.npz"))
    for c, k, o in zip(z["ctrs"], z["keys"], z["outs"]):
        assert np.array_equal(oracle.philox(c, k), o)


def test_philox_lanes_uniform(oracle):
    """Chi-square of the top byte of 40k Philox draws (each lane)."""
    outs = np.stack([oracle.philox([i, 7, 0, 0], [42, 0]) for i in range(10000)])
    for lane in range(4):
        hist = np.bincount(outs[:, lane] >> 24, minlength=256)
        exp = len(outs) / 256.0
        chi2 = float(((hist - exp) ** 2 / exp).sum())
        assert chi2 < 340.0, (lane, chi2)  # 255 dof, p ~ 3e-4


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*_s8.npz"))))
def test_golden_walks(oracle, path):
    z = np.load(path)
    cfg = _cfg_from(oracle, z)
    n = len(z["hashes"])
    r = oracle.walk(z["beg"], z["csr"], cfg, 0, n, paths=True)
    assert np.array_equal(r["hashes"], z["hashes"])
    assert np.array_equal(r["lens"], z["lens"])
    assert np.array_equal(r["paths"], z["paths"])
    assert r["stats"]["steps"] == int(z["steps"])


def test_paths_follow_edges(oracle):
    beg, csr = oracle.rmat_graph(10, 8, seed=3)
    cfg = oracle.make_cfg(algo=oracle.ALG_NODE2VEC, maxhops=30, p=2.0, q=0.5, seed=7)
    V = len(beg) - 1
    r = oracle.walk(beg, csr, cfg, 0, V, paths=True)
    for w in range(0, V, 37):
        L = int(r["lens"][w])
        p = r["paths"][w, :L]
        assert p[0] == w
        for a, b in zip(p[:-1], p[1:]):
            adj = csr[int(beg[a]):int(beg[a + 1])]
            assert b in adj
        assert oracle.path_hash(p) == int(r["hashes"][w])


def test_termination_length_distribution(oracle):
    """SOPR with termination 0.15, max 20: mean length ~ (1-0.85^20)/0.15."""
    beg, csr = oracle.rmat_graph(11, 16, seed=1)
    V = len(beg) - 1
    cfg = oracle.make_cfg(algo=oracle.ALG_SOPR, maxhops=20, alpha=0.2, term_prob=0.15, seed=42, wps=4)
    r = oracle.walk(beg, csr, cfg, 0, 4 * V, paths=False)
    deg = np.diff(beg.astype(np.int64))
    live = np.repeat(deg > 0, 4)
    mean = (r["lens"][live].astype(np.float64) - 1).mean()
    expect = (1 - 0.85 ** 20) / 0.15
    assert abs(mean - expect) < 0.08, mean


def test_dead_end_rule(oracle):
    """A walker reaching a vertex without out-edges stops there
    (engine/engine.hpp:196-199: hop = maxhop-1, next vertex 0)."""
    beg = np.array([0, 1, 2, 2], dtype=np.uint64)   # 0->1, 1->2, 2 has no out-edge
    csr = np.array([1, 2], dtype=np.uint32)
    cfg = oracle.make_cfg(algo=oracle.ALG_NODE2VEC, maxhops=10, p=1.0, q=1.0, seed=1)
    r = oracle.walk(beg, csr, cfg, 0, 3, paths=True, finals=True)
    assert list(r["paths"][0, :r["lens"][0]]) == [0, 1, 2]
    assert list(r["finals"][0]) == [2, 0, 10]
    assert r["lens"][2] == 1 and list(r["finals"][2]) == [2, 0, 10]
    assert r["stats"]["dead_ends"] == 3


def test_single_source_init(oracle):
    cfg = oracle.make_cfg(algo=oracle.ALG_SOSR, init_mode=oracle.INIT_SINGLE_SOURCE, numwalks=10)
    L = oracle.lib()
    srcs = [L.oracle_walker_source(cfg, 100, w) for w in range(10)]
    assert srcs == [1] * 5 + [3] * 5


def test_walker_range_beyond_sources_is_rejected(oracle):
    beg, csr = oracle.rmat_graph(8, 8, seed=1)
    V = len(beg) - 1
    cfg = oracle.make_cfg(algo=oracle.ALG_SOPR, maxhops=5, wps=2)
    oracle.walk(beg, csr, cfg, 2 * V - 4, 4, paths=False)
    with pytest.raises(ValueError):
        oracle.walk(beg, csr, cfg, 2 * V - 4, 5, paths=False)


def test_block_splitters(oracle):
    beg, csr = oracle.rmat_graph(12, 16, seed=1)
    vb, eb = oracle.split_equal_edge_mass(beg, 8)
    assert len(vb) == 9 and vb[0] == 0 and vb[-1] == len(beg) - 1
    assert np.all(np.diff(vb.astype(np.int64)) > 0)
    assert np.array_equal(eb, beg[vb.astype(np.int64)])
    mass = np.diff(eb.astype(np.int64))
    assert mass.max() < 2.5 * mass.mean()
    vr, er = oracle.split_blocks_reference(beg, 64 * 1024)
    assert vr[0] == 0 and vr[-1] == len(beg) - 1
    assert np.all(np.diff(er.astype(np.int64)[:-1]) <= 64 * 1024 // 4)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_step.so")),
                    reason="reference harness not built (needs the GOWalker sources)")
@pytest.mark.parametrize("algo", [0, 1])
def test_reference_harness_matches_oracle(oracle, tmp_path, algo):
    """The reference's own CPU step, fed the same Philox stream, takes the same
    trials as the oracle (directed graph: dead ends included)."""
    V = 150
    src, dst = oracle.rmat_edges(8, 0, 6 << 8, seed=11)
    keep = (src < V) & (dst < V)
    beg, csr = oracle.build_csr(V, src[keep], dst[keep], symmetric=False)
    beg2, csr2, vb, eb = oracle.harness_graph(beg, csr)
    base = str(tmp_path / "g")
    oracle.write_dataset(base, beg2, csr2)
    oracle.write_blocks(base, 1, vb, eb)
    starts = [(v, V + v, v, 0, V + v, v) for v in range(V)]
    with mp.get_context("spawn").Pool(1) as pool:
        _, res = pool.apply(oracle.ref_scenario, (base, algo, 0.7, 1.9, 0.25, 12, 1, 99, starts))
    cfg = oracle.make_cfg(algo=algo, maxhops=12, p=0.7, q=1.9, alpha=0.25, seed=99, keying=oracle.KEY_TRIAL)
    for v in range(V):
        moves, _, trace, final = oracle.walk_traced(beg, csr, cfg, v, v, v, 0)
        run, rtrace, _, _ = res[v]
        dead = 1 if (moves < 12 and final[1] == 0 and final[2] == 12) else 0
        assert np.array_equal(trace, rtrace), v
        assert run == moves + dead, v


def test_product_splitters_match_oracle(oracle):
    from gowalker_b200 import preprocess as P
    beg, csr = oracle.rmat_graph(12, 16, seed=1)
    for nb in (1, 3, 8, 64):
        a = P.split_equal_edge_mass(beg, nb)
        b = oracle.split_equal_edge_mass(beg, nb)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for bs in (16 * 1024, 64 * 1024):
        a = P.split_blocks(beg, bs)
        b = oracle.split_blocks_reference(beg, bs)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_dataset_files_roundtrip(oracle, tmp_path):
    from gowalker_b200 import preprocess as P
    beg, csr = oracle.rmat_graph(10, 8, seed=2)
    base = str(tmp_path / "g")
    P.write_dataset(base, beg, csr)
    assert os.path.getsize(base + ".meta") == 16
    assert P.read_meta(base) == (len(beg) - 1, len(csr), 0)
    b2, c2 = P.load_dataset(base)
    assert np.array_equal(b2, beg) and np.array_equal(c2, csr)
    vb, eb = P.split_equal_edge_mass(beg, 4)
    P.write_blocks(base, 64, vb, eb)
    v2, e2 = P.load_blocks(base, 64)
    assert np.array_equal(v2, vb) and np.array_equal(e2, eb)
    # oracle writer produces byte-identical files
    base2 = str(tmp_path / "h")
    oracle.write_dataset(base2, beg, csr)
    for ext in (".beg", ".csr", ".meta"):
        assert open(base + ext, "rb").read() == open(base2 + ext, "rb").read()
    with open(base + ".meta", "wb") as f:
        f.write(b"\0" * 5)
    with pytest.raises(ValueError):
        P.load_dataset(base)


def test_mlp_oracle_gradient_by_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, M.NPARAMS)
    x = rng.normal(0, 1, (20, M.IN))
    t = rng.normal(0, 1, 20)
    _, g = M.loss_and_grad(p, x, t)
    for idx in rng.choice(M.NPARAMS, 12, replace=False):
        pp = p.copy()
        pp[idx] += 1e-6
        lp, _ = M.loss_and_grad(pp, x, t)
        pp[idx] -= 2e-6
        lm, _ = M.loss_and_grad(pp, x, t)
        assert abs((lp - lm) / 2e-6 - g[idx]) < 1e-5 * max(1.0, abs(g[idx]))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_step_unmod.so")),
                    reason="reference harness not built (needs the GOWalker sources)")
@pytest.mark.parametrize("algo", [0, 1])
def test_transition_law_chi_square(oracle, tmp_path, algo):
    """Transition frequencies out of one (prev, cur) state against the analytic
    second-order law (engine/engine.hpp:209-258, 334-375): the oracle (the
    engine's stream) and the reference's own CPU step fed the Philox stream
    follow it; the unmodified reference does not.  That outcome is recorded,
    not fixed: its RandNum::inlineRandPair (util/util.hpp:291-301) builds
    rand_val by reading the low 32 bits of a 64-bit integer as a float."""
    from scipy.stats import chisquare
    V = 200
    src, dst = oracle.rmat_edges(8, 0, 8 << 8, seed=3)
    keep = (src < V) & (dst < V)
    beg, csr = oracle.build_csr(V, src[keep], dst[keep], symmetric=True)
    # vertices 0..V-1 in block 0; V+v, a copy of v's adjacency that nothing
    # points to, in block 1: a walker at (V+p, c) takes one step inside block 0
    beg2, csr2, _, _ = oracle.harness_graph(beg, csr)
    E = int(beg[-1])
    base = str(tmp_path / "g")
    oracle.write_dataset(base, beg2, csr2)
    oracle.write_blocks(base, 1, np.array([0, V, 2 * V], dtype=np.uint32), np.array([0, E, 2 * E], dtype=np.uint64))
    deg = np.diff(beg.astype(np.int64))
    c = int(np.argsort(deg)[-3])
    nc = csr[beg[c]:beg[c + 1]]
    p = int(max(nc, key=lambda y: len(np.intersect1d(nc, csr[beg[y]:beg[y + 1]]))))
    found = np.isin(nc, csr[beg[p]:beg[p + 1]])
    assert 0 < found.sum() < len(nc)
    if algo == 0:  # Node2vec p=0.5, q=2: weight 1 in N(prev), 1/q outside (x == V+p never occurs)
        w = np.where(found, 1.0, 0.5)
    else:          # SOPR alpha 0.2: (1-alpha)/deg(cur) + alpha/deg(prev) in N(prev)
        w = 0.8 / deg[c] + np.where(found, 0.2 / deg[p], 0.0)
    prob = w / w.sum()
    n = 30000
    starts = [(i, V + p, c, 0, 1, 0) for i in range(n)]

    def pvalue(nxt):
        assert np.all(nxt >= 0)
        counts = np.array([np.sum(nxt == x) for x in nc])
        return chisquare(counts, prob * counts.sum()).pvalue

    res = {}
    for unmod in (False, True):
        with mp.get_context("spawn").Pool(1) as pool:
            res[unmod] = pool.apply(oracle.ref_single_steps, (base, algo, 0.5, 2.0, 0.2, 12345, starts, unmod))
    cfg = oracle.make_cfg(algo=algo, maxhops=1, p=0.5, q=2.0, alpha=0.2, seed=777)
    ours = np.array([oracle.walk_traced(beg2, csr2, cfg, i, V + p, c, 0, cap=16)[1][0] for i in range(n)])
    assert pvalue(ours) > 1e-3
    assert pvalue(res[False]) > 1e-3
    assert pvalue(res[True]) < 1e-4


@pytest.mark.parametrize("sort", [False, True])
@pytest.mark.parametrize("case", range(6))
def test_convert_edges_pinned_by_streaming_converter(oracle, sort, case):
    """The vectorised converter restatement equals a line-by-line replay of
    the reference's streaming converter (graph_converter.hpp:167-263) on
    source-sorted lists with self loops, repeats, gaps, a first source > 0
    and a largest id that only appears as a destination."""
    rng = np.random.default_rng(100 + case)
    nv = [5, 17, 64, 300, 1000, 40][case]
    n = [8, 40, 500, 3000, 2000, 200][case]
    src = np.sort(rng.integers(case % 3, nv - 1, n)).astype(np.uint32)
    dst = rng.integers(0, nv, n).astype(np.uint32)
    loops = rng.random(n) < 0.1
    dst[loops] = src[loops]
    rep = rng.random(n) < 0.2  # repeat the previous edge
    rep[0] = False
    for i in np.nonzero(rep)[0]:
        if src[i] == src[i - 1]:
            dst[i] = dst[i - 1]
    dst[-1] = nv - 1 if src[-1] != nv - 1 else 0  # largest id as a destination only
    edges = list(zip(src.tolist(), dst.tolist()))
    b1, c1, n1 = oracle.convert_stream(edges, sort=sort)
    b2, c2, n2 = oracle.convert_edges(src, dst, 0, symmetric=False, sort=sort)
    assert n1 == n2
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    if sort:
        oracle.check_csr(b2, c2)


def test_convert_edges_dedup_symmetric_is_build_csr(oracle):
    rng = np.random.default_rng(7)
    src = rng.integers(0, 500, 20000).astype(np.uint32)
    dst = rng.integers(0, 500, 20000).astype(np.uint32)
    b1, c1 = oracle.build_csr(500, src, dst, symmetric=True)
    b2, c2, nv = oracle.convert_edges(src, dst, 500, symmetric=True, dedup=True)
    assert nv == 500 and np.array_equal(b1, b2) and np.array_equal(c1, c2)
    with pytest.raises(ValueError):
        oracle.convert_edges(src, dst, 499)


def test_split_equal_edge_mass_integer_targets(oracle):
    """The equal-edge-mass cut targets are floor(k*E/nblocks) in integers."""
    beg = np.array([0, 3, 3, 10, 11, 20, 20, 21], dtype=np.uint64)
    vb, eb = oracle.split_equal_edge_mass(beg, 3)
    # targets 7 and 14: first offsets >= them are beg[3]=10 and beg[5]=20
    assert vb.tolist() == [0, 3, 5, 7] and eb.tolist() == [0, 10, 20, 21]


def test_sa_log_accuracy(oracle):
    """The fixed-step log of a 32-bit draw the annealing acceptance uses is
    within a few ulp of libm."""
    import math
    rng = np.random.default_rng(2)
    for z in list(rng.integers(1, 1 << 32, 3000)) + [1, 2, 3, 0xFFFFFFFF, 1 << 31, 0xB504F333]:
        z = int(z)
        want = math.log(z * 2.0 ** -32)
        got = oracle.sa_log_draw(z)
        assert abs(got - want) <= 4e-16 * max(abs(want), 1e-300) + 1e-300, z
    assert oracle.sa_log_draw(0) == -math.inf and oracle.sa_log_draw((1 << 32) - 1) < 0


def test_sa_choice_properties(oracle):
    rng = np.random.default_rng(4)
    c = rng.integers(0, 100, (20, 20)).astype(np.uint32)
    c[3, 3] = c[7, 3] = 100000
    s = oracle.sa_choose_blocks(c, [], 6, 1, 0)
    assert len(set(s.tolist())) == 6 and s.max() < 20
    assert 3 in s  # the block the hot walkers wait for
    assert np.array_equal(s, oracle.sa_choose_blocks(c, [], 6, 1, 0))
    assert sorted(oracle.sa_choose_blocks(c, [], 25, 1, 0).tolist()) == list(range(20))


def test_web_degrees_power_law(oracle):
    """Out-degrees of the web-shaped graph: at least floor(dmin), a power-law
    tail P(D >= d) ~ d^-1.1 (density exponent 2.1), capped."""
    deg = oracle.web_degrees(200000, 6.0, 1.1, 65536, 1).astype(np.float64)
    assert deg.min() == 6 and deg.max() <= 65536
    for a, b in [(20, 200), (50, 2000)]:
        slope = np.log((deg >= b).mean() / (deg >= a).mean()) / np.log(b / a)
        assert abs(slope + 1.1) < 0.05, slope


def test_alias_tables_reproduce_weights(oracle):
    beg, csr = oracle.rmat_graph(10)
    rng = np.random.default_rng(1)
    w = rng.lognormal(0.0, 1.5, len(csr)).astype(np.float32)
    prob, alias = oracle.build_alias(beg, w)
    V = len(beg) - 1
    for v in rng.choice(V, 200, replace=False):
        h, d = int(beg[v]), int(beg[v + 1] - beg[v])
        if d == 0:
            continue
        got = np.zeros(d)
        np.add.at(got, np.arange(d), prob[h:h + d])
        np.add.at(got, alias[h:h + d].astype(np.int64), 1.0 - prob[h:h + d].astype(np.float64))
        want = w[h:h + d].astype(np.float64) / w[h:h + d].astype(np.float64).sum() * d
        assert np.abs(got - want).max() < 1e-5 * max(1.0, want.max())
    with pytest.raises(ValueError):
        bad = w.copy()
        bad[5] = 0.0
        oracle.build_alias(beg, bad)


def test_weighted_oracle_equal_weights_is_unweighted(oracle):
    beg, csr = oracle.rmat_graph(11)
    cfg = oracle.make_cfg(algo=0, maxhops=15, p=2.0, q=0.5, seed=9)
    al = oracle.build_alias(beg, np.full(len(csr), 3.5, np.float32))
    a = oracle.walk(beg, csr, cfg, 0, 2048, alias=al)
    b = oracle.walk(beg, csr, cfg, 0, 2048)
    assert np.array_equal(a["paths"], b["paths"]) and np.array_equal(a["hashes"], b["hashes"])


def test_weighted_node2vec_transition_law_chi_square(oracle):
    """Second-order transitions of the weighted oracle follow
    P(x | prev, cur) ~ w(cur, x) * (1/p if x == prev, 1 if x in N(prev), 1/q else)."""
    import math
    rng = np.random.default_rng(4)
    V = 40
    src = rng.integers(0, V, 600)
    dst = rng.integers(0, V, 600)
    beg, csr = oracle.build_csr(V, src, dst, symmetric=True)
    w = rng.uniform(0.2, 4.0, len(csr)).astype(np.float32)
    p, q = 2.0, 0.5
    cfg = oracle.make_cfg(algo=0, maxhops=4, p=p, q=q, seed=17, wps=4000)
    nz = np.nonzero(np.diff(beg.astype(np.int64)))[0]
    r = oracle.walk(beg, csr, cfg, 0, V * 4000, alias=oracle.build_alias(beg, w))
    P, L = r["paths"], r["lens"]
    counts = {}
    for row, n in zip(P, L):
        for t in range(2, n):
            key = (int(row[t - 2]), int(row[t - 1]))
            counts.setdefault(key, {}).setdefault(int(row[t]), 0)
            counts[key][int(row[t])] += 1
    tested = 0
    for (a, b), obs in sorted(counts.items(), key=lambda kv: -sum(kv[1].values()))[:25]:
        nb = csr[beg[b]:beg[b + 1]]
        wb = w[beg[b]:beg[b + 1]].astype(np.float64)
        na = set(csr[beg[a]:beg[a + 1]].tolist())
        bias = np.array([1 / p if x == a else (1.0 if x in na else 1 / q) for x in nb])
        pr = wb * bias / (wb * bias).sum()
        n = sum(obs.values())
        chi = sum((obs.get(int(x), 0) - n * px) ** 2 / (n * px) for x, px in zip(nb, pr))
        dof = len(nb) - 1
        # chi-square upper tail bound: mean dof, sd sqrt(2 dof); 5 sd is far beyond chance
        assert chi < dof + 5 * math.sqrt(2 * dof) + 10, ((a, b), chi, dof)
        tested += 1
    assert tested == 25 and len(nz) == V


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_step.so")),
                    reason="reference harness not built (needs the GOWalker sources)")
@pytest.mark.parametrize("nb", [6, 20, 64])
def test_max_choose_blocks_matches_reference(oracle, tmp_path, nb):
    """The oracle's restatement of GOWalker's block choice takes the decision
    the reference's own GOwalker_scheduler_t::max_choose_blocks
    (engine/schedule.hpp:70-138, compiled from its sources) takes, on random
    and adversarial bucket-count matrices: not-full and full caches, zero
    threshold at and below the best score, all-zero counts, equal scores
    among at most 16 uncached blocks, shared smallest links."""
    import schedule_cases as SC
    # one vertex per block: the scheduler's nblocks is nb
    beg = np.arange(nb + 1, dtype=np.uint64)
    csr = ((np.arange(nb) + 1) % nb).astype(np.uint32)
    base = str(tmp_path / "g")
    oracle.write_dataset(base, beg, csr)
    oracle.write_blocks(base, 1, np.arange(nb + 1, dtype=np.uint32), beg.copy())
    cases = SC.cases(nb, seed=nb)
    assert len(cases) >= 30
    with mp.get_context("spawn").Pool(1) as pool:
        res = pool.apply(oracle.ref_choose_blocks, (base, cases))
    acts = set()
    for (counts, cached, nslots, zt), (chose, after) in zip(cases, res):
        want = SC.ref_to_decision(cached, chose, after)
        got = oracle.max_choose_blocks(counts, cached, nslots, zt)
        assert got == want, (cached, nslots, zt)
        acts.add(got[0])
    assert acts == {0, 1, 2}


def test_schedule_replay_zero_mode_and_incident_eviction(oracle):
    """The CPU schedule replay's options: GOWalker's zero mode ends the
    loading at the first iteration whose best score is at or below the
    threshold and leaves every remaining step to the mapped tail (loaded plus
    tail steps = every step of the walks, for any threshold and either
    eviction rule), and a higher threshold loads no more blocks."""
    beg, csr = oracle.rmat_graph(13, 12, seed=5)
    nb = 16
    vb, eb = oracle.split_equal_edge_mass(beg, nb)
    cfg = oracle.make_cfg(algo=0, maxhops=40, p=0.5, q=2.0, seed=9)
    reqs, nent = oracle.walk_requirements(beg, csr, cfg, vb, 0, len(beg) - 1)
    total = oracle.walk(beg, csr, cfg, 0, len(beg) - 1, paths=False)["stats"]["steps"]
    loads = {}
    for ev in (False, True):
        for zt in (0, 40, 200):
            for pf in (False, True):
                st, _ = oracle.sched_replay(reqs, nent, nb, 5, prefetch=pf, zero_threshold=zt, evict_incident=ev,
                                            zero_tail=zt > 0)
                assert st["steps"] + st["zc_steps"] == total, (ev, zt, pf)
                assert (st["zc_steps"] > 0) == (zt > 0) or zt == 0
                loads[(ev, zt, pf)] = st["loads"]
    for ev in (False, True):
        for pf in (False, True):
            assert loads[(ev, 200, pf)] <= loads[(ev, 40, pf)] <= loads[(ev, 0, pf)]

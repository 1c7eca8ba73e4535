"""GPU tests of SOWalker's annealing block choice (GW_POLICY_SA): the device
choice equals the oracle's restatement bit for bit, and out-of-core walks
under it are those of the oracle."""
import numpy as np
import pytest

from test_gpu_ooc import graph, run_ooc

pytestmark = pytest.mark.gpu


def skewed_counts(rng, nb):
    """Walker counts per (prev, cur) pair: a diagonal-heavy band plus a few
    hot pairs and empty rows, like a bucket table mid-run."""
    c = rng.integers(0, 50, (nb, nb))
    c[np.arange(nb), np.arange(nb)] += rng.integers(100, 5000, nb)
    hot = rng.integers(0, nb, (max(nb // 4, 1), 2))
    c[hot[:, 0], hot[:, 1]] += rng.integers(1000, 100000, len(hot))
    c[rng.random(nb) < 0.1, :] = 0
    return c.astype(np.uint32)


@pytest.mark.parametrize("nb,k,ncached", [(8, 3, 0), (8, 3, 3), (16, 5, 2), (64, 15, 15), (64, 15, 7),
                                          (150, 40, 40), (300, 30, 30), (64, 64, 10), (64, 1, 1)])
@pytest.mark.parametrize("call", [0, 3])
def test_sa_choice_matches_oracle(gw, oracle, nb, k, ncached, call):
    rng = np.random.default_rng(nb * 1000 + k * 10 + ncached)
    counts = skewed_counts(rng, nb)
    cached = rng.choice(nb, ncached, replace=False).astype(np.uint32)
    got = gw.sa_choose_blocks(counts, cached, k, seed=42 + call, call=call)
    want = oracle.sa_choose_blocks(counts, cached, k, 42 + call, call)
    assert np.array_equal(got, want)
    assert len(set(got.tolist())) == min(k, nb)


def test_sa_choice_zero_counts_and_bad_args(gw, oracle):
    counts = np.zeros((10, 10), np.uint32)
    got = gw.sa_choose_blocks(counts, [], 4, seed=1)
    assert np.array_equal(got, oracle.sa_choose_blocks(counts, [], 4, 1, 0))
    with pytest.raises(gw.GwError):
        gw.sa_choose_blocks(counts, [10], 4)  # cached block out of range


@pytest.mark.parametrize("algo,prefetch", [(0, 0), (1, 0), (0, 1)])
def test_ooc_sa_policy_same_walks(gw, oracle, algo, prefetch):
    beg, csr = graph(oracle, scale=13, ef=10, sym=True, cap=7000, seed=9)
    V = len(beg) - 1
    from gowalker_b200.preprocess import split_equal_edge_mass
    from test_gpu_ooc import cache_for
    vb, eb = split_equal_edge_mass(beg, 16)
    eng = gw.WalkEngine(algorithm=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, seed=5, walkpersource=1,
                        record_paths=0, cache_size=cache_for(beg, eb, 5), prefetch=prefetch)
    eng.set_host_graph(beg, csr, vb, eb)
    eng.init_walkers(algo, 1, 5)
    st = eng.run(gw.GW_POLICY_SA)
    cfg = oracle.make_cfg(algo=algo, maxhops=30, p=0.5, q=2.0, alpha=0.2, seed=5, wps=1)
    ref = oracle.walk(beg, csr, cfg, 0, V, paths=False)
    assert np.array_equal(eng.hashes(), ref["hashes"])
    assert st["steps"] == ref["stats"]["steps"]
    assert st["block_loads"] >= 5
    eng.close()
    e0, s0 = run_ooc(gw, beg, csr, 16, 5, algo=algo, maxhops=30, paths=0, policy=0)
    assert np.array_equal(e0.hashes(), ref["hashes"])
    e0.close()

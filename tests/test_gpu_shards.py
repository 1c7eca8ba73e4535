"""Walker-id shards (gw_init_walker_range): the population split by id
range, each shard walked on its own, gives exactly the walks of the whole
population -- in-core and out-of-core, every init mode.  The walker ids are
the reference's (engine/walk.hpp:32-49: v*walkpersource + i)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _walk(gw, beg, csr, algo, shard=None, blocks=None, init_mode=0, numwalks=0, wps=2, cache=1 << 34, **kw):
    eng = gw.WalkEngine(algorithm=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2, term_prob=0.1 if algo else 0.0,
                        seed=77, walkpersource=wps, record_paths=1, init_mode=init_mode, numwalks=numwalks,
                        cache_size=cache, **kw)
    vb, eb = (None, None) if blocks is None else blocks
    eng.set_host_graph(beg, csr, vb, eb)
    if shard is None:
        eng.init_walkers(algo, wps, 77)
    else:
        eng.init_walkers(algo, wps, 77, first=shard[0], count=shard[1])
    st = eng.run()
    out = (eng.hashes(), eng.paths(), st)
    eng.close()
    return out


@pytest.mark.parametrize("algo,init_mode", [(0, 0), (1, 0), (2, 1), (0, 2)])
def test_shards_union_equals_whole_incore(gw, oracle, algo, init_mode):
    beg, csr = oracle.rmat_graph(13, 16, seed=3)
    V = len(beg) - 1
    nw = 5000 if init_mode else 0
    H, (P, L), st = _walk(gw, beg, csr, algo, init_mode=init_mode, numwalks=nw)
    n = len(H)
    cuts = [0, n // 3, n // 3 + 1, (2 * n) // 3, n]
    steps = 0
    for a, b in zip(cuts[:-1], cuts[1:]):
        h, (p, l), s = _walk(gw, beg, csr, algo, shard=(a, b - a), init_mode=init_mode, numwalks=nw)
        assert np.array_equal(h, H[a:b]) and np.array_equal(p, P[a:b]) and np.array_equal(l, L[a:b])
        steps += s["steps"]
    assert steps == st["steps"]
    # the oracle agrees on a shard's walkers by their global ids
    cfg = oracle.make_cfg(algo=algo, maxhops=25, p=0.5, q=2.0, alpha=0.2, term_prob=0.1 if algo else 0.0, seed=77,
                          wps=2, init_mode=init_mode, numwalks=nw)
    ids = np.arange(cuts[1], cuts[3], dtype=np.uint32)
    assert np.array_equal(oracle.walk_ids(beg, csr, cfg, ids)["hashes"], H[cuts[1]:cuts[3]])


def test_shards_union_equals_whole_out_of_core(gw, oracle):
    beg, csr = oracle.rmat_graph(13, 16, seed=4)
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, 8)
    slot = ((int(np.diff(eb.astype(np.int64)).max()) + 3) & ~3) * 4
    cache = len(beg) * 8 + 4 * slot
    H, (P, _), _ = _walk(gw, beg, csr, 0, blocks=(vb, eb), cache=cache, wps=1)
    n = len(H)
    for a, b in ((0, 1000), (1000, n)):
        h, (p, _), s = _walk(gw, beg, csr, 0, shard=(a, b - a), blocks=(vb, eb), cache=cache, wps=1, prefetch=1)
        assert s["block_loads"] > 0
        assert np.array_equal(h, H[a:b]) and np.array_equal(p, P[a:b])


def test_shard_bounds_rejected(gw, oracle):
    beg, csr = oracle.rmat_graph(8, 8, seed=1)
    eng = gw.WalkEngine(algorithm=0, maxhops=5, walkpersource=1)
    eng.set_host_graph(beg, csr)
    V = len(beg) - 1
    for first, count in ((V, 1), (0, V + 1), (V - 1, 2), (3, 0)):
        with pytest.raises(gw.GwError):
            eng.init_walkers(0, 1, 1, first=first, count=count)
    eng.init_walkers(0, 1, 1, first=V - 1, count=1)
    assert eng.num_walkers() == 1
    eng.close()

"""GPU parity tests of the preprocessing entry points: gw_edges_csr (edge list
-> CSR on the device) against the oracle's converter restatement, and
gw_split_blocks against the oracle's splitters.  Integer data: every
comparison is equality."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLAG_SETS = [dict(symmetric=s, sort=o, dedup=d) for s in (False, True) for o in (False, True) for d in (False, True)]


def messy_edges(rng, nv, n):
    """Unsorted list with self loops, repeats and hubs."""
    src = rng.integers(0, nv, n).astype(np.uint32)
    dst = rng.integers(0, nv, n).astype(np.uint32)
    hub = rng.random(n) < 0.2
    src[hub] = rng.integers(0, 4, int(hub.sum()))
    loops = rng.random(n) < 0.05
    dst[loops] = src[loops]
    rep = np.nonzero(rng.random(n) < 0.1)[0]
    rep = rep[rep > 0]
    src[rep], dst[rep] = src[rep - 1], dst[rep - 1]
    return src, dst


def device_csr(gw, src, dst, nverts=0, **flags):
    g = gw.DeviceGraph.from_edges(src, dst, nverts=nverts, **flags)
    beg, csr = g.to_host()
    return beg, csr, g.nverts


@pytest.mark.parametrize("flags", FLAG_SETS, ids=lambda f: "".join(k[0] for k, v in f.items() if v) or "plain")
@pytest.mark.parametrize("nv,n", [(50, 400), (3000, 100000), (1 << 17, 1 << 21)])
def test_edges_csr_matches_converter(gw, oracle, flags, nv, n):
    rng = np.random.default_rng(nv + n)
    src, dst = messy_edges(rng, nv, n)
    b1, c1, n1 = device_csr(gw, src, dst, **flags)
    b2, c2, n2 = oracle.convert_edges(src, dst, 0, **flags)
    assert n1 == n2
    assert np.array_equal(b1, b2)
    assert np.array_equal(c1, c2)


def test_edges_csr_device_input_and_given_nverts(gw, oracle):
    import torch
    rng = np.random.default_rng(3)
    src, dst = messy_edges(rng, 5000, 200000)
    ds = torch.from_numpy(src.view(np.int32)).cuda()
    dd = torch.from_numpy(dst.view(np.int32)).cuda()
    b1, c1, n1 = device_csr(gw, ds, dd, nverts=6000, symmetric=True, sort=True)
    b2, c2, n2 = oracle.convert_edges(src, dst, 6000, symmetric=True, sort=True)
    assert n1 == n2 == 6000
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    assert int(b1[5000]) == len(c1)  # vertices past the largest id are empty


def test_edges_csr_edge_cases(gw, oracle):
    L = gw.load()
    # empty list, all self loops
    for src, dst in [(np.zeros(0, np.uint32), np.zeros(0, np.uint32)),
                     (np.arange(10, dtype=np.uint32), np.arange(10, dtype=np.uint32))]:
        b, c, nv = device_csr(gw, src, dst)
        assert nv == 0 and b.tolist() == [0] and len(c) == 0
        b, c, nv = device_csr(gw, src, dst, nverts=12)
        assert nv == 12 and not b.any() and len(c) == 0
    # out of range: an id >= nverts, or 2^32-1 with nverts taken from the data
    src = np.array([0, 7], np.uint32)
    dst = np.array([1, 2], np.uint32)
    with pytest.raises(gw.GwError):
        gw.DeviceGraph.from_edges(src, dst, nverts=7)
    with pytest.raises(gw.GwError):
        gw.DeviceGraph.from_edges(np.array([0xFFFFFFFF], np.uint32), np.array([1], np.uint32))
    db, dc, ne, nv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint32()
    assert L.gw_edges_csr(None, None, 0, 0, 8, ctypes.byref(db), ctypes.byref(dc), ctypes.byref(ne),
                          ctypes.byref(nv)) == -1


def test_edges_csr_rmat_scale20_equals_device_generator(gw, oracle):
    """The C1 graph (R-MAT scale 20, 16 samples per vertex) built two ways on
    the device -- from the counter-based sampler, and from its sample list
    through the converter -- is the same CSR."""
    scale = 20
    g = gw.DeviceGraph(scale)
    b1, c1 = g.to_host()
    src, dst = oracle.rmat_edges(scale, 0, 16 << scale, 1)
    b2, c2, nv = device_csr(gw, src, dst, nverts=1 << scale, symmetric=True, dedup=True)
    assert nv == 1 << scale
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)


@pytest.mark.parametrize("block_mb", [1, 4, 16, 64])
def test_split_reference_matches_restatement(gw, oracle, block_mb):
    beg, csr = oracle.rmat_graph(16)
    vb, eb = gw.split_blocks_device(beg, len(beg) - 1, gw.GW_SPLIT_REFERENCE, (block_mb << 20) // 16)
    rv, re_ = oracle.split_blocks_reference(beg, (block_mb << 20) // 16)
    assert np.array_equal(vb, rv) and np.array_equal(eb, re_)


def test_split_reference_hub_and_tiny_blocks(gw, oracle):
    """Degenerate sizes: a vertex with more edges than a block, blocks of one
    vertex (block size < 16 bytes), and a block-size 0 corner."""
    deg = np.array([1, 500, 2, 0, 0, 3, 900, 1, 1, 0, 7], dtype=np.uint64)
    beg = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint64)
    for bs in [0, 4, 8, 15, 16, 100, 400, 2000, 4000, 1 << 20]:
        vb, eb = gw.split_blocks_device(beg, len(beg) - 1, gw.GW_SPLIT_REFERENCE, bs)
        rv, re_ = oracle.split_blocks_reference(beg, bs)
        assert np.array_equal(vb, rv), bs
        assert np.array_equal(eb, re_), bs
    with pytest.raises(gw.GwError):
        gw.split_blocks_device(beg, len(beg) - 1, gw.GW_SPLIT_REFERENCE, 4, cap=3)


@pytest.mark.parametrize("nblocks", [1, 2, 7, 64, 1000])
def test_split_equal_edges_matches_restatement(gw, oracle, nblocks):
    beg, csr = oracle.rmat_graph(14)
    g = gw.DeviceGraph.from_edges(*oracle.rmat_edges(14, 0, 16 << 14, 1), nverts=1 << 14, symmetric=True,
                                  dedup=True)
    for vb, eb in (gw.split_blocks_device(beg, len(beg) - 1, gw.GW_SPLIT_EQUAL_EDGES, nblocks),
                   g.split(gw.GW_SPLIT_EQUAL_EDGES, nblocks)):
        rv, re_ = oracle.split_equal_edge_mass(beg, nblocks)
        assert np.array_equal(vb, rv) and np.array_equal(eb, re_)


@pytest.mark.parametrize("window,local,dmin", [(64, 800, 6.0), (4096, 500, 3.5), (3, 1000, 2.0)])
def test_web_graph_matches_oracle(gw, oracle, window, local, dmin):
    """The web-shaped generator (power-law out-degrees drawn with the
    fixed-step log/exp, local and R-MAT-distributed destinations) against the
    oracle's restatement."""
    scale, V = 14, 12000
    g = gw.DeviceGraph.web(scale, V, dmin=dmin, local_permille=local, window=window, seed=7)
    b1, c1 = g.to_host()
    b2, c2 = oracle.web_graph(scale, V, dmin=dmin, local_permille=local, window=window, seed=7)
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    assert np.diff(b1.astype(np.int64)).min() >= 1  # every vertex keeps an out-edge


@pytest.mark.parametrize("maker", ["rmat", "web"])
def test_generator_thinning_matches_oracle(gw, oracle, maker):
    scale, V, n = 12, 3000, 40000
    if maker == "rmat":
        full = gw.DeviceGraph(scale, nverts=V, nsamples=n, seed=3, symmetric=False)
        s, d = oracle.rmat_edges(scale, 0, n, 3)
        keep = (s < V) & (d < V)
        b0, c0 = oracle.build_csr(V, s[keep], d[keep], symmetric=False)
    else:
        full = gw.DeviceGraph.web(scale, V, window=100, seed=3)
        b0, c0 = oracle.web_graph(scale, V, window=100, seed=3)
    assert full.nedges == len(c0)
    target = len(c0) - len(c0) // 7
    if maker == "rmat":
        thin = gw.DeviceGraph(scale, nverts=V, nsamples=n, seed=3, symmetric=False, target_edges=target)
    else:
        thin = gw.DeviceGraph.web(scale, V, window=100, seed=3, target_edges=target)
    b1, c1 = thin.to_host()
    b2, c2 = oracle.thin_sorted(b0, c0, target)
    assert np.array_equal(b1, b2) and np.array_equal(c1, c2)
    with pytest.raises(gw.GwError):
        if maker == "rmat":
            gw.DeviceGraph(scale, nverts=V, nsamples=n, seed=3, symmetric=False, target_edges=len(c0) + 1)
        else:
            gw.DeviceGraph.web(scale, V, window=100, seed=3, target_edges=len(c0) + 1)

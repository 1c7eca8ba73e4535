"""gw_walk_noalloc: the walk for callers that cannot let the library allocate
device memory (a host that owns all device memory through its own pool, a
runtime that forbids allocation after start-up).  The caller passes the CSR
and the output buffers; the library's only other memory is a fixed 256-byte
array.  Its walks must equal those of the allocating entry point (gw_run),
bit for bit, on consecutive calls that share that array."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(gw, cfg, dg, nwalkers, paths, fill=0):
    import torch
    L = gw.load()
    hashes = torch.full((nwalkers,), fill, dtype=torch.int64, device="cuda")
    lens = torch.full((nwalkers,), fill, dtype=torch.int32, device="cuda")
    prows = torch.full((nwalkers, cfg.maxhops + 1), fill, dtype=torch.int32, device="cuda") if paths else None
    st = gw.GwStats()
    rc = L.gw_walk_noalloc(ctypes.byref(cfg), ctypes.c_void_p(dg.beg_ptr), ctypes.c_void_p(dg.csr_ptr), dg.nverts,
                           dg.nedges, nwalkers, ctypes.c_void_p(hashes.data_ptr()), ctypes.c_void_p(lens.data_ptr()),
                           ctypes.c_void_p(prows.data_ptr() if paths else 0), None, ctypes.byref(st))
    assert rc == 0, rc
    out = (hashes.cpu().numpy().view(np.uint64), lens.cpu().numpy().view(np.uint32),
           prows.cpu().numpy().view(np.uint32) if paths else None)
    return out, st


@pytest.mark.parametrize("algo,maxhops,term,wps,p,q", [(1, 20, 0.15, 2, 0.5, 2.0), (0, 30, 0.0, 1, 2.0, 0.5)])
def test_noalloc_matches_gw_run_twice(gw, algo, maxhops, term, wps, p, q):
    dg = gw.DeviceGraph(13, edgefactor=16, seed=7)
    cfg = gw.default_config(algorithm=algo, maxhops=maxhops, term_prob=term, walkpersource=wps, p=p, q=q,
                            alpha=0.2, seed=11, record_paths=1)
    eng = gw.WalkEngine(cfg)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    eng.init_walkers(algo, wps, 11)
    ref_stats = eng.run()
    ref_paths, ref_lens = eng.paths()
    ref_hashes = eng.hashes()
    n = eng.num_walkers()
    eng.close()
    # the second call reuses the scratch the first one left behind; its
    # output buffers start filled with ones, as a reused caller buffer may be
    for fill in (0, -1):
        (h, l, pr), st = _noalloc(gw, cfg, dg, n, paths=True, fill=fill)
        assert np.array_equal(h, ref_hashes)
        assert np.array_equal(l, ref_lens)
        assert np.array_equal(pr, ref_paths)
        assert st.steps == ref_stats["steps"] and st.walkers == n
    dg.free()


def test_noalloc_rejects_bad_sizes(gw):
    import torch
    dg = gw.DeviceGraph(10, edgefactor=8, seed=3)
    L = gw.load()
    cfg = gw.default_config(algorithm=0, maxhops=10, walkpersource=1)
    buf = torch.zeros(dg.nverts, dtype=torch.int64, device="cuda")
    common = (ctypes.c_void_p(dg.beg_ptr), ctypes.c_void_p(dg.csr_ptr), dg.nverts, dg.nedges)
    # population does not match the configuration
    assert L.gw_walk_noalloc(ctypes.byref(cfg), *common, dg.nverts + 1, ctypes.c_void_p(buf.data_ptr()),
                             ctypes.c_void_p(buf.data_ptr()), None, None, None) == -1
    # 2^32 walkers or more: walker ids are 32-bit
    wps = (1 << 32) // dg.nverts + 1
    big = gw.default_config(algorithm=0, maxhops=10, walkpersource=wps)
    assert dg.nverts * wps > 0xFFFFFFFF
    assert L.gw_walk_noalloc(ctypes.byref(big), *common, dg.nverts * wps, ctypes.c_void_p(buf.data_ptr()),
                             ctypes.c_void_p(buf.data_ptr()), None, None, None) == -1
    dg.free()

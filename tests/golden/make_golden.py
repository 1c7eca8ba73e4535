"""Generate the golden walk fixtures under tests/golden/.

Run from the repository root on a machine that has the GOWalker sources, after
`make -C oracle all` built the reference step harness (oracle/_ref):

    python tests/golden/make_golden.py

For every fixture the walks come from the oracle (oracle/gw_oracle.c) and are
first checked, trial by trial, against the reference's own
graph_engine::sidewalkupdate / SOPR_sidewalkupdate (engine/engine.hpp:158-404)
driven through the Philox shim (oracle/ref_step_harness.cu).  The script stops
if the two disagree, so a committed fixture is pinned to the reference's code.
"""
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, graph (scale, edgefactor, symmetric, nverts cap), walk config
    ("n2v_sym_s8", (8, 8, True, None), dict(algo=O.ALG_NODE2VEC, maxhops=20, p=2.0, q=0.5, wps=2)),
    ("n2v_dir_s8", (8, 6, False, 200), dict(algo=O.ALG_NODE2VEC, maxhops=20, p=0.5, q=2.0, wps=1)),
    ("sopr_sym_s8", (8, 8, True, None), dict(algo=O.ALG_SOPR, maxhops=20, alpha=0.2, wps=2)),
    ("sosr_dir_s8", (8, 6, False, 200), dict(algo=O.ALG_SOSR, maxhops=15, alpha=0.3, wps=1)),
]
SEED = 42


def graph(scale, ef, symmetric, cap):
    V = (1 << scale) if cap is None else cap
    src, dst = O.rmat_edges(scale, 0, ef << scale, seed=1)
    keep = (src < V) & (dst < V)
    return O.build_csr(V, src[keep], dst[keep], symmetric)


def verify_against_reference(name, beg, csr, wc):
    """Trial-by-trial equality of oracle and reference step for every walker."""
    beg2, csr2, vb, eb = O.harness_graph(beg, csr)
    tmp = tempfile.mkdtemp(prefix="gw_golden_")
    base = os.path.join(tmp, "g")
    O.write_dataset(base, beg2, csr2)
    O.write_blocks(base, 1, vb, eb)
    V = len(beg) - 1
    starts = [(v, V + v, v, 0, V + v, v) for v in range(V)]
    args = (base, wc["algo"], wc.get("p", 0.5), wc.get("q", 2.0), wc.get("alpha", 0.2), wc["maxhops"], 1, SEED,
            starts)
    with mp.get_context("spawn").Pool(1) as pool:
        _, res = pool.apply(O.ref_scenario, args)
    cfg = O.make_cfg(algo=wc["algo"], maxhops=wc["maxhops"], p=wc.get("p", 0.5), q=wc.get("q", 2.0),
                     alpha=wc.get("alpha", 0.2), seed=SEED, keying=O.KEY_TRIAL)
    trials = 0
    for v in range(V):
        moves, _, trace, final = O.walk_traced(beg, csr, cfg, v, v, v, 0)
        run, rtrace, _, _ = res[v]
        dead = 1 if (moves < wc["maxhops"] and final[1] == 0 and final[2] == wc["maxhops"]) else 0
        if not (np.array_equal(trace, rtrace) and run == moves + dead):
            raise SystemExit("%s: oracle and reference disagree at walker %d" % (name, v))
        trials += len(trace)
    return trials


def main():
    for name, (scale, ef, sym, cap), wc in CASES:
        beg, csr = graph(scale, ef, sym, cap)
        trials = verify_against_reference(name, beg, csr, wc)
        V = len(beg) - 1
        cfg = O.make_cfg(algo=wc["algo"], maxhops=wc["maxhops"], p=wc.get("p", 0.5), q=wc.get("q", 2.0),
                         alpha=wc.get("alpha", 0.2), term_prob=0.0, seed=SEED, wps=wc["wps"])
        r = O.walk(beg, csr, cfg, 0, V * wc["wps"], paths=True)
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"), beg=beg, csr=csr, paths=r["paths"], lens=r["lens"],
            hashes=r["hashes"], algo=wc["algo"], maxhops=wc["maxhops"], p=np.float32(wc.get("p", 0.5)),
            q=np.float32(wc.get("q", 2.0)), alpha=np.float32(wc.get("alpha", 0.2)), wps=wc["wps"], seed=SEED,
            steps=r["stats"]["steps"], reference_trials_checked=trials)
        print("%s: V=%d E=%d walkers=%d steps=%d reference trials checked=%d" %
              (name, V, len(csr), V * wc["wps"], r["stats"]["steps"], trials))
    # Philox known answers from the oracle (regression pins; the GPU test
    # also checks the device generator against curand's Philox4_32_10).
    ctrs = np.array([[0, 0, 0, 0], [1, 2, 3, 4], [0xFFFFFFFF] * 4, [7, 80, 3, 0x524D4154]], dtype=np.uint32)
    keys = np.array([[0, 0], [42, 0], [0xFFFFFFFF, 0xFFFFFFFF], [1, 0]], dtype=np.uint32)
    outs = np.stack([O.philox(c, k) for c, k in zip(ctrs, keys)])
    np.savez_compressed(os.path.join(OUT, "philox.npz"), ctrs=ctrs, keys=keys, outs=outs)


if __name__ == "__main__":
    main()

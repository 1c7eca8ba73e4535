"""Whole-run checksums of the in-core workloads, computed by the oracle on
the CPU, for tests/golden/config_checksums.json.

For each workload the graph is built by the oracle's R-MAT restatement
(counter-based samples, symmetrised, deduplicated, sorted) and every walker
is walked by the oracle's restatement of the reference step
(engine/engine.hpp:158-404) under the Philox stream.  Recorded: the graph's
size and SHA-256 of its offsets and neighbour ids (so a test can show the
device generator built the same graph), and the run's sum of path hashes
(mod 2^64), steps and trials.

    python tests/golden/make_config_checksums.py [c1] [c2]

C2 takes several minutes on 8 host threads (about 430 M steps)."""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

WORKLOADS = {
    "c1": dict(scale=20, ef=16, algo=0, maxhops=80, wps=1, p=2.0, q=0.5, alpha=0.2, term=0.0, seed=42),
    "c2": dict(scale=24, ef=16, algo=1, maxhops=20, wps=4, p=0.5, q=2.0, alpha=0.2, term=0.15, seed=42),
}
OUT = os.path.join(HERE, "config_checksums.json")


def graph_digest(beg, csr):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(beg, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(csr, dtype=np.uint32).tobytes())
    return h.hexdigest()


def main(names):
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name in names:
        w = WORKLOADS[name]
        t0 = time.time()
        beg, csr = O.rmat_graph(w["scale"], w["ef"], seed=1, symmetric=True)
        V = len(beg) - 1
        print("%s: graph V=%d E=%d in %.0fs" % (name, V, len(csr), time.time() - t0), flush=True)
        cfg = O.make_cfg(algo=w["algo"], maxhops=w["maxhops"], p=w["p"], q=w["q"], alpha=w["alpha"],
                         term_prob=w["term"], seed=w["seed"], wps=w["wps"])
        n = V * w["wps"]
        hsum, steps, trials = 0, 0, 0
        chunk = 1 << 22
        t0 = time.time()
        for s in range(0, n, chunk):
            r = O.walk(beg, csr, cfg, s, min(chunk, n - s), paths=False)
            hsum = (hsum + int(r["hashes"].sum(dtype=np.uint64))) & 0xFFFFFFFFFFFFFFFF
            steps += r["stats"]["steps"]
            trials += r["stats"]["trials"]
        print("%s: %d walkers, %d steps in %.0fs" % (name, n, steps, time.time() - t0), flush=True)
        data[name] = dict(w, vertices=V, edges=len(csr), graph_sha256=graph_digest(beg, csr), walkers=n,
                          path_hash_sum=str(hsum), steps=steps, trials=trials)
        json.dump(data, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c1", "c2"])

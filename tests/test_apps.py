"""The Node2vec / SOPR / SOSR apps (gowalker_b200/apps): GOWalker's flags and
defaults (apps/Node2vec.cu:35-135), block files, and walks through the app
equal to the oracle's."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "gowalker_b200", "apps", "bin")


@pytest.fixture(scope="module")
def apps():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gowalker_b200", "host")], check=True)
    return BIN


@pytest.fixture(scope="module")
def dataset(tmp_path_factory, oracle):
    from gowalker_b200 import preprocess as P
    d = tmp_path_factory.mktemp("ds")
    beg, csr = oracle.rmat_graph(11, 8, seed=4)
    base = str(d / "g")
    P.write_dataset(base, beg, csr)
    return base, beg, csr


def run(apps, app, *args, check=True):
    out = subprocess.run([os.path.join(apps, app)] + [str(a) for a in args], capture_output=True, text=True,
                         timeout=600, cwd=os.path.dirname(args[0]) if args and os.path.isabs(str(args[0])) else None)
    if check:
        assert out.returncode == 0, out.stderr
    return out


def config(apps, app, base, *flags):
    out = run(apps, app, base + ".txt", "skip", "print-config", *flags)
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_help(apps):
    out = run(apps, "Node2vec", "x", "h")
    assert "walkpersource" in out.stdout and "length" in out.stdout


def test_defaults_and_rules(apps, dataset):
    base, beg, csr = dataset
    V = len(beg) - 1
    c = config(apps, "Node2vec", base)
    assert c["base_name"] == base
    assert abs(c["p"] - 0.5) < 1e-7 and abs(c["q"] - 2.0) < 1e-7 and abs(c["alpha"] - 0.2) < 1e-7
    assert c["maxhops"] == 30 and c["blocksize"] == 1024 << 20 and c["cache_size"] == 4 << 30
    assert c["numwalks"] == V and c["walkpersource"] == 1 and c["init_mode"] == 0
    assert c["zero_threshold"] == 0
    c = config(apps, "Node2vec", base, "walkpersource", 3, "length", 80, "p", 2, "q", 0.5)
    assert c["numwalks"] == 3 * V and c["maxhops"] == 80 and abs(c["p"] - 2.0) < 1e-7
    c = config(apps, "Node2vec", base, "numwalks", 1000)          # numwalks given: walkpersource = 0
    assert c["numwalks"] == 1000 and c["walkpersource"] == 0 and c["init_mode"] == 2
    c = config(apps, "Node2vec", base, "zero", "blocksize", 256)  # zero_threshold = blocksize/128/24
    assert c["zero_threshold"] == (256 << 20) // 128 // 24
    c = config(apps, "SOPR", base)                               # SOPR: all walkers at vertex 1
    assert c["algorithm"] == 1 and c["init_mode"] == 1 and c["numwalks"] == V
    c = config(apps, "SOSR", base, "persource", "termination", 0.15, "--seed=7", "learned")
    assert c["algorithm"] == 2 and c["init_mode"] == 0 and abs(c["term_prob"] - 0.15) < 1e-7
    assert c["seed"] == 7 and c["learned"] == 1


def test_block_files_follow_reference_splitter(apps, dataset, oracle):
    base, beg, csr = dataset
    config(apps, "Node2vec", base, "blocksize", 1)
    from gowalker_b200 import preprocess as P
    v, e = P.load_blocks(base, 1)
    vr, er = oracle.split_blocks_reference(beg, 1 << 20)
    assert np.array_equal(v, vr) and np.array_equal(e, er)


def test_node2vec_requires_one_scheduler(apps, dataset):
    base, _, _ = dataset
    out = run(apps, "Node2vec", base + ".txt", "skip")
    assert "Please select one walker" in out.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("app,algo,extra,ocfg", [
    ("Node2vec", 0, ["GOWalker", "gpu", "p", 2, "q", 0.5, "length", 25, "walkpersource", 2], dict(wps=2, p=2.0, q=0.5)),
    ("SOPR", 1, ["GOWalker", "length", 20, "termination", 0.15], dict(init_mode=1, numwalks=None, term_prob=0.15)),
    ("SOSR", 2, ["GOWalker", "length", 20, "persource", "termination", 0.15], dict(wps=1, term_prob=0.15)),
])
def test_app_walks_match_oracle(apps, dataset, oracle, tmp_path, app, algo, extra, ocfg):
    base, beg, csr = dataset
    V = len(beg) - 1
    pfile = tmp_path / "paths.txt"
    out = run(apps, app, base + ".txt", "skip", "seed", 9, "paths", pfile, *extra)
    assert "walks:" in out.stdout
    maxhops = int(extra[extra.index("length") + 1])
    kw = dict(algo=algo, maxhops=maxhops, seed=9, p=ocfg.get("p", 0.5), q=ocfg.get("q", 2.0), alpha=0.2,
              term_prob=ocfg.get("term_prob", 0.0), wps=ocfg.get("wps", 1), init_mode=ocfg.get("init_mode", 0))
    n = V * kw["wps"]
    if kw["init_mode"] == 1:
        kw["numwalks"] = V
        n = V
    ref = oracle.walk(beg, csr, oracle.make_cfg(**kw), 0, n, paths=True)
    lines = open(pfile).read().splitlines()
    assert len(lines) == n
    for w in range(0, n, max(1, n // 300)):
        L = int(ref["lens"][w])
        assert lines[w].split() == [str(x) for x in ref["paths"][w, :L]], w
    metrics = open(os.path.join(os.path.dirname(base), "randgraph_metrics.txt")).read()
    assert ".0_Total_time=" in metrics and ".1_GPUTime=" in metrics and ".steps=" in metrics


@pytest.mark.gpu
def test_weighted_node2vec_app_matches_oracle(apps, dataset, oracle, tmp_path):
    """`weighted` reads <base>.wht and the walks follow the weights."""
    from gowalker_b200 import preprocess as P
    base, beg, csr = dataset
    wbase = str(tmp_path / "gw")
    P.write_dataset(wbase, beg, csr)
    w = np.random.default_rng(6).lognormal(0.0, 1.0, len(csr)).astype(np.float32)
    P.write_weights(wbase, w)
    pfile = tmp_path / "paths.txt"
    run(apps, "Node2vec", wbase + ".txt", "skip", "weighted", "seed", 3, "paths", pfile, "GOWalker", "p", 2,
        "q", 0.5, "length", 15)
    V = len(beg) - 1
    ref = oracle.walk(beg, csr, oracle.make_cfg(algo=0, maxhops=15, seed=3, p=2.0, q=0.5), 0, V, paths=True,
                      alias=oracle.build_alias(beg, w))
    lines = open(pfile).read().splitlines()
    assert len(lines) == V
    for i in range(0, V, max(1, V // 300)):
        L = int(ref["lens"][i])
        assert lines[i].split() == [str(x) for x in ref["paths"][i, :L]], i

#!/usr/bin/env python3
"""Walk-engine benchmark: walk steps/s on one B200 (per rank), JSON on one line.

Workload (default, `--config c3`): out-of-core Node2vec (p=0.5, q=2, length
80, one walker per vertex, walk seed 42) on the 41.6 M-vertex, 1.47 B-edge
directed R-MAT graph (scale 26, ids >= 41.6 M rejected, thinned to exactly
1.47 B edges, generator seed 1), split into 64 equal-edge-mass blocks held in
pinned host memory, device block cache capped at 1.5 GB.  Two arms run after
one another on the same engine, K times each: GOWalker's block choice
(plain) and the learned demand predictor (learned), both with GOWalker's zero
mode (the tail read through mapped host memory, `--no-zero-copy` to turn it
off); value = the learned arm's steps/s, the plain arm beside it with both
arms' H2D bytes per step, and the walks of both arms must be identical.

One bench step = one full run of every walker of the workload (gw_run).
Other workloads: `--config c2` (in-core SOPR, scale 24), `c1` (in-core
Node2vec, scale 20), `c1w` (weighted), `c4`, `c5`, `c3s` (C3 at 1/16 size),
`prep` (edge list -> CSR).  In-core lines time the graph resident in HBM
(value) and end to end through the C ABI with the CSR copied from pinned host
memory and the walks read back (e2e).

Under torchrun every rank walks one walker-id shard of the same population
(walkers are independent: no data-path collective); value = all ranks' steps
/ the slowest rank's time.

`--impl reference` times the oracle (the reference CPU step rule restated in
C, OpenMP over all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c2": dict(name="C2: SOPR alpha=0.2, termination 0.15, max length 20, 4 walkers/vertex, "
                    "R-MAT scale 24 ef 16 symmetrised, in-core",
               scale=24, ef=16, algo=1, maxhops=20, wps=4, p=0.5, q=2.0, alpha=0.2, term=0.15),
    "c1": dict(name="C1: Node2vec p=2 q=0.5 length 80, 1 walker/vertex, R-MAT scale 20 ef 16 symmetrised, in-core",
               scale=20, ef=16, algo=0, maxhops=80, wps=1, p=2.0, q=0.5, alpha=0.2, term=0.0),
    "c1w": dict(name="C1 weighted: Node2vec p=2 q=0.5 length 80, 1 walker/vertex, R-MAT scale 20 ef 16 symmetrised, "
                     "edge weights lognormal(0, 1) (torch generator seed 1), in-core",
                scale=20, ef=16, algo=0, maxhops=80, wps=1, p=2.0, q=0.5, alpha=0.2, term=0.0, weighted=True),
    "c3": dict(name="C3: out-of-core Node2vec p=0.5 q=2 length 80, 1 walker/vertex, directed R-MAT scale 26 "
                    "rejecting ids >= 41.6M, thinned to 1.47B edges, 64 equal-edge-mass blocks, 1.5 GB device cache",
               scale=26, nverts=41_600_000, target=1_470_000_000, nsamples=2_600_000_000, ef=0, algo=0, maxhops=80,
               wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, nblocks=64, cache=1_500_000_000, ooc=True),
    "c3s": dict(name="C3 at 1/16 size (profiling case): out-of-core Node2vec p=0.5 q=2 length 80, 1 walker/vertex, "
                     "directed R-MAT scale 22 rejecting ids >= 2.6M, thinned to 91.875M edges, 64 equal-edge-mass "
                     "blocks, 93.75 MB device cache",
                scale=22, nverts=2_600_000, target=91_875_000, nsamples=162_500_000, ef=0, algo=0, maxhops=80,
                wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, nblocks=64, cache=93_750_000, ooc=True),
    "c4": dict(name="C4: out-of-core SOPR/SOSR transition rule (alpha 0.2, termination 0.15, max length 20), 2 walkers "
                    "per vertex, undirected R-MAT scale 26 rejecting ids >= 65.6M, symmetrised and thinned to 3.6B "
                    "directed edges, 128 equal-edge-mass blocks, 4 GB device cache",
               scale=26, nverts=65_600_000, target=3_600_000_000, nsamples=2_100_000_000, ef=0, algo=1, maxhops=20,
               wps=2, p=0.5, q=2.0, alpha=0.2, term=0.15, nblocks=128, cache=4_000_000_000, ooc=True, sym=True),
    "c5": dict(name="C5: out-of-core Node2vec p=0.5 q=2 length 80, 1 walker/vertex, web-shaped graph: 133.6M vertices, "
                    "5.5B directed edges, out-degree power law P(D>=d)=(d/6.8)^-1.1 (exponent 2.1, cap 65,536), 80% "
                    "of edges within +-65,536 of the source id, the rest to R-MAT (scale 28) destinations, 256 "
                    "equal-edge-mass blocks, 8 GB device cache",
               scale=28, nverts=133_600_000, target=5_500_000_000, nsamples=0, ef=0, algo=0, maxhops=80,
               wps=1, p=0.5, q=2.0, alpha=0.2, term=0.0, nblocks=256, cache=8_000_000_000, ooc=True, web=True,
               dmin=6.8, tail=1.1, max_degree=65536, local_permille=800, window=65536),
    "c5s": dict(name="C5 at 1/16 size (profiling case): out-of-core Node2vec p=0.5 q=2 length 80, 1 walker/vertex, "
                     "web-shaped graph, 8.35M vertices, 343.75M edges, 256 equal-edge-mass blocks, 500 MB device cache",
                scale=24, nverts=8_350_000, target=343_750_000, nsamples=0, ef=0, algo=0, maxhops=80, wps=1, p=0.5,
                q=2.0, alpha=0.2, term=0.0, nblocks=256, cache=500_000_000, ooc=True, web=True, dmin=6.8, tail=1.1,
                max_degree=65536, local_permille=800, window=65536),
    "prep": dict(name="edge list -> CSR on the device (gw_edges_csr): R-MAT scale 24 ef 16 sample list "
                      "(268,435,456 u32 pairs, (a,b,c,d) = (0.57,0.19,0.19,0.05)), symmetrised, deduplicated, sorted",
                 scale=24, ef=16, prep=True),
}
L2_BYTES = 126 * 1024 * 1024


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_bytes_per_step(workload):
    """dram bytes per walk step from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "walk_incore_%s.md" % workload)
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_step:\s*([0-9.]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers

def build_graph(gw, wl):
    t0 = time.time()
    if wl.get("ooc"):
        nsamples = wl["nsamples"]
        for _ in range(4):
            try:
                if wl.get("web"):
                    dg = gw.DeviceGraph.web(wl["scale"], wl["nverts"], dmin=wl["dmin"], tail=wl["tail"],
                                            max_degree=wl["max_degree"], local_permille=wl["local_permille"],
                                            window=wl["window"], seed=1, target_edges=wl["target"])
                else:
                    dg = gw.DeviceGraph(wl["scale"], nverts=wl["nverts"], nsamples=nsamples, seed=1,
                                        symmetric=bool(wl.get("sym")), target_edges=wl["target"])
                break
            except gw.GwError as exc:
                if exc.status != -1:
                    raise
                nsamples = int(nsamples * 1.2)  # too few unique edges: sample more
                wl["dmin"] = wl.get("dmin", 1.0) * 1.1
        else:
            raise RuntimeError("could not reach the target edge count")
        log("graph: V=%d E=%d from %d samples, built on device in %.1fs" % (dg.nverts, dg.nedges, nsamples,
                                                                           time.time() - t0))
        return dg
    dg = gw.DeviceGraph(wl["scale"], edgefactor=wl["ef"], seed=1, symmetric=True)
    log("graph: V=%d E=%d built on device in %.1fs" % (dg.nverts, dg.nedges, time.time() - t0))
    return dg


def host_graph(dg):
    beg_t, csr_t = dg.to_host(pinned=True)
    beg = beg_t.numpy().view(np.uint64)
    csr = csr_t.numpy().view(np.uint32)[: dg.nedges]
    return beg_t, csr_t, beg, csr


def oracle_sample(O, beg, csr, wl, seed, target_s, nchunks=32, threads=0, alias=None):
    """Time the oracle on an evenly spread sample of the workload's walkers,
    sized to take about target_s seconds.  Returns (steps, seconds, stats,
    walkers, description)."""
    V = len(beg) - 1
    nwalk = V * wl["wps"]
    cfg = O.make_cfg(algo=wl["algo"], maxhops=wl["maxhops"], p=wl["p"], q=wl["q"], alpha=wl["alpha"],
                     term_prob=wl["term"], seed=seed, wps=wl["wps"])
    # calibration
    t0 = time.time()
    r = O.walk(beg, csr, cfg, nwalk // 3, 20000, paths=False, nthreads=threads, alias=alias)
    dt = max(time.time() - t0, 1e-3)
    per_walker = dt / 20000
    count = int(max(nchunks * 64, min(nwalk, target_s / per_walker)))
    chunk = max(1, count // nchunks)
    starts = [int(i * (nwalk - chunk) / max(nchunks - 1, 1)) for i in range(nchunks)]
    tot = {k: 0 for k in r["stats"]}
    t0 = time.time()
    for s in starts:
        rr = O.walk(beg, csr, cfg, s, chunk, paths=False, nthreads=threads, alias=alias)
        for k, v in rr["stats"].items():
            tot[k] += v
    secs = time.time() - t0
    desc = "%d walkers in %d evenly spaced runs of %d (of %d)" % (chunk * nchunks, nchunks, chunk, nwalk)
    return tot["steps"], secs, tot, chunk * nchunks, desc


def algorithmic_bytes(stats, walkers, paths, weighted=False):
    """Bytes the walk must move: 32-B sectors for (beg[cur], beg[cur+1]), one csr
    sector per trial, the distinct sectors of each trial's search of N(prev),
    plus the per-walker outputs (hash 8 B, length 4 B, path entries 4 B).
    Weighted walks read one more sector per trial (the alias-table entry)."""
    b = 32 * (stats["off_sectors"] + stats["trials"] * (2 if weighted else 1) + stats["search_sectors"])
    b += 12 * walkers
    if paths:
        b += 4 * (stats["steps"] + walkers)
    return b


# ---------------------------------------------------------------- arms

def run_reference_arm(args, wl):
    """The reference's CPU walk step (oracle port) on the host cores."""
    import gowalker_b200 as gw
    from oracle import oracle as O
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dg = build_graph(gw, wl)
    _, _, beg, csr = host_graph(dg)[:4]
    alias = None
    if wl.get("weighted"):
        import torch
        g = torch.Generator(device="cuda")
        g.manual_seed(1)
        w = torch.empty(dg.nedges, dtype=torch.float32, device="cuda").log_normal_(0.0, 1.0, generator=g)
        alias = O.build_alias(beg, w.cpu().numpy())
    dg.free()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_sample(O, beg, csr, wl, 42, 0.5, threads=threads, alias=alias)
    steps = secs = 0.0
    desc = ""
    for _ in range(args.steps):
        s, t, _, _, desc = oracle_sample(O, beg, csr, wl, 42, args.ref_seconds, threads=threads, alias=alias)
        steps += s
        secs += t
    v = steps / secs
    # the metric of this workload's own line (the out-of-core pair's by default)
    metric = ("walk steps/sec on 1 B200, learned vs plain schedule (bit-exact); H2D bytes/step"
              if wl.get("ooc") and args.policy == "pair" else "walk steps/sec")
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+fp32/fp64 compares",
            "data": "synthetic", "config": {"workload": wl["name"]},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": "per step: " + desc},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_prep_reference(args, wl):
    """The converter restatement (numpy, one thread) on a bounded prefix of
    the same sample list, per step."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = wl["ef"] << wl["scale"]
    V = 1 << wl["scale"]
    src, dst = rmat_edges_torch(wl["scale"], n, 1)
    src, dst = src.cpu().numpy().view(np.uint32), dst.cpu().numpy().view(np.uint32)
    for _ in range(args.warmup):
        prep_cpu_baseline(src, dst, V, 0.5)
    vals = [prep_cpu_baseline(src, dst, V, args.ref_seconds) for _ in range(args.steps)]
    v = sum(x["value"] for x in vals) / len(vals)
    line = {"impl": "reference", "metric": "edge-list samples converted/sec", "value": v, "unit": "samples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * args.ref_seconds, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 ids, u64 keys", "data": "synthetic",
            "config": {"workload": wl["name"]},
            "cpu_baseline": dict(vals[-1], value=v),
            "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


PCIE_GEN5_X16_GBS = 64.0  # nominal host-link peak per direction, for context


def cpu_model():
    """Host CPU model name (for the CPU baseline's record)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measure_h2d_peak(device, nbytes=1 << 30, reps=4):
    """Host-link peak of this box: the best of `reps` pinned host -> device
    copies of `nbytes`, timed with CUDA events (GB/s)."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device=device)
    best = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d.copy_(h, non_blocking=True)
        e1.record()
        e1.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del h, d
    torch.cuda.empty_cache()
    return best


def rank_shard(rank, world, n):
    """Walker ids [first, first+count) of rank `rank`: the population split
    into `world` contiguous id ranges (the reference's ids, engine/walk.hpp:
    32-49), sizes differing by at most one."""
    q, r = divmod(n, world)
    first = rank * q + min(rank, r)
    return first, q + (1 if rank < r else 0)


def combine_hash_sums(dist, local, device):
    """Sum (mod 2^64) of the ranks' path-hash sums: with walker-id shards it
    equals the checksum of the whole population walked in one process.  Every
    rank must call it."""
    if dist is None:
        return int(local) & 0xFFFFFFFFFFFFFFFF
    import torch
    world = dist.get_world_size()
    v = torch.tensor([int(local) & 0xFFFFFFFF, int(local) >> 32], dtype=torch.int64, device=device)
    out = [torch.zeros_like(v) for _ in range(world)]
    dist.all_gather(out, v)
    return sum(int(t[0]) | (int(t[1]) << 32) for t in out) & 0xFFFFFFFFFFFFFFFF


def init_dist():
    """torch.distributed over NCCL when launched by torchrun (RANK/WORLD_SIZE
    in the environment), with a short timeout; returns (dist or None, rank,
    world, local)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world <= 1:
        return None, rank, world, local
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return dist, rank, world, local


POLICIES = {"plain": 0, "learned": 1, "sa": 2}


def run_ooc_bench(args, wl):
    """Out-of-core workload: blocks in pinned host memory, device cache capped.
    Default: the plain and the learned block policy, run after one another K
    times each on the same engine; value = the learned arm's steps/s."""
    import torch
    import gowalker_b200 as gw
    dist, rank, world, local = init_dist()
    dev = torch.device("cuda", local)
    peak_h2d = measure_h2d_peak(dev)
    dg = build_graph(gw, wl)
    beg_t, csr_t, beg, csr = host_graph(dg)
    dg.free()
    from gowalker_b200.preprocess import split_equal_edge_mass
    vb, eb = split_equal_edge_mass(beg, wl["nblocks"])
    arms = ["plain", "learned"] if args.policy == "pair" else [args.policy]
    V = len(beg) - 1
    # GOWalker's zero mode: its threshold is blocksize / 128 / 24 walkers
    # (apps/Node2vec.cu:100-108), the block size here the largest block's bytes
    zero_threshold = int(4 * int(np.diff(eb.astype(np.int64)).max()) / 128 / 24) if args.zero_copy else 0
    zero_threshold = int(zero_threshold * args.zero_scale)
    first, count = rank_shard(rank, world, V * wl["wps"])
    eng = gw.WalkEngine(algorithm=wl["algo"], maxhops=wl["maxhops"], p=wl["p"], q=wl["q"], alpha=wl["alpha"],
                        term_prob=wl["term"], seed=42, walkpersource=wl["wps"], record_paths=0,
                        cache_size=wl["cache"], zero_copy=1 if args.zero_copy else 0, zero_threshold=zero_threshold,
                        strict_blocks=1 if args.strict_blocks else 0,
                        prefetch=0 if args.no_prefetch else 1, compress_blocks=0 if args.no_compress else 1,
                        learned_mode=args.learned_mode, device=local)
    eng.set_host_graph(beg_t, csr_t[: len(csr)], vb, eb)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=local)
    h_hash = np.zeros(count, dtype=np.uint64)
    L = gw.load()
    import ctypes

    def one(arm, timed=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        eng.init_walkers(wl["algo"], wl["wps"], 42, first=first, count=count)
        st = eng.run(POLICIES[arm])
        ev[1].record(stream)
        # the run's result back in host memory: every walker's path hash
        eng._check(L.gw_path_hashes(eng.h, 0, count, ctypes.c_void_p(h_hash.ctypes.data)))
        ev[2].record(stream)
        if timed is not None:
            timed.append((ev, st, int(h_hash.sum(dtype=np.uint64))))
        return st

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        for arm in arms:
            one(arm)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    rec = {arm: [] for arm in arms}
    for _ in range(args.steps):
        for arm in arms:
            one(arm, rec[arm])
    barrier()
    clk = clocks.stop()
    res = {}
    for arm in arms:
        run_ms = sum(ev[0].elapsed_time(ev[1]) for ev, _, _ in rec[arm])
        e2e_ms = sum(ev[0].elapsed_time(ev[2]) for ev, _, _ in rec[arm])
        sts = [st for _, st, _ in rec[arm]]
        steps = sum(st["steps"] for st in sts)
        h2d = sum(st["h2d_bytes"] for st in sts)
        run_ms, e2e_ms, steps_all, h2d_all = reduce_rank_times(dist, run_ms, e2e_ms, steps, h2d, "cuda")
        hsum = combine_hash_sums(dist, rec[arm][-1][2], dev)
        res[arm] = dict(
            value=steps_all / (run_ms / 1e3), e2e=steps_all / (e2e_ms / 1e3), ms_per_run=run_ms / args.steps,
            h2d_bytes_per_run=h2d_all / args.steps, h2d_bytes_per_walk_step=h2d_all / max(steps_all, 1),
            steps_per_run=steps_all / args.steps, block_loads_per_run=sum(s["block_loads"] for s in sts) / args.steps,
            iterations_per_run=sum(s["iterations"] for s in sts) / args.steps,
            launches=sum(s["launches"] for s in sts), path_hash_sum=str(hsum),
            zero_copy_steps_per_run=sum(s["zero_copy_steps"] for s in sts) / args.steps,
            kernel_ms_per_run=sum(s["kernel_ms"] for s in sts) / args.steps,
            bucket_ms_per_run=sum(s["bucket_ms"] for s in sts) / args.steps,
            learned_iterations_per_run=sum(s["learned_iterations"] for s in sts) / args.steps,
            reverted_runs=sum(s["policy_reverted"] for s in sts),
            learned_parts=[s["learned_parts"] for s in sts])
        # the copy stream: busy time of the block copies, and the block bytes
        # (H2D bytes less the mapped sectors of the tail) over that time
        copy_ms = sum(s["copy_ms"] for s in sts)
        block_bytes = sum(s["h2d_bytes"] - 32 * s["zero_copy_sectors"] for s in sts)
        res[arm]["copy_stream"] = {
            "busy_ms_per_run": copy_ms / args.steps,
            "busy_frac": copy_ms / max(sum(ev[0].elapsed_time(ev[1]) for ev, _, _ in rec[arm]), 1e-9),
            "block_gb_per_s_while_busy": block_bytes / max(copy_ms / 1e3, 1e-9) / 1e9,
            "nominal_pcie_gen5_x16_gbs": PCIE_GEN5_X16_GBS}
        if arm == "learned":
            res[arm]["pred_error"] = sts[-1]["pred_error"]
            res[arm]["persist_error"] = sts[-1]["persist_error"]
            res[arm]["train_loss"] = sts[-1]["train_loss"]
    head = "learned" if "learned" in res else arms[0]
    r = res[head]
    if rank == 0:
        link = r["h2d_bytes_per_run"] / (r["ms_per_run"] / 1e3) / 1e9
        line = {"metric": "walk steps/sec on 1 B200, learned vs plain schedule (bit-exact); H2D bytes/step"
                          if args.policy == "pair" else "walk steps/sec",
                "value": r["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_run"], "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int32 gathers, fp32/fp64 accept compares",
                "data": "synthetic",
                "config": {"workload": wl["name"], "arms": arms, "headline_arm": head,
                           "residency": "both blocks (reference rule)" if args.strict_blocks else
                                        "current block until N(prev) is needed",
                           "prefetch": not args.no_prefetch, "compressed_blocks": not args.no_compress,
                           "zero_copy_tail": {"on": bool(args.zero_copy), "zero_threshold_walkers": zero_threshold},
                           "learned_mode": {0: "automatic: forecast eviction and zero-copy switch, then the "
                                               "switch alone, then the faster",
                                            1: "forecast eviction", 2: "zero-copy switch priced by measured costs",
                                            3: "forecast eviction and zero-copy switch"}[args.learned_mode],
                           "vertices": V, "edges": len(csr), "blocks": wl["nblocks"], "cache_bytes": wl["cache"],
                           "walkers": V * wl["wps"], "graph_in": "pinned host memory",
                           "l2": "every run copies the graph's blocks from the host into a 1.5 GB-class device "
                                 "cache far larger than L2; no flush",
                           "parallelism": "walker-id shards, one per rank" if world > 1 else "1 GPU",
                           "walk_seed": 42, "generator_seed": 1},
                "gpu_launches": sum(res[a]["launches"] for a in arms),
                "e2e": {"value": r["e2e"], "unit": "steps/s", "h2d_bytes_per_step": int(r["h2d_bytes_per_run"]),
                        "d2h_bytes_per_step": 8 * V * wl["wps"],
                        "note": "per step: one full run through the C ABI from pinned host blocks (cold device "
                                "cache), then every walker's 64-bit path hash read back to host memory"},
                "h2d_bytes_per_walk_step": r["h2d_bytes_per_walk_step"],
                "arms": res,
                "roofline": {"bound": "host-link", "achieved": link, "peak": peak_h2d, "unit": "GB/s",
                             "frac": link / peak_h2d, "traffic": None,
                             "peak_source": "measured: best pinned 1 GiB host-to-device copy in this run",
                             "nominal_pcie_gen5_x16": PCIE_GEN5_X16_GBS,
                             "kernel": "block copies (cudaMemcpyAsync of compressed blocks) overlapped with "
                                       "k_walk_ooc"},
                "walks_identical_across_arms": len({res[a]["path_hash_sum"] for a in arms}) == 1}
        if "plain" in res and "learned" in res:
            line["learned_over_plain"] = {
                "steps_per_s": res["learned"]["value"] / res["plain"]["value"],
                "h2d_bytes_per_step": res["learned"]["h2d_bytes_per_walk_step"] / res["plain"]["h2d_bytes_per_walk_step"],
                "target": "steps/s >= 1.3, H2D bytes/step <= 0.75"}
        if clk:
            line["clocks"] = clk
        if args.cpu_seconds > 0:
            from oracle import oracle as O
            threads = os.cpu_count() or 1
            s_steps, s_secs, _, _, s_desc = oracle_sample(O, beg, csr, wl, 42, args.cpu_seconds, threads=threads)
            line["cpu_baseline"] = {"value": s_steps / s_secs, "unit": "steps/s", "cores": threads, "kind": "port",
                                    "cpu_model": cpu_model(), "sample": s_desc}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def rmat_edges_torch(scale, n, seed, abc=(0.57, 0.19, 0.19)):
    """Seeded R-MAT sample list generated on the device with torch's RNG:
    `scale` quadrant choices per sample (a: (0,0), b: (0,1), c: (1,0),
    d: (1,1)).  Returns int32 device tensors (ids < 2^scale)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    a, b, c = abc
    src = torch.zeros(n, dtype=torch.int32, device="cuda")
    dst = torch.zeros(n, dtype=torch.int32, device="cuda")
    for _ in range(scale):
        u = torch.rand(n, device="cuda", generator=g)
        src.mul_(2).add_((u >= a + b).to(torch.int32))
        dst.mul_(2).add_((((u >= a) & (u < a + b)) | (u >= a + b + c)).to(torch.int32))
        del u
    return src, dst


def run_prep_bench(args, wl):
    """gw_edges_csr on the workload's sample list: value with the list resident
    in HBM; e2e from pinned host arrays to the CSR back in pinned host memory."""
    import ctypes
    import torch
    import gowalker_b200 as gw
    torch.cuda.set_device(0)
    L = gw.load()
    n = wl["ef"] << wl["scale"]
    V = 1 << wl["scale"]
    flags = gw.GW_EDGES_SYMMETRIC | gw.GW_EDGES_SORT | gw.GW_EDGES_DEDUP
    src, dst = rmat_edges_torch(wl["scale"], n, 1)
    h_src = torch.empty(n, dtype=torch.int32, pin_memory=True)
    h_dst = torch.empty(n, dtype=torch.int32, pin_memory=True)
    h_src.copy_(src)
    h_dst.copy_(dst)
    torch.cuda.synchronize()

    def convert(ps, pd):
        db, dc, ne, nv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64(), ctypes.c_uint32()
        st = L.gw_edges_csr(ctypes.c_void_p(ps), ctypes.c_void_p(pd), n, V, flags, ctypes.byref(db),
                            ctypes.byref(dc), ctypes.byref(ne), ctypes.byref(nv))
        if st != 0:
            raise gw.GwError(st, "gw_edges_csr failed")
        return db.value, dc.value, int(ne.value)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), out

    for _ in range(args.warmup):
        db, dc, ne = convert(src.data_ptr(), dst.data_ptr())
        L.gw_device_free(ctypes.c_void_p(db))
        L.gw_device_free(ctypes.c_void_p(dc))
    clocks = ClockSampler(0)
    clocks.start()
    dev_ms = []
    for _ in range(args.steps):
        ms, (db, dc, ne) = timed(lambda: convert(src.data_ptr(), dst.data_ptr()))
        dev_ms.append(ms)
        L.gw_device_free(ctypes.c_void_p(db))
        L.gw_device_free(ctypes.c_void_p(dc))
    h_beg = torch.empty(V + 1, dtype=torch.int64, pin_memory=True)
    h_csr = torch.empty(ne, dtype=torch.int32, pin_memory=True)

    def e2e_step():
        db, dc, ne2 = convert(h_src.data_ptr(), h_dst.data_ptr())
        L.gw_memcpy(ctypes.c_void_p(h_beg.data_ptr()), ctypes.c_void_p(db), (V + 1) * 8)
        L.gw_memcpy(ctypes.c_void_p(h_csr.data_ptr()), ctypes.c_void_p(dc), ne2 * 4)
        L.gw_device_free(ctypes.c_void_p(db))
        L.gw_device_free(ctypes.c_void_p(dc))
        return ne2

    e2e_ms = []
    for _ in range(args.steps):
        ms, ne2 = timed(e2e_step)
        assert ne2 == ne
        e2e_ms.append(ms)
    clk = clocks.stop()
    ms = sum(dev_ms) / len(dev_ms)
    ems = sum(e2e_ms) / len(e2e_ms)
    # Least traffic a conversion can have: read the pairs once (8 B per
    # sample), write the offsets and the kept neighbour ids once.
    min_bytes = 8 * n + 8 * (V + 1) + 4 * ne
    peaks, peak_kind = measured_peaks()
    hbm = peaks["hbm_gbs"]
    achieved = min_bytes / (ms / 1e3) / 1e9
    line = {"metric": "edge-list samples converted/sec", "value": n / (ms / 1e3), "unit": "samples/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 ids, u64 keys", "data": "synthetic",
            "config": {"workload": wl["name"], "vertices": V, "samples": n, "edges_out": ne,
                       "l2": "inputs larger than L2 (2 GB of pairs)"},
            "gpu_launches": 2,
            "library_launches": "CUB radix sort (8-bit digits over the 2 x bit_length(V-1) bits of the packed "
                                "(src, dst) key), unique, scan",
            "e2e": {"value": n / (ems / 1e3), "unit": "samples/s", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * (V + 1) + 4 * ne},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None, "peak_source": peak_kind,
                         "note": "achieved counts the least I/O of a conversion (pairs in, CSR out); the radix "
                                 "sort's digit passes read and write every key again"}}
    if clk:
        line["clocks"] = clk
    if args.cpu_seconds > 0:
        line["cpu_baseline"] = prep_cpu_baseline(h_src.numpy().view(np.uint32), h_dst.numpy().view(np.uint32), V,
                                                 args.cpu_seconds)
    print(json.dumps(line), flush=True)
    return 0


def prep_cpu_baseline(src, dst, V, target_s):
    """The oracle's converter (numpy, one thread) on a prefix of the sample
    list sized to take about target_s seconds."""
    from oracle import oracle as O
    k = 1 << 18
    t0 = time.time()
    O.convert_edges(src[:k], dst[:k], V, symmetric=True, dedup=True)
    dt = max(time.time() - t0, 1e-3)
    k = int(min(len(src), max(k, k * target_s / dt)))
    t0 = time.time()
    O.convert_edges(src[:k], dst[:k], V, symmetric=True, dedup=True)
    dt = time.time() - t0
    return {"value": k / dt, "unit": "samples/s", "cores": 1, "kind": "port",
            "sample": "first %d of the samples, symmetrised + deduplicated + sorted" % k}


def reduce_rank_times(dist, ms, ms2, steps, e2e_steps, device):
    """Whole-job figures from every rank's own: the slowest rank's times (max)
    and all ranks' steps (sum), so value = all steps / the max time.  Every
    rank must call it (two all-reduces, in the same order everywhere)."""
    if dist is None:
        return ms, ms2, float(steps), float(e2e_steps)
    import torch
    tmax = torch.tensor([ms, ms2], dtype=torch.float64, device=device)
    tsum = torch.tensor([float(steps), float(e2e_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tmax[1]), float(tsum[0]), float(tsum[1])


def necessary_bytes(stats, walkers, paths):
    """Bytes a walk step cannot avoid moving (oracle counts on a sample): the
    32-B sector(s) of (beg[cur], beg[cur+1]), the sector of the accepted
    candidate, the distinct sectors of the accepted trial's search of N(prev)
    when its verdict needed one, the path entry (when recorded), and each
    walker's hash and length.  Rejected trials need not read their
    candidates (a warp decides them from positions), so they add nothing."""
    b = 32 * (stats["off_sectors"] + stats["steps"] + stats["acc_sectors"]) + 12 * walkers
    if paths:
        b += 4 * (stats["steps"] + walkers)
    return b


def golden_checksum(config):
    """The oracle's whole-run checksum of an in-core workload
    (tests/golden/config_checksums.json), or None."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "config_checksums.json")) as f:
            return json.load(f).get(config)
    except (OSError, ValueError):
        return None


def run_ours(args, wl):
    """In-core workload: the graph resident in HBM (value) or copied from
    pinned host blocks every step with the walks read back (e2e).  Under
    torchrun every rank walks its own walker-id shard of the one population
    on its own copy of the graph (no data-path collective)."""
    import ctypes
    import torch
    import gowalker_b200 as gw

    dist, rank, world, local = init_dist()
    dev = torch.device("cuda", local)
    seed = 42
    paths = 1 if args.paths else 0
    L = gw.load()
    rate, rate_ms = ctypes.c_double(), ctypes.c_float()
    if L.gw_philox_rate(local, 4096, ctypes.byref(rate), ctypes.byref(rate_ms)) != 0:
        raise gw.GwError(-2, "gw_philox_rate failed")

    dg = build_graph(gw, wl)
    total = dg.nverts * wl["wps"]
    first, count = rank_shard(rank, world, total)
    cfgkw = dict(algorithm=wl["algo"], maxhops=wl["maxhops"], p=wl["p"], q=wl["q"], alpha=wl["alpha"],
                 term_prob=wl["term"], seed=seed, walkpersource=wl["wps"], record_paths=paths, device=local,
                 cache_size=1 << 40)
    eng = gw.WalkEngine(**cfgkw)
    eng.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=local)
    d_w = None
    if wl.get("weighted"):
        g = torch.Generator(device="cuda")
        g.manual_seed(1)
        d_w = torch.empty(dg.nedges, dtype=torch.float32, device="cuda").log_normal_(0.0, 1.0, generator=g)
        eng.set_device_weights(d_w.data_ptr())

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident runs
    for _ in range(args.warmup):
        eng.init_walkers(wl["algo"], wl["wps"], seed, first=first, count=count)
        eng.run()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    steps = 0
    kernel_ms = 0.0
    launches = 0
    trials = 0
    variant = -1
    coop = [0, 0, 0, 0]
    for _ in range(args.steps):
        eng.init_walkers(wl["algo"], wl["wps"], seed, first=first, count=count)
        st = eng.run()
        for i, k in enumerate(("coop_small_steps", "coop_small_attempts", "coop_large_steps", "coop_large_attempts")):
            coop[i] += st[k]
        steps += st["steps"]
        kernel_ms += st["kernel_ms"]
        trials += st["trials"]
        variant = st["kernel_variant"]
        chunk = st["walker_chunk"]
        launches += st["launches"]
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    hash_sum, steps_last = eng.checksum()

    # ---- the plain form for comparison: one launch per hop, same walks
    hop_arm = None
    if args.launch_per_hop:
        eng3 = gw.WalkEngine(**dict(cfgkw, launch_mode=gw.GW_LAUNCH_PER_HOP))
        eng3.set_device_graph(dg.nverts, dg.nedges, dg.beg_ptr, dg.csr_ptr)
        stream3 = torch.cuda.ExternalStream(eng3.stream_handle(), device=local)
        for _ in range(args.warmup):
            eng3.init_walkers(wl["algo"], wl["wps"], seed, first=first, count=count)
            eng3.run()
        barrier()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream3)
        hop_steps = hop_kernel_ms = 0
        for _ in range(args.steps):
            eng3.init_walkers(wl["algo"], wl["wps"], seed, first=first, count=count)
            st3 = eng3.run()
            hop_steps += st3["steps"]
            hop_kernel_ms += st3["kernel_ms"]
        h1.record(stream3)
        barrier()
        hop_ms = h0.elapsed_time(h1)
        hop_hash, _ = eng3.checksum()
        eng3.close()
        hop_ms, _, hop_all, _ = reduce_rank_times(dist, hop_ms, 0.0, hop_steps, 0, "cuda")
        hop_arm = {"value": hop_all / (hop_ms / 1000.0), "unit": "steps/s", "ms_per_run": hop_ms / args.steps,
                   "kernel_ms_per_run": hop_kernel_ms / args.steps, "launches_per_run": wl["maxhops"],
                   "same_walks": hop_hash == hash_sum}

    # ---- end to end through the C ABI: host blocks in, the walks out
    beg_t, csr_t, beg, csr = host_graph(dg)
    eng2 = gw.WalkEngine(**cfgkw)
    eng2.set_host_graph(beg_t, csr_t[: dg.nedges])
    h_w = None
    if d_w is not None:
        h_w = torch.empty(dg.nedges, dtype=torch.float32, pin_memory=True)
        h_w.copy_(d_w)
        eng2.set_host_weights(h_w)
    stride = wl["maxhops"] + 1
    out_rows = torch.empty((count, stride) if paths else (1,), dtype=torch.int32, pin_memory=True)
    out_lens = torch.empty(count, dtype=torch.int32, pin_memory=True)
    out_hash = torch.empty(count, dtype=torch.int64, pin_memory=True)
    stream2 = torch.cuda.ExternalStream(eng2.stream_handle(), device=local)

    def e2e_step():
        eng2.cache_reset()
        eng2.init_walkers(wl["algo"], wl["wps"], seed, first=first, count=count)
        st2 = eng2.run()
        if paths:
            eng2._check(L.gw_get_paths(eng2.h, 0, count, ctypes.c_void_p(out_rows.data_ptr()),
                                       ctypes.c_void_p(out_lens.data_ptr())))
        else:
            eng2._check(L.gw_path_lengths(eng2.h, 0, count, ctypes.c_void_p(out_lens.data_ptr())))
        eng2._check(L.gw_path_hashes(eng2.h, 0, count, ctypes.c_void_p(out_hash.data_ptr())))
        return st2

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream2)
    e2e_steps = h2d = 0
    for _ in range(args.steps):
        st2 = e2e_step()
        e2e_steps += st2["steps"]
        h2d += st2["h2d_bytes"]
    f1.record(stream2)
    barrier()
    ms2 = f0.elapsed_time(f1)
    d2h = count * (12 + (4 * stride if paths else 0))
    hs2 = int(out_hash.numpy().view(np.uint64).sum(dtype=np.uint64))
    if hs2 != hash_sum:
        log("warning: e2e checksum differs from the device-resident run")

    # max over ranks; the population's checksum from the shards'
    ms, ms2, steps_all, e2e_all = reduce_rank_times(dist, ms, ms2, steps, e2e_steps, "cuda")
    pop_hash = combine_hash_sums(dist, hash_sum, dev)
    pop_steps = int(reduce_rank_times(dist, 0.0, 0.0, steps_last, 0, "cuda")[2])

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        value = steps_all / (ms / 1000.0)
        line = {
            "metric": "walk steps/sec", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int32 gathers, fp32/fp64 accept compares", "data": "synthetic",
            "config": {"workload": wl["name"], "vertices": dg.nverts, "edges": dg.nedges, "walkers": total,
                       "csr_bytes": (dg.nverts + 1) * 8 + dg.nedges * 4,
                       "l2": "inputs larger than L2 (CSR %.2f GB vs 126 MB L2); no flush"
                             % (((dg.nverts + 1) * 8 + dg.nedges * 4) / 1e9),
                       "paths_recorded": bool(paths), "walk_seed": seed, "generator_seed": 1,
                       "parallelism": "walker-id shards, one per rank" if world > 1 else "1 GPU"},
            "gpu_launches": launches,
            "e2e": {"value": e2e_all / (ms2 / 1000.0), "unit": "steps/s",
                    "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h * world,
                    "note": "per step: the CSR copied from pinned host blocks and validated, every walker run, "
                            "then %s read back into pinned host memory"
                            % ("every path row, length and hash" if paths else "every path length and hash")},
            "checksum": {"path_hash_sum": pop_hash, "steps_per_run": pop_steps},
            "trials_per_step": trials / max(steps, 1),
            "kernel_variant": variant,
            "walker_chunk": chunk,
            "hard_steps": {"by_position": coop[0] // args.steps, "by_position_attempts": coop[1] // args.steps,
                           "by_search": coop[2] // args.steps, "by_search_attempts": coop[3] // args.steps},
        }
        if hop_arm is not None:
            hop_arm["persistent_over_per_hop"] = value / hop_arm["value"]
            line["one_launch_per_hop"] = hop_arm
        gold = golden_checksum(args.config)
        if gold is not None and "path_hash_sum" in gold:
            line["checksum"]["oracle_path_hash_sum"] = int(gold["path_hash_sum"])
            line["checksum"]["matches_oracle"] = (pop_hash == int(gold["path_hash_sum"]) and
                                                  pop_steps == gold["steps"])
        if clk:
            line["clocks"] = clk
        # roofline of the step kernel: the bytes a step cannot avoid (oracle
        # counts on a sample of the workload) over the kernel's time
        from oracle import oracle as O
        O.lib()
        threads = os.cpu_count() or 1
        alias = O.build_alias(beg, h_w.numpy()) if h_w is not None else None
        s_steps, s_secs, s_stats, s_walk, s_desc = oracle_sample(O, beg, csr, wl, seed, args.cpu_seconds,
                                                                 threads=threads, alias=alias)
        bpstep = necessary_bytes(s_stats, s_walk, paths) / max(s_steps, 1)
        if alias is not None:
            bpstep += 32.0  # the accepted candidate's alias-table entry
        kernel_s = kernel_ms / 1000.0 / args.steps
        steps_per_launch = steps / args.steps
        achieved = bpstep * steps_per_launch / kernel_s / 1e9
        dram_ps = profile_bytes_per_step(args.config)
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                            "frac": achieved / peaks["hbm_gbs"],
                            "traffic": (dram_ps * steps_per_launch) if dram_ps else None,
                            "peak_source": peak_kind,
                            "algorithmic_bytes_per_step": bpstep,
                            "bytes_model": "offsets sector + accepted candidate sector + the accepted trial's "
                                           "N(prev) search sectors + path entry + hash and length per walker",
                            "sector_model_bytes_per_step": algorithmic_bytes(s_stats, s_walk, paths,
                                                                             weighted=alias is not None)
                                                           / max(s_steps, 1),
                            "kernel_ms_per_launch": kernel_ms / args.steps,
                            "kernel": "k_walk_incore (weighted)" if h_w is not None else "k_walk_incore"}
        if dram_ps:
            line["roofline"]["dram_bytes_per_step"] = dram_ps
            line["roofline"]["dram_frac"] = dram_ps * steps_per_launch / kernel_s / 1e9 / peaks["hbm_gbs"]
        trial_rate = trials / args.steps / kernel_s
        line["issue_roofline"] = {"achieved": trial_rate, "peak": rate.value, "unit": "trials/s",
                                  "frac": trial_rate / rate.value,
                                  "peak_source": "measured in this run: gw_philox_rate, the step kernels' keyed "
                                                 "Philox4x32-10 alone, best of 3 launches (%.1f ms)" % rate_ms.value,
                                  "note": "every rejection trial evaluates at least one Philox draw"}
        line["cpu_baseline"] = {"value": s_steps / s_secs, "unit": "steps/s", "cores": threads, "kind": "port",
                                "cpu_model": cpu_model(), "sample": s_desc}
        print(json.dumps(line), flush=True)
    eng.close()
    eng2.close()
    dg.free()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--scale", type=int, default=None, help="override the graph scale (smaller smoke runs)")
    ap.add_argument("--paths", type=int, default=1, help="record full paths (1) or hashes only (0)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--policy", default="pair", choices=["pair", "plain", "learned", "sa"],
                    help="block policy (out-of-core): both GOWalker's rule and the learned predictor (pair), or "
                         "one of GOWalker's rule, the learned predictor, SOWalker's annealing")
    ap.add_argument("--no-compress", action="store_true",
                    help="out-of-core: copy plain neighbour lists (default: compressed, decoded on the device)")
    ap.add_argument("--no-zero-copy", dest="zero_copy", action="store_false",
                    help="out-of-core: keep loading blocks to the end (default: GOWalker's zero mode -- once no "
                         "block scores above blocksize/3072 walkers, every walker finishes reading mapped host "
                         "memory)")
    ap.add_argument("--learned-mode", type=int, default=0,
                    help="out-of-core learned policy parts: 1 forecast eviction, 2 zero-copy switch priced by "
                         "measured costs, 3 both (default 0: automatic -- both, then the switch alone, then the "
                         "faster)")
    ap.add_argument("--zero-scale", type=float, default=1.0,
                    help="out-of-core: multiply GOWalker's zero-mode threshold by this factor (default 1)")
    ap.add_argument("--launch-per-hop", action="store_true",
                    help="in-core: also time the plain one-launch-per-hop form (same walks) beside the persistent "
                         "kernel")
    ap.add_argument("--no-prefetch", action="store_true",
                    help="out-of-core: take each block choice in its own iteration (default: one iteration "
                         "ahead, the copy overlapped with the step)")
    ap.add_argument("--strict-blocks", action="store_true",
                    help="out-of-core: run a walker only when both its blocks are resident (the reference's rule)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.config])
    if args.scale:
        wl["scale"] = args.scale
        wl["name"] = wl["name"].replace("scale %d" % WORKLOADS[args.config]["scale"], "scale %d" % args.scale)
    if args.warmup < 3:
        log("note: fewer than 3 warm-up steps")
    if args.impl == "reference":
        if wl.get("prep"):
            return run_prep_reference(args, wl)
        return run_reference_arm(args, wl)
    if wl.get("prep"):
        return run_prep_bench(args, wl)
    if wl.get("ooc"):
        return run_ooc_bench(args, wl)
    return run_ours(args, wl)


if __name__ == "__main__":
    sys.exit(main())

"""Bucket-count matrices for the block-choice tests: the (prev block, cur
block) walker counts, the scheduler's cached list, the slot count and the
zero threshold that GOwalker_scheduler_t::max_choose_blocks
(engine/schedule.hpp:70-138) decides from.  Seeded; shared by the test of the
oracle against the reference's own scheduler and the test of the device
kernel against the oracle."""
import numpy as np


def scores(counts, cached, nslots):
    """max_choose_blocks' score of every uncached block, in block order."""
    c = np.asarray(counts).astype(np.int64)
    nb = c.shape[0]
    cl = np.array(cached, dtype=np.int64)
    cs = set(int(x) for x in cached)
    full = len(cached) >= nslots
    out = []
    for i in range(nb):
        if i in cs:
            continue
        links = c[i, cl] + c[cl, i] if len(cl) else np.zeros(0, dtype=np.int64)
        if full:
            out.append(int(links.sum() - (links.min() if len(links) else 0xFFFFFFFF)))
        else:
            out.append(int(links.sum() + c[i, i]))
    return out


def _unique_top(counts, cached, nslots):
    """True when the best score of the uncached blocks is taken by one block
    only (the reference's std::sort leaves the order of equal scores open
    beyond 16 uncached blocks)."""
    sc = sorted(scores(counts, cached, nslots), reverse=True)
    return len(sc) < 2 or sc[0] != sc[1]


def cases(nb, seed, n_random=40, ties_anywhere=False):
    """Returns a list of (counts u32 nb x nb, cached list, nslots, zero_threshold)."""
    rng = np.random.default_rng(seed)
    out = []

    def add(counts, cached, nslots, zt=0):
        counts = np.asarray(counts, dtype=np.uint32).reshape(nb, nb)
        cached = [int(x) for x in cached]
        uncached = nb - len(cached)
        if uncached == 0:
            return  # the reference reads block_score[0] of an empty list there
        if not ties_anywhere and uncached > 16 and not _unique_top(counts, cached, nslots):
            return
        out.append((counts, cached, nslots, zt))

    for k in range(n_random):
        nslots = int(rng.integers(2, max(3, nb - 1)))
        full = k % 2 == 0
        ncached = nslots if full else int(rng.integers(0, nslots))
        ncached = min(ncached, nb - 1)
        cached = rng.permutation(nb)[:ncached]
        kind = k % 5
        if kind == 0:  # dense, wide range
            counts = rng.integers(0, 1 << 20, (nb, nb))
        elif kind == 1:  # sparse: most buckets empty
            counts = rng.integers(0, 1000, (nb, nb)) * (rng.random((nb, nb)) < 0.05)
        elif kind == 2:  # heavy diagonal (walkers staying inside a block)
            counts = rng.integers(0, 50, (nb, nb)) + np.diag(rng.integers(0, 1 << 16, nb))
        elif kind == 3:  # power-law bucket sizes
            counts = (rng.pareto(1.2, (nb, nb)) * 100).astype(np.int64)
        else:  # walkers only between cached blocks and one or two others
            counts = np.zeros((nb, nb), dtype=np.int64)
            for c in cached:
                for o in rng.integers(0, nb, 2):
                    counts[c, o] += int(rng.integers(1, 5000))
                    counts[o, c] += int(rng.integers(0, 5000))
        zt = 0 if k % 3 else int(np.percentile(counts, 90)) * 2
        add(np.minimum(counts, 1 << 24), cached, nslots, zt)
    # all zero: nothing qualifies
    add(np.zeros((nb, nb)), list(range(min(2, nb - 1))), 4)
    # walkers only inside cached blocks: every uncached block scores 0
    z = np.zeros((nb, nb), dtype=np.int64)
    cl = list(range(min(3, nb - 1)))
    for c in cl:
        z[c, c] = 100
    add(z, cl, 3)
    # the threshold exactly at the best score (strict '>') and one below it
    c = rng.integers(0, 100, (nb, nb))
    cl = list(range(0, nb, 3))[: max(1, min(nb // 3, nb - 1))]
    for ns in (len(cl), len(cl) + 1):
        best = max(scores(c, cl, ns))
        add(c, cl, ns, best)
        add(c, cl, ns, max(best - 1, 0))
    # equal scores: uncached blocks with identical links (lowest id wins when
    # at most 16 are uncached; beyond that only the device test checks them)
    t = np.ones((nb, nb), dtype=np.int64) * 7
    keep = max(1, nb - 12)
    add(t, list(range(min(keep, nb - 1))), max(2, min(keep, nb - 1)))
    add(t, list(range(min(keep, nb - 1))), nb)
    # full cache, the smallest link shared by several cached blocks (first position wins)
    s = rng.integers(10, 20, (nb, nb))
    cl = [int(x) for x in rng.permutation(nb)[: max(2, min(nb // 2, nb - 1))]]
    for c2 in cl[::2]:
        s[:, c2] = 1
        s[c2, :] = 1
    add(s, cl, len(cl))
    return out


def ref_to_decision(before, chose, after):
    """(action, block, position) from the reference scheduler's list before
    and after max_choose_blocks."""
    before = [int(x) for x in before]
    after = [int(x) for x in after]
    if not chose:
        assert after == before
        return (0, -1, -1)
    if len(after) == len(before) + 1:
        assert after[:-1] == before
        return (1, after[-1], len(before))
    assert len(after) == len(before)
    diff = [j for j in range(len(before)) if before[j] != after[j]]
    assert len(diff) == 1
    return (2, after[diff[0]], diff[0])

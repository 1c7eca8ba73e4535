"""GOWalker's block choice on the device (k_schedule through
gw_plain_choose_block) against the oracle's restatement of
GOwalker_scheduler_t::max_choose_blocks (engine/schedule.hpp:70-138), which a
CPU test pins to the reference's own scheduler.  Index-exact on (action,
block, position); covers the block counts of every out-of-core workload (64,
128 and 256 blocks: C3, C4, C5) and the 1024-block maximum."""
import numpy as np
import pytest

import schedule_cases as SC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nb", [1, 2, 6, 20, 64, 128, 256])
def test_plain_choice_matches_oracle(gw, oracle, nb):
    if nb == 1:
        # one block, nothing cached: it is the only candidate
        c = np.array([[5]], dtype=np.uint32)
        assert gw.plain_choose_block(c, [], 2) == oracle.max_choose_blocks(c, [], 2) == (1, 0, 0)
        return
    cases = SC.cases(nb, seed=1000 + nb, n_random=60, ties_anywhere=True)
    acts = set()
    for counts, cached, nslots, zt in cases:
        got = gw.plain_choose_block(counts, cached, nslots, zt)
        want = oracle.max_choose_blocks(counts, cached, nslots, zt)
        assert got == want, (nb, cached, nslots, zt)
        acts.add(got[0])
    # (with 2 blocks at most one is cached, below every slot count: no replace)
    assert {1, 2} <= acts if nb > 2 else 1 in acts


def test_plain_choice_largest_table(gw, oracle):
    """1024 blocks (the block table's limit), a full cache of 88 slots (C5's
    8 GB cache holds about that many), skewed counts."""
    rng = np.random.default_rng(5)
    nb = 1024
    for k in range(3):
        counts = (rng.pareto(1.1, (nb, nb)) * 50).astype(np.uint32)
        cached = rng.permutation(nb)[:88]
        nslots = 88 if k else 200
        got = gw.plain_choose_block(counts, cached, nslots)
        assert got == oracle.max_choose_blocks(counts, cached, nslots), k


def test_plain_choice_rejects_bad_lists(gw):
    c = np.ones((8, 8), dtype=np.uint32)
    for cached in ([8], [1, 1]):
        with pytest.raises(gw.GwError):
            gw.plain_choose_block(c, cached, 4)

"""Host-side planning of the batched SIMPLE (no GPU): the tile lists of the
persistent stage kernels and the Krylov team tables, called through the C
ABI (cfdb_batch_plan_tiles, cfdb_batch_plan_teams)."""
import itertools

import numpy as np
import pytest

from cfdapp_b200 import cfdb


@pytest.mark.parametrize("tile", [32, 100, 1024])
def test_tiles_cover_every_item_once(tile):
    rng = np.random.default_rng(3)
    counts = rng.integers(0, 5000, size=17)
    counts[4] = 0
    first, tc, ts = cfdb.plan_tiles(counts, tile)
    assert first[0] == 0 and np.all(np.diff(first) == -(-counts // tile))
    for k, c in enumerate(counts):
        seg = slice(first[k], first[k + 1])
        assert np.all(tc[seg] == k)
        assert np.array_equal(ts[seg], np.arange(0, c, tile))
    assert tc.size == first[-1]


def test_tiles_reject_bad_arguments():
    with pytest.raises(cfdb.CfdbError):
        cfdb.plan_tiles([10, -1], 32)
    with pytest.raises(cfdb.CfdbError):
        cfdb.plan_tiles([10], 0)


def _greedy(weight, cells, active, nblocks, minc):
    """Pure-Python statement of the team rule, for the test."""
    n = len(weight)
    blocks = [1 if (active[k] and cells[k] > 0) else 0 for k in range(n)]
    cap = [max(1, cells[k] // minc) for k in range(n)]
    left = nblocks - sum(blocks)
    while left > 0:
        best, bw = -1, -1.0
        for k in range(n):
            if blocks[k] == 0 or blocks[k] >= cap[k]:
                continue
            if weight[k] / blocks[k] > bw:
                best, bw = k, weight[k] / blocks[k]
        if best < 0:
            break
        blocks[best] += 1
        left -= 1
    return blocks


def test_teams_follow_the_highest_weight_per_block_rule():
    rng = np.random.default_rng(5)
    sides = rng.choice([64, 96, 128, 192, 256, 384, 512], size=64)
    cells = (sides * sides).astype(np.int64)
    active = np.ones(64, dtype=np.int32)
    active[[3, 9]] = 0
    weight = cells.astype(np.float64) ** 1.5
    tf, bc = cfdb.plan_teams(weight, cells, active, 296, 2048)
    blocks = np.diff(tf)
    assert list(blocks) == _greedy(weight, cells, active, 296, 2048)
    assert blocks[3] == 0 and blocks[9] == 0
    assert np.all(blocks[active == 1] >= 1)
    assert np.all(blocks <= np.maximum(1, cells // 2048))
    assert tf[-1] <= 296
    for k in range(64):
        assert np.all(bc[tf[k]:tf[k + 1]] == k)
    assert np.all(bc[tf[-1]:] == -1)


def test_teams_minimise_the_largest_weight_per_block():
    """On a small case the greedy rule's worst weight per block equals the
    optimum found by exhaustive search."""
    weight = np.array([9.0, 4.0, 1.0, 6.0])
    cells = np.array([10 ** 6] * 4, dtype=np.int64)
    active = np.ones(4, dtype=np.int32)
    nb = 9
    tf, _ = cfdb.plan_teams(weight, cells, active, nb, 1)
    got = max(weight / np.diff(tf))
    best = min(max(weight / np.array(b)) for b in itertools.product(range(1, nb), repeat=4)
               if sum(b) <= nb)
    assert got == pytest.approx(best)


def test_teams_refuse_more_active_cases_than_blocks():
    with pytest.raises(cfdb.CfdbError):
        cfdb.plan_teams(np.ones(5), np.full(5, 4096), np.ones(5), 4)
    tf, bc = cfdb.plan_teams(np.ones(5), np.full(5, 4096), [1, 0, 1, 0, 1], 3)
    assert list(np.diff(tf)) == [1, 0, 1, 0, 1] and list(bc) == [0, 2, 4]

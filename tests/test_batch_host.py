"""Host side of the batched build (no GPU): the synthetic workload of seeded
random tables."""
import numpy as np

import helpers as H


def _batch():
    return __import__("importlib").import_module("2048endgametablebase_b200.batch")


def _connected(cells):
    cells = set(cells)
    seen, todo = {(3, 3)}, [(3, 3)]
    while todo:
        r, c = todo.pop()
        for dr, dc in ((0, 1), (0, -1), (1, 0), (-1, 0)):
            q = (r + dr, c + dc)
            if q in cells and q not in seen:
                seen.add(q)
                todo.append(q)
    return seen == cells


def test_random_tables_shape_and_determinism():
    B = _batch()
    a = B.random_tables(64)
    b = B.random_tables(64)
    assert [t.name for t in a] == [t.name for t in b]
    assert all(np.array_equal(x.seeds, y.seeds) for x, y in zip(a, b))
    pats = __import__("importlib").import_module("2048endgametablebase_b200.patterns")
    sizes, targets = set(), set()
    for t in a:
        k = len(t.cells)
        sizes.add(k)
        targets.add(t.target)
        assert 6 <= k <= 10 and (3, 3) in t.cells and len(set(t.cells)) == k
        assert _connected(t.cells)
        mask = t.masks[0]
        free = {(3 - r) * 4 + (3 - c) for r, c in t.cells}
        for nib in range(16):
            assert ((mask >> (4 * nib)) & 0xF) == (0 if nib in free else 0xF)
        assert len(t.seeds) == k * (k - 1)
        sums = {pats.tile_sum(int(s)) for s in t.seeds}
        assert len(sums) == 1
        s0 = sums.pop()
        assert (t.steps, t.docheck) == pats.steps_and_docheck(s0, t.target, 48)
        for s in t.seeds:
            assert (int(s) & mask) == mask
    assert targets <= {6, 7, 8, 9} and len(targets) == 4
    assert len(sizes) >= 4


def test_make_table_seeds_are_two_tiles():
    B = _batch()
    t = B.make_table("x", [(3, 3), (3, 2), (2, 3)], 5)
    assert len(t.seeds) == 6
    for s in t.seeds:
        free = [(int(s) >> (4 * k)) & 0xF for k in (0, 1, 4)]
        assert sorted(free) == [0, 1, 2]

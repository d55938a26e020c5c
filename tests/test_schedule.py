"""Persistent launch schedule (host side, no GPU): units of a launch cut at
MC-step boundaries over the resident CTAs by McNaughton's wrap-around rule.

The kernel relies on three properties checked here: every unit's steps are
covered once and in order, a piece only waits for steps that run on a CTA
numbered lower (so every wait ends), and no CTA gets more than the balanced
share plus one step of one unit."""
import numpy as np
import pytest

from gpudock_b200 import lib


def _check(cost, steps, m):
    pieces, off = lib.schedule_pieces(cost, steps, m)
    used = len(off) - 1
    assert used <= m
    total = float(np.dot(cost, steps))
    if total == 0:
        assert used == 0 and len(pieces) == 0
        return pieces, off
    C = max(max(c * s for c, s in zip(cost, steps)), total / m)
    machine_of = np.repeat(np.arange(used), np.diff(off))
    # coverage, in order, each step once
    for u, n in enumerate(steps):
        mine = pieces[pieces[:, 0] == u]
        if n == 0:
            assert len(mine) == 0
            continue
        order = np.argsort(mine[:, 1])
        lo, hi = mine[order, 1], mine[order, 2]
        assert lo[0] == 0 and hi[-1] == n
        assert np.all(hi[:-1] == lo[1:]) and np.all(hi > lo)
    # waits: exactly the pieces that do not start at step 0, and each waits
    # for a piece on a lower-numbered CTA
    assert np.array_equal(pieces[:, 3] != 0, pieces[:, 1] > 0)
    for k in np.nonzero(pieces[:, 3])[0]:
        u, lo = pieces[k, 0], pieces[k, 1]
        pred = np.nonzero((pieces[:, 0] == u) & (pieces[:, 2] == lo))[0]
        assert len(pred) == 1 and machine_of[pred[0]] < machine_of[k]
    # balance: each end of a CTA's share is cut within half a step of its
    # ideal place, so no CTA is more than one step above the balanced length
    loads = np.zeros(used)
    for (u, lo, hi, _), mch in zip(pieces, machine_of):
        loads[mch] += cost[u] * (hi - lo)
    assert loads.max() <= C + max(cost) + 1e-9 * C
    assert loads.sum() == pytest.approx(total)
    return pieces, off


def test_equal_units_more_than_machines():
    # 275 units of 20 steps on 148 CTAs: 37 or 38 unit-steps each instead of
    # two waves (40)
    pieces, off = _check([1.0] * 275, [20] * 275, 148)
    assert len(off) - 1 == 148
    per = [sum(p[2] - p[1] for p in pieces[off[m]:off[m + 1]]) for m in range(148)]
    assert min(per) >= 37 and max(per) <= 38
    # a CTA runs at most one late piece, last
    for m in range(148):
        w = pieces[off[m]:off[m + 1], 3]
        assert w[:-1].sum() == 0


@pytest.mark.parametrize("seed", range(6))
def test_random_costs(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 400))
    cost = rng.uniform(0.2, 5.0, n)
    steps = rng.integers(0, 60, n)
    steps[rng.random(n) < 0.05] = 0
    m = int(rng.integers(1, 200))
    _check(cost, steps, m)


def test_edges():
    _check([], [], 4)
    _check([1.0], [0], 4)
    _check([1.0], [1], 8)       # one unit, one step
    _check([3.0, 1.0], [5, 5], 1)
    pieces, off = _check([1.0] * 4, [10] * 4, 16)  # fewer units than CTAs
    assert (pieces[:, 3] == 0).all()
    with pytest.raises(lib.GdError):
        lib.schedule_pieces([1.0], [3], 0)
    with pytest.raises(lib.GdError):
        lib.schedule_pieces([0.0], [3], 2)


def _check_queue(cost, steps, m, tail):
    """Schedules with a shared queue: the machines' pieces cover each unit's
    first steps[u] - tail steps (as the plain schedule does), the queue holds
    each remaining step once as a one-step piece, a unit's queue steps come in
    order and after its own machine part, and every piece but a unit's first
    waits."""
    pieces, off, nq = lib.schedule_queue(cost, steps, m, tail)
    assert len(off) == m + 1 and off[m] + nq == len(pieces)
    head = [max(0, s - tail) for s in steps]
    static, queue = pieces[:off[m]], pieces[off[m]:]
    ref, ref_off = lib.schedule_pieces(cost, head, m)
    assert np.array_equal(static, ref)
    assert np.array_equal(off[:len(ref_off)], ref_off) and (off[len(ref_off) - 1:] == ref_off[-1]).all()
    assert (queue[:, 2] - queue[:, 1] == 1).all()
    assert np.array_equal(queue[:, 3] != 0, queue[:, 1] > 0)
    assert np.array_equal(static[:, 3] != 0, static[:, 1] > 0)
    for u, n in enumerate(steps):
        q = queue[queue[:, 0] == u, 1]
        assert list(q) == list(range(head[u], n))
    # the queue takes every unit's first queued step before any unit's second
    rank = np.array([s - head[u] for u, s in queue[:, :2]])
    assert (np.diff(rank) >= 0).all()
    return pieces, off, nq


def test_queue_ensemble():
    # 275 units of 20 steps on 148 CTAs, the last 2 steps of each in the queue
    pieces, off, nq = _check_queue([1.0] * 275, [20] * 275, 148, 2)
    assert nq == 550
    per = np.diff(off)
    assert per.min() >= 1


@pytest.mark.parametrize("seed", range(4))
def test_queue_random(seed):
    rng = np.random.default_rng(200 + seed)
    n = int(rng.integers(1, 300))
    cost = rng.uniform(0.2, 5.0, n)
    steps = rng.integers(0, 30, n)
    _check_queue(cost, steps, int(rng.integers(1, 200)), int(rng.integers(0, 5)))


def test_queue_edges():
    _check_queue([1.0], [1], 8, 2)       # the whole unit in the queue
    _check_queue([1.0] * 3, [2] * 3, 2, 2)
    pieces, off, nq = _check_queue([1.0] * 5, [10] * 5, 3, 0)
    assert nq == 0
    with pytest.raises(lib.GdError):
        lib.schedule_queue([1.0], [3], 2, -1)

"""Binomial checkpointing schedule of the capped adjoint tape (host only).

dglm_adjoint_schedule returns the schedule the library runs: the
checkpoints the recording places (spine) and the backward pass's actions.
A simulation of the slots checks that every advance starts from the state
it claims, that every chunk is reversed exactly once and in reverse order,
and that the number of chunk advances equals the optimum of the binomial
recursion restated here (Griewank and Walther, revolve, 2000):
    cost(1, f) = 0, cost(n, 0) = n (n - 1) / 2,
    cost(n, f) = min(cost(n, f - 1), min_m  m + cost(n - m, f - 1) + cost(m, f)).
"""
import functools

import numpy as np
import pytest

from exadglm_b200 import capi


@functools.lru_cache(maxsize=None)
def cost(n, f):
    if n == 1:
        return 0
    if f == 0:
        return n * (n - 1) // 2
    best = cost(n, f - 1)
    for m in range(1, n):
        best = min(best, m + cost(n - m, f - 1) + cost(m, f))
    return best


def simulate(nsteps, leaf, slots, prestored):
    spine, acts, adv = capi.adjoint_schedule(nsteps, leaf, slots, prestored)
    n = -(-nsteps // leaf)
    held = {0: 0}
    if prestored:
        for q, c in enumerate(spine):
            held[q] = int(c)
    assert spine[0] == 0 and len(spine) <= slots
    assert list(spine) == sorted(set(int(c) for c in spine)), "spine chunks ascend"
    reversed_order, chunk_adv, step_adv = [], 0, 0
    for kind, src, chunk, count, dst in acts:
        assert held.get(int(src)) == chunk, (kind, src, chunk, held)
        if kind == 0:
            assert count >= 1 and chunk + count < n
            assert dst == -1 or 0 < dst < slots
            held[int(dst)] = int(chunk + count)
            chunk_adv += count
            step_adv += min((chunk + count) * leaf, nsteps) - chunk * leaf
        else:
            assert kind == 1 and count == 1
            reversed_order.append(int(chunk))
    assert reversed_order == list(range(n - 1, -1, -1))
    assert step_adv == adv
    return n, chunk_adv, spine


@pytest.mark.parametrize("nsteps,leaf,slots", [
    (1, 1, 1), (7, 1, 1), (7, 1, 2), (10, 1, 3), (37, 1, 4), (37, 3, 4), (50, 5, 2),
    (64, 1, 8), (100, 7, 5), (120, 1, 120), (500, 10, 10), (500, 4, 40), (333, 11, 3),
])
def test_schedule_is_valid_and_optimal(nsteps, leaf, slots):
    n, adv, spine = simulate(nsteps, leaf, slots, prestored=False)
    f = min(slots - 1, n - 1)
    assert adv == cost(n, f)
    # with the recording's checkpoints in place, the advances along the
    # spine are saved: exactly the spine's last chunk
    n2, adv2, spine2 = simulate(nsteps, leaf, slots, prestored=True)
    assert adv2 == adv - int(spine2[-1])


def test_known_costs():
    assert cost(5, 0) == 10
    assert all(cost(n, n - 1) == n - 1 for n in range(1, 30))
    # more slots never cost more
    for n in range(1, 40):
        assert all(cost(n, f) >= cost(n, f + 1) for f in range(0, 10))
    # the library agrees on the table at sizes the recursion reaches quickly
    for n, f in [(12, 1), (12, 2), (30, 3), (45, 5)]:
        _, acts, _ = capi.adjoint_schedule(n, 1, f + 1, prestored=False)
        assert int(sum(r[3] for r in acts if r[0] == 0)) == cost(n, f)


def test_schedule_rejects_bad_arguments():
    with pytest.raises(capi.DglmError, match="positive"):
        capi.adjoint_schedule(0, 1, 1)
    with pytest.raises(capi.DglmError, match="positive"):
        capi.adjoint_schedule(10, 1, 0)

"""Binomial checkpointing schedule (SWESimulators.Adjoint.Revolve), checked
by replaying it on integer 'states' without a GPU."""

import pytest

torch = pytest.importorskip("torch")

from SWESimulators.Adjoint import Revolve  # noqa: E402


def replay(rv):
    slots, cur, reversed_, advances, peak = {}, None, [], 0, 0
    for act in rv.actions:
        kind = act[0]
        if kind == "takeshot":
            _, slot, step = act
            assert cur == step or (cur is None and step == 0)
            slots[slot] = step
            cur = step
            peak = max(peak, len(slots))
        elif kind == "restore":
            _, slot, step = act
            assert slots[slot] == step
            cur = step
        elif kind == "advance":
            _, a, b = act
            assert cur == a and b > a
            advances += b - a
            cur = b
        else:
            _, n = act
            assert cur == n
            reversed_.append(n)
            cur = n + 1
    return reversed_, advances, peak


@pytest.mark.parametrize("n, s", [(1, 1), (5, 1), (10, 2), (30, 3), (64, 5), (100, 10), (57, 57), (200, 400)])
def test_schedule_reverses_every_step_once_in_order(n, s):
    rv = Revolve(n, s)
    reversed_, advances, peak = replay(rv)
    assert reversed_ == list(range(n - 1, -1, -1))
    assert peak <= min(s, n)
    assert advances == int(rv.F[rv.s - 1, n])
    assert rv.forward_steps() == advances + n


def test_cost_matches_brute_force_minimum():
    # the recursion against an exhaustive search over first split points
    import functools

    @functools.lru_cache(maxsize=None)
    def best(c, t):
        if t <= 1:
            return 0
        if c == 0:
            return t * (t - 1) // 2
        return min(m + best(c - 1, t - m) + best(c, m) for m in range(1, t))

    for c in range(0, 5):
        for t in range(1, 40):
            assert Revolve(t, c + 1).F[min(c, t - 1) if t > 1 else 0, t] == best(min(c, max(t - 1, 0)), t)


def test_more_slots_never_cost_more():
    costs = [Revolve(120, s).forward_steps() for s in (1, 2, 4, 8, 16, 120)]
    assert costs == sorted(costs, reverse=True)
    assert costs[-1] == 2 * 120 - 1          # every state stored: one forward pass + one step per reversal

"""The binomial checkpoint schedule of eup_adjoint_run, built on the host by
eup_adjoint_plan (no GPU): its forward-step count against an independent dynamic
program over every split (small cases) and against the closed form
t(n, c) = r n - C(c + r, r - 1) of Griewank & Walther (large cases)."""
from functools import lru_cache
from math import comb

import pytest


@lru_cache(maxsize=None)
def best(n, free):
    """Fewest forward steps to reverse n steps from a stored state with `free` more slots."""
    if n == 1:
        return 0
    if free == 0:
        return n * (n - 1) // 2
    return min(m + best(m, free) + best(n - m, free - 1) for m in range(1, n))


def closed_form(n, c):
    if n <= 1:
        return 0
    if c <= 1:
        return n * (n - 1) // 2
    r = 0
    while comb(c + r, c) < n:
        r += 1
    return r * n - comb(c + r, r - 1)


@pytest.mark.parametrize("n,c", [(1, 1), (2, 1), (7, 1), (15, 2), (40, 3), (60, 4), (100, 3), (150, 8), (64, 64)])
def test_schedule_is_optimal_small(eup, n, c):
    p = eup.adjoint_plan(n, c)
    assert p["forward_steps"] == best(n, c - 1)
    assert p["recomputed_steps"] == p["forward_steps"] - (n - 1)


@pytest.mark.parametrize("n,c,r", [(4000, 64, 3), (10000, 8, 8), (2000, 8, 6), (2500, 16, 4), (4000, 128, 2)])
def test_schedule_attains_the_closed_form(eup, n, c, r):
    p = eup.adjoint_plan(n, c)
    assert p["forward_steps"] == closed_form(n, c)
    assert p["repetitions"] == r


def test_plan_defaults_and_errors(eup):
    assert eup.adjoint_plan(4000, 0) == eup.adjoint_plan(4000, 64)
    # more slots than steps: every state stored, nothing recomputed
    assert eup.adjoint_plan(10, 50)["recomputed_steps"] == 0
    with pytest.raises(eup.EupError):
        eup.adjoint_plan(0, 4)

"""The binomial checkpointing schedule of the adjoint runs
(lbm_adjoint_schedule, a dry run of the schedule lbm_adjoint_backward
follows with binomial_checkpoints > 0): Griewank's revolve bounds, no
device needed."""
import math

import pytest

import lbm_b200 as L


def least_repetitions(n, c):
    r = 1
    while math.comb(c + r, c) < n:
        r += 1
    return r


def test_no_checkpoints_recomputes_every_prefix():
    for n in (1, 2, 7, 30):
        s = L.adjoint_schedule(n, 0)
        assert s["recompute_steps"] == n * (n + 1) // 2 and s["peak_checkpoints"] == 0


def test_enough_checkpoints_store_every_step_once():
    for n in (2, 7, 30):
        s = L.adjoint_schedule(n, n - 1)
        assert s["recompute_steps"] == 2 * n - 1 and s["peak_checkpoints"] == n - 1


@pytest.mark.parametrize("n,c", [(100, 3), (1000, 10), (2000, 20), (5000, 25), (5000, 8)])
def test_revolve_bounds(n, c):
    s = L.adjoint_schedule(n, c)
    r = least_repetitions(n, c)
    assert s["peak_checkpoints"] <= c
    # every step is run at most r times by the advances plus once as a leaf
    assert s["recompute_steps"] <= (r + 1) * n
    # fewer slots never make it cheaper
    assert s["recompute_steps"] <= L.adjoint_schedule(n, max(c - 1, 0))["recompute_steps"]


def test_schedule_rejects_bad_arguments():
    with pytest.raises(L.LBMError):
        L.adjoint_schedule(0, 3)


def fewest_recomputations(n, c):
    """Exhaustive search over every split of the recursive schedule (the
    fewest forward steps it can recompute)."""
    import functools

    @functools.lru_cache(maxsize=None)
    def best(l, k):
        if l == 1:
            return 1
        if k == 0:
            return l * (l + 1) // 2
        return min(l1 + best(l - l1, k - 1) + best(l1, k) for l1 in range(1, l))
    return best(n, c)


@pytest.mark.parametrize("n,c", [(20, 1), (60, 2), (100, 3), (120, 5), (150, 10)])
def test_schedule_is_near_the_fewest_recomputations(n, c):
    got = L.adjoint_schedule(n, c)["recompute_steps"]
    want = fewest_recomputations(n, c)
    assert want <= got <= 1.05 * want, (got, want)

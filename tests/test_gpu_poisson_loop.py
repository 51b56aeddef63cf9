"""The device-side Poisson loop: a CUDA graph whose conditional WHILE node
runs segment after segment (check_interval sweeps, the convergence test and a
one-thread decide kernel), with no host round trip between segments; the host
looks at the solver state once per launch (at most 64 segments).  It runs the
same kernels in the same order as the host-driven loop (LBM_POISSON_LOOP=0),
so fields are bitwise equal and every step takes the same number of sweeps:
natural exits, replayed counts, the dual residual, the mixed box, the slip
walls and the periodic box, and the sweep cap's error."""
import os

import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu
SHAPE = (16, 12, 10)


def run(loop, periodic, precision="fp64", dual=False, replay=None, steps=3, check=100, tol=1e-6, cap=0,
        fail=False, form="kinetic"):
    os.environ["LBM_POISSON_LOOP"] = "1" if loop else "0"
    try:
        p, f = laplace_case(SHAPE, DD=8.0, noise=1e-4, seed=5)
        p.periodic_x = periodic
        g = L.InamuroCUDA(p, f, precision=precision)
        g.set_poisson(check_interval=check, tolerance=tol, dual=dual, max_sweeps=cap, fail_on_limit=fail)
        if form != "kinetic":
            g.set_poisson_form(form)
        st = g.step_replay(replay) if replay else g.step(steps)
        out = g.download_fields()
        tm = g.timing()
        g.close()
        return [int(s["iterations"]) for s in st], out, tm
    finally:
        os.environ.pop("LBM_POISSON_LOOP", None)


@pytest.mark.parametrize("periodic", [0, 1], ids=["slip_x", "periodic_x"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_loop_is_the_host_loop(periodic, precision):
    sa, fa, _ = run(False, periodic, precision)
    sb, fb, tb = run(True, periodic, precision)
    assert sa == sb and max(sa) > 100, (sa, sb)
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k


@pytest.mark.parametrize("check", [100, 3])
def test_device_loop_dual_residual(check):
    """Dual residual: the first segment (one plain sweep fewer) runs from the
    host, the rest in the device loop; check interval 3 alternates the h
    buffer every segment (the loop's nested IF node)."""
    sa, fa, _ = run(False, 0, dual=True, check=check, tol=1e-4)
    sb, fb, _ = run(True, 0, dual=True, check=check, tol=1e-4)
    assert sa == sb, (sa, sb)
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k


def test_device_loop_replay_and_long_steps():
    """Replayed counts (the loop stops at the count), including a step longer
    than one launch's 64 segments (the host relaunches the loop)."""
    plan = [300, 7000, 100]
    sa, fa, _ = run(False, 1, replay=plan)
    sb, fb, _ = run(True, 1, replay=plan)
    assert sa == sb == plan
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k


@pytest.mark.parametrize("form", ["scalar", "scalar-rb"])
def test_device_loop_scalar_forms(form):
    sa, fa, _ = run(False, 1, form=form, tol=1e-8)
    sb, fb, _ = run(True, 1, form=form, tol=1e-8)
    assert sa == sb, (sa, sb)
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k


def test_device_loop_sweep_cap():
    """The sweep cap stops the device loop at the same check as the host loop:
    LBM_ERR_POISSON_BUDGET with fail_on_limit, else the capped count."""
    sa, fa, _ = run(False, 0, tol=1e-14, cap=500)
    sb, fb, _ = run(True, 0, tol=1e-14, cap=500)
    assert sa == sb and max(sa) == 500 and all(s <= 500 for s in sa), (sa, sb)
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k
    with pytest.raises(L.LBMError) as e:
        run(True, 0, tol=1e-14, cap=500, fail=True)
    assert e.value.status == 3


def batch_run(loop, replay=None, steps=2):
    from tests.test_gpu_batch import CAP, uneven_cases
    os.environ["LBM_POISSON_LOOP"] = "1" if loop else "0"
    try:
        cases = uneven_cases()
        b = L.Batch([p for p, _ in cases], [f for _, f in cases])
        b.set_poisson(max_sweeps=CAP, fail_on_limit=True)
        st = b.step_replay(replay) if replay else b.step(steps)
        counts = [[int(s["iterations"]) for s in row] for row in st]
        fields = [b.download_fields(i) for i in range(len(cases))]
        return counts, fields
    finally:
        os.environ.pop("LBM_POISSON_LOOP", None)


@pytest.mark.parametrize("replay", [None, [[300, 200, 7000, 100, 300]]], ids=["natural", "replay"])
def test_batch_device_loop_is_the_host_loop(replay):
    """The batch's device-side loop (segments until no instance is active,
    64 per launch) against one segment graph per host round trip: the same
    per-instance sweep counts and bitwise equal fields."""
    ca, fa = batch_run(False, replay)
    cb, fb = batch_run(True, replay)
    assert ca == cb, (ca, cb)
    for i, (x, y) in enumerate(zip(fa, fb)):
        for k in L.FIELDS:
            assert np.array_equal(x[k], y[k]), (i, k)

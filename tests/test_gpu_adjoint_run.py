"""Gradients through whole FP64 steps (lbm_adjoint_*): the implicit adjoint
of the Poisson solve, the step adjoints chained backwards, checkpoints with
recomputation.

The objective mirrors the adjoint calibration workload on a small periodic
box: J = 0.5 sum (phi_T - phi_target)^2, phi_target the final phi of a run
with k_f raised by 5 % (plus fixed random weights on rho_T, u_T and p_T, so
that every final field's adjoint path is exercised).  Directional
derivatives from the reverse pass are checked against FP64 centred finite
differences of forward runs (step 1e-6 of each field's scale) along seeded
random directions of the loaded phi, rho, u, p and along k_f, to 1e-6
relative.  The loaded rho enters J only through the O(k_g) capillary terms
of the first g collision, so its directional derivative is small against J:
at step 1e-6 the forward runs' rounding (the last bits of J move with the
inputs, ~1e-10 of that derivative per 1e-16 of J) is of the order of the
tolerance, so that direction uses step 1e-5 (truncation ~1e-10 relative).
The finite-difference runs replay the base run's sweep counts, so
J is a smooth function of the inputs; the base run's Poisson exit (relative
change 1e-11 between checks) and the adjoint solve's (1e-13) make the
implicit derivative and that of the replayed run agree far below 1e-6.
Seven steps with checkpoints every three: two recomputed intervals and a
partial one.  The same checks run on the reference's x slip walls (the
transposed overwrite and mirrored stencils, and the adjoint of the gauged
solve whose sweeps drift along the constant mode)."""
import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu
SHAPE = (20, 16, 12)
STEPS = 7
KINT = 3
FD_STEP = 1e-6
TOL = 1e-6


def setup_case(periodic=1):
    p, f = laplace_case(SHAPE, DD=7.0, noise=1e-4, seed=21)
    p.periodic_x = periodic
    rng = np.random.default_rng(5)
    shp = f["phi"].shape
    f["u"] = 0.005 * np.sin(2 * np.pi * np.arange(SHAPE[0]) / SHAPE[0])[None, None, :] * np.ones(shp)
    f["w"] = 0.002 * rng.standard_normal(shp)
    return p, f


def poisson(obj):
    obj.set_poisson(check_interval=100, tolerance=1e-11, max_sweeps=400000, fail_on_limit=1)


def final_fields(p, f, sweeps=None):
    a = L.Adjoint(p, checkpoint_interval=KINT)
    poisson(a)
    a.forward(f, STEPS, sweeps)
    out = {k: a.download(k) for k in L.FIELDS}
    counts = a.sweeps()
    a.close()
    return out, counts


class Objective:
    def __init__(self, p, f):
        rng = np.random.default_rng(77)
        pt = L.make_params(**{k: getattr(p, k) for k, _ in L.Params._fields_})
        pt.k_f = p.k_f * 1.05
        self.target = final_fields(pt, f)[0]["phi"]
        shp = f["phi"].shape
        self.w_rho = 1e-3 * rng.standard_normal(shp)
        self.w_u = 1e-1 * rng.standard_normal(shp)
        self.w_p = 1e-1 * rng.standard_normal(shp)

    def value(self, y):
        return (0.5 * np.sum((y["phi"] - self.target) ** 2) + np.sum(self.w_rho * y["rho"]) +
                np.sum(self.w_u * y["u"]) + np.sum(self.w_p * y["p"]))

    def adjoint(self, y):
        return {"phi": y["phi"] - self.target, "rho": self.w_rho, "u": self.w_u, "p": self.w_p}


def make_run(periodic):
    p, f = setup_case(periodic)
    obj = Objective(p, f)
    a = L.Adjoint(p, checkpoint_interval=KINT, check_interval=50, tolerance=1e-13, max_sweeps=2000000)
    poisson(a)
    a.forward(f, STEPS)
    y = {k: a.download(k) for k in L.FIELDS}
    sweeps = a.sweeps()
    grads, stats = a.backward(obj.adjoint(y))
    return p, f, obj, y, sweeps, grads, stats, a


@pytest.fixture(scope="module")
def run():
    return make_run(1)


@pytest.fixture(scope="module")
def run_walls():
    return make_run(0)


def fd(p, f, obj, sweeps, field=None, d=None, kf=False, step=FD_STEP):
    vals = []
    for sgn in (1.0, -1.0):
        pp = L.make_params(**{k: getattr(p, k) for k, _ in L.Params._fields_})
        ff = dict(f)
        if kf:
            h = step * p.k_f
            pp.k_f = p.k_f + sgn * h
        else:
            h = step
            ff[field] = f[field] + sgn * h * d
        vals.append(obj.value(final_fields(pp, ff, sweeps)[0]))
    return (vals[0] - vals[1]) / (2 * h)


def test_forward_matches_the_solver(run):
    """The adjoint object's forward run is the FP64 solver's run."""
    p, f, obj, y, sweeps, grads, stats, a = run
    g = L.InamuroCUDA(p, f, precision="fp64")
    g.set_poisson(check_interval=100, tolerance=1e-11, max_sweeps=400000, fail_on_limit=True)
    st = g.step(STEPS)
    assert [int(s["iterations"]) for s in st] == sweeps
    for k in L.FIELDS:
        assert np.array_equal(g.download(k), y[k]), k


@pytest.mark.parametrize("field,seed,step", [("phi", 1, FD_STEP), ("phi", 2, FD_STEP), ("rho", 3, 1e-5),
                                             ("u", 4, FD_STEP), ("p", 5, FD_STEP)])
def test_gradient_matches_finite_differences(run, field, seed, step):
    p, f, obj, y, sweeps, grads, stats, a = run
    rng = np.random.default_rng(seed)
    scale = max(float(np.max(np.abs(f[field]))), 1e-2)
    d = scale * rng.standard_normal(f[field].shape)
    want = fd(p, f, obj, sweeps, field, d, step=step)
    got = float(np.sum(grads[field] * d))
    assert abs(got - want) <= TOL * abs(want), (field, got, want)


def test_kappa_f_gradient_matches_finite_differences(run):
    p, f, obj, y, sweeps, grads, stats, a = run
    want = fd(p, f, obj, sweeps, kf=True)
    got = stats["grad_kappa_f"]
    assert abs(got - want) <= TOL * abs(want), (got, want)


def test_reverse_pass_bookkeeping(run):
    p, f, obj, y, sweeps, grads, stats, a = run
    assert stats["forward_steps"] == STEPS and stats["recompute_steps"] == STEPS
    assert stats["forward_sweeps"] == sum(sweeps) and stats["adjoint_sweeps"] > 0
    # p enters only through its mean (the gauge target): its gradient is uniform
    gp = grads["p"]
    assert np.ptp(gp) <= 1e-12 * max(np.max(np.abs(gp)), 1e-300)
    # a second reverse pass on the same forward run gives the same gradient
    g2, s2 = a.backward(obj.adjoint(y))
    for k in L.FIELDS:
        assert np.array_equal(g2[k], grads[k]), k
    assert s2["grad_kappa_f"] == stats["grad_kappa_f"]


def test_slip_walls_forward_matches_the_solver(run_walls):
    p, f, obj, y, sweeps, grads, stats, a = run_walls
    assert p.periodic_x == 0
    g = L.InamuroCUDA(p, f, precision="fp64")
    g.set_poisson(check_interval=100, tolerance=1e-11, max_sweeps=400000, fail_on_limit=True)
    st = g.step(STEPS)
    assert [int(s["iterations"]) for s in st] == sweeps
    for k in L.FIELDS:
        assert np.array_equal(g.download(k), y[k]), k


@pytest.mark.parametrize("field,seed,step", [("phi", 1, FD_STEP), ("phi", 2, FD_STEP), ("u", 4, FD_STEP),
                                             ("p", 5, FD_STEP)])
def test_slip_walls_gradient_matches_finite_differences(run_walls, field, seed, step):
    p, f, obj, y, sweeps, grads, stats, a = run_walls
    rng = np.random.default_rng(seed)
    scale = max(float(np.max(np.abs(f[field]))), 1e-2)
    d = scale * rng.standard_normal(f[field].shape)
    want = fd(p, f, obj, sweeps, field, d, step=step)
    got = float(np.sum(grads[field] * d))
    assert abs(got - want) <= TOL * abs(want), (field, got, want)


def test_slip_walls_kappa_f_gradient_matches_finite_differences(run_walls):
    p, f, obj, y, sweeps, grads, stats, a = run_walls
    want = fd(p, f, obj, sweeps, kf=True)
    got = stats["grad_kappa_f"]
    assert abs(got - want) <= TOL * abs(want), (got, want)
    gp = grads["p"]
    assert np.ptp(gp) <= 1e-12 * max(np.max(np.abs(gp)), 1e-300)


def test_slip_walls_krylov_adjoint_matches_the_sweeps(run_walls):
    """BiCGSTAB on the walls' adjoint system (consistent: E^T B = E^T and the
    right-hand side has zero sum) reaches the transposed sweeps' solution."""
    p, f, obj, y, sweeps, grads, stats, a = run_walls
    b = L.Adjoint(p, checkpoint_interval=KINT, check_interval=50, tolerance=1e-13, max_sweeps=2000000,
                  krylov=True, krylov_tolerance=1e-11)
    poisson(b)
    b.forward(f, STEPS)
    g2, s2 = b.backward(obj.adjoint(y))
    for k in L.FIELDS:
        scale = float(np.max(np.abs(grads[k])))
        assert float(np.max(np.abs(g2[k] - grads[k]))) <= 1e-7 * scale, k
    assert abs(s2["grad_kappa_f"] - stats["grad_kappa_f"]) <= 1e-7 * abs(stats["grad_kappa_f"])
    b.close()


@pytest.mark.parametrize("slots", [1, 2])
def test_binomial_checkpointing_matches_uniform(run, slots):
    """Binomial checkpointing (revolve) recomputes the same states bitwise and
    runs the same step adjoints in the same order: the gradient is bitwise the
    uniform schedule's, and the recomputed steps are the dry schedule's."""
    p, f, obj, y, sweeps, grads, stats, a = run
    b = L.Adjoint(p, check_interval=50, tolerance=1e-13, max_sweeps=2000000, binomial_checkpoints=slots)
    poisson(b)
    b.forward(f, STEPS)
    assert b.sweeps() == sweeps
    g2, s2 = b.backward(obj.adjoint(y))
    for k in L.FIELDS:
        assert np.array_equal(g2[k], grads[k]), (slots, k)
    assert s2["grad_kappa_f"] == stats["grad_kappa_f"]
    assert s2["recompute_steps"] == L.adjoint_schedule(STEPS, slots)["recompute_steps"]
    b.close()


def test_krylov_adjoint_solve_matches_the_sweeps(run):
    """The adjoint Poisson problem solved by BiCGSTAB (krylov=True) gives the
    gradient of the transposed sweeps (which the finite-difference tests
    check) to 1e-7, in a fraction of the applications."""
    p, f, obj, y, sweeps, grads, stats, a = run
    b = L.Adjoint(p, checkpoint_interval=KINT, check_interval=50, tolerance=1e-13, max_sweeps=2000000,
                  krylov=True, krylov_tolerance=1e-11)
    poisson(b)
    b.forward(f, STEPS)
    g2, s2 = b.backward(obj.adjoint(y))
    for k in L.FIELDS:
        scale = float(np.max(np.abs(grads[k])))
        assert float(np.max(np.abs(g2[k] - grads[k]))) <= 1e-7 * scale, k
    assert abs(s2["grad_kappa_f"] - stats["grad_kappa_f"]) <= 1e-7 * abs(stats["grad_kappa_f"])
    assert s2["adjoint_sweeps"] * 3 <= stats["adjoint_sweeps"], (s2["adjoint_sweeps"], stats["adjoint_sweeps"])
    b.close()


@pytest.mark.parametrize("krylov", [False, True])
def test_nonfinite_adjoint_rhs_is_an_error(krylov):
    """A NaN in the final fields' adjoint reaches the adjoint Poisson problem's
    right-hand side: both the transposed sweeps and BiCGSTAB report
    LBM_ERR_NONFINITE instead of returning a NaN gradient as a success."""
    p, f = setup_case()
    a = L.Adjoint(p, checkpoint_interval=KINT, krylov=krylov)
    poisson(a)
    a.forward(f, 2)
    lam_p = np.zeros(f["phi"].shape)
    lam_p[1, 2, 3] = np.nan
    with pytest.raises(L.LBMError) as e:
        a.backward({"p": lam_p})
    assert e.value.status == 2, str(e.value)
    a.close()


def test_mixed_forward_adjoint_against_fp64_fd(run):
    """The adjoint run over the mixed box (FP32 populations; the reverse pass
    differentiates the FP64 step at the mixed forward's states): dJ/dk_f and
    dJ/dphi_0 along a seeded direction against centred finite differences of
    the FP64 forward (replayed sweep counts).  The gradient carries the mixed
    forward's error, so the bar is 1e-5 relative instead of the FP64 run's
    1e-6 (measured: 6.8e-7 along k_f, 3.2e-8 along phi_0); the errors are
    printed."""
    p, f, obj, y, sweeps, grads, stats, a = run
    m = L.Adjoint(p, checkpoint_interval=KINT, check_interval=50, tolerance=1e-13, max_sweeps=2000000,
                  precision="mixed")
    poisson(m)
    m.forward(f, STEPS, sweeps)
    assert m.sweeps() == sweeps
    ym = {k: m.download(k) for k in L.FIELDS}
    gm, sm = m.backward(obj.adjoint(ym))
    m.close()
    fd_kf = fd(p, f, obj, sweeps, kf=True)
    d = np.random.default_rng(1).standard_normal(f["phi"].shape)
    fd_phi = fd(p, f, obj, sweeps, field="phi", d=d)
    e_kf = abs(sm["grad_kappa_f"] - fd_kf) / abs(fd_kf)
    e_phi = abs(float(np.sum(gm["phi"] * d)) - fd_phi) / abs(fd_phi)
    print(f"\nmixed-forward adjoint vs FP64 FD: k_f {e_kf:.3e}, phi_0 {e_phi:.3e}")
    assert e_kf <= 1e-5 and e_phi <= 1e-5, (e_kf, e_phi)

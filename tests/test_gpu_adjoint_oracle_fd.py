"""Gradients of the GPU adjoint against centred finite differences of the
reference CPU solver's arithmetic: the FP64 oracle (oracle/lbm_oracle.c, the
bit-exact restatement of CPU/Inamuro.cpp), not this library's own forward.

Box 16^3, one tanh drop (rho_L/rho_G = 50, seeded phi noise), three steps,
on both x boundaries: periodic, and the reference's own slip walls.  J = 0.5 sum (phi_T - phi_target)^2, phi_target the oracle's final phi
with k_f raised by 5 %.  The oracle's natural exits (relative change 1e-11,
check 100) fix the sweep counts; the GPU forward and every oracle run of a
finite difference replay them, so J is a smooth function of the inputs.
dJ/dk_f and dJ/dphi_0 along three seeded directions from the GPU reverse pass
(adjoint solve by transposed sweeps to 1e-13) agree with the oracle's centred
differences (step 1e-6) to 1e-6 relative."""
import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import laplace_case, oracle_params

pytestmark = pytest.mark.gpu
SHAPE = (16, 16, 16)
STEPS = 3
H = 1e-6
TOL = 1e-6


def oracle_final_phi(p, f, sweeps=None, kf=None):
    prm = oracle_params(p)
    if kf is not None:
        prm["k_f"] = kf
    o = pyoracle.Oracle(p.shape, prm, f, tol=1e-11, max_sweeps=2_000_000, periodic_x=bool(p.periodic_x))
    counts = []
    for s in range(STEPS):
        info = o.step(0 if sweeps is None else sweeps[s])
        counts.append(int(info["sweeps"]))
    phi = o.fields()["phi"]
    o.close()
    return phi, counts


@pytest.fixture(scope="module", params=[1, 0], ids=["periodic_x", "slip_x"])
def case(request):
    p, f = laplace_case(SHAPE, DD=8.0, noise=1e-4, seed=41)
    p.periodic_x = request.param
    target, _ = oracle_final_phi(p, f, kf=p.k_f * 1.05)
    _, sweeps = oracle_final_phi(p, f)
    a = L.Adjoint(p, checkpoint_interval=2, check_interval=100, tolerance=1e-13, max_sweeps=2_000_000)
    a.set_poisson(check_interval=100, tolerance=1e-11, max_sweeps=2_000_000, fail_on_limit=1)
    a.forward(f, STEPS, sweeps)
    phi_T = a.download("phi")
    grads, stats = a.backward({"phi": phi_T - target})
    a.close()
    return p, f, target, sweeps, phi_T, grads, stats


def J(phi, target):
    return 0.5 * float(np.sum((phi - target) ** 2))


def test_gpu_forward_is_the_oracle_forward(case):
    p, f, target, sweeps, phi_T, grads, stats = case
    phi_o, counts = oracle_final_phi(p, f, sweeps)
    assert counts == sweeps
    assert float(np.max(np.abs(phi_T - phi_o))) <= 1e-12 * float(np.max(np.abs(phi_o)))


def test_kappa_f_gradient_against_oracle_fd(case):
    p, f, target, sweeps, phi_T, grads, stats = case
    h = H * p.k_f
    jp = J(oracle_final_phi(p, f, sweeps, kf=p.k_f + h)[0], target)
    jm = J(oracle_final_phi(p, f, sweeps, kf=p.k_f - h)[0], target)
    fd = (jp - jm) / (2 * h)
    assert abs(stats["grad_kappa_f"] - fd) <= TOL * abs(fd), (stats["grad_kappa_f"], fd)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_phi0_gradient_against_oracle_fd(case, seed):
    p, f, target, sweeps, phi_T, grads, stats = case
    d = 0.05 * np.random.default_rng(seed).standard_normal(f["phi"].shape)
    vals = []
    for sgn in (1.0, -1.0):
        ff = dict(f)
        ff["phi"] = f["phi"] + sgn * H * d
        vals.append(J(oracle_final_phi(p, ff, sweeps)[0], target))
    fd = (vals[0] - vals[1]) / (2 * H)
    got = float(np.sum(grads["phi"] * d))
    assert abs(got - fd) <= TOL * abs(fd), (got, fd)

"""The oracle's restatement of the reference's scalar Poisson form
(scalarPressureJacobiKernel, GPU/InamuroCUDA.cu:864-901): run to a tight
tolerance, its p satisfies the scalar equation
(sum_{q=1..14} p(x - c_q) - 14 p) / 5 = scale rho s up to the constant the
gauge absorbs and its checkerboard component, with the x neighbours mirrored
at the slip walls, and keeps the gauge target as its mean.  The Jacobi sweep
maps the checkerboard chi = (-1)^(x+y+z) to -chi (every neighbour has the
other colour), so at the even sweep counts of its checks it never takes up
the right-hand side's chi component: the residual is exactly that component."""
import numpy as np
import pytest

from oracle import pyoracle
from tests.helpers import laplace_case, oracle_params

CX = np.array([0, 1, 0, 0, -1, 0, 0, 1, -1, 1, 1, -1, 1, -1, -1])
CY = np.array([0, 0, 1, 0, 0, -1, 0, 1, 1, -1, 1, -1, -1, 1, -1])
CZ = np.array([0, 0, 0, 1, 0, 0, -1, 1, 1, 1, -1, -1, -1, -1, 1])


def neighbour_sum(p, periodic):
    lz, ly, lx = p.shape
    x = np.arange(lx)
    out = np.zeros_like(p)
    for q in range(1, 15):
        xs = x - CX[q]
        if periodic:
            xs = xs % lx
        else:
            xs = np.where(xs < 0, 1, np.where(xs >= lx, lx - 2, xs))
        shifted = np.roll(p, (CZ[q], CY[q]), axis=(0, 1))[:, :, xs]
        out += shifted
    return out


@pytest.mark.parametrize("periodic", [False, True])
def test_scalar_restatement_solves_the_scalar_equation(periodic):
    shape = (14, 10, 8)
    p, f = laplace_case(shape, DD=5.0, noise=1e-4, seed=9)
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(shape[2]) / shape[2])[:, None, None] * np.ones_like(f["w"])
    f["p"] = 1e-3 * np.ones_like(f["phi"])
    o = pyoracle.Oracle(shape, oracle_params(p), f, tol=1e-13, max_sweeps=2000000, periodic_x=periodic,
                        poisson_form=1, scalar_source_scale=2.0)
    info = o.step()
    fl = o.fields()
    d = o.derivatives()
    s = d[6] + d[10] + d[14]   # projected u_x + v_y + w_z (D_UX, D_VY, D_WZ)
    lap = (neighbour_sum(fl["p"], periodic) - 14.0 * fl["p"]) / 5.0
    resid = lap - 2.0 * fl["rho"] * s
    # components along the constant and chi, projected with the weights under
    # which the mirrored stencil is symmetric (1/2 on the wall planes)
    lz, ly, lx = fl["p"].shape
    w = np.ones(lx)
    if not periodic:
        w[0] = w[-1] = 0.5
    w = np.broadcast_to(w, fl["p"].shape)
    chi = (-1.0) ** np.add.outer(np.add.outer(np.arange(lz), np.arange(ly)), np.arange(lx))
    proj = lambda a, v: float(np.sum(w * a * v) / np.sum(w))
    rhs = 2.0 * fl["rho"] * s
    resid -= proj(resid, 1.0)
    assert np.max(np.abs(resid + proj(rhs, chi) * chi)) <= 1e-8 * np.max(np.abs(rhs))
    resid -= proj(resid, chi) * chi
    assert np.max(np.abs(resid)) <= 1e-8 * np.max(np.abs(2.0 * fl["rho"] * s))
    assert abs(fl["p"].mean() - info["gauge_target"]) <= 1e-15
    assert abs(info["gauge_target"] - 1e-3) <= 1e-15

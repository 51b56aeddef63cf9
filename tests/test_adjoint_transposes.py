"""The transposes the slip-wall adjoint kernels use (adjoint_fp64.cu,
lbm_device.cuh: slip_T, tpull, stencil_T, the correction's x part), restated
in numpy with the kernels' index rules and checked by dot-product tests
<y, F x> = <F^T y, x> against the forward maps on a tiny box (no GPU):

* F = W R, the pull x - c_q followed by the x slip overwrite
  (CPU/Inamuro.cpp:589-623); its transpose by the kernels' rule: cell x reads
  population q of y at x + c_q, 0 when that neighbour is a wall cell whose q
  is overwritten, plus the overwritten partner's value when q is the one
  copied (tpull);
* the gradient and laplacian stencils with mirrored x neighbours
  (CPU/Inamuro.hpp:213-314): the transpose gathers from x - c_k without
  wrapping x, plus the wall cells' mirrored reads at x = 1 and lx - 2
  (stencil_T);
* the x difference of the velocity correction with mirrored neighbours
  (CPU/Inamuro.cpp:794-823): wall cells contribute nothing."""
import numpy as np
import pytest

CX = np.array([0, 1, 0, 0, -1, 0, 0, 1, -1, 1, 1, -1, 1, -1, -1])
CY = np.array([0, 0, 1, 0, 0, -1, 0, 1, 1, -1, 1, -1, -1, 1, -1])
CZ = np.array([0, 0, 0, 1, 0, 0, -1, 1, 1, 1, -1, -1, -1, -1, 1])
BOUNCE_LEFT = {1: 4, 7: 8, 9: 14, 10: 13, 12: 11}
BOUNCE_RIGHT = {v: k for k, v in BOUNCE_LEFT.items()}
SHAPE = (4, 3, 6)   # lz, ly, lx


def pull_bounce(h):
    v = np.stack([np.roll(h[q], (CZ[q], CY[q], CX[q]), axis=(0, 1, 2)) for q in range(15)])
    for q, m in BOUNCE_LEFT.items():
        v[q][:, :, 0] = v[m][:, :, 0]
    for q, m in BOUNCE_RIGHT.items():
        v[q][:, :, -1] = v[m][:, :, -1]
    return v


def tpull(y):
    """The kernels' rule, cell by cell."""
    lz, ly, lx = SHAPE
    out = np.zeros_like(y)
    for q in range(15):
        for z in range(lz):
            for yy in range(ly):
                for x in range(lx):
                    n = ((z + CZ[q]) % lz, (yy + CY[q]) % ly, (x + CX[q]) % lx)
                    v = y[q][n]
                    if CX[q] == 1:
                        if x == lx - 1:
                            v = 0.0
                        elif x == lx - 2:
                            v += y[BOUNCE_LEFT[q]][n]
                    elif CX[q] == -1:
                        if x == 0:
                            v = 0.0
                        elif x == 1:
                            v += y[BOUNCE_RIGHT[q]][n]
                    out[q, z, yy, x] = v
    return out


def mirror_x(x, d, lx):
    x += d
    return 1 if x < 0 else (lx - 2 if x >= lx else x)


def stencil(f, k_weight):
    """sum_k w(k) f(x + c_k), x mirrored, y and z periodic (k = 1..14)."""
    lz, ly, lx = SHAPE
    out = np.zeros_like(f)
    for z in range(lz):
        for y in range(ly):
            for x in range(lx):
                out[z, y, x] = sum(k_weight(k) * f[(z + CZ[k]) % lz, (y + CY[k]) % ly, mirror_x(x, CX[k], lx)]
                                   for k in range(1, 15))
    return out


def stencil_T(a, k_weight):
    """The kernels' rule: gather from x - c_k without wrapping x, plus the
    wall cells' mirrored reads (x = 0 reads x = 1 for c_x = -1, x = lx - 1
    reads x = lx - 2 for c_x = +1)."""
    lz, ly, lx = SHAPE
    out = np.zeros_like(a)
    for z in range(lz):
        for y in range(ly):
            for x in range(lx):
                s = 0.0
                for k in range(1, 15):
                    zz, yy = (z - CZ[k]) % lz, (y - CY[k]) % ly
                    xc = x - CX[k]
                    if 0 <= xc < lx:
                        s += k_weight(k) * a[zz, yy, xc]
                    if CX[k] == -1 and x == 1:
                        s += k_weight(k) * a[zz, yy, 0]
                    if CX[k] == 1 and x == lx - 2:
                        s += k_weight(k) * a[zz, yy, lx - 1]
                out[z, y, x] = s
    return out


def xdiff(p, inv2rho):
    lx = SHAPE[2]
    out = np.zeros_like(p)
    for x in range(lx):
        out[:, :, x] = (p[:, :, mirror_x(x, 1, lx)] - p[:, :, mirror_x(x, -1, lx)]) * inv2rho[:, :, x]
    return out


def xdiff_T(la, inv2rho):
    """The correction adjoint's x part: t receives -la/(2 rho) from x - 1 and
    +la/(2 rho) from x + 1, interior cells only (no wrap)."""
    lx = SHAPE[2]
    out = np.zeros_like(la)
    g = la * inv2rho
    for x in range(lx):
        if x - 1 >= 1:
            out[:, :, x] += g[:, :, x - 1]
        if x + 1 <= lx - 2:
            out[:, :, x] -= g[:, :, x + 1]
    return out


def dot_ok(fx, y, x, fty):
    lhs, rhs = float(np.sum(y * fx)), float(np.sum(fty * x))
    return abs(lhs - rhs) <= 1e-12 * (np.sum(np.abs(y * fx)) + 1.0), (lhs, rhs)


def test_transposed_pull_with_slip_walls():
    rng = np.random.default_rng(0)
    h = rng.standard_normal((15,) + SHAPE)
    y = rng.standard_normal((15,) + SHAPE)
    ok, vals = dot_ok(pull_bounce(h), y, h, tpull(y))
    assert ok, vals


@pytest.mark.parametrize("which", ["x", "y", "z", "lap"])
def test_mirrored_stencil_transposes(which):
    w = {"x": lambda k: CX[k] / 10.0, "y": lambda k: CY[k] / 10.0, "z": lambda k: CZ[k] / 10.0,
         "lap": lambda k: 1.0 / 5.0}[which]
    rng = np.random.default_rng(1)
    f = rng.standard_normal(SHAPE)
    a = rng.standard_normal(SHAPE)
    ok, vals = dot_ok(stencil(f, w), a, f, stencil_T(a, w))
    assert ok, vals


def test_mirrored_correction_transpose():
    rng = np.random.default_rng(2)
    p = rng.standard_normal(SHAPE)
    la = rng.standard_normal(SHAPE)
    inv2rho = 1.0 / (2.0 * (0.5 + rng.random(SHAPE)))
    # u = u* - xdiff(p): the adjoint of p is -xdiff^T
    ok, vals = dot_ok(-xdiff(p, inv2rho), la, p, -xdiff_T(la, inv2rho))
    assert ok, vals

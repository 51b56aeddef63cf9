"""The algebra behind two Poisson solvers, restated in numpy on tiny boxes
(no GPU): the kinetic map K of one sweep (pull x - c_q, the x slip overwrite
of CPU/Inamuro.cpp:589-623, the relaxation hv - omega (hv - E sum hv)),
b = -(E/3) s.

* Slip walls make (I - K) h = b inconsistent: the sweeps drift along E (the
  uniform-p null vector) and the gauge removes the drift at every check.  The
  bordered system (I - K) h + delta E = b, sum_x p(h) = N target, which the
  Krylov form solves on the walls, has the gauged sweeps' limit as its
  solution.
* The refinement form's corrections e_1 = r = K H + b - H,
  e_(k+1) = K e_k + r make H + e_k the state after k sweeps from H; rounding
  the corrections to FP32 costs an error of the order of the corrections'
  size, not of h's."""
import numpy as np

CX = np.array([0, 1, 0, 0, -1, 0, 0, 1, -1, 1, 1, -1, 1, -1, -1])
CY = np.array([0, 0, 1, 0, 0, -1, 0, 1, 1, -1, 1, -1, -1, 1, -1])
CZ = np.array([0, 0, 0, 1, 0, 0, -1, 1, 1, 1, -1, -1, -1, -1, 1])
E = np.array([2 / 9] + [1 / 9] * 6 + [1 / 72] * 8)[:, None, None, None]
BOUNCE_LEFT = {1: 4, 7: 8, 9: 14, 10: 13, 12: 11}
BOUNCE_RIGHT = {v: k for k, v in BOUNCE_LEFT.items()}


def case(walls, shape=(5, 4, 6), seed=3):
    lz, ly, lx = shape
    z, y, x = np.meshgrid(np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    r = np.sqrt((x - (lx - 1) / 2) ** 2 + (y - (ly - 1) / 2) ** 2 + (z - (lz - 1) / 2) ** 2)
    rho = 0.02 + 0.98 * 0.5 * (1 - np.tanh(r - 1.5))
    om = 1.0 / (1.0 / rho + 0.5)
    s = np.random.default_rng(seed).standard_normal(shape) * 1e-3
    s -= s.mean()

    def pulled(h):
        v = np.stack([np.roll(h[q], (CZ[q], CY[q], CX[q]), axis=(0, 1, 2)) for q in range(15)])
        if walls:
            for q, m in BOUNCE_LEFT.items():
                v[q][:, :, 0] = v[m][:, :, 0]
            for q, m in BOUNCE_RIGHT.items():
                v[q][:, :, -1] = v[m][:, :, -1]
        return v

    def K(h):
        v = pulled(h)
        return v - om * (v - E * v.sum(0))

    b = -(E / 3.0) * s
    return K, lambda h: pulled(h).sum(0), b


def test_bordered_system_is_the_gauged_sweeps_limit():
    K, P, b = case(walls=True)
    n = b[0].size
    target = 0.37
    # the sweeps, gauged every 100 sweeps, to their limit
    h = E * target * np.ones_like(b)
    for _ in range(400):
        for _ in range(100):
            h = K(h) + b
        shift = P(h).mean() - target
        h = h - E * shift
    p_sweeps = P(h)
    drift = (K(h) + b - h).mean(axis=(1, 2, 3)) / E[:, 0, 0, 0]
    assert np.ptp(drift) < 1e-9 * np.abs(b).max() and abs(drift[0]) > 1e-9, drift   # a uniform drift E delta

    # BiCGSTAB on the bordered system, unknowns (h, delta), row scaled by N
    def A(x):
        hh, d = x
        return hh - K(hh) + d * E, P(hh).sum()

    def dot(a, c):
        return float((a[0] * c[0]).sum() + a[1] * c[1])

    x = (E * target * np.ones_like(b), 0.0)
    Ax = A(x)
    r = (b - Ax[0], n * target - Ax[1])
    r0, pp, rho_old = r, r, dot(r, r)
    bn = np.sqrt((b * b).sum())
    for _ in range(3000):
        v = A(pp)
        al = rho_old / dot(r0, v)
        sv = (r[0] - al * v[0], r[1] - al * v[1])
        t = A(sv)
        w = dot(t, sv) / dot(t, t)
        x = (x[0] + al * pp[0] + w * sv[0], x[1] + al * pp[1] + w * sv[1])
        r = (sv[0] - w * t[0], sv[1] - w * t[1])
        if np.sqrt(dot(r, r)) < 1e-13 * bn:
            break
        rho_new = dot(r0, r)
        be = rho_new / rho_old * al / w
        rho_old = rho_new
        pp = (r[0] + be * (pp[0] - w * v[0]), r[1] + be * (pp[1] - w * v[1]))
    p_kr = P(x[0])
    scale = np.abs(p_sweeps - target).max()
    assert np.abs(p_kr - p_sweeps).max() <= 1e-8 * scale, np.abs(p_kr - p_sweeps).max() / scale
    assert abs(p_kr.mean() - target) < 1e-12
    # delta is the sweeps' drift per sweep
    assert abs(x[1] - drift[0]) <= 1e-6 * abs(drift[0]), (x[1], drift[0])


def test_refinement_corrections_are_sweeps():
    for walls in (True, False):
        K, P, b = case(walls=walls)
        H = E * 0.4 * np.ones_like(b) + 1e-3 * np.random.default_rng(1).standard_normal(b.shape)
        r = K(H) + b - H
        # exact arithmetic: H + e_k is k sweeps from H
        e, h = r, K(H) + b
        for _ in range(20):
            e = K(e) + r
            h = K(h) + b
        assert np.abs(H + e - h).max() <= 1e-14 * np.abs(h).max()
        # FP32 corrections: the error scales with |e|, not with |h|
        e32, r32 = r.astype(np.float32), r.astype(np.float32)
        for _ in range(20):
            e32 = (K(e32.astype(np.float64)) + r32).astype(np.float32)
        err = np.abs(H + e32 - h).max()
        assert err <= 1e-5 * np.abs(e).max(), (err, np.abs(e).max())
        assert err <= 1e-8 * np.abs(h).max()

"""Adjoints of the explicit FP64 kernels (lbm_collide/moments/correct_backward).

Each backward call is checked by the dot-product test against centred finite
differences of the matching forward call (the solver's own FP64 kernel): for a
random direction d of one input and random output adjoints lam,
    <lam, (F(x + e d) - F(x - e d)) / (2 e)>  ==  <d, B(lam)>.
With e = 1e-6 of each field's scale the truncation error is O(e^2) and the
rounding error O(1e-16 / e), so both sides agree to ~1e-10 of the sum of the
terms' magnitudes; the tolerance is 1e-7 of that sum.  Forward calls are also
checked against numpy restatements (moments, correction), and a chained
collide -> moments gradient against finite differences.  Every test runs on
both x boundaries: periodic, and the reference's slip walls (the overwrite of
the incoming populations at x = 0 and lx-1 after the pull, and the mirrored
x neighbours of the stencils and the correction)."""
import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPE = (20, 12, 10)     # lx, ly, lz: partial CTA tiles in x and y
EPS = 1e-6
TOL = 1e-7
CX = np.array([0, 1, 0, 0, -1, 0, 0, 1, -1, 1, 1, -1, 1, -1, -1])
CY = np.array([0, 0, 1, 0, 0, -1, 0, 1, 1, -1, 1, -1, -1, 1, -1])
CZ = np.array([0, 0, 0, 1, 0, 0, -1, 1, 1, 1, -1, -1, -1, -1, 1])


def dev(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def ptr(t):
    return t.data_ptr()


BCS = pytest.mark.parametrize("periodic", [1, 0], ids=["periodic_x", "slip_x"])
BOUNCE_LEFT = {1: 4, 7: 8, 9: 14, 10: 13, 12: 11}     # incoming at x = 0 <- its mirror
BOUNCE_RIGHT = {v: k for k, v in BOUNCE_LEFT.items()}  # incoming at x = lx-1 <- its mirror


def state(seed=3, periodic=1):
    """A droplet box with an interface (the sine branch of rho(phi) is
    active), a random small velocity and random populations."""
    p, f = laplace_case(SHAPE, DD=8.0, noise=1e-3, seed=seed)
    p.periodic_x = periodic
    rng = np.random.default_rng(seed)
    shp = f["phi"].shape
    n = f["phi"].size
    x = {k: dev(f[k]) for k in ("phi", "rho", "p")}
    for k in ("u", "v", "w"):
        x[k] = dev(0.01 * rng.standard_normal(shp))
    x["fin"] = dev(f["phi"].ravel()[None, :] / 15.0 + 0.01 * rng.standard_normal((15, n)))
    x["gin"] = dev(1.0 / 15.0 + 0.01 * rng.standard_normal((15, n)))
    return p, x


def zeros_like(t):
    return torch.zeros_like(t)


def rand_like(t, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(t.shape, dtype=torch.float64, device="cuda", generator=g)


def scale_of(t):
    s = float(t.abs().max())
    return s if s > 0 else 1.0


def dot_check(fwd, x, lam, grads, names, seed=100):
    """Dot-product test of the input fields `names`: fwd(x) -> dict of outputs."""
    for i, k in enumerate(names):
        d = rand_like(x[k], seed + i) * scale_of(x[k])
        xp = dict(x)
        xm = dict(x)
        xp[k] = x[k] + EPS * d
        xm[k] = x[k] - EPS * d
        yp, ym = fwd(xp), fwd(xm)
        terms = [(lam[o] * (yp[o] - ym[o]) / (2 * EPS)) for o in lam]
        lhs = float(sum(t.sum() for t in terms))
        mag = float(sum(t.abs().sum() for t in terms))
        rhs = float((d * grads[k]).sum())
        assert mag > 0, k
        assert abs(lhs - rhs) <= TOL * mag, (k, lhs, rhs, mag)


def set_taus(p):
    p.tauf, p.taug = 0.8, 0.7   # 1 - 1/tau != 0: the populations' own path is exercised
    return p


# ---- collide ----------------------------------------------------------------
COLLIDE_IN = ("fin", "gin", "phi", "rho", "u", "v", "w")
COLLIDE_OUT = ("fout", "gout", "dux", "dvy", "dwz")


def collide_fwd(p, x):
    y = {"fout": zeros_like(x["fin"]), "gout": zeros_like(x["gin"])}
    for k in ("dux", "dvy", "dwz"):
        y[k] = zeros_like(x["phi"])
    L.collide_forward(p, *[ptr(x[k]) for k in COLLIDE_IN], *[ptr(y[k]) for k in COLLIDE_OUT])
    return y


def collide_bwd(p, x, lam):
    gr = {k: zeros_like(x[k]) for k in COLLIDE_IN}
    L.collide_backward(p, *[ptr(x[k]) for k in COLLIDE_IN], *[ptr(lam[k]) for k in COLLIDE_OUT],
                       *[ptr(gr[k]) for k in COLLIDE_IN])
    return gr


@BCS
def test_collide_backward_is_the_transposed_jacobian(periodic):
    p, x = state(periodic=periodic)
    set_taus(p)
    y = collide_fwd(p, x)
    lam = {k: rand_like(y[k], 7 + i) for i, k in enumerate(COLLIDE_OUT)}
    gr = collide_bwd(p, x, lam)
    dot_check(lambda xx: collide_fwd(p, xx), x, lam, gr, COLLIDE_IN)


# Inputs each collide output depends on (f does not see rho, g does not see phi).
DEPS = {"fout": ("fin", "phi", "u", "v", "w"), "gout": ("gin", "rho", "u", "v", "w"),
        "dux": ("u",), "dvy": ("v",), "dwz": ("w",)}


@BCS
def test_collide_backward_per_output(periodic):
    """One output adjoint at a time (the others zero), so that a wrong term
    cannot hide behind another output's; inputs the output does not depend on
    get exactly zero."""
    p, x = state(seed=5, periodic=periodic)
    set_taus(p)
    y = collide_fwd(p, x)
    for j, o in enumerate(COLLIDE_OUT):
        lam = {k: (rand_like(y[k], 30 + j) if k == o else zeros_like(y[k])) for k in COLLIDE_OUT}
        gr = collide_bwd(p, x, lam)
        dot_check(lambda xx: collide_fwd(p, xx), x, lam, gr, DEPS[o], seed=200 + 10 * j)
        for k in COLLIDE_IN:
            if k not in DEPS[o]:
                assert not bool(gr[k].any()), (o, k)


# ---- moments ----------------------------------------------------------------
MOM_OUT = ("phi", "rho", "u", "v", "w")


def moments_fwd(p, x):
    y = {k: x["f"].new_zeros(x["f"].shape[1:]) for k in MOM_OUT}
    L.moments_forward(p, ptr(x["f"]), ptr(x["g"]), *[ptr(y[k]) for k in MOM_OUT])
    return y


def pulled(a, shape, periodic):
    """The pull stream x - c_q of every population, then (slip walls) the
    overwrite of the incoming ones by their mirrors (CPU/Inamuro.cpp:589-623)."""
    v = [np.roll(a[q].reshape(shape), (CZ[q], CY[q], CX[q]), axis=(0, 1, 2)) for q in range(15)]
    if not periodic:
        for q, m in BOUNCE_LEFT.items():
            v[q][:, :, 0] = v[m][:, :, 0]
        for q, m in BOUNCE_RIGHT.items():
            v[q][:, :, -1] = v[m][:, :, -1]
    return v


def moments_numpy(p, f, g, shape):
    fv, gv = pulled(f, shape, p.periodic_x), pulled(g, shape, p.periodic_x)
    phi = sum(fv[q] for q in range(15))
    u = sum(CX[q] * gv[q] for q in range(15))
    v = sum(CY[q] * gv[q] for q in range(15))
    w = sum(CZ[q] * gv[q] for q in range(15))
    arg = (phi - (p.fei_L + p.fei_G) / 2) / (p.fei_L - p.fei_G) * np.pi
    rho = (p.rho_L - p.rho_G) / 2 * (np.sin(arg) + 1) + p.rho_G
    rho = np.where(phi <= p.fei_G, p.rho_G, np.where(phi >= p.fei_L, p.rho_L, rho))
    return {"phi": phi, "rho": rho, "u": u, "v": v, "w": w}


@BCS
def test_moments_forward_and_backward(periodic):
    p, s = state(seed=9, periodic=periodic)
    x = {"f": s["fin"], "g": s["gin"]}
    y = moments_fwd(p, x)
    want = moments_numpy(p, x["f"].cpu().numpy(), x["g"].cpu().numpy(), s["phi"].shape)
    for k in MOM_OUT:
        got = y[k].cpu().numpy().reshape(s["phi"].shape)
        assert np.max(np.abs(got - want[k])) <= 1e-13 * max(np.max(np.abs(want[k])), 1e-300), k
    phi = y["phi"].cpu().numpy()
    assert np.any((phi > p.fei_G) & (phi < p.fei_L)), "the interface branch of rho(phi) must be active"
    lam = {k: rand_like(y[k], 40 + i) for i, k in enumerate(MOM_OUT)}
    gr = {"f": zeros_like(x["f"]), "g": zeros_like(x["g"])}
    L.moments_backward(p, ptr(y["phi"]), *[ptr(lam[k]) for k in MOM_OUT], ptr(gr["f"]), ptr(gr["g"]))
    dot_check(lambda xx: moments_fwd(p, xx), x, lam, gr, ("f", "g"))


# ---- correction -------------------------------------------------------------
def correct_fwd(p, x):
    y = {k: x[k].clone() for k in ("u", "v", "w")}
    L.correct_forward(p, ptr(y["u"]), ptr(y["v"]), ptr(y["w"]), ptr(x["p"]), ptr(x["rho"]))
    return y


@BCS
def test_correct_forward_and_backward(periodic):
    p, x = state(seed=11, periodic=periodic)
    x["p"] = x["p"] + dev(1e-3 * np.random.default_rng(4).standard_normal(tuple(x["p"].shape)))
    y = correct_fwd(p, x)
    pn, rn = x["p"].cpu().numpy(), x["rho"].cpu().numpy()
    for k, ax in (("u", 2), ("v", 1), ("w", 0)):
        grad = np.roll(pn, -1, axis=ax) - np.roll(pn, 1, axis=ax)
        if ax == 2 and not periodic:
            grad[:, :, 0] = 0.0     # mirrored neighbours: x = 0 reads x = 1 on both sides
            grad[:, :, -1] = 0.0
        want = x[k].cpu().numpy() - grad * (1.0 / (2.0 * rn))
        assert np.max(np.abs(y[k].cpu().numpy() - want)) <= 1e-15 * max(np.max(np.abs(want)), 1e-300), k
    lam = {k: rand_like(y[k], 50 + i) for i, k in enumerate(("u", "v", "w"))}
    gr = {k: lam[k] for k in ("u", "v", "w")}   # the adjoints of u*, v*, w* are those of u, v, w
    gr["p"], gr["rho"] = zeros_like(x["p"]), zeros_like(x["rho"])
    L.correct_backward(p, ptr(x["p"]), ptr(x["rho"]), ptr(lam["u"]), ptr(lam["v"]), ptr(lam["w"]), ptr(gr["p"]),
                       ptr(gr["rho"]))
    dot_check(lambda xx: correct_fwd(p, xx), x, lam, gr, ("u", "v", "w", "p", "rho"))


# ---- chained: collide then moments (the explicit part of a step) -------------
@BCS
def test_collide_then_moments_gradient(periodic):
    """J = <c, phi' + rho' + u' + v' + w'> after collide -> moments; the
    gradient by moments_backward then collide_backward against finite
    differences of the chained forward calls."""
    p, x = state(seed=13, periodic=periodic)
    set_taus(p)
    y = collide_fwd(p, x)
    m = moments_fwd(p, {"f": y["fout"], "g": y["gout"]})
    lam_m = {k: rand_like(m[k], 60 + i) for i, k in enumerate(MOM_OUT)}
    lam_c = {"fout": zeros_like(y["fout"]), "gout": zeros_like(y["gout"])}
    L.moments_backward(p, ptr(m["phi"]), *[ptr(lam_m[k]) for k in MOM_OUT], ptr(lam_c["fout"]),
                       ptr(lam_c["gout"]))
    for k in ("dux", "dvy", "dwz"):
        lam_c[k] = zeros_like(y[k])
    gr = collide_bwd(p, x, lam_c)

    def chain(xx):
        yy = collide_fwd(p, xx)
        return moments_fwd(p, {"f": yy["fout"], "g": yy["gout"]})

    dot_check(chain, x, lam_m, gr, COLLIDE_IN, seed=300)


def test_slip_wall_adjoint_differs_from_periodic():
    """The walls change the transposes: the same state and output adjoints give
    different input adjoints next to the walls and the same ones in the
    interior (x = 3 .. lx-4, out of reach of the wall cells' reads)."""
    grads = []
    for periodic in (1, 0):
        p, x = state(seed=17, periodic=periodic)
        set_taus(p)
        y = collide_fwd(p, x)
        lam = {k: rand_like(y[k], 70 + i) for i, k in enumerate(COLLIDE_OUT)}
        grads.append(collide_bwd(p, x, lam))
    lz, ly, lx = state()[1]["phi"].shape
    for k in ("phi", "u"):
        a = grads[0][k].reshape(lz, ly, lx).cpu().numpy()
        b = grads[1][k].reshape(lz, ly, lx).cpu().numpy()
        assert np.array_equal(a[:, :, 3:lx - 3], b[:, :, 3:lx - 3]), k
        assert not np.allclose(a[:, :, 0], b[:, :, 0]), k

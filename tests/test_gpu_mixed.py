"""Mixed precision (FP32 populations as rest-state deviations, FP64 pressure
accumulation, reductions and exit test) against the FP64 oracle.

Tolerance: 1e-5 norm-wise relative error in phi, rho, u, v, w and p after
each step when both run the same sweep counts (replay of the oracle's
counts; a relative-change exit can stop one check earlier or later, a 1e-3
effect on p)."""
import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import fixture, fields_dict, laplace_case, oracle_params, params_from_text, rel_err

pytestmark = pytest.mark.gpu
TOL = {"phi": 1e-5, "rho": 1e-5, "u": 1e-5, "v": 1e-5, "w": 1e-5, "p": 1e-5}
CAP = 60000


def mixed_vs_oracle(p, f, steps, dual=False):
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, dual=dual, max_sweeps=CAP)
    g = L.InamuroCUDA(p, f, precision="mixed")
    g.set_poisson(dual=dual, max_sweeps=CAP, fail_on_limit=True)
    errs = []
    for _ in range(steps):
        info = o.step()
        st = g.step_replay([int(info["sweeps"])])[0]
        assert st["iterations"] == info["sweeps"]
        gf, of = g.download_fields(), o.fields()
        errs.append({k: rel_err(gf[k], of[k]) for k in L.FIELDS})
        # the FP64 rest population carries sum(phi) exactly; what differs is
        # the FP32 populations' share of the flux through the slip walls
        assert abs(st["mass"] - info["mass"]) <= 1e-9 * abs(info["mass"])
    g.close()
    return errs


@pytest.mark.parametrize("name", ["step_single_tanh", "step_two_sharp", "step_example_16x32x32"])
def test_mixed_matches_fp64_oracle(name):
    fx = fixture(name)
    p = params_from_text(fx["params_text"])
    for s, e in enumerate(mixed_vs_oracle(p, fields_dict(fx["init"]), len(fx["sweeps"]))):
        for k, v in e.items():
            assert v <= TOL[k], f"step {s + 1} {k}: {v:.3e}"


def test_mixed_laplace_32():
    fx = fixture("step_laplace_32")
    p = params_from_text(fx["params_text"])
    for s, e in enumerate(mixed_vs_oracle(p, fields_dict(fx["init"]), 2)):
        for k, v in e.items():
            assert v <= TOL[k], f"step {s + 1} {k}: {v:.3e}"


def test_mixed_dual_residual_runs():
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    errs = mixed_vs_oracle(p, fields_dict(fx["init"]), 2, dual=True)
    for k, v in errs[-1].items():
        assert v <= TOL[k], (k, v)


def test_mixed_natural_exit_close_to_fp64():
    """Without replay the mixed run picks its own exits; sweep counts agree to
    within one check interval and phi, u stay within 1e-4."""
    p, f = laplace_case((24, 20, 16), DD=8.0, noise=1e-4)
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(16) / 16)[:, None, None] * np.ones_like(f["w"])
    a = L.InamuroCUDA(p, f, precision="mixed")
    b = L.InamuroCUDA(p, f, precision="fp64")
    for g in (a, b):
        g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    for _ in range(3):
        sa, sb = a.step(1)[0], b.step(1)[0]
        assert abs(int(sa["iterations"]) - int(sb["iterations"])) <= 100
    fa, fb = a.download_fields(), b.download_fields()
    for k in ("phi", "u", "v", "w"):
        assert rel_err(fa[k], fb[k]) <= 1e-4, k


def test_mixed_field_statistics_and_ghosts():
    p, f = laplace_case((16, 12, 10), DD=6.0)
    g = L.InamuroCUDA(p, f, precision="mixed")
    g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    g.step(1)
    phi = g.download("phi")
    st = g.field_statistics("phi")
    assert st["valid_count"] == phi.size
    assert abs(st["sum"] - phi.sum()) <= 1e-9 * np.abs(phi).sum()
    gh = g.download_ghosted("rho")
    assert np.all(gh[0] == p.rho_G) and np.all(gh[-1] == p.rho_G)


@pytest.mark.parametrize("zlen,periodic", [("32", 0), ("5", 0), ("1", 0), ("32", 1)])
def test_two_sweep_pass_matches_single_sweeps(zlen, periodic, monkeypatch):
    """The temporally blocked pass (two sweeps per launch, 2.5-D z march with a
    shared-memory plane ring) gives the same steps as single-sweep launches:
    same sweep counts, fields equal to FP32 rounding; z runs that do not divide
    the box (5), single-plane runs (1) and periodic x included."""
    p, f = laplace_case((64, 40, 24), DD=12.0, noise=1e-4)
    p.periodic_x = periodic
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[:, None, None] * np.ones_like(f["w"])
    monkeypatch.setenv("LBM_SWEEP2_ZLEN", "0")
    a = L.InamuroCUDA(p, f, precision="mixed")
    monkeypatch.setenv("LBM_SWEEP2_ZLEN", zlen)
    b = L.InamuroCUDA(p, f, precision="mixed")
    for g in (a, b):
        g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    for _ in range(3):
        sa, sb = a.step(1)[0], b.step(1)[0]
        assert sa["iterations"] == sb["iterations"]
    fa, fb = a.download_fields(), b.download_fields()
    for k in L.FIELDS:
        assert rel_err(fb[k], fa[k]) <= 1e-6, k
    # the fused launches really ran: fewer launches for the same sweeps
    ta, tb = a.timing(), b.timing()
    assert ta["sweep_kernels"] == tb["sweep_kernels"]
    assert tb["kernel_launches"] < ta["kernel_launches"]


@pytest.mark.parametrize("zlen,periodic", [("16", 0), ("5", 0), ("1", 0), ("16", 1)])
def test_zmarch_collide_matches_plane_collide(zlen, periodic, monkeypatch):
    """The z-marching collide (macro fields staged in a shared-memory plane
    ring) computes the same cells as the plane-per-CTA collide: after the
    first step (equilibrium start, no reductions involved) phi and rho are
    bitwise equal; later steps differ only through the order of the source
    sum, inside FP32 rounding (1e-6; 1e-5 for the small zero-mean p).  z runs that do not divide the box (5),
    single-plane runs (1) and periodic x are covered."""
    p, f = laplace_case((64, 40, 24), DD=12.0, noise=1e-4)
    p.periodic_x = periodic
    f["u"] = 0.005 * np.cos(2 * np.pi * np.arange(40) / 40)[None, :, None] * np.ones_like(f["u"])
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[:, None, None] * np.ones_like(f["w"])
    monkeypatch.setenv("LBM_COLLIDE_ZLEN", "0")
    a = L.InamuroCUDA(p, f, precision="mixed")
    monkeypatch.setenv("LBM_COLLIDE_ZLEN", zlen)
    b = L.InamuroCUDA(p, f, precision="mixed")
    for g in (a, b):
        g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
        g.step_replay([300])
    fa, fb = a.download_fields(), b.download_fields()
    assert np.array_equal(fa["phi"], fb["phi"]) and np.array_equal(fa["rho"], fb["rho"])
    for _ in range(3):
        a.step_replay([300])
        b.step_replay([300])
    fa, fb = a.download_fields(), b.download_fields()
    for k in L.FIELDS:
        assert rel_err(fb[k], fa[k]) <= (1e-5 if k == "p" else 1e-6), k


def test_mixed_periodic_x_against_periodic_oracle():
    """Periodic x (not a reference mode): the mixed box against the FP64
    oracle run with periodic x, equal sweep counts; sum(phi) conserved to
    1e-12 of the loaded phi's FP64 sum (FP64 rest population, the stream a
    permutation of the stored FP32 moving populations)."""
    p, f = laplace_case((32, 24, 16), DD=8.0, noise=1e-4)
    p.periodic_x = 1
    f["u"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[None, :, None] * np.ones_like(f["u"])
    f["v"] = 0.01 * np.cos(2 * np.pi * np.arange(32) / 32)[None, None, :] * np.ones_like(f["v"])
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, max_sweeps=CAP, periodic_x=True)
    g = L.InamuroCUDA(p, f, precision="mixed")
    g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    masses = []
    for _ in range(3):
        info = o.step()
        masses.append(g.step_replay([int(info["sweeps"])])[0]["mass"])
    gf, of = g.download_fields(), o.fields()
    for k in ("phi", "rho", "p"):
        assert rel_err(gf[k], of[k]) <= TOL[k], k
    # velocity components against the velocity scale (a component that stays
    # near zero has no meaningful relative error of its own)
    vscale = max(float(np.max(np.abs(of[k]))) for k in ("u", "v", "w"))
    for k in ("u", "v", "w"):
        assert float(np.max(np.abs(gf[k] - of[k]))) <= 1e-5 * vscale, k
    m0 = float(np.sum(f["phi"]))
    assert max(abs(m - m0) for m in masses) <= 1e-12 * abs(m0)

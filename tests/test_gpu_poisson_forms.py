"""Poisson forms (lbm_set_poisson_form) and the reference's own GPU program.

* The scalar form (the reference's --poisson scalar, GPU/InamuroCUDA.cu:864-901)
  against the oracle's restatement of it: same sweep counts at natural exits,
  fields within the FP64 bar (1e-10 relative; the device sums run in another
  order than the oracle's x-outer loops).
* The red-black SOR form reaches the Jacobi sweeps' fixed point (tight
  tolerance on both: fields within 1e-8) in a fraction of the sweeps.
* The one-pass form with each accelerator, and source-aware init on the
  kinetic form, against the oracle's FP64 restatements (sweep counts and
  fields to the FP64 bar).
* The Krylov form (BiCGSTAB) reaches the kinetic form's fixed point (tight
  tolerance on both: fields within 1e-8) in a fraction of its applications.
* oracle/_ref/lbm_gpu_ref, the reference's GPU program compiled from its
  sources, against the reference's GPU/main.cpp over this library
  (oracle/_ref/lbm_gpu_dropin) on the same params.in with the split, fused
  and one-pass Poisson flags and the accelerators (source-aware h init,
  relaxation scales, Anderson-m1, two-grid correction): Tecplot fields to
  float32 rounding and the same sweep count at every step.
* With --poisson scalar the reference program does not solve the scalar
  equation: after each Jacobi sweep its loop still runs the split form's
  bounce + computePressure on the unchanged h (the block after the sweep is
  guarded only by !use_onepass_poisson, GPU/InamuroCUDA.cu:2307-2329), so p is
  reset to sum_q h = its start value every sweep.  The test records that
  behaviour (p stays 0 from the zero start, each solve exits at its first
  check); this library's scalar form solves the equation its kernel states
  (pinned to the oracle above)."""
import csv
import os
import subprocess

import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import laplace_case, oracle_params, rel_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_REF = os.path.join(ROOT, "oracle", "_ref", "lbm_gpu_ref")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "lbm_gpu_dropin")
SHAPE = (16, 12, 10)


def case(periodic):
    p, f = laplace_case(SHAPE, DD=6.0, noise=1e-4, seed=3)
    p.periodic_x = int(periodic)
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(SHAPE[2]) / SHAPE[2])[:, None, None] * np.ones_like(f["w"])
    return p, f


def gpu_box(p, f, form, tol, cap=400000):
    g = L.InamuroCUDA(p, f, precision="fp64")
    g.set_poisson(check_interval=100, tolerance=tol, max_sweeps=cap, fail_on_limit=True)
    g.set_poisson_form(form)
    return g


@pytest.mark.parametrize("periodic", [False, True])
def test_scalar_form_matches_oracle(periodic):
    p, f = case(periodic)
    g = gpu_box(p, f, "scalar", 1e-3)
    o = pyoracle.Oracle(SHAPE, oracle_params(p), f, tol=1e-3, periodic_x=periodic, poisson_form=1)
    for step in range(3):
        want = o.step()
        got = g.step(1)[0]
        assert got["iterations"] == want["sweeps"], step
        assert got["converged"] == 1
    of, gf = o.fields(), g.download_fields()
    for k in L.FIELDS:
        assert rel_err(gf[k], of[k]) <= 1e-10, k


ACCELS = [{}, {"fixed_point_relax": 0.8}, {"pressure_relax_scale": 0.9}, {"anderson_m1": 1}, {"two_grid": 1},
          {"source_aware_init": 1, "source_aware_scale": 0.5}]


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("accel", ACCELS, ids=["plain", "omega", "relax", "anderson", "twogrid", "source"])
def test_onepass_matches_oracle(periodic, accel):
    """The one-pass form and each accelerator against the oracle's FP64
    restatement (poisson_onepass in oracle/lbm_oracle.c): the same sweep
    count at every natural exit and fields within the FP64 bar (1e-10;
    Anderson 1e-9: its mixing coefficient comes from sums in another order)."""
    p, f = case(periodic)
    g = gpu_box(p, f, "onepass", 1e-3)
    g.set_poisson_accel(**accel)
    o = pyoracle.Oracle(SHAPE, oracle_params(p), f, tol=1e-3, periodic_x=periodic, poisson_form=2, accel=accel)
    for step in range(3):
        want = o.step()
        got = g.step(1)[0]
        assert got["iterations"] == want["sweeps"], step
    of, gf = o.fields(), g.download_fields()
    tol = 1e-9 if accel.get("anderson_m1") else 1e-10
    for k in L.FIELDS:
        assert rel_err(gf[k], of[k]) <= tol, k


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("acc", [{"source_aware_init": 1, "source_aware_scale": 0.5}, {"two_grid": 1}],
                         ids=["source", "twogrid"])
def test_kinetic_accelerators_match_oracle(periodic, acc):
    """Source-aware init and two-grid correction on the kinetic form against
    the oracle (the correction adds E_q c to the next sweep's post-collision
    h here and to the pre-collision h there: equal up to rounding)."""
    p, f = case(periodic)
    g = gpu_box(p, f, "kinetic", 1e-3)
    g.set_poisson_accel(**acc)
    o = pyoracle.Oracle(SHAPE, oracle_params(p), f, tol=1e-3, periodic_x=periodic, accel=acc)
    for step in range(3):
        assert g.step(1)[0]["iterations"] == o.step()["sweeps"], step
    of, gf = o.fields(), g.download_fields()
    for k in L.FIELDS:
        assert rel_err(gf[k], of[k]) <= 1e-10, k


def test_red_black_reaches_the_jacobi_fixed_point():
    p, f = case(True)
    a = gpu_box(p, f, "scalar", 1e-12)
    b = gpu_box(p, f, "scalar-rb", 1e-12)
    assert 1.0 < b.poisson_form()["omega"] < 2.0
    sa = [s["iterations"] for s in a.step(2)]
    sb = [s["iterations"] for s in b.step(2)]
    assert all(x * 3 <= y for x, y in zip(sb, sa)), (sa, sb)
    fa, fb = a.download_fields(), b.download_fields()
    for k in ("p", "u", "v", "w"):
        assert rel_err(fb[k], fa[k]) <= 1e-8, k
    for k in ("phi", "rho"):
        assert rel_err(fb[k], fa[k]) <= 1e-12, k


@pytest.mark.parametrize("periodic", [True, False], ids=["periodic_x", "slip_x"])
def test_krylov_reaches_the_kinetic_fixed_point(periodic):
    """BiCGSTAB on (I - K) h = b converges to the kinetic form's fixed point:
    both run to tight tolerances (relative change 1e-12 between checks;
    residual 1e-10, near the method's rounding floor of ~1e-11 here) and agree
    to 1e-8, the Krylov form in a fraction of the kinetic map's
    applications.  With the slip walls the singular system is inconsistent
    (the wall overwrite is not a permutation): the sweeps drift along the
    constant mode and the gauge removes it, and BiCGSTAB runs on the bordered
    system of that gauged fixed point."""
    p, f = case(periodic)
    a = gpu_box(p, f, "kinetic", 1e-12, cap=2000000)
    b = gpu_box(p, f, "krylov", 1e-10, cap=2000000)
    sa = [s["iterations"] for s in a.step(2)]
    sb = b.step(2)
    assert all(s["converged"] == 1 and s["relative_error"] < 1e-10 for s in sb)
    assert all(y["iterations"] * 4 <= x for x, y in zip(sa, sb)), (sa, [y["iterations"] for y in sb])
    fa, fb = a.download_fields(), b.download_fields()
    for k in L.FIELDS:
        assert rel_err(fb[k], fa[k]) <= 1e-8, k
    with pytest.raises(L.LBMError) as e:
        b.step_replay([100])
    assert e.value.status == 4 and "replay" in str(e.value)


@pytest.mark.parametrize("periodic", [True, False], ids=["periodic_x", "slip_x"])
@pytest.mark.parametrize("degree", [4, 8])
def test_krylov_polynomial_form_reaches_the_same_fixed_point(degree, periodic):
    """BiCGSTAB on the polynomially preconditioned system (I - K^m) h =
    (I + ... + K^(m-1)) b (lbm_poisson_accel.krylov_degree = m) reaches the
    kinetic form's fixed point as the plain system does (fields within 1e-8
    of the kinetic form run to 1e-12); with the slip walls the bordered
    system's drift column is m times the sweeps' drift and h the same."""
    p, f = case(periodic)
    a = gpu_box(p, f, "kinetic", 1e-12, cap=2000000)
    b = gpu_box(p, f, "krylov", 1e-10, cap=2000000)
    b.set_poisson_accel(krylov_degree=degree)
    a.step(2)
    sb = b.step(2)
    assert all(s["converged"] == 1 for s in sb)
    fa, fb = a.download_fields(), b.download_fields()
    for k in L.FIELDS:
        assert rel_err(fb[k], fa[k]) <= 1e-8, k
    with pytest.raises(L.LBMError) as e:
        b.set_poisson_accel(krylov_degree=17)
    assert e.value.status == 4


def test_accelerators_through_python():
    """lbm_set_poisson_accel from Python: the one-pass form with every
    accelerator converges; the kinetic form refuses the one-pass-only
    settings at the next step; invalid values are refused by the setter and
    leave the settings unchanged."""
    p, f = case(True)
    g = gpu_box(p, f, "onepass", 1e-3)
    g.set_poisson_accel(anderson_m1=1, two_grid=1, spatial_diagnostics=1, source_aware_init=1,
                        fixed_point_relax=0.9)
    st = g.step(2)
    assert all(s["converged"] == 1 for s in st)
    k = gpu_box(p, f, "kinetic", 1e-3)
    k.set_poisson_accel(anderson_m1=1)
    with pytest.raises(L.LBMError) as e:
        k.step(1)
    assert e.value.status == 4 and "one-pass" in str(e.value)
    k.set_poisson_accel(anderson_m1=0, two_grid=1)
    assert k.step(1)[0]["converged"] == 1
    with pytest.raises(L.LBMError) as e:
        k.set_poisson_accel(fixed_point_relax=-1.0)
    assert e.value.status == 4


def test_scalar_form_rejections():
    p, f = case(True)
    m = L.InamuroCUDA(p, f, precision="mixed")
    with pytest.raises(L.LBMError) as e:
        m.set_poisson_form("scalar")
    assert e.value.status == 4
    p2, f2 = laplace_case((16, 11, 10), DD=6.0)
    g = L.InamuroCUDA(p2, f2, precision="fp64")
    with pytest.raises(L.LBMError) as e:
        g.set_poisson_form("scalar-rb")
    assert e.value.status == 4 and "even" in str(e.value)
    g2 = L.InamuroCUDA(p, f, precision="fp64")
    g2.set_poisson(dual=True)
    g2.set_poisson_form("scalar")
    with pytest.raises(L.LBMError) as e:
        g2.step(1)
    assert e.value.status == 4 and "kinetic" in str(e.value)


PARAMS = """16 32 32
1
3
1
50.0 1.0
1.0 1.0
0.008 0.00016
0.5 0.0005
0.035
1.0
6.7
0.09714 0.01134
0.092 0.015
8.0
"""


def tecplot_points(path, n):
    raw = open(path, "rb").read()
    data = np.frombuffer(raw[len(raw) - 36 * n:], dtype=np.dtype([("xyz", "<i4", 3), ("val", "<f4", 6)]))
    return data["xyz"], data["val"]


def final_counts(path):
    finals = {}
    for r in csv.DictReader(open(path)):
        if r["converged"] == "1":
            finals[int(r["step"])] = int(r["iteration"])
    return finals


def run_program(exe, d, pf, flags):
    d.mkdir()
    args = [exe, "--mode", "gpu", "--params", str(pf), "--steps", "3", "--write-output", "--output-steps",
            "3", "--no-roofline", "--poisson-diagnostics", "diag.csv"] + flags
    r = subprocess.run(args, cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (exe, r.stdout[-2000:] + r.stderr[-2000:])
    return d


@pytest.mark.skipif(not (os.path.exists(GPU_REF) and os.path.exists(DROPIN)),
                    reason="reference GPU program or drop-in CLI not built (needs the reference sources)")
@pytest.mark.parametrize("flags", [["--poisson", "split"],
                                   ["--poisson", "fused", "--pressure-boundary", "fused"],
                                   ["--poisson", "split", "--source-aware-hh-init", "--source-aware-hh-scale", "0.5"],
                                   ["--poisson", "onepass"],
                                   ["--poisson", "onepass", "--poisson-fixed-point-relax", "0.8"],
                                   ["--poisson", "onepass", "--pressure-relax-scale", "0.9"],
                                   ["--poisson", "onepass", "--source-aware-hh-init"],
                                   ["--poisson", "onepass", "--poisson-anderson-m1"],
                                   ["--poisson", "onepass", "--poisson-two-grid-correction",
                                    "--poisson-two-grid-strength", "0.5"],
                                   ["--poisson", "split", "--poisson-two-grid-correction"],
                                   ["--poisson", "split", "--poisson-spatial-diagnostics"],
                                   ["--poisson", "onepass", "--poisson-spatial-diagnostics",
                                    "--poisson-two-grid-correction"]])
def test_reference_gpu_program_matches_dropin(tmp_path, flags):
    pf = tmp_path / "params.in"
    pf.write_text(PARAMS)
    outs = {name: run_program(exe, tmp_path / name, pf, flags) for name, exe in (("ref", GPU_REF), ("ours", DROPIN))}
    n = 16 * 32 * 32
    xr, vr = tecplot_points(outs["ref"] / "out" / "3D000000003.plt", n)
    xo, vo = tecplot_points(outs["ours"] / "out" / "3D000000003.plt", n)
    assert np.array_equal(xr, xo)
    for j, name in enumerate(("u", "v", "w", "rho", "fei", "press")):
        scale = float(np.max(np.abs(vr[:, j])))
        err = float(np.max(np.abs(vo[:, j].astype(np.float64) - vr[:, j])))
        assert err <= 2e-6 * max(scale, 1e-30), (name, err, scale)
    assert final_counts(outs["ours"] / "diag.csv") == final_counts(outs["ref"] / "diag.csv")
    # the spatial columns of every check row (block fraction to 1e-9: the
    # reference sums its blocks with atomicAdd)
    ref_rows = list(csv.DictReader(open(outs["ref"] / "diag.csv")))
    our_rows = list(csv.DictReader(open(outs["ours"] / "diag.csv")))
    assert len(ref_rows) == len(our_rows)
    for a, b in zip(ref_rows, our_rows):
        assert (a["block_size"], a["block_count"]) == (b["block_size"], b["block_count"])
        fa, fb = a["block_low_frequency_fraction"], b["block_low_frequency_fraction"]
        assert (fa == "") == (fb == "")
        if fa:
            assert abs(float(fa) - float(fb)) <= 1e-9 * max(abs(float(fa)), 1e-300), (a["iteration"], fa, fb)


@pytest.mark.skipif(not os.path.exists(GPU_REF), reason="reference GPU program not built (needs the reference sources)")
def test_reference_scalar_option_keeps_its_start_pressure(tmp_path):
    pf = tmp_path / "params.in"
    pf.write_text(PARAMS)
    d = run_program(GPU_REF, tmp_path / "ref", pf, ["--poisson", "scalar"])
    _, v = tecplot_points(d / "out" / "3D000000003.plt", 16 * 32 * 32)
    assert np.all(v[:, 5] == 0.0)
    assert final_counts(d / "diag.csv") == {1: 100, 2: 100, 3: 100}


def varcoef_residual_np(pv, rho, s, periodic):
    """numpy restatement of the variable-coefficient operator of the
    "varcoef-rb" form: r = A p - (s - mean_W s), A p = 6 sum_q E_q k_q
    (p(x + c_q) - p(x)), k_q the mean of 1/rho at x and x + c_q, x mirrored at
    slip walls (x = -1 -> 1, x = lx -> lx - 2), y and z periodic; W = 1/2 on
    the wall planes.  Arrays (lz, ly, lx).  Returns (r, W)."""
    lz, ly, lx = pv.shape
    xs = np.arange(lx)

    def shift(a, cx, cy, cz):
        ix = xs + cx
        if periodic:
            ix %= lx
        else:
            ix = np.where(ix < 0, 1, np.where(ix >= lx, lx - 2, ix))
        a = a[:, :, ix]
        return np.roll(np.roll(a, -cy, axis=1), -cz, axis=0)

    W = np.ones_like(pv)
    if not periodic:
        W[:, :, 0] = W[:, :, -1] = 0.5
    rhs = s - np.sum(W * s) / np.sum(W)
    inv = 1.0 / rho
    ap = np.zeros_like(pv)
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    dirs += [(a, b, c) for a in (1, -1) for b in (1, -1) for c in (1, -1)]
    for cx_, cy_, cz_ in dirs:
        e = 1.0 / 9.0 if abs(cx_) + abs(cy_) + abs(cz_) == 1 else 1.0 / 72.0
        k = 0.5 * (inv + shift(inv, cx_, cy_, cz_))
        ap += 6.0 * e * k * (shift(pv, cx_, cy_, cz_) - pv)
    return ap - rhs, W, rhs


@pytest.mark.parametrize("periodic", [False, True])
def test_varcoef_rb_solves_its_equation(periodic):
    """The variable-coefficient red-black form solves div((1/rho) grad p) = s
    on the step's own source (the oracle's projected source of the same
    collision) to its residual tolerance, p gauged to the step's target."""
    p, f = case(periodic)
    f["u"] = 0.01 * np.sin(2 * np.pi * np.arange(SHAPE[0]) / SHAPE[0])[None, None, :] * np.ones_like(f["u"])
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, tol=1e-12, max_sweeps=400000, periodic_x=periodic)
    o.step()
    d = o.derivatives()   # u_x (mean-projected) at 6, v_y at 10, w_z at 14
    s = d[6] + d[10] + d[14]
    rho_o = o.fields()["rho"]
    g = gpu_box(p, f, "varcoef-rb", 1e-12)
    st = g.step(1)[0]
    assert st["converged"] == 1 and st["fixed_point_evaluated"] == 1
    assert st["fixed_point_h_relative"] < 1e-12
    got = g.download_fields()
    assert rel_err(got["rho"], rho_o) <= 1e-13
    r, W, rhs = varcoef_residual_np(got["p"], got["rho"], s, periodic)
    assert float(np.sum(W * np.abs(r))) <= 1e-10 * float(np.sum(W * np.abs(rhs)))
    assert abs(float(np.mean(got["p"])) - float(np.mean(f["p"]))) <= 1e-12
    g.close()


@pytest.mark.parametrize("periodic", [False, True])
def test_varcoef_rb_error_against_kinetic_fixed_point(periodic, capsys):
    """Reported, not claimed: the variable-coefficient scalar form against the
    kinetic form's fixed point (both converged to 1e-12 from the same state,
    one step).  The test records the errors in p and u and checks only that
    the form tracks the kinetic solution's scale (error below 1)."""
    p, f = case(periodic)
    f["u"] = 0.01 * np.sin(2 * np.pi * np.arange(SHAPE[0]) / SHAPE[0])[None, None, :] * np.ones_like(f["u"])
    out = {}
    for form in ("kinetic", "varcoef-rb"):
        g = gpu_box(p, f, form, 1e-12)
        g.step(1)
        out[form] = g.download_fields()
        g.close()
    errs = {k: rel_err(out["varcoef-rb"][k], out["kinetic"][k]) for k in ("p", "u", "v", "w")}
    with capsys.disabled():
        print(f"\nvarcoef-rb vs kinetic fixed point (periodic_x={int(periodic)}): " +
              ", ".join(f"{k} {v:.3e}" for k, v in errs.items()))
    assert all(np.isfinite(v) and v < 1.0 for v in errs.values()), errs

"""FP64 CUDA path (through the C ABI) against the oracle and the reference.

Tolerances: the FP64 kernels keep the reference's per-cell operation order
without FMA, so fields differ from the reference only through sin() and the
order of the global sums; the bar is 1e-10 norm-wise relative error
(max|gpu - ref| / max|ref|) per field and identical per-step sweep counts.
"""
import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import fixture, fields_dict, laplace_case, oracle_params, params_from_text, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


# Every solve in this file is capped (60000 sweeps, a multiple of every check
# interval used) so that a case that never meets its exit test fails instead of
# looping: the reference's own loop is unbounded.
CAP = 60000


def solver(p, f=None):
    g = L.InamuroCUDA(p, f)
    g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    return g


def run_pair(p, f, steps, dual=False, check_interval=100, tol=1e-3, replay=None):
    g = solver(p, f)
    g.set_poisson(check_interval=check_interval, tolerance=tol, dual=dual, max_sweeps=CAP,
                  fail_on_limit=True)
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, check_interval=check_interval, tol=tol, dual=dual,
                        max_sweeps=CAP)
    out = []
    for s in range(steps):
        if replay is None:
            gs = g.step(1)[0]
            os_ = o.step()
        else:
            gs = g.step_replay([replay[s]])[0]
            os_ = o.step(replay=replay[s])
        out.append((gs, os_, g.download_fields(), o.fields()))
    g.close()
    return out


def assert_fields_close(gf, of, tol=TOL, what=""):
    for k in L.FIELDS:
        e = rel_err(gf[k], of[k])
        assert e <= tol, f"{what} {k}: rel err {e:.3e}"


@pytest.mark.parametrize("name", ["step_single_tanh", "step_two_sharp", "step_example_16x32x32"])
def test_fp64_matches_reference_fixture(name):
    fx = fixture(name)
    p = params_from_text(fx["params_text"])
    g = solver(p, fields_dict(fx["init"]))
    for s in range(len(fx["sweeps"])):
        st = g.perform_time_step_gpu()
        assert st["iterations"] == fx["sweeps"][s], f"step {s + 1}"
        assert st["converged"] == 1
        gf = g.download_fields()
        if "fields" in fx.files:
            ref = fields_dict(fx["fields"][s])
        else:
            ref = None
        for i, k in enumerate(L.FIELDS):
            got = gf[k].reshape(-1)[fx["sample_index"]]
            want = fx["samples"][s, i]
            scale = max(np.max(np.abs(want)), 1e-300)
            assert np.max(np.abs(got - want)) / scale <= TOL, (k, s)
            if ref is not None:
                assert rel_err(gf[k], ref[k]) <= TOL, (k, s)
        assert abs(st["mass"] - fx["mass"][s]) <= 1e-11 * abs(fx["mass"][s])
    g.close()


def test_fp64_first_step_near_bitwise():
    """One step on a tiny non-cubic box: per-cell arithmetic is the
    reference's, so agreement is at rounding level."""
    fx = fixture("step_single_tanh")
    p = params_from_text(fx["params_text"])
    (gs, os_, gf, of), = run_pair(p, fields_dict(fx["init"]), 1)
    assert gs["iterations"] == os_["sweeps"]
    assert_fields_close(gf, of, tol=1e-13, what="step1")


def test_fp64_laplace_32_sweep_counts_and_fields():
    """Laplace static droplet, 32^3, the reference's own 100/4200 sweeps."""
    fx = fixture("step_laplace_32")
    p = params_from_text(fx["params_text"])
    res = run_pair(p, fields_dict(fx["init"]), 2)
    for s, (gs, os_, gf, of) in enumerate(res):
        assert gs["iterations"] == fx["sweeps"][s] == os_["sweeps"]
        assert_fields_close(gf, of, what=f"step{s + 1}")


@pytest.mark.parametrize("shape,ci", [((9, 7, 5), 100), ((20, 6, 11), 3), ((16, 16, 4), 50)])
def test_fp64_odd_shapes_and_check_intervals(shape, ci):
    p, f = laplace_case(shape, DD=4.0, noise=1e-4, seed=shape[0])
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(shape[2]) / shape[2])[:, None, None] * np.ones_like(f["w"])
    for gs, os_, gf, of in run_pair(p, f, 3, check_interval=ci):
        assert gs["iterations"] == os_["sweeps"]
        assert_fields_close(gf, of)


@pytest.mark.parametrize("ci", [100, 4, 3, 2])
def test_fp64_dual_residual_matches_oracle(ci):
    """Dual exit: relative change AND kinetic fixed-point residual < tol."""
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    for gs, os_, gf, of in run_pair(p, fields_dict(fx["init"]), 2, dual=True, check_interval=ci):
        assert gs["iterations"] == os_["sweeps"]
        assert gs["fixed_point_evaluated"] == 1 and gs["converged"] == 1
        assert abs(gs["fixed_point_relative"] - os_["fp_rel"]) <= 1e-8 * abs(os_["fp_rel"])
        assert abs(gs["relative_error"] - os_["relative_error"]) <= 1e-8 * abs(os_["relative_error"])
        assert_fields_close(gf, of)


def test_fp64_dual_residual_floor_matches_oracle():
    """Step 3 of the two-drop case never meets the dual exit: the kinetic
    fixed-point residual stalls at 1.066e-3 (an undamped period-2 parity mode
    of the D3Q15 stream) while the pressure has stopped changing.  Replayed for
    2000 sweeps, both implementations report the same floor."""
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    res = run_pair(p, fields_dict(fx["init"]), 3, dual=True, replay=[500, 500, 2000])
    gs, os_, gf, of = res[-1]
    assert 1.0e-3 < os_["fp_rel"] < 1.1e-3
    assert abs(gs["fixed_point_relative"] - os_["fp_rel"]) <= 1e-8 * os_["fp_rel"]
    assert gs["pressure_converged"] == 1 and gs["fixed_point_converged"] == 0
    assert_fields_close(gf, of)


def test_fp64_replay_forces_counts():
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    replay = [200, 700, 300]
    for s, (gs, os_, gf, of) in enumerate(run_pair(p, fields_dict(fx["init"]), 3, replay=replay)):
        assert gs["iterations"] == replay[s] == os_["sweeps"]
        assert_fields_close(gf, of)


def test_ghosted_layout_roundtrip():
    p, f = laplace_case((8, 6, 5), DD=3.0)
    g = solver(p)
    gh = {}
    rng = np.random.default_rng(3)
    for k in L.FIELDS:
        a = rng.normal(size=(p.lz + 2, p.ly, p.lx))
        a[1:-1] = f[k]
        gh[k] = a
    g.load_fields_ghosted(gh)
    for k in L.FIELDS:
        assert np.array_equal(g.download_ghosted(k), gh[k])
    g.step(1)
    o = pyoracle.Oracle(p.shape, oracle_params(p), f)
    o.step()
    of = o.fields()
    for k in L.FIELDS:
        out = g.download_ghosted(k)
        assert np.array_equal(out[0], gh[k][0]) and np.array_equal(out[-1], gh[k][-1])
        assert rel_err(out[1:-1], of[k]) <= TOL


def test_download_hh_is_E_times_p():
    p, f = laplace_case((8, 6, 5), DD=3.0)
    g = solver(p, f)
    assert np.all(g.download_hh() == 0.0)
    g.step(1)
    hh = g.download_hh().reshape(-1, 15)
    pp = g.download("p").reshape(-1)
    E = np.array([2 / 9] + [1 / 9] * 6 + [1 / 72] * 8)
    assert np.array_equal(hh, pp[:, None] * E[None, :])


def test_nonfinite_source_is_an_error_and_handle_recovers():
    p, f = laplace_case((8, 6, 5), DD=3.0)
    bad = {k: v.copy() for k, v in f.items()}
    bad["u"][2, 3, 4] = np.nan
    g = solver(p, bad)
    with pytest.raises(L.LBMError) as e:
        g.step(1)
    assert e.value.status == 2 and "source" in str(e.value)
    g.load_fields(f)
    st = g.step(1)[0]
    assert st["converged"] == 1


def test_iteration_limit_fallback_and_budget_error():
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    g = solver(p, fields_dict(fx["init"]))
    g.set_poisson(check_interval=100, tolerance=1e-12, max_sweeps=300)
    st = g.step(1)[0]
    assert st["iterations"] == 300 and st["converged"] == 0
    g.set_poisson(check_interval=100, tolerance=1e-12, max_sweeps=300, fail_on_limit=True)
    with pytest.raises(L.LBMError) as e:
        g.step(1)
    assert e.value.status == 3
    with pytest.raises(L.LBMError) as e2:
        g.set_poisson(check_interval=100, tolerance=1e-3, max_sweeps=250)
    assert e2.value.status == 4


def test_deterministic_repeat():
    """Fixed-order reductions: two runs are bitwise identical."""
    p, f = laplace_case((24, 20, 16), DD=8.0, noise=1e-4)
    outs = []
    for _ in range(2):
        g = solver(p, f)
        st = g.step(2)
        outs.append((g.download_fields(), [s["iterations"] for s in st]))
        g.close()
    assert outs[0][1] == outs[1][1]
    for k in L.FIELDS:
        assert np.array_equal(outs[0][0][k], outs[1][0][k])


def test_full_size_256_translation_and_mirror():
    """256^3, two drops (R = 32, 96 cells apart, rho ratio 100).  (a) With the
    +-0.02 approach velocity, a z shift of the initial condition shifts the
    result (periodic z) up to the rounding of reordered global sums.  (b) For
    resting drops the state is mirror-symmetric about the mid plane z = 128:
    phi even, w odd, to rounding."""
    n = 256
    p = L.make_params(lx=n, ly=n, lz=n, rho_L=100.0, rho_G=1.0, mu_L=10.0, mu_G=0.1, k_f=0.06,
                      k_g=6e-6, DD=64.0, init_tanh=1, interface_width=2.0, init_velocity=0.02,
                      init_center_x=128.0, init_separation=48.0)
    f = L.init_droplets(p)
    g = solver(p, f)
    st = g.step(1)[0]
    a = g.download_fields()
    shifted = {k: np.roll(v, 7, axis=0) for k, v in f.items()}
    g.load_fields(shifted)
    st2 = g.step(1)[0]
    b = g.download_fields()
    assert st["iterations"] == st2["iterations"]
    for k in L.FIELDS:
        assert rel_err(np.roll(a[k], 7, axis=0), b[k]) <= 1e-11, k
    rest = dict(f)
    rest["w"] = np.zeros_like(f["w"])
    g.load_fields(rest)
    g.step(2)
    c = g.download_fields()
    g.close()
    # plane k <-> plane 256 - k (planes 1..255; plane 0 and 128 map to themselves)
    assert rel_err(c["phi"][1:][::-1], c["phi"][1:]) <= 1e-11
    assert rel_err(-c["w"][1:][::-1], c["w"][1:]) <= 1e-9
    assert np.max(np.abs(c["w"])) > 0.0


@pytest.mark.parametrize("zlen,periodic", [("32", 0), ("7", 0), ("32", 1)])
def test_fp64_two_sweep_pass_is_bitwise(zlen, periodic, monkeypatch):
    """The FP64 temporally blocked pass (two sweeps per launch) keeps every
    cell's arithmetic, so it reproduces single-sweep launches bit for bit
    (slip walls and periodic x)."""
    p, f = laplace_case((64, 16, 20), DD=8.0, noise=1e-4)
    p.periodic_x = periodic
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(20) / 20)[:, None, None] * np.ones_like(f["w"])
    monkeypatch.setenv("LBM_SWEEP2_ZLEN", "0")
    a = solver(p, f)
    monkeypatch.setenv("LBM_SWEEP2_ZLEN", zlen)
    b = solver(p, f)
    for _ in range(3):
        assert a.step(1)[0]["iterations"] == b.step(1)[0]["iterations"]
    fa, fb = a.download_fields(), b.download_fields()
    for k in L.FIELDS:
        assert np.array_equal(fa[k], fb[k]), k
    assert b.timing()["kernel_launches"] < a.timing()["kernel_launches"]


@pytest.mark.parametrize("zlen,minb,periodic", [("16", "2", 0), ("5", "1", 0), ("1", "2", 0), ("16", "2", 1)])
def test_fp64_zmarch_collide_matches_plane_collide(zlen, minb, periodic, monkeypatch):
    """The z-marching FP64 collide (macro fields staged in a shared-memory
    plane ring) evaluates every cell with the same operations as the plane
    collide: phi and rho after the first step are bitwise equal; later steps
    differ only through the order of the source sum (FP64 rounding).  z runs
    that do not divide the box (5), single-plane runs (1), both register
    budgets and periodic x are covered."""
    p, f = laplace_case((64, 40, 24), DD=12.0, noise=1e-4)
    p.periodic_x = periodic
    f["u"] = 0.005 * np.cos(2 * np.pi * np.arange(40) / 40)[None, :, None] * np.ones_like(f["u"])
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[:, None, None] * np.ones_like(f["w"])
    monkeypatch.setenv("LBM_COLLIDE_ZLEN", "0")
    a = L.InamuroCUDA(p, f)
    monkeypatch.setenv("LBM_COLLIDE_ZLEN", zlen)
    monkeypatch.setenv("LBM_COLLIDE_MINB", minb)
    b = L.InamuroCUDA(p, f)
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
        assert rel_err(fb[k], fa[k]) <= 1e-12, k


def test_fp64_periodic_x_matches_periodic_oracle_and_conserves_mass():
    """Periodic x (not a reference mode; the configs' periodic boxes): the FP64
    box against the oracle run with periodic x (same sweep counts, fields to
    1e-10), and the phi sum conserved to 1e-12 relative over the steps (with
    the reference's slip walls the scheme itself does not conserve it)."""
    p, f = laplace_case((32, 24, 16), DD=8.0, noise=1e-4)
    p.periodic_x = 1
    f["u"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[None, :, None] * np.ones_like(f["u"])
    f["v"] = 0.01 * np.cos(2 * np.pi * np.arange(32) / 32)[None, None, :] * np.ones_like(f["v"])
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, max_sweeps=CAP, periodic_x=True)
    g = solver(p, f)
    masses = []
    for _ in range(3):
        info = o.step()
        st = g.step(1)[0]
        assert st["iterations"] == info["sweeps"]
        masses.append(st["mass"])
    gf, of = g.download_fields(), o.fields()
    for k in L.FIELDS:
        assert rel_err(gf[k], of[k]) <= 1e-10, k
    assert max(abs(m - masses[0]) for m in masses) <= 1e-12 * abs(masses[0])


def test_exact_division_matches_ieee_division():
    """The FP64 Poisson kernels take their 15 quotients by tau_h per cell from
    one reciprocal (two Markstein remainder corrections, exact_div.cuh).
    Against CUDA's IEEE division on 2^32 pseudo-random operand pairs
    (relaxation times, densities, stencil constants and arbitrary normal
    divisors) every quotient must be bit-identical."""
    assert L.selftest_division(1 << 32, seed=20261203) == 0

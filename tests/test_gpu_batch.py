"""Batched boxes (lbm_batch_*): many uneven mixed-precision boxes advanced
together.  Each instance must step exactly as the same box alone: the batch
evaluates every cell with the single box's cell functions, so after the first
step (no reductions involved) phi and rho are bitwise equal to a single-box
run with the plane kernels, and later steps differ only through the order of
the FP64 sums (tolerance 1e-6; 1e-5 for the small zero-mean p).  Natural exits give each instance its own
sweep count, equal to the single box's; against the FP64 oracle each instance
meets the mixed bar (1e-5)."""
import numpy as np
import pytest

import bench
import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import laplace_case, oracle_params, rel_err

pytestmark = pytest.mark.gpu
CAP = 60000


def uneven_cases():
    """Five boxes of different shapes and physics; lx = 40 and 24 leave
    partial CTA tiles in x, lz = 5 a partial z run."""
    shapes = [(40, 32, 24), (32, 48, 16), (24, 16, 40), (64, 24, 5), (16, 40, 32)]
    cases = []
    for k, shp in enumerate(shapes):
        p, f = laplace_case(shp, DD=min(shp) * 0.5, noise=1e-4, seed=k + 1,
                            rho=(20.0 * (k + 1), 1.0), kappa=(0.03 + 0.015 * k, 6e-6))
        f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(shp[2]) / shp[2])[:, None, None] * np.ones_like(f["w"])
        cases.append((p, f))
    return cases


def single(p, f, monkeypatch):
    monkeypatch.setenv("LBM_COLLIDE_ZLEN", "0")
    monkeypatch.setenv("LBM_SWEEP2_ZLEN", "0")
    g = L.InamuroCUDA(p, f, precision="mixed")
    g.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    return g


def test_batch_matches_single_boxes_replayed(monkeypatch):
    cases = uneven_cases()
    b = L.Batch([p for p, _ in cases], [f for _, f in cases])
    b.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    singles = [single(p, f, monkeypatch) for p, f in cases]
    counts = [300, 200, 400, 100, 300]
    stats = b.step_replay([counts])[0]
    for i, g in enumerate(singles):
        st = g.step_replay([counts[i]])[0]
        assert stats[i]["iterations"] == counts[i] == st["iterations"]
        assert np.array_equal(b.download(i, "phi"), g.download("phi")), i
        assert np.array_equal(b.download(i, "rho"), g.download("rho")), i
        assert abs(stats[i]["mass"] - st["mass"]) <= 1e-12 * abs(st["mass"])
    for _ in range(2):
        b.step_replay([counts])
        for i, g in enumerate(singles):
            g.step_replay([counts[i]])
    for i, g in enumerate(singles):
        fb, fs = b.download_fields(i), g.download_fields()
        for k in L.FIELDS:
            assert rel_err(fb[k], fs[k]) <= (1e-5 if k == "p" else 1e-6), (i, k)


def test_batch_natural_exit_per_instance(monkeypatch):
    cases = uneven_cases()[:3]
    b = L.Batch([p for p, _ in cases], [f for _, f in cases])
    b.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    singles = [single(p, f, monkeypatch) for p, f in cases]
    total = 0
    for _ in range(2):
        stats = b.step(1)[0]
        for i, g in enumerate(singles):
            st = g.step(1)[0]
            assert stats[i]["iterations"] == st["iterations"], i
            assert stats[i]["converged"] == 1
        total += sum(s["iterations"] for s in stats)
    its = [s["iterations"] for s in stats]
    assert len(set(its)) > 1, "instances should leave the Poisson loop at different checks"
    t = b.timing()
    assert t["steps"] == 2 and t["sweeps"] == total


def test_batch_against_fp64_oracle():
    cases = uneven_cases()[1:3]
    b = L.Batch([p for p, _ in cases], [f for _, f in cases])
    b.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    oracles = [pyoracle.Oracle(p.shape, oracle_params(p), f, max_sweeps=CAP) for p, f in cases]
    for _ in range(2):
        infos = [o.step() for o in oracles]
        b.step_replay([[int(x["sweeps"]) for x in infos]])
    for i, o in enumerate(oracles):
        of, gf = o.fields(), b.download_fields(i)
        for k in ("phi", "rho", "u", "v", "w"):
            assert rel_err(gf[k], of[k]) <= 1e-5, (i, k)
        assert rel_err(gf["p"], of["p"]) <= 1e-4, i


def test_batch_tuning_changes_no_result():
    cases = uneven_cases()
    ps, fs = [p for p, _ in cases], [f for _, f in cases]
    a = L.Batch(ps, fs)
    b = L.Batch(ps, fs)
    for x in (a, b):
        x.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    chosen = b.tune()
    assert (chosen["tile_x"], chosen["tile_y"]) in ((32, 8), (16, 16), (8, 32))
    assert chosen["zrun"] in (1, 2, 4, 8) and chosen["ctas_per_sm"] in (2, 4, 8) and chosen["sweep_ms"] > 0
    assert chosen["sweep2_zrun"] in (0, 8, 16, 32)
    assert b.tuning()["zrun"] == chosen["zrun"]
    counts = [[200] * len(ps)] * 2
    a.step_replay(counts)
    b.step_replay(counts)
    for i in range(len(ps)):
        assert np.array_equal(a.download(i, "phi"), b.download(i, "phi")) or \
            rel_err(b.download(i, "phi"), a.download(i, "phi")) <= 1e-6
        assert rel_err(b.download(i, "p"), a.download(i, "p")) <= 1e-5


def test_batch_sweep_cap_is_reported():
    cases = uneven_cases()[:2]
    b = L.Batch([p for p, _ in cases], [f for _, f in cases])
    b.set_poisson(max_sweeps=100, fail_on_limit=True)
    with pytest.raises(L.LBMError) as e:
        b.step(1)
    assert e.value.status == 3 and "limit" in str(e.value)


def test_batch_workload_steps_and_conserves_mass():
    """Eight instances of the batched droplet-oscillation workload (periodic
    boxes) step with natural exits; every instance converges and keeps its
    mass (phi sum) to 1e-12 of the loaded phi's FP64 sum: the rest population
    is kept in FP64 as phi minus the stored moving populations, and the
    stream only permutes the stored FP32 values."""
    params, fields = bench.batch_workload(8, seed=11)
    assert all(p.periodic_x == 1 for p in params)
    b = L.Batch(params, fields)
    b.set_poisson(max_sweeps=CAP, fail_on_limit=True)
    s1 = b.step(1)[0]
    s3 = b.step(2)[-1]
    for i, (a, c) in enumerate(zip(s1, s3)):
        m0 = float(np.sum(fields[i]["phi"]))
        assert a["converged"] == 1 and c["converged"] == 1
        assert abs(a["mass"] - m0) <= 1e-12 * abs(m0)
        assert abs(c["mass"] - m0) <= 1e-12 * abs(m0)


@pytest.mark.parametrize("zrun2", [8, 3])
def test_batch_two_sweep_pass_matches_single_sweeps(zrun2):
    """Two plain sweeps per launch (temporal blocking on 16 x 8 tiles, any box
    side: partial x and z tiles included) evaluate every cell as single sweeps
    do, so the instances' fields are bitwise equal."""
    cases = uneven_cases()
    ps, fs = [p for p, _ in cases], [f for _, f in cases]
    a = L.Batch(ps, fs)
    b = L.Batch(ps, fs)
    a.set_tuning(32, 8, 4, 4, 0)
    b.set_tuning(32, 8, 4, 4, zrun2)
    counts = [[300, 200, 400, 100, 300]] * 2
    for x in (a, b):
        x.set_poisson(max_sweeps=CAP, fail_on_limit=True)
        x.step_replay(counts)
    for i in range(len(ps)):
        fa, fb = a.download_fields(i), b.download_fields(i)
        for k in L.FIELDS:
            assert np.array_equal(fa[k], fb[k]), (i, k)
    assert b.timing()["fused_sweeps"] > 0 and a.timing()["fused_sweeps"] == 0

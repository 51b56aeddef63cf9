"""Drop-in check with the reference's own front end.

oracle/_ref/lbm_gpu_dropin is the reference's GPU/main.cpp and GPU/Inamuro.cpp,
compiled unchanged against include/InamuroCUDA.hpp (this library's drop-in
InamuroCUDA) by oracle/Makefile.  Its --mode gpu runs this library, its
--mode cpu the reference's own CPU solver; both write the reference's Tecplot
output (float32 fields), which must agree to float32 rounding, and the GPU
run's per-check diagnostics CSV must show the oracle's sweep counts."""
import csv
import os
import subprocess

import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import oracle_params

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "lbm_gpu_dropin")

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
    """The last n points of a Tecplot file written by Inamuro::writeTecplotBinary:
    per point 3 int32 coordinates then u, v, w, rho, fei, press as float32."""
    raw = open(path, "rb").read()
    data = np.frombuffer(raw[len(raw) - 36 * n:], dtype=np.dtype([("xyz", "<i4", 3), ("val", "<f4", 6)]))
    return data["xyz"], data["val"]


def run(args, cwd):
    r = subprocess.run([DROPIN] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in CLI not built (needs the reference sources)")
def test_reference_main_gpu_mode_matches_its_cpu_mode(tmp_path):
    pf = tmp_path / "params.in"
    pf.write_text(PARAMS)
    gdir, cdir = tmp_path / "gpu", tmp_path / "cpu"
    gdir.mkdir()
    cdir.mkdir()
    common = ["--params", str(pf), "--steps", "3", "--write-output", "--output-steps", "3", "--no-roofline"]
    out_g = run(["--mode", "gpu", "--poisson-diagnostics", "diag.csv"] + common, gdir)
    assert "GPU wall_total_ms=" in out_g
    run(["--mode", "cpu"] + common, cdir)
    n = 16 * 32 * 32
    xg, vg = tecplot_points(gdir / "out" / "3D000000003.plt", n)
    xc, vc = tecplot_points(cdir / "out" / "3D000000003.plt", n)
    assert np.array_equal(xg, xc)
    for j, name in enumerate(("u", "v", "w", "rho", "fei", "press")):
        scale = float(np.max(np.abs(vc[:, j])))
        err = float(np.max(np.abs(vg[:, j].astype(np.float64) - vc[:, j])))
        assert err <= 2e-6 * scale, (name, err, scale)
    # per-check CSV rows: the converged row of each step carries the oracle's count
    rows = list(csv.DictReader(open(gdir / "diag.csv")))
    finals = {}
    for r in rows:
        if r["converged"] == "1":
            finals[int(r["step"])] = int(r["iteration"])
    p = L.params_load(str(pf))
    o = pyoracle.Oracle(p.shape, oracle_params(p), L.init_droplets(p))
    for s in (1, 2, 3):
        assert finals[s] == o.step()["sweeps"], s
    # every check of a step appears, in order
    by_step = [int(r["iteration"]) for r in rows if r["step"] == "1"]
    assert by_step == list(range(100, finals[1] + 1, 100))


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in CLI not built (needs the reference sources)")
def test_reference_main_production_flags(tmp_path):
    """The reference's `make run` flag set (GPU/Makefile:25-29) is accepted and
    the dual exit is reported in its CSV."""
    pf = tmp_path / "params.in"
    pf.write_text(PARAMS)
    run(["--mode", "gpu", "--params", str(pf), "--steps", "2", "--poisson", "split",
         "--pressure-boundary", "split", "--poisson-dual-residual", "--poisson-deterministic-reductions",
         "--poisson-check-interval", "100", "--poisson-tolerance", "1e-3", "--poisson-iteration-limit", "0",
         "--no-roofline", "--poisson-diagnostics", "d.csv"], tmp_path)
    rows = list(csv.DictReader(open(tmp_path / "d.csv")))
    assert rows and all(r["dual_residual_enabled"] == "1" and r["fixed_point_evaluated"] == "1" for r in rows)
    assert rows[-1]["converged"] == "1" and float(rows[-1]["fixed_point_relative"]) < 1e-3


CPU_DROPIN = os.path.join(ROOT, "oracle", "_ref", "lbm_cpu_dropin")
LBM_SIM = os.path.join(ROOT, "oracle", "_ref", "lbm_sim")
CPU_PARAMS = """16 24 16
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
enable_progress=0   # key=value switches of the CPU tree
output_dir=out/
"""


@pytest.mark.skipif(not (os.path.exists(CPU_DROPIN) and os.path.exists(LBM_SIM)),
                    reason="CPU-tree programs not built (need the reference sources)")
def test_reference_cpu_program_over_gpu_solver_matches_reference(tmp_path):
    """The reference's CPU/main.cpp and CPU/Inamuro.cpp, unchanged, over the
    drop-in InamuroSolver (GPU steps) against the reference's own CPU program
    on the same params.in: equal Tecplot fields to float32 rounding and the
    same step_diagnostics.csv (columns, sweep counts, statistics to the
    file's 11 digits)."""
    outs = {}
    for name, exe in (("gpu", CPU_DROPIN), ("cpu", LBM_SIM)):
        d = tmp_path / name
        d.mkdir()
        (d / "params.in").write_text(CPU_PARAMS)
        r = subprocess.run([exe, "params.in"], cwd=d, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        outs[name] = d / "out"
    n = 16 * 24 * 16
    for step in (0, 1, 2):
        xg, vg = tecplot_points(outs["gpu"] / f"3D{step:09d}.plt", n)
        xc, vc = tecplot_points(outs["cpu"] / f"3D{step:09d}.plt", n)
        assert np.array_equal(xg, xc)
        for j in range(6):
            scale = float(np.max(np.abs(vc[:, j])))
            assert float(np.max(np.abs(vg[:, j].astype(np.float64) - vc[:, j]))) <= 2e-6 * max(scale, 1e-30), (step, j)
    rows = {k: list(csv.reader(open(v / "step_diagnostics.csv"))) for k, v in outs.items()}
    assert rows["gpu"][0] == rows["cpu"][0]
    assert len(rows["gpu"]) == len(rows["cpu"]) == 5
    head = rows["cpu"][0]
    for rg, rc in zip(rows["gpu"][1:], rows["cpu"][1:]):
        cpu_row = dict(zip(head, rc))
        for k, name in enumerate(head):
            if name in ("step_time_ms", "pressure_solve_ms"):
                continue
            a, b = float(rg[k]), float(rc[k])
            # a mean is a sum in another order: against the field's scale (a
            # zero-mean field's mean is pure rounding)
            scale = float(cpu_row[name[:-len("mean")] + "abs_max"]) if name.endswith("_mean") else abs(b)
            assert abs(a - b) <= 1e-9 * max(scale, 1e-12), (rg[0], name, a, b)

"""Output formats.  The Tecplot binary writer (include/lbm_b200_tecplot.hpp) against the
reference's own writer (Inamuro::writeTecplotBinary, CPU/Inamuro.cpp:865-1013,
run from its sources by oracle/_ref/ref_cpu_harness): the same bytes for the
same fields.  Host only."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_harness")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference harness not built (needs the reference sources)")
@pytest.mark.parametrize("shape", [(6, 5, 4), (16, 12, 10)])
def test_tecplot_bytes_match_the_reference_writer(tmp_path, shape):
    lx, ly, lz = shape
    rng = np.random.default_rng(lx * 100 + ly)
    fields = rng.standard_normal((6, lz, ly, lx))
    fields[1] = 1.0 + np.abs(fields[1])   # rho > 0
    raw = tmp_path / "fields.bin"
    fields.tofile(raw)
    params = tmp_path / "params.in"
    params.write_text(f"{lx} {ly} {lz}\n1\n1\n1\n50.0 1.0\n1.0 1.0\n0.008 0.00016\n0.5 0.0005\n0.035\n1.0\n6.7\n"
                      "0.09714 0.01134\n0.092 0.015\n8.0\n")
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    r = subprocess.run([HARNESS, "--params", str(params), "--tecplot", str(ref_dir), "--init", str(raw)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    exe = tmp_path / "tecplot_write"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "tecplot_write.cpp"), "-o", str(exe)], check=True)
    ours = tmp_path / "ours.plt"
    subprocess.run([str(exe), str(lx), str(ly), str(lz), str(raw), str(ours)], check=True)
    want = (ref_dir / "3D000000000.plt").read_bytes()
    assert ours.read_bytes() == want


def test_poisson_csv_writer_format(tmp_path):
    """lbm_b200::PoissonCsv (include/lbm_b200_diagnostics.hpp): the reference
    GPU program's per-check CSV header (GPU/InamuroCUDA.cu:2610-2682) and rows,
    with the columns a check did not evaluate left empty."""
    exe = tmp_path / "poisson_csv"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "poisson_csv.cpp"), "-o", str(exe)], check=True)
    out = tmp_path / "p.csv"
    subprocess.run([str(exe), str(out)], check=True)
    lines = out.read_text().splitlines()
    assert lines[0].split(",") == [
        "step", "iteration", "pressure_l1_delta", "pressure_l1_norm", "relative_error",
        "fixed_point_h_l1", "fixed_point_h_scale", "fixed_point_h_relative",
        "fixed_point_p_l1", "fixed_point_p_scale", "fixed_point_p_relative",
        "fixed_point_relative", "fixed_point_evaluated", "pressure_converged", "fixed_point_converged",
        "dual_residual_enabled", "converged", "block_low_frequency_fraction", "block_size", "block_count"]
    assert lines[1] == "3,200,0.25,4,0.0625,,,,,,,,0,0,0,0,0,,0,0"
    assert lines[2] == "3,300,0.25,4,0.0625,1.5,,,,,,0.5,1,1,0,0,1,0.125,4,27"

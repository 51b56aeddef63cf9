"""Device-side step diagnostics (lbm_diagnostics_snapshot,
Inamuro::collectDiagnostics of CPU/Inamuro.cpp:412-507) and the reference's
step_diagnostics.csv format (include/lbm_b200_diagnostics.hpp,
CPU/InamuroSolver.cpp:262-334).

min, max, abs_max and the NaN/Inf/valid counts are order-independent and
must equal numpy's on the downloaded fields exactly; the mean is a sum in a
fixed device order (relative 1e-12 against numpy's pairwise sum); the
velocity magnitude may differ from numpy's sqrt(u*u + v*v + w*w) by FMA
contraction in its last bits (1e-15)."""
import os
import subprocess

import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAMES = ("rho", "fei", "u", "v", "w", "velocity_magnitude", "p")
HEADER_STATS = ("rho", "fei", "u", "v", "w", "vel_mag", "p")


def expected(fields):
    u, v, w = fields["u"], fields["v"], fields["w"]
    src = {"rho": fields["rho"], "fei": fields["phi"], "u": u, "v": v, "w": w,
           "velocity_magnitude": np.sqrt(u * u + v * v + w * w), "p": fields["p"]}
    out = {}
    for k, a in src.items():
        a = a.ravel()
        fin = a[np.isfinite(a)]
        out[k] = {"min": fin.min(), "max": fin.max(), "abs_max": np.abs(fin).max(), "mean": fin.mean(),
                  "nan_count": int(np.isnan(a).sum()), "inf_count": int(np.isinf(a).sum()), "valid_count": fin.size}
    return out


def check(got, exp, exact_tol=0.0):
    for k in NAMES:
        tol = 1e-15 if k == "velocity_magnitude" else exact_tol
        for s in ("min", "max", "abs_max"):
            assert abs(got[k][s] - exp[k][s]) <= tol * max(abs(exp[k][s]), 1e-300), (k, s)
        assert abs(got[k]["mean"] - exp[k]["mean"]) <= 1e-12 * max(exp[k]["abs_max"], 1e-300), k
        for s in ("nan_count", "inf_count", "valid_count"):
            assert got[k][s] == exp[k][s], (k, s)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_snapshot_matches_host_statistics(precision):
    p, f = laplace_case((32, 24, 16), DD=8.0, noise=1e-4)
    f["u"] = 0.01 * np.sin(2 * np.pi * np.arange(24) / 24)[None, :, None] * np.ones_like(f["u"])
    g = L.InamuroCUDA(p, f, precision=precision)
    g.set_poisson(max_sweeps=60000, fail_on_limit=True)
    g.step(2)
    check(g.diagnostics(), expected(g.download_fields()))


@pytest.mark.parametrize("precision", [0, 1])
def test_step_diagnostics_csv_has_reference_columns(tmp_path, precision):
    exe = tmp_path / "step_diag_csv"
    lib_dir = os.path.join(ROOT, "lbm_b200")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "step_diag_csv.cpp"), "-o", str(exe), "-L", lib_dir,
                    "-llbm_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    csv_path, bin_path = tmp_path / "step_diagnostics.csv", tmp_path / "fields.bin"
    r = subprocess.run([str(exe), str(csv_path), str(bin_path), str(precision)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = csv_path.read_text().splitlines()
    header = lines[0].split(",")
    want = ["time_step", "step_time_ms", "pressure_solve_call_count", "prev_pressure_iterations",
            "pressure_iterations", "pressure_hit_max_iter", "pressure_solve_ms"]
    for n in HEADER_STATS:
        want += [f"{n}_{s}" for s in ("min", "max", "mean", "abs_max", "nan_count", "inf_count")]
    assert header == want
    assert len(lines) == 4
    row0 = lines[1].split(",")
    assert row0[:7] == ["0", "0", "0", "0", "0", "0", "0"]
    last = lines[3].split(",")
    assert int(last[0]) == 2 and int(last[2]) == 2 and int(last[4]) > 0 and last[5] == "0"
    # statistics columns of the last row against the dumped final fields
    raw = np.fromfile(bin_path, dtype=np.float64)
    n = raw.size // 6
    fields = {k: raw[i * n:(i + 1) * n] for i, k in enumerate(L.FIELDS)}
    exp = expected(fields)
    vals = last[7:]
    for j, k in enumerate(NAMES):
        mn, mx, mean, amax, nan, inf = vals[6 * j:6 * j + 6]
        # 11 significant digits in the file (scientific, precision 10)
        for got, ref in ((mn, "min"), (mx, "max"), (mean, "mean"), (amax, "abs_max")):
            assert abs(float(got) - exp[k][ref]) <= 1e-9 * max(abs(exp[k][ref]), exp[k]["abs_max"], 1e-300), (k, ref)
        assert int(nan) == exp[k]["nan_count"] and int(inf) == exp[k]["inf_count"]

"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Run here (where the reference checkout exists), never on the GPU box:

    python tests/golden/make_golden.py

It builds oracle/_ref (oracle/Makefile compiles the reference's own
CPU/Inamuro.cpp, GPU/Inamuro.cpp and common.cpp with a small harness) and
records:

  init_*.npz   params.in text -> parsed parameters and initial fields of the
               reference GPU-tree Inamuro constructor (params parser + droplet
               initial condition, GPU/Inamuro.cpp:24-115, 491-566).
  step_*.npz   initial fields (from the droplet init, plus seeded phi noise)
               -> per-step fields and Poisson sweep counts of the reference
               CPU solver (CPU/Inamuro.cpp:347-363).  Small boxes keep full
               FP64 fields; larger ones keep SHA-256 digests of the raw FP64
               bytes, sampled values and the sweep counts.

The params files are written by this script (the reference's 14-line format);
physical constants follow the reference examples and the droplet benchmark
configurations (Laplace test: rho_L/rho_G = 50, a = 1, b = 6.7, T = 0.035,
kappa_f = 0.06, kappa_g = 6e-6, tau = 1, mu = 0.1 rho).
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import pyoracle  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
FIELDS = ("phi", "rho", "u", "v", "w", "p")


def params_text(shape, rho=(50.0, 1.0), tau=(1.0, 1.0), mu=(0.008, 0.00016), kappa=(0.5, 0.0005),
                T=0.035, a=1.0, b=6.7, fei_mm=(0.09714, 0.01134), fei_lg=(0.092, 0.015), DD=8.0,
                steps=20, extra=""):
    lx, ly, lz = shape
    lines = [f"{lx} {ly} {lz}", "1", str(steps), "20",
             f"{rho[0]!r} {rho[1]!r}", f"{tau[0]!r} {tau[1]!r}", f"{mu[0]!r} {mu[1]!r}",
             f"{kappa[0]!r} {kappa[1]!r}", repr(T), repr(a), repr(b),
             f"{fei_mm[0]!r} {fei_mm[1]!r}", f"{fei_lg[0]!r} {fei_lg[1]!r}", repr(DD)]
    return "\n".join(lines) + "\n" + extra


LAPLACE = dict(rho=(50.0, 1.0), mu=(5.0, 0.1), kappa=(0.06, 6e-6))

INIT_CASES = {
    "init_two_sharp": dict(shape=(12, 10, 8), DD=4.0),
    "init_single_tanh": dict(shape=(12, 10, 8), DD=5.0,
                             extra="init_mode=single_droplet init_profile=tanh interface_width=2.0 "
                                   "init_velocity=0.01\n"),
    "init_two_tanh_offset": dict(shape=(12, 10, 16), DD=4.0,
                                 extra="init_mode=two_droplets init_profile=tanh interface_width=1.5\n"
                                       "init_center_x=5.5 init_center_y=4.0 init_center_z=8.0\n"
                                       "init_separation=3.5 init_offset_x=2.0 init_velocity=0.02\n"),
    # CPU-tree output switches (line-wise, '#' comments) mixed with GPU-tree tokens.
    "init_mixed_styles": dict(shape=(10, 12, 8), DD=6.0,
                              extra="# output switches of the CPU solver\n"
                                    "enable_timing=1               # comment\n"
                                    "enable_tecplot_output=0\n"
                                    "output_dir=out/\n"
                                    "init_mode=single_droplet\n"
                                    "init_profile=unknown_profile\n"
                                    "init_center_x=3 init_center_z=2.5\n"),
}

STEP_CASES = {
    # tiny non-cubic box, single tanh drop, Laplace-test physics, seeded noise
    "step_single_tanh": dict(shape=(12, 10, 8), DD=6.0, steps=3, noise=1e-4, seed=11, full=True,
                             phys=LAPLACE,
                             extra="init_mode=single_droplet init_profile=tanh interface_width=2.0 "
                                   "init_velocity=0.0\n"),
    # two sharp drops moving along z (the reference's default initial condition)
    "step_two_sharp": dict(shape=(16, 12, 10), DD=4.0, steps=3, noise=0.0, seed=0, full=True,
                           phys={}, extra=""),
    # reference example physics (GPU/params.in) on its 16x32x32 box
    "step_example_16x32x32": dict(shape=(16, 32, 32), DD=8.0, steps=2, noise=0.0, seed=0, full=False,
                                  phys={}, extra=""),
    # the Laplace static-droplet configuration: 32^3, R = 8, W = 4 (tanh(2(r-R)/W)
    # == tanh((r-R)/2)), noise 1e-4, rho_L/rho_G = 50
    "step_laplace_32": dict(shape=(32, 32, 32), DD=16.0, steps=2, noise=1e-4, seed=2024, full=False,
                            phys=LAPLACE,
                            extra="init_mode=single_droplet init_profile=tanh interface_width=2.0 "
                                  "init_velocity=0.0\n"),
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed: {r.stderr[-2000:]}")
    return r


def sample_index(n, k=256, seed=7):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False))


def make_init(name, case, tmp):
    text = params_text(case["shape"], DD=case["DD"], extra=case.get("extra", ""))
    pf = os.path.join(tmp, name + ".in")
    open(pf, "w").write(text)
    out = os.path.join(tmp, name + ".bin")
    run([os.path.join(REF, "ref_init_harness"), pf, out])
    lx, ly, lz = case["shape"]
    n, plane = lx * ly * lz, lx * ly
    raw = np.fromfile(out)
    fields = raw[:6 * n].reshape(6, lz, ly, lx)
    ghosts = raw[6 * n:6 * n + 12 * plane].reshape(6, 2, ly, lx)
    prm = raw[6 * n + 12 * plane:]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), params_text=text, parsed=prm,
                        fields=fields, ghosts=ghosts)
    print(name, "ok")


def make_step(name, case, tmp):
    text = params_text(case["shape"], DD=case["DD"], extra=case.get("extra", ""), **case["phys"])
    pf = os.path.join(tmp, name + ".in")
    open(pf, "w").write(text)
    # Initial fields: the reference GPU-tree init of this params file, plus noise on phi.
    ib = os.path.join(tmp, name + "_init.bin")
    run([os.path.join(REF, "ref_init_harness"), pf, ib])
    lx, ly, lz = case["shape"]
    n = lx * ly * lz
    init = np.fromfile(ib)[:6 * n].reshape(6, lz, ly, lx).copy()
    if case["noise"] > 0:
        rng = np.random.default_rng(case["seed"])
        init[0] += rng.uniform(-case["noise"], case["noise"], size=init[0].shape)
    init_file = os.path.join(tmp, name + "_noisy.bin")
    init.tofile(init_file)
    outdir = os.path.join(tmp, name)
    os.makedirs(outdir, exist_ok=True)
    run([os.path.join(REF, "ref_cpu_harness"), "--params", pf, "--steps", str(case["steps"]),
         "--out", outdir, "--init", init_file])
    summ = np.loadtxt(os.path.join(outdir, "summary.txt"), ndmin=2)
    steps = []
    for s in range(1, case["steps"] + 1):
        steps.append(np.fromfile(os.path.join(outdir, f"step{s:04d}.bin")).reshape(6, lz, ly, lx))
    steps = np.stack(steps)
    idx = sample_index(n)
    payload = dict(params_text=text, init=init, sweeps=summ[:, 1].astype(np.int64),
                   ref_ms=summ[:, 2], sample_index=idx,
                   samples=steps.reshape(case["steps"], 6, n)[:, :, idx],
                   digests=np.array([[sha(steps[s, f]) for f in range(6)]
                                     for s in range(case["steps"])]),
                   mass=steps[:, 0].sum(axis=(1, 2, 3)))
    if case["full"]:
        payload["fields"] = steps
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **payload)
    print(name, "sweeps", summ[:, 1].astype(int).tolist(), "ref ms", summ[:, 2].round(1).tolist())


def main():
    pyoracle.build()
    only = set(sys.argv[1:])
    with tempfile.TemporaryDirectory() as tmp:
        for name, case in INIT_CASES.items():
            if not only or name in only:
                make_init(name, case, tmp)
        for name, case in STEP_CASES.items():
            if not only or name in only:
                make_step(name, case, tmp)


if __name__ == "__main__":
    main()

"""Benchmark of the Inamuro two-phase D3Q15 droplet step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--impl ours|reference]

Workload (the head-on binary droplet collision): 256^3 box, two spheres R = 32
whose centres are 96 cells apart, approaching at +-0.02 (lattice units),
rho_L/rho_G = 100, a = 1, b = 6.7, T = 0.035, kappa_f = 0.06, kappa_g = 6e-6,
tau_f = tau_g = 1, mu = 0.1 rho (nu = 0.1 in both phases), tanh interface with
W = 4 (interface_width = 2), seeded uniform noise of amplitude 1e-4 on phi.
The collision runs along z: x carries the reference's slip walls.  The Poisson
stop is the contract shared by every reference entry point (check every 100
sweeps, relative pressure change below 1e-3; the reference's WHILE_BASELINE.md); --dual adds
the GPU production switch's kinetic fixed-point residual.  Inputs are synthetic;
the box (about 14 GB of FP64 state) is far larger than L2, so no flush is
needed between timed steps.

A step is one full time step including its Poisson solve.  The metric is
MLUPS with Poisson sweeps counted: cells * (steps + sweeps) / time / 1e6.

--impl reference times the reference's own CPU solver (oracle/_ref, built from
the unmodified reference sources) on the host cores with a bounded sample of
the same 256^3 workload: one non-Poisson step part plus a few kinetic sweeps,
extrapolated to the sweeps-per-step of the GPU run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS (Poisson sweeps counted) of the Inamuro D3Q15 droplet step"
UNIT = "MLUPS"
N_SIDE = 256
# Algorithmic bytes per cell of one kinetic Poisson sweep (FP64: 30 pops +
# rho, s, p_in, p_out; mixed: FP32 pops).
SWEEP_BYTES = {"fp64": 272.0, "mixed": 144.0}
# What the sweep kernels actually have to move per cell (p is not stored per
# sweep): FP64 15x8 read + 15x8 write + rho, s; mixed 15x4 + 15x4 + omega, s.
COMPULSORY_BYTES = {"fp64": 256.0, "mixed": 128.0}
# Algorithmic bytes per cell of the non-Poisson kernels: collide (K4), moments
# (K1) and correction (C), FP64 and mixed.
PHASE_BYTES = {"collide_ms": {"fp64": 528.0, "mixed": 264.0},
               "moments_ms": {"fp64": 280.0, "mixed": 140.0},
               "correct_ms": {"fp64": 64.0, "mixed": 36.0}}
# Mean sweeps per step of the 256^3 head-on workload, FP64, steps 6-25 of the
# default run (measured on B200 with this bench: 3655); the reference arm's
# CPU sample is extrapolated to it (the reference needs ~2.3 s per sweep on
# one core, so a full step of ~3655 sweeps is not run).
DEFAULT_SWEEPS_PER_STEP = 3655.0
# The head-on workload as the reference's own params.in (GPU-tree grammar,
# GPU/Inamuro.cpp:24-115): 14 positional entries, then the initial-condition
# keys.  Written from constants so that the reference arm needs nothing of
# this repository's library.
WORKLOAD = {"rho_L": 100.0, "rho_G": 1.0, "tauf": 1.0, "taug": 1.0, "mu_L": 10.0, "mu_G": 0.1,
            "k_f": 0.06, "k_g": 6e-6, "T": 0.035, "a": 1.0, "b": 6.7, "fei_max": 0.09714,
            "fei_min": 0.01134, "fei_L": 0.092, "fei_G": 0.015, "DD": 64.0}


def workload_params(n=N_SIDE):
    import lbm_b200 as L
    w = WORKLOAD
    p = L.make_params(lx=n, ly=n, lz=n, rho_L=w["rho_L"], rho_G=w["rho_G"], mu_L=w["mu_L"], mu_G=w["mu_G"],
                      tauf=w["tauf"], taug=w["taug"], k_f=w["k_f"], k_g=w["k_g"], T=w["T"], a=w["a"], b=w["b"],
                      DD=w["DD"], init_single_droplet=0, init_tanh=1, interface_width=2.0,
                      init_velocity=0.02, init_center_x=n / 2.0, init_separation=48.0)
    assert (p.fei_max, p.fei_min, p.fei_L, p.fei_G) == (w["fei_max"], w["fei_min"], w["fei_L"], w["fei_G"])
    return p


def workload_params_text(n=N_SIDE, init_keys=True):
    """The head-on workload as a params.in of the reference (positional
    entries of CPU/Inamuro.cpp:38-53; with init_keys the GPU tree's
    initial-condition tokens, GPU/Inamuro.cpp:56-103)."""
    w = WORKLOAD
    text = (f"{n} {n} {n}\n1\n20\n20\n{w['rho_L']!r} {w['rho_G']!r}\n{w['tauf']!r} {w['taug']!r}\n"
            f"{w['mu_L']!r} {w['mu_G']!r}\n{w['k_f']!r} {w['k_g']!r}\n{w['T']!r}\n{w['a']!r}\n{w['b']!r}\n"
            f"{w['fei_max']!r} {w['fei_min']!r}\n{w['fei_L']!r} {w['fei_G']!r}\n{w['DD']!r}\n")
    if init_keys:
        text += (f"init_mode=two_droplets init_profile=tanh init_velocity=0.02 interface_width=2.0 "
                 f"init_center_x={n / 2.0!r} init_separation=48.0\n")
    return text


def reference_inputs(n, tmp, seed=1234):
    """Inputs of the reference arm without this repository's library: the
    reference's own GPU-tree initial condition (oracle/_ref/ref_init_harness,
    GPU/Inamuro.cpp:491-566 compiled from its sources) plus the workload's
    seeded phi noise.  Returns (params path, init path)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_init_harness")
    if not os.path.exists(exe):
        raise FileNotFoundError("reference init harness not built (oracle/_ref missing)")
    gpf = os.path.join(tmp, "params_gpu_tree.in")
    with open(gpf, "w") as fh:
        fh.write(workload_params_text(n, init_keys=True))
    pf = os.path.join(tmp, "params.in")
    with open(pf, "w") as fh:
        fh.write(workload_params_text(n, init_keys=False))
    raw = os.path.join(tmp, "ref_init.bin")
    r = subprocess.run([exe, gpf, raw], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference init harness failed: {r.stderr[-300:]}")
    cells = n * n * n
    fields = np.fromfile(raw, dtype=np.float64, count=6 * cells).reshape(6, n, n, n)
    rng = np.random.default_rng(seed)
    fields[0] += rng.uniform(-1e-4, 1e-4, size=(n, n, n))
    ib = os.path.join(tmp, "init.bin")
    fields.tofile(ib)
    return pf, ib


def workload_fields(p, seed=1234):
    import lbm_b200 as L
    f = L.init_droplets(p)
    rng = np.random.default_rng(seed)
    f["phi"] = f["phi"] + rng.uniform(-1e-4, 1e-4, size=f["phi"].shape)
    return f


BATCH_SIDES = (32, 48, 64, 80, 96)


def batch_workload(n_instances=64, seed=2024, noise=1e-4):
    """Batched droplet oscillation: n_instances independent periodic boxes, each side
    drawn uniformly from {32, 48, 64, 80, 96}; one ellipsoidal drop per box
    with semi-axes R(1+e), R, R/(1+e) along x, y, z, R ~ U[6, min side / 4],
    e ~ U[0.1, 0.4], centred; rho_L/rho_G log-uniform in [10, 1000] (rho_G =
    1); kappa_f ~ U[0.03, 0.1]; otherwise the Laplace-test physics (a = 1,
    b = 6.7, T = 0.035, kappa_g = 6e-6, tau = 1, mu = 0.1 rho, tanh interface
    W = 4, seeded phi noise).  The ellipsoid is built here (the reference's
    initializer only makes spheres): phi = phi_min + (phi_max - phi_min) *
    0.5 * (1 - tanh(2 (r_e - R) / W)), r_e = R * |(x/a, y/b, z/c)|.
    Returns (params list, fields list)."""
    import lbm_b200 as L
    rng = np.random.default_rng(seed)
    params, fields = [], []
    for _ in range(n_instances):
        lx, ly, lz = (int(rng.choice(BATCH_SIDES)) for _ in range(3))
        R = float(rng.uniform(6.0, min(lx, ly, lz) / 4.0))
        e = float(rng.uniform(0.1, 0.4))
        ratio = float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0))))
        kf = float(rng.uniform(0.03, 0.1))
        p = L.make_params(lx=lx, ly=ly, lz=lz, rho_L=ratio, rho_G=1.0, mu_L=0.1 * ratio, mu_G=0.1, tauf=1.0,
                          taug=1.0, k_f=kf, k_g=6e-6, T=0.035, a=1.0, b=6.7, DD=2.0 * R,
                          init_single_droplet=1, init_tanh=1, interface_width=2.0, init_velocity=0.0,
                          periodic_x=1)
        axes = (R * (1.0 + e), R, R / (1.0 + e))
        z, y, x = np.meshgrid(np.arange(lz) - (lz - 1) / 2.0, np.arange(ly) - (ly - 1) / 2.0,
                              np.arange(lx) - (lx - 1) / 2.0, indexing="ij")
        re = R * np.sqrt((x / axes[0]) ** 2 + (y / axes[1]) ** 2 + (z / axes[2]) ** 2)
        frac = 0.5 * (1.0 - np.tanh(2.0 * (re - R) / 4.0))
        phi = p.fei_min + frac * (p.fei_max - p.fei_min) + rng.uniform(-noise, noise, size=frac.shape)
        rho = p.rho_G + frac * (p.rho_L - p.rho_G)
        zero = np.zeros_like(phi)
        params.append(p)
        fields.append({"phi": phi, "rho": rho, "u": zero, "v": zero, "w": zero, "p": zero})
    return params, fields


def coalescence_workload(n=256, R=28.0, side=60.0, speed=0.01, ratio=1000.0, kf=0.06, seed=4242, noise=1e-4):
    """Three-droplet coalescence: an n^3 periodic box, three drops of radius R
    centred on an equilateral triangle of side `side` in the plane z = n/2
    (centroid at the box centre), each moving towards the centroid at
    `speed`; rho_L/rho_G = ratio (rho_G = 1), mu = 0.1 rho, kappa_f = kf,
    otherwise the Laplace-test physics (a = 1, b = 6.7, T = 0.035,
    kappa_g = 6e-6, tau = 1, tanh interfaces W = 4, seeded phi noise).  Each
    drop's profile is phi = phi_min + (phi_max - phi_min) * 0.5 (1 - tanh(2 (r
    - R) / W)); where profiles overlap the largest is kept, and the velocity is
    that of the drop whose profile is kept, scaled by it.  Built here: the
    reference's initializer makes one or two drops on the z axis.  Returns
    (params, fields)."""
    import lbm_b200 as L
    p = L.make_params(lx=n, ly=n, lz=n, rho_L=ratio, rho_G=1.0, mu_L=0.1 * ratio, mu_G=0.1, tauf=1.0, taug=1.0,
                      k_f=kf, k_g=6e-6, T=0.035, a=1.0, b=6.7, DD=2.0 * R, init_single_droplet=1, init_tanh=1,
                      interface_width=2.0, init_velocity=0.0, periodic_x=1)
    c = (n - 1) / 2.0
    rc = side / np.sqrt(3.0)             # centroid-to-vertex distance
    centres = [(c + rc * np.cos(a), c + rc * np.sin(a), c) for a in (np.pi / 2, np.pi / 2 + 2 * np.pi / 3,
                                                                        np.pi / 2 + 4 * np.pi / 3)]
    frac = np.zeros((n, n, n))
    u = np.zeros((n, n, n))
    v = np.zeros((n, n, n))
    x = np.arange(n, dtype=np.float64)
    for cx_, cy_, cz_ in centres:
        r = np.sqrt((x[None, None, :] - cx_) ** 2 + (x[None, :, None] - cy_) ** 2 + (x[:, None, None] - cz_) ** 2)
        fr = 0.5 * (1.0 - np.tanh(2.0 * (r - R) / 4.0))
        take = fr > frac
        dx, dy = c - cx_, c - cy_
        norm = np.hypot(dx, dy)
        u = np.where(take, speed * dx / norm * fr, u)
        v = np.where(take, speed * dy / norm * fr, v)
        frac = np.maximum(frac, fr)
        del r, fr, take
    rng = np.random.default_rng(seed)
    phi = p.fei_min + frac * (p.fei_max - p.fei_min) + rng.uniform(-noise, noise, size=frac.shape)
    rho = p.rho_G + frac * (p.rho_L - p.rho_G)
    return p, {"phi": phi, "rho": rho, "u": u, "v": v, "w": np.zeros_like(phi), "p": np.zeros_like(phi)}


def adjoint_workload(n=64, e=0.0, kf_scale=1.0, seed=31, noise=1e-4):
    """Adjoint calibration box: n^3 periodic, one drop R = n/4 at the centre
    (semi-axes R(1+e), R, R/(1+e); e = 0 a sphere), tanh interface W = 4,
    rho_L/rho_G = 100, mu = 0.1 rho, a = 1, b = 6.7, T = 0.035,
    kappa_f = 0.06 kf_scale, kappa_g = 6e-6, tau = 1, at rest, seeded phi
    noise.  Returns (params, fields)."""
    import lbm_b200 as L
    R = n / 4.0
    p = L.make_params(lx=n, ly=n, lz=n, rho_L=100.0, rho_G=1.0, mu_L=10.0, mu_G=0.1, tauf=1.0, taug=1.0,
                      k_f=0.06 * kf_scale, k_g=6e-6, T=0.035, a=1.0, b=6.7, DD=2.0 * R, init_single_droplet=1,
                      init_tanh=1, interface_width=2.0, init_velocity=0.0, periodic_x=1)
    axes = (R * (1.0 + e), R, R / (1.0 + e))
    c = (n - 1) / 2.0
    z, y, x = np.meshgrid(np.arange(n) - c, np.arange(n) - c, np.arange(n) - c, indexing="ij")
    re = R * np.sqrt((x / axes[0]) ** 2 + (y / axes[1]) ** 2 + (z / axes[2]) ** 2)
    frac = 0.5 * (1.0 - np.tanh(2.0 * (re - R) / 4.0))
    rng = np.random.default_rng(seed)
    phi = p.fei_min + frac * (p.fei_max - p.fei_min) + rng.uniform(-noise, noise, size=frac.shape)
    rho = p.rho_G + frac * (p.rho_L - p.rho_G)
    zero = np.zeros_like(phi)
    return p, {"phi": phi, "rho": rho, "u": zero, "v": zero, "w": zero, "p": zero}


def config_dict(n, precision, dual=False):
    return {"workload": f"head-on binary droplet collision {n}^3, 2 x R=32 drops 96 apart, "
                        f"+-0.02, rho_L/rho_G=100",
            "box": [n, n, n], "cells": n ** 3, "precision": precision,
            "poisson": {"check_interval": 100, "tolerance": 1e-3, "dual_residual": dual},
            "l2": "inputs larger than L2 (14 GB FP64 state vs 126 MB L2)",
            "parallelism": "replicas (one box per GPU)"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------- CPU sample
def reference_cpu_samples(n, sample_sweeps=3, reps=1, nonpoisson_reps=None):
    """Runs the reference CPU solver (oracle/_ref/ref_cpu_harness, built from
    the unmodified reference sources) on the n^3 workload, inputs from the
    reference's own initial condition (reference_inputs): `reps` times
    `sample_sweeps` kinetic sweeps, the first `nonpoisson_reps` (default all)
    preceded by one non-Poisson step part.  Returns
    ([(seconds_nonpoisson or None, seconds_per_sweep), ...], cells, wall_s)
    or raises."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_harness")
    if not os.path.exists(exe):
        raise FileNotFoundError("reference harness not built (oracle/_ref missing)")
    with tempfile.TemporaryDirectory() as tmp:
        pf, ib = reference_inputs(n, tmp)
        cmd = [exe, "--params", pf, "--sample-sweeps", str(sample_sweeps), "--out", tmp, "--init", ib,
               "--sample-reps", str(reps)]
        if nonpoisson_reps is not None:
            cmd += ["--nonpoisson-reps", str(nonpoisson_reps)]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed: {r.stderr[-300:]}")
        cells, reps_out = None, []
        for line in open(os.path.join(tmp, "sample.txt")):
            parts = line.split()
            if parts[0] == "cells":
                cells = float(parts[1])
            elif parts[0] == "rep":
                t_np = float(parts[2]) / 1e3
                reps_out.append((t_np if t_np >= 0 else None, float(parts[3]) / 1e3 / max(sample_sweeps, 1)))
    return reps_out, cells, wall


def cpu_value(cells, t_np, t_sw, sweeps_per_step):
    """MLUPS (sweeps counted) of a step with `sweeps_per_step` sweeps."""
    return cells * (1.0 + sweeps_per_step) / (t_np + sweeps_per_step * t_sw) / 1e6


def cpu_baseline_entry(n, reps_out, cells, wall, sweeps_per_step, sample_sweeps, value=None):
    nps = [r[0] for r in reps_out if r[0] is not None]
    t_np = statistics.median(nps)
    t_sw = statistics.median(r[1] for r in reps_out)
    v = cpu_value(cells, t_np, t_sw, sweeps_per_step) if value is None else value
    sample = (f"reference CPU solver (CPU/Inamuro.cpp, g++ -O3, single-threaded) on the {n}^3 "
              f"workload (inputs from the reference's own init + seeded noise), {len(reps_out)} rep(s) of "
              f"{sample_sweeps} kinetic sweeps ({t_sw:.2f} s each) and {len(nps)} non-Poisson step part(s) "
              f"({t_np:.2f} s), extrapolated to {sweeps_per_step:.0f} sweeps/step (B200 FP64 measurement of "
              f"this workload); harness wall {wall:.1f} s incl. setup")
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample,
            "seconds_per_sweep": t_sw, "seconds_nonpoisson": t_np, "extrapolated": True,
            "sweeps_per_step_extrapolated_to": sweeps_per_step, "sweeps_timed_per_rep": sample_sweeps}


# ---------------------------------------------------------------- reference GPU
def _program_run(exe, d, pf, steps, timeout):
    """One run of a GPU/main.cpp front end (the reference's own program or the
    same main.cpp over this library): wall ms of its step loop (its
    wall_total_ms) and the sweeps of each step (its Poisson CSV)."""
    os.makedirs(d)
    cmd = [exe, "--mode", "gpu", "--params", pf, "--steps", str(steps), "--poisson", "split",
           "--poisson-diagnostics", "diag.csv", "--no-roofline"]
    r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} exited {r.returncode}: {(r.stdout + r.stderr)[-300:]}")
    ms = None
    for tok in r.stdout.split():
        if tok.startswith("wall_total_ms="):
            ms = float(tok.split("=", 1)[1])
    if ms is None:
        raise RuntimeError(f"{os.path.basename(exe)}: no wall_total_ms in its output")
    import csv
    sweeps = {}
    for row in csv.DictReader(open(os.path.join(d, "diag.csv"))):
        s = int(row["step"])
        sweeps[s] = max(sweeps.get(s, 0), int(row["iteration"]))
    return ms, [sweeps[s] for s in sorted(sweeps)]


def reference_gpu_leg(n=N_SIDE, steps=1, timeout=900):
    """The reference's own FP64 GPU step (GPU/InamuroCUDA.cu, compiled from its
    unmodified sources for sm_100a: oracle/_ref/lbm_gpu_ref) beside this
    library behind the same front end (the reference's GPU/main.cpp over
    include/InamuroCUDA.hpp: oracle/_ref/lbm_gpu_dropin), on the same
    noise-free head-on params.in (the reference's own initial condition), the
    reference CLI's strict production settings (split kinetic form, check 100,
    tolerance 1e-3, unbounded), `steps` steps; the per-step sweep counts must
    agree.  Host wall clock of each program's step loop (its wall_total_ms).
    MLUPS with sweeps counted = cells (steps + sweeps) / wall."""
    ref = os.path.join(ROOT, "oracle", "_ref", "lbm_gpu_ref")
    ours = os.path.join(ROOT, "oracle", "_ref", "lbm_gpu_dropin")
    missing = [os.path.basename(x) for x in (ref, ours) if not os.path.exists(x)]
    if missing:
        return {"unavailable": "not built: " + ", ".join(missing)}
    cells = float(n) ** 3
    out = {"box": [n, n, n], "steps": steps,
           "config": f"head-on {n}^3 params.in without noise, --poisson split, check 100, tolerance 1e-3"}
    with tempfile.TemporaryDirectory() as tmp:
        pf = os.path.join(tmp, "params.in")
        with open(pf, "w") as fh:
            fh.write(workload_params_text(n, init_keys=True))
        for name, exe in (("reference", ref), ("ours", ours)):
            ms, sw = _program_run(exe, os.path.join(tmp, name), pf, steps, timeout)
            out[name] = {"wall_ms": ms, "sweeps_per_step": sw,
                         "mlups": cells * (steps + sum(sw)) / (ms / 1e3) / 1e6,
                         "mlups_reference_definition": cells * steps / (ms / 1e3) / 1e6}
    out["sweeps_equal"] = out["reference"]["sweeps_per_step"] == out["ours"]["sweeps_per_step"]
    out["ratio"] = out["ours"]["mlups"] / out["reference"]["mlups"]
    return out


# ---------------------------------------------------------------- helpers
def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = os.environ.get("LBM_BENCH_BACKEND", "nccl")
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def read_traffic(precision):
    """DRAM bytes per sweep (256^3) from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"sweep_{precision}_256.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_sweep_256:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- arms
def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.size
    try:
        # the non-Poisson part (~11 s on one core) is timed in the first two
        # reps only, so the W + K reps of sweeps fit a few minutes
        reps_out, cells, wall = reference_cpu_samples(n, args.sample_sweeps, args.warmup + args.steps,
                                                      nonpoisson_reps=2)
    except Exception as e:  # harness missing or failed: report, do not crash the driver
        print(json.dumps({"impl": "reference", "unavailable": str(e)[:200]}))
        return 0
    t_np = statistics.median(r[0] for r in reps_out if r[0] is not None)
    timed = reps_out[args.warmup:] or reps_out
    vals = [cpu_value(cells, t_np, t_sw, args.sweeps_per_step) for _, t_sw in timed]
    value = statistics.median(vals)
    step_s = statistics.median(t_np + args.sweeps_per_step * t_sw for _, t_sw in timed)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(n, "fp64"), "impl": "reference",
            "cpu_baseline": cpu_baseline_entry(n, reps_out, cells, wall, args.sweeps_per_step,
                                               args.sample_sweeps, value=value),
            "timing": "ms_per_step is extrapolated: per rep, sample_sweeps sweeps are timed and a step is "
                      "t_nonpoisson + sweeps_per_step x t_sweep (not run in full: ~2.3 s per sweep)",
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_leg(args, precision, world, rank, local, p, f, e2e: bool):
    """Times K steps (after W warm-up steps) of one precision on this rank."""
    import lbm_b200 as L
    g = L.InamuroCUDA(p, f, precision=precision, device=local)
    g.set_poisson(check_interval=100, tolerance=1e-3, dual=args.dual, max_sweeps=args.max_sweeps)
    for _ in range(args.warmup):   # includes the first, equilibrium-initialised step
        g.step(1)
    g.synchronize()
    barrier(world)
    g.reset_timing()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    stats = g.step(args.steps)
    g.synchronize()
    wall = time.perf_counter() - t0
    barrier(world)
    clk = clocks.stop()
    tm = g.timing()
    cells = float(p.lx * p.ly * p.lz)
    dev_s = sum(s["device_ms"] for s in stats) / 1e3
    sweeps = sum(s["iterations"] for s in stats)
    t_max = dist_max(dev_s, world)
    units_all = dist_sum(cells * (args.steps + sweeps), world)
    leg = {"value": units_all / t_max / 1e6, "ms_per_step": t_max * 1e3 / args.steps,
           "sweeps_per_step": sweeps / args.steps,
           "converged_steps": int(sum(s["converged"] for s in stats)),
           "mlups_reference_definition": cells * args.steps * world / t_max / 1e6,
           "gpu_launches": int(dist_sum(tm["kernel_launches"], world)),
           "clocks": clk, "wall_s": wall,
           "phase_ms_per_step": {k: tm[k] / max(tm["steps"], 1) for k in
                                 ("collide_ms", "moments_ms", "prep_ms", "poisson_ms", "correct_ms")}}
    # roofline of the dominant kernel (the kinetic sweep): average launch time
    # over the timed region = Poisson device time / sweep-kernel launches
    # (sweep-equivalents: a two-sweep launch counts twice, so this is the
    # device time per sweep whether or not sweeps are fused)
    sweep_ms = tm["poisson_ms"] / max(tm["sweep_kernels"], 1)
    achieved = SWEEP_BYTES[precision] * cells / (sweep_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    # A two-sweep launch moves the populations through DRAM once for two
    # sweeps: its compulsory bytes per sweep are half a single sweep's.
    fused = tm["fused_sweeps"] / max(tm["sweep_kernels"], 1)
    compulsory = COMPULSORY_BYTES[precision] * (1.0 - 0.5 * fused)
    leg["roofline"] = {"bound": "hbm", "kernel": f"sweep ({precision})", "achieved": achieved,
                       "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                       "traffic": read_traffic(precision), "bytes_per_cell": SWEEP_BYTES[precision],
                       "fraction_of_sweeps_in_two_sweep_passes": fused,
                       "compulsory_bytes_per_cell_per_sweep": compulsory,
                       "frac_compulsory": compulsory * cells / (sweep_ms / 1e3) / 1e9 / peak,
                       "avg_ms_per_sweep": sweep_ms,
                       "note": "frac uses the per-sweep byte model (one DRAM pass per sweep); "
                               "two-sweep passes beat it, frac_compulsory is against what the "
                               "launches actually have to move"}
    # the collide+stream kernel (K4: stencils, f and g collision, pull
    # stream), one launch per step, from the same timed steps
    col_ms = tm["collide_ms"] / max(tm["steps"], 1)
    col_bytes = PHASE_BYTES["collide_ms"][precision]
    leg["roofline_collide"] = {"bound": "hbm", "kernel": f"collide ({precision})",
                               "achieved": col_bytes * cells / (col_ms / 1e3) / 1e9, "peak": peak,
                               "unit": "GB/s", "frac": col_bytes * cells / (col_ms / 1e3) / 1e9 / peak,
                               "bytes_per_cell": col_bytes, "avg_launch_ms": col_ms}
    if e2e:
        # end to end through the public API with host buffers: upload the
        # initial fields from pinned host memory, run K steps, download all six
        # fields after every step
        import torch
        pinned = {k: torch.from_numpy(np.ascontiguousarray(f[k])).pin_memory() for k in L.FIELDS}
        outs = {k: torch.empty(f[k].shape, dtype=torch.float64).pin_memory() for k in L.FIELDS}
        nbytes = 6 * p.lx * p.ly * p.lz * 8
        g.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        g.load_fields({k: pinned[k].numpy() for k in L.FIELDS})
        e_sweeps = 0
        for _ in range(args.steps):
            e_sweeps += g.step(1)[0]["iterations"]
            for k in L.FIELDS:
                g.download(k, outs[k].numpy())
        g.synchronize()
        e_wall = time.perf_counter() - t0
        barrier(world)
        e_units = dist_sum(cells * (args.steps + e_sweeps), world)
        leg["e2e"] = {"value": e_units / dist_max(e_wall, world) / 1e6, "unit": UNIT,
                      "h2d_bytes_per_step": nbytes // args.steps, "d2h_bytes_per_step": nbytes,
                      "steps": args.steps, "sweeps": e_sweeps,
                      "note": "fresh run from the host initial condition: one H2D upload of the six "
                              "fields (amortised per step) + K steps + D2H of all six fields after "
                              "each step, host wall clock"}
    g.close()
    return leg


def accuracy_probe(n, steps, sweeps):
    """Mixed against FP64 on the bench workload, outside the timed region: both
    precisions advance `steps` steps from the same initial fields with the same
    replayed sweep count per step (so the comparison is not blurred by where
    each run's 1e-3 exit falls), then the norm-wise relative error
    max|mixed - fp64| / max|fp64| per field.  The FP64 path matches the FP64
    oracle to ~1e-15, so these are the errors against the oracle.  Mass drift:
    max over steps k of |M_k - M_1| / |M_1|, M_k = sum(phi) after step k (the
    step's FP64 device reduction), for each precision."""
    import lbm_b200 as L
    p = workload_params(n)
    p.periodic_x = 1        # the configuration's periodic box: no slip-wall mass flux
    f = workload_fields(p)
    out = {"box": [n, n, n], "steps": steps, "sweeps_per_step": sweeps, "x_boundary": "periodic"}
    fields, drift = {}, {}
    for prec in ("fp64", "mixed"):
        s = L.InamuroCUDA(p, f, precision=prec)
        d, m1 = 0.0, None
        for _ in range(steps):
            st = s.step_replay([sweeps])[0]
            m1 = st["mass"] if m1 is None else m1
            d = max(d, abs(st["mass"] - m1) / abs(m1))
        fields[prec] = s.download_fields()
        drift[prec] = d
        s.close()
    out["rel_err_mixed_vs_fp64"] = {
        k: float(np.max(np.abs(fields["mixed"][k] - fields["fp64"][k])) /
                 max(float(np.max(np.abs(fields["fp64"][k]))), 1e-300)) for k in L.FIELDS}
    out["mass_drift"] = drift
    return out


def run_batch(args):
    print(json.dumps(batch_measure(args)))
    return 0


def batch_measure(args):
    """The batched droplet oscillation (64 uneven periodic boxes, mixed
    precision): autotune the batched kernels, W warm-up steps, K timed steps
    (natural Poisson exits per instance), device time from the batch's CUDA
    events.  MLUPS with sweeps counted = sum_i cells_i (steps + sweeps_i) / t.
    Roofline: the sweep-equivalent bytes (144 B per cell and sweep) and the
    bytes the launches must move (128 B for a single sweep, 64 B per sweep in
    a two-sweep pass) over the Poisson device time."""
    import lbm_b200 as L
    params, fields = batch_workload(args.batch_instances, seed=args.batch_seed)
    cells = [p.lx * p.ly * p.lz for p in params]
    b = L.Batch(params, fields)
    b.set_poisson(100, 1e-3, max_sweeps=args.max_sweeps)
    t0 = time.perf_counter()
    tuning = b.tune()
    tune_s = time.perf_counter() - t0
    if args.warmup:
        b.step(args.warmup)
    b.reset_timing()
    clk = ClockSampler(0)
    clk.start()
    t0 = time.perf_counter()
    stats = b.step(args.steps)
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    t = b.timing()
    dev_ms = t["collide_ms"] + t["moments_ms"] + t["prep_ms"] + t["poisson_ms"] + t["correct_ms"]
    swept = sum(cells[i] * sum(stats[s][i]["iterations"] for s in range(args.steps)) for i in range(len(cells)))
    updates = sum(cells) * args.steps + swept
    value = updates / (dev_ms / 1e3) / 1e6
    peak, kind = measured_peaks()
    sweep_gbs = SWEEP_BYTES["mixed"] * swept / (t["poisson_ms"] / 1e3) / 1e9
    fused = t["fused_sweeps"] / max(t["sweep_kernels"], 1)
    compulsory = COMPULSORY_BYTES["mixed"] * (1.0 - 0.5 * fused)
    comp_gbs = compulsory * swept / (t["poisson_ms"] / 1e3) / 1e9
    line = {"metric": "MLUPS (Poisson sweeps counted) of the batched droplet oscillation", "value": value,
            "unit": "MLUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded uneven boxes, ellipsoidal drops, random noise 1e-4 on phi)",
            "config": {"workload": f"batched droplet oscillation, {len(cells)} periodic boxes with sides from "
                                   f"{{32,48,64,80,96}}, ellipsoids R(1+e),R,R/(1+e), rho ratio 10-1000, "
                                   f"kappa_f 0.03-0.1", "instances": len(cells), "cells": sum(cells),
                       "poisson": {"check_interval": 100, "tolerance": 1e-3}, "seed": args.batch_seed,
                       "l2": "inputs larger than L2"},
            "tuning": tuning, "tune_s": tune_s,
            "sweeps_per_step_mean": swept / sum(cells) / args.steps,
            "phase_ms_per_step": {k: t[k] / args.steps for k in
                                  ("collide_ms", "moments_ms", "prep_ms", "poisson_ms", "correct_ms")},
            "roofline": {"bound": "hbm", "kernel": "batched sweep (mixed)", "achieved": sweep_gbs, "peak": peak,
                         "unit": "GB/s", "frac": sweep_gbs / peak, "peak_kind": kind,
                         "bytes_per_cell": SWEEP_BYTES["mixed"],
                         "fraction_of_sweeps_in_two_sweep_passes": fused,
                         "compulsory_bytes_per_cell_per_sweep": compulsory, "frac_compulsory": comp_gbs / peak,
                         "note": "sweep-equivalent bytes of the instances' own sweeps over the Poisson device "
                                 "time, checks and finalisations included; frac_compulsory against what the "
                                 "launches must move"},
            "gpu_launches": t["kernel_launches"], "clocks": clocks, "wall_s": wall,
            "converged": all(st["converged"] for st in stats[-1])}
    b.close()
    return line


def run_adjoint(args):
    print(json.dumps(adjoint_measure(args)))
    return 0


def adjoint_measure(args):
    """Adjoint calibration (FP64, periodic n^3, bounded sample of the
    2000-step run): J = 0.5 sum (phi_T - phi_target)^2, phi_target the final
    phi of a run from an ellipsoidal drop (e = 0.2) with kappa_f + 5 %.  W
    warm-up steps on a separate box, then one forward run of K steps
    (checkpoints every min(100, K) steps) and its reverse pass (recomputation
    included), timed on the wall clock around the synchronous calls; the
    gradient along kappa_f and along seeded random directions of phi_0 is
    checked against centred finite differences (step 1e-6) of replayed runs."""
    import lbm_b200 as L
    n, K = args.adjoint_size, args.steps
    tol_f, tol_a = args.adjoint_forward_tol, args.adjoint_tol
    p, f = adjoint_workload(n)
    pt, ft = adjoint_workload(n, e=0.2, kf_scale=1.05)

    def forward(pp, ff, sweeps=None):
        a = L.Adjoint(pp, checkpoint_interval=min(100, K), check_interval=100, tolerance=tol_a,
                      krylov=args.adjoint_krylov, krylov_tolerance=args.adjoint_krylov_tol)
        a.set_poisson(check_interval=100, tolerance=tol_f, max_sweeps=args.max_sweeps, fail_on_limit=1)
        a.forward(ff, K, sweeps)
        return a

    if args.warmup:
        w = L.InamuroCUDA(p, f, precision="fp64")
        w.set_poisson(check_interval=100, tolerance=tol_f, max_sweeps=args.max_sweeps, fail_on_limit=True)
        w.step(args.warmup)
        w.close()
    tgt = forward(pt, ft)
    target = tgt.download("phi")
    tgt.close()
    clk = ClockSampler(0)
    clk.start()
    a = forward(p, f)
    phi_T = a.download("phi")
    grads, st = a.backward({"phi": phi_T - target})
    clocks = clk.stop()
    sweeps = a.sweeps()
    J = 0.5 * float(np.sum((phi_T - target) ** 2))

    def J_of(pp, ff):
        b = forward(pp, ff, sweeps)
        v = 0.5 * float(np.sum((b.download("phi") - target) ** 2))
        b.close()
        return v

    checks = []
    h = 1e-6
    pp = [L.make_params(**{k: getattr(p, k) for k, _ in L.Params._fields_}) for _ in range(2)]
    pp[0].k_f, pp[1].k_f = p.k_f * (1 + h), p.k_f * (1 - h)
    fd = (J_of(pp[0], f) - J_of(pp[1], f)) / (2 * h * p.k_f)
    checks.append({"along": "kappa_f", "adjoint": st["grad_kappa_f"], "fd": fd,
                   "rel_err": abs(st["grad_kappa_f"] - fd) / abs(fd)})
    rng = np.random.default_rng(7)
    for i in range(args.adjoint_directions):
        d = 0.05 * rng.standard_normal(f["phi"].shape)
        vals = []
        for sgn in (1.0, -1.0):
            ff = dict(f)
            ff["phi"] = f["phi"] + sgn * h * d
            vals.append(J_of(p, ff))
        fd = (vals[0] - vals[1]) / (2 * h)
        got = float(np.sum(grads["phi"] * d))
        checks.append({"along": f"phi_0 direction {i}", "adjoint": got, "fd": fd, "rel_err": abs(got - fd) / abs(fd)})
    cells = n ** 3
    fwd_s, bwd_s = st["forward_ms"] / 1e3, st["backward_ms"] / 1e3
    fwd_updates = cells * (K + st["forward_sweeps"])
    bwd_updates = cells * (2 * st["recompute_steps"] + st["forward_sweeps"] + st["adjoint_sweeps"])
    line = {"metric": "MLUPS (Poisson sweeps counted) of the adjoint calibration run (forward + reverse pass)",
            "value": (fwd_updates + bwd_updates) / (fwd_s + bwd_s) / 1e6, "unit": "MLUPS", "n_gpus": 1,
            "steps": K, "warmup": args.warmup, "ms_per_step": (st["forward_ms"] + st["backward_ms"]) / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded phi noise 1e-4; target from an ellipsoidal drop e=0.2, kappa_f +5%)",
            "config": {"workload": f"adjoint calibration {n}^3 periodic, R={n // 4}, rho_L/rho_G=100, "
                                   f"{K} of 2000 steps (bounded sample), checkpoints every {min(100, K)} steps",
                       "poisson": {"forward_tolerance": tol_f, "adjoint_tolerance": tol_a, "check_interval": 100,
                                   "adjoint_solver": "BiCGSTAB" if args.adjoint_krylov else "transposed sweeps",
                                   "adjoint_krylov_tolerance": args.adjoint_krylov_tol if args.adjoint_krylov else None},
                       "l2": "per-step state larger than L2" if cells * 288 > 126e6 else "state fits in L2"},
            "forward_mlups": fwd_updates / fwd_s / 1e6, "reverse_mlups": bwd_updates / bwd_s / 1e6,
            "adjoint_forward_time_ratio": bwd_s / fwd_s,
            "forward_ms": st["forward_ms"], "backward_ms": st["backward_ms"],
            "sweeps_per_step": {"forward": st["forward_sweeps"] / K, "adjoint": st["adjoint_sweeps"] / K},
            "objective": J, "gradient_checks": checks,
            "max_rel_err": max(c["rel_err"] for c in checks), "clocks": clocks}
    a.close()
    return line


def run_coalescence_adjoint(args):
    """Bounded sample of the large adjoint configuration: the three-drop
    coalescence (coalescence_workload, rho_L/rho_G = 1000) on an n^3 periodic
    box, a forward run of K steps over the mixed box (FP32 populations, FP64
    rest population, pressure and reductions; lbm_adjoint_cfg.precision = 1)
    with binomial checkpointing, and its reverse pass (adjoint Poisson solves
    by transposed sweeps, or BiCGSTAB with --adjoint-krylov), for each of
    --coalescence-samples kappa_f values drawn
    uniformly from [0.04, 0.08].  Objective J = 0.5 sum (phi_T - phi_target)^2,
    phi_target the final phi of the first sample's forward run with kappa_f
    + 5 %.  Reported: MLUPS (sweeps counted) of forward and reverse, the
    reverse/forward time ratio, the device memory in use after the reverse
    pass (its checkpoint slots are still held), the binomial schedule's
    recomputation, and for the first sample dJ/dk_f against a centred finite
    difference of the FP64 forward (replayed sweep counts)."""
    import torch
    import lbm_b200 as L
    n, K = args.size, args.steps
    rng = np.random.default_rng(77)
    kfs = [float(k) for k in rng.uniform(0.04, 0.08, size=args.coalescence_samples)]
    slots = args.binomial_slots
    tol_f = args.adjoint_forward_tol
    # --coalescence-cap: each forward step stops at this many sweeps, converged
    # or not (the reference's poisson_iteration_limit); at rho_L/rho_G = 1000
    # the liquid's diffusivity 1/(3 rho) makes a converged solve take millions
    # of sweeps, so a bounded sample caps it and the gradient is then that of
    # an unconverged solve (its finite-difference error says how far)
    fail = 0 if args.coalescence_cap else 1
    if args.coalescence_cap:
        args.max_sweeps = args.coalescence_cap
    free0, total = torch.cuda.mem_get_info()
    out = {"metric": "MLUPS (sweeps counted) of the coalescence adjoint sample (forward + reverse)", "unit": "MLUPS",
           "n_gpus": 1, "steps": K, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 populations + f64 pressure/reductions (forward); f64 adjoint",
           "data": "synthetic (three seeded tanh drops, rho ratio 1000, phi noise 1e-4)",
           "config": {"workload": f"three-drop coalescence {n}^3 periodic, R=28, triangle side 60 in z=n/2, "
                                  f"approach 0.01, rho_L/rho_G={args.coalescence_ratio:g}; {K} of 5000 steps "
                                  f"(bounded sample)",
                      "kappa_f": kfs, "binomial_checkpoints": slots,
                      "poisson": {"forward_tolerance": tol_f, "forward_sweep_cap": args.coalescence_cap or None,
                                  "adjoint_solver": "BiCGSTAB" if args.adjoint_krylov else "transposed sweeps",
                                  "adjoint_tolerance": args.adjoint_tol,
                                  "adjoint_krylov_tolerance": args.adjoint_krylov_tol}},
           "samples": []}
    target = None
    for i, kf in enumerate(kfs):
        p, f = coalescence_workload(n, kf=kf, ratio=args.coalescence_ratio)
        if target is None:
            pt, ft = coalescence_workload(n, kf=kf * 1.05, ratio=args.coalescence_ratio)
            a = L.Adjoint(pt, binomial_checkpoints=slots, check_interval=100, tolerance=args.adjoint_tol,
                          krylov=args.adjoint_krylov, krylov_tolerance=args.adjoint_krylov_tol, precision="mixed")
            a.set_poisson(check_interval=100, tolerance=tol_f, max_sweeps=args.max_sweeps, fail_on_limit=fail)
            a.forward(ft, K)
            target = a.download("phi")
            a.close()
            del pt, ft
        a = L.Adjoint(p, binomial_checkpoints=slots, check_interval=100, tolerance=args.adjoint_tol,
                      krylov=args.adjoint_krylov, krylov_tolerance=args.adjoint_krylov_tol, precision="mixed")
        a.set_poisson(check_interval=100, tolerance=tol_f, max_sweeps=args.max_sweeps, fail_on_limit=fail)
        a.forward(f, K)
        phi_T = a.download("phi")
        grads, st = a.backward({"phi": phi_T - target})
        free1, _ = torch.cuda.mem_get_info()
        sweeps = a.sweeps()
        a.close()
        cells = float(n) ** 3
        fwd_s, bwd_s = st["forward_ms"] / 1e3, st["backward_ms"] / 1e3
        fwd_updates = cells * (K + st["forward_sweeps"])
        bwd_updates = cells * (2 * st["recompute_steps"] + st["forward_sweeps"] + st["adjoint_sweeps"])
        rec = {"kappa_f": kf, "forward_mlups": fwd_updates / fwd_s / 1e6, "reverse_mlups": bwd_updates / bwd_s / 1e6,
               "adjoint_forward_time_ratio": bwd_s / fwd_s, "forward_ms": st["forward_ms"],
               "backward_ms": st["backward_ms"], "forward_sweeps_per_step": st["forward_sweeps"] / K,
               "adjoint_matvecs_per_step": st["adjoint_sweeps"] / K, "recompute_steps": st["recompute_steps"],
               "device_gb_in_use_after_reverse": (total - free1) / 1e9, "grad_kappa_f": st["grad_kappa_f"],
               "objective": 0.5 * float(np.sum((phi_T - target) ** 2)), "updates": fwd_updates + bwd_updates}
        if i == 0 and args.coalescence_fd:
            h = 1e-6 * kf
            vals = []
            for sgn in (1.0, -1.0):
                pp, ff = coalescence_workload(n, kf=kf + sgn * h, ratio=args.coalescence_ratio)
                b = L.InamuroCUDA(pp, ff, precision="fp64")
                b.set_poisson(check_interval=100, tolerance=tol_f, max_sweeps=args.max_sweeps)
                b.step_replay(sweeps)
                vals.append(0.5 * float(np.sum((b.download("phi") - target) ** 2)))
                b.close()
                del pp, ff
            fd = (vals[0] - vals[1]) / (2 * h)
            rec["fd_kappa_f_fp64"] = fd
            rec["rel_err_vs_fp64_fd"] = abs(st["grad_kappa_f"] - fd) / abs(fd)
        out["samples"].append(rec)
        print(json.dumps({"sample": i, **rec}), flush=True)
        del p, f, grads
    tot_f = sum(s["forward_ms"] for s in out["samples"])
    tot_b = sum(s["backward_ms"] for s in out["samples"])
    upd = sum(s["updates"] for s in out["samples"])
    out["value"] = upd / ((tot_f + tot_b) / 1e3) / 1e6
    out["forward_mlups_mean"] = float(np.mean([s["forward_mlups"] for s in out["samples"]]))
    out["adjoint_forward_time_ratio"] = tot_b / tot_f
    out["ms_per_step"] = (tot_f + tot_b) / K / len(kfs)
    out["device_gb_before"] = (total - free0) / 1e9
    print(json.dumps(out))
    return 0


def run_poisson_forms(args):
    """The head-on workload in FP64 with each Poisson form (kinetic: the
    production solve; scalar: the reference's scalar Jacobi form; scalar-rb:
    red-black SOR of the same scalar equation), natural exits at the 1e-3
    contract: W warm-up steps, K timed steps per form from the same initial
    fields, device time from the handle's CUDA events.  Reports sweeps per
    step, MLUPS (sweeps counted and the reference definition), the Poisson
    phase's bandwidth on the form's algorithmic bytes (kinetic 272 B, scalar 32
    B per cell and sweep: p in, p out, rho, s) and the error of each form's
    fields after the run against the kinetic form's."""
    import lbm_b200 as L
    n = args.size
    p = workload_params(n)
    f = workload_fields(p)
    cells = float(n ** 3)
    peak, peak_kind = measured_peaks()
    out, fields = {}, {}
    for form in ("kinetic", "scalar", "scalar-rb"):
        g = L.InamuroCUDA(p, f, precision="fp64")
        g.set_poisson(check_interval=100, tolerance=1e-3, max_sweeps=args.max_sweeps)
        g.set_poisson_form(form)
        g.step(args.warmup)
        g.reset_timing()
        clk = ClockSampler(0)
        clk.start()
        stats = g.step(args.steps)
        clocks = clk.stop()
        tm = g.timing()
        dev_s = sum(st["device_ms"] for st in stats) / 1e3
        sweeps = sum(st["iterations"] for st in stats)
        bytes_cell = SWEEP_BYTES["fp64"] if form == "kinetic" else 32.0
        gbs = bytes_cell * cells * sweeps / (tm["poisson_ms"] / 1e3) / 1e9
        out[form] = {"mlups": cells * (args.steps + sweeps) / dev_s / 1e6,
                     "mlups_reference_definition": cells * args.steps / dev_s / 1e6,
                     "ms_per_step": dev_s * 1e3 / args.steps, "sweeps_per_step": sweeps / args.steps,
                     "poisson_ms_per_step": tm["poisson_ms"] / args.steps,
                     "poisson_gbs": gbs, "poisson_frac": gbs / peak, "bytes_per_cell_sweep": bytes_cell,
                     "converged_steps": int(sum(st["converged"] for st in stats)),
                     "omega": g.poisson_form()["omega"], "gpu_launches": tm["kernel_launches"], "clocks": clocks}
        fields[form] = g.download_fields()
        g.close()
    for form in ("scalar", "scalar-rb"):
        out[form]["rel_err_vs_kinetic"] = {k: float(np.max(np.abs(fields[form][k] - fields["kinetic"][k])) /
                                                    np.max(np.abs(fields["kinetic"][k]))) for k in ("phi", "u", "w", "p")}
    out["scalar-rb"]["rel_err_vs_scalar"] = {k: float(np.max(np.abs(fields["scalar-rb"][k] - fields["scalar"][k])) /
                                                      np.max(np.abs(fields["scalar"][k]))) for k in ("phi", "u", "w", "p")}
    line = {"metric": "MLUPS (Poisson sweeps counted) of the Inamuro D3Q15 droplet step per Poisson form",
            "value": out["scalar-rb"]["mlups_reference_definition"], "unit": "MLUPS (reference definition)",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config_dict(n, "fp64"), poisson={"check_interval": 100, "tolerance": 1e-3}),
            "peak": peak, "peak_kind": peak_kind, "forms": out}
    print(json.dumps(line))
    return 0


def run_krylov(args):
    """The kinetic Poisson fixed point by the kinetic sweeps (relative change
    < --kinetic-tol between checks 100 sweeps apart, default --krylov-tol)
    and by BiCGSTAB (residual < --krylov-tol) at each polynomial degree, FP64,
    the head-on workload at --size with the x boundary of --krylov-boundary
    (the reference's slip walls by default): W warm-up steps, K timed steps
    each, device time from the handle's CUDA events; reports sweeps
    (kinetic-map applications) per step, the Poisson time per step and the
    forms' difference after the run.  --krylov-truth-tol t > 0 also runs the
    highest degree to residual t and reports every form's error against it
    (how far each stop leaves p and u from the fixed point)."""
    import lbm_b200 as L
    n = args.size
    p = workload_params(n)
    p.periodic_x = 1 if args.krylov_boundary == "periodic" else 0
    f = workload_fields(p)
    tol = args.krylov_tol
    ktol = args.kinetic_tol if args.kinetic_tol > 0 else tol
    out, fields = {}, {}
    degrees = [int(d) for d in args.krylov_degrees.split(",")]
    forms = ["kinetic"] + [f"krylov_d{d}" for d in degrees]
    if args.krylov_truth_tol > 0:
        forms.append("truth")
    for form in forms:
        g = L.InamuroCUDA(p, f, precision="fp64")
        ftol = ktol if form == "kinetic" else (args.krylov_truth_tol if form == "truth" else tol)
        g.set_poisson(check_interval=100, tolerance=ftol, max_sweeps=args.max_sweeps, fail_on_limit=True)
        if form == "truth":
            form = f"krylov_d{max(degrees)}_truth"
        g.set_poisson_form("kinetic" if form == "kinetic" else "krylov")
        if form != "kinetic":
            g.set_poisson_accel(krylov_degree=int(form.split("_d")[1].split("_")[0]))
        g.step(args.warmup)
        g.reset_timing()
        clk = ClockSampler(0)
        clk.start()
        stats = g.step(args.steps)
        clocks = clk.stop()
        tm = g.timing()
        out[form] = {"sweeps_per_step": sum(st["iterations"] for st in stats) / args.steps,
                     "poisson_ms_per_step": tm["poisson_ms"] / args.steps,
                     "ms_per_step": sum(st["device_ms"] for st in stats) / args.steps,
                     "final_relative": stats[-1]["relative_error"], "clocks": clocks}
        fields[form] = g.download_fields()
        g.close()

    def rel(a, b):
        return {k: float(np.max(np.abs(a[k] - b[k])) / max(float(np.max(np.abs(b[k]))), 1e-300)) for k in L.FIELDS}

    truth = next((form for form in fields if form.endswith("_truth")), None)
    diff = {form: rel(fields[form], fields["kinetic"]) for form in fields if form not in ("kinetic", truth)}
    timed = [form for form in out if form not in ("kinetic", truth)]
    best = min(timed, key=lambda k: out[k]["poisson_ms_per_step"])
    for form in timed:
        out[form]["speedup_vs_kinetic"] = out["kinetic"]["poisson_ms_per_step"] / out[form]["poisson_ms_per_step"]
    if truth:
        for form in out:
            if form != truth:
                out[form]["error_vs_truth"] = rel(fields[form], fields[truth])
    line = {"metric": "Poisson time per step to the kinetic fixed point, kinetic sweeps vs BiCGSTAB",
            "value": out["kinetic"]["poisson_ms_per_step"] / out[best]["poisson_ms_per_step"], "best": best,
            "unit": "speed-up (x)", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config_dict(n, "fp64"), boundary_x=args.krylov_boundary, tolerance=tol,
                           kinetic_tolerance=ktol, truth_tolerance=args.krylov_truth_tol or None),
            "forms": out, "rel_diff_krylov_vs_kinetic": diff}
    print(json.dumps(line))
    return 0


def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    n = args.size
    p = workload_params(n)
    f = workload_fields(p, seed=1234 + rank)
    legs = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    res = {}
    for prec in legs:
        res[prec] = run_leg(args, prec, world, rank, local, p, f, e2e=(prec == legs[0] and not args.no_e2e))
    head = res[legs[0]]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            reps_out, cells, cwall = reference_cpu_samples(n, args.sample_sweeps, 1)
            cpu = cpu_baseline_entry(n, reps_out, cells, cwall, head["sweeps_per_step"], args.sample_sweeps)
        except Exception as e:
            cpu = {"value": None, "unavailable": str(e)[:200]}

    if rank == 0:
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if legs[0] == "fp64" else "f32+f64",
                "data": "synthetic (seeded droplet initial condition, random noise 1e-4 on phi)",
                "config": config_dict(n, legs[0], args.dual),
                "sweeps_per_step": head["sweeps_per_step"],
                "converged_steps": head["converged_steps"],
                "mlups_reference_definition": head["mlups_reference_definition"],
                "gpu_launches": sum(r["gpu_launches"] for r in res.values()),
                "clocks": head["clocks"], "roofline": head["roofline"],
                "phase_ms_per_step": head["phase_ms_per_step"], "wall_s": head["wall_s"],
                "e2e": head.get("e2e"), "cpu_baseline": cpu, "roofline_collide": head.get("roofline_collide")}
        if "mixed" in res and legs[0] != "mixed":
            m = res["mixed"]
            line["mixed"] = {k: m[k] for k in ("value", "ms_per_step", "sweeps_per_step", "converged_steps",
                                               "roofline", "clocks", "phase_ms_per_step")}
            line["mixed"]["dtype"] = "f32 populations + f64 pressure sums/reductions"
            line["mixed"]["stated_error"] = ("<= 1e-5 norm-wise relative error in phi, rho, u, v, w and p vs "
                                             "the FP64 oracle on equal sweep counts, sum(phi) conserved to "
                                             "1e-12 on periodic boxes (tests/test_gpu_mixed.py, "
                                             "tests/test_gpu_parity_large.py)")
            line["speedup_mixed_vs_fp64"] = m["value"] / head["value"]
            if world == 1 and not args.no_accuracy:
                try:
                    line["mixed"]["accuracy"] = accuracy_probe(n, 3, 1000)
                except Exception as e:
                    line["mixed"]["accuracy"] = {"unavailable": str(e)[:200]}
        if world == 1 and not args.no_extras:
            extra_legs(args, line)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def refine_measure(n=64, steps=2, tol=1e-10):
    """The mixed box at a tight Poisson stop (relative change `tol`, check
    100) on the head-on workload at n^3 with the reference's slip walls: the
    FP64 box to 1e-12 as the fixed point, then the FP64 box, the mixed box by
    iterative refinement (LBM_POISSON_REFINE) and the plain mixed box (capped
    at 4x the FP64 box's sweeps; its relative change stalls near 1e-7) to
    `tol`.  Reports sweeps and Poisson ms per step, and each run's max-norm
    relative error in p, u and phi against the fixed point."""
    import lbm_b200 as L
    p = workload_params(n)
    p.DD, p.init_separation = n / 4.0, n / 2.0
    p.periodic_x = 0
    f = workload_fields(p)
    runs = {}
    fields = {}
    cap = 0
    for name, prec, form, t in (("fp64_fixed_point", "fp64", "kinetic", 1e-12), ("fp64", "fp64", "kinetic", tol),
                                ("mixed_refine", "mixed", "refine", tol), ("mixed_plain", "mixed", "kinetic", tol)):
        g = L.InamuroCUDA(p, f, precision=prec)
        limit = cap if name == "mixed_plain" else 10_000_000
        g.set_poisson(check_interval=100, tolerance=t, max_sweeps=limit, fail_on_limit=False)
        if form != "kinetic":
            g.set_poisson_form(form)
        st = g.step(steps)
        tm = g.timing()
        sw = [int(s["iterations"]) for s in st]
        runs[name] = {"sweeps_per_step": sw, "converged": [int(s["converged"]) for s in st],
                      "poisson_ms_per_step": tm["poisson_ms"] / steps,
                      "ms_per_sweep": tm["poisson_ms"] / max(1, sum(sw))}
        fields[name] = g.download_fields()
        g.close()
        if name == "fp64":
            cap = 4 * (max(sw) // 100 + 1) * 100
    ref = fields["fp64_fixed_point"]
    for name in ("fp64", "mixed_refine", "mixed_plain"):
        runs[name]["rel_err_vs_fixed_point"] = {
            k: float(np.max(np.abs(fields[name][k] - ref[k])) / max(float(np.max(np.abs(ref[k]))), 1e-300))
            for k in ("p", "u", "phi")}
    runs["speedup_refine_vs_fp64"] = runs["fp64"]["poisson_ms_per_step"] / runs["mixed_refine"]["poisson_ms_per_step"]
    runs["config"] = {"workload": f"head-on droplet pair {n}^3 (R={n / 8:g}, {n / 2:g} apart, +-0.02, "
                                  f"rho_L/rho_G=100), slip walls", "steps": steps, "tolerance": tol,
                      "check_interval": 100}
    return runs


def extra_legs(args, line):
    """Bounded samples of the other measurements, in the default line: the
    reference's own GPU step beside this library's (reference_gpu), the
    adjoint calibration run with its adjoint/forward cost and finite-difference
    checks (adjoint), the batched droplet oscillation (batch), and the mixed
    box at a tight Poisson stop by iterative refinement (refine)."""
    import copy
    try:
        # 128^3, one step: the reference program needs ~20 ms per sweep at
        # 256^3 (a 256^3 step of 20 000 sweeps takes it 408 s)
        line["reference_gpu"] = reference_gpu_leg(min(args.size, 128), 1)
    except Exception as e:
        line["reference_gpu"] = {"unavailable": str(e)[:300]}
    try:
        a = copy.copy(args)
        a.steps, a.warmup, a.adjoint_krylov = 2, 1, True
        r = adjoint_measure(a)
        line["adjoint"] = {k: r[k] for k in ("value", "unit", "steps", "forward_mlups", "reverse_mlups",
                                             "adjoint_forward_time_ratio", "forward_ms", "backward_ms",
                                             "sweeps_per_step", "gradient_checks", "max_rel_err", "config")}
        line["adjoint"]["sample"] = "2 of the 2000 steps of the 64^3 calibration run, BiCGSTAB adjoint solve"
    except Exception as e:
        line["adjoint"] = {"unavailable": str(e)[:300]}
    try:
        b = copy.copy(args)
        b.steps, b.warmup = 2, 1
        r = batch_measure(b)
        line["batch"] = {k: r[k] for k in ("value", "unit", "steps", "ms_per_step", "sweeps_per_step_mean",
                                           "roofline", "tuning", "gpu_launches", "converged", "config")}
    except Exception as e:
        line["batch"] = {"unavailable": str(e)[:300]}
    try:
        line["refine"] = refine_measure()
    except Exception as e:
        line["refine"] = {"unavailable": str(e)[:300]}


def run_phase_timing(args):
    """Per-kernel device times of the step's non-Poisson kernels with a fixed
    number of sweeps per step (replay), one JSON line per precision: the
    measurement behind the collide/moments/correction roofline fractions."""
    import lbm_b200 as L
    p = workload_params(args.size)
    f = workload_fields(p)
    cells = args.size ** 3
    peak, kind = measured_peaks()
    for prec in (["fp64", "mixed"] if args.precision == "both" else [args.precision]):
        s = L.InamuroCUDA(p, f, precision=prec)
        s.step_replay([args.phase_sweeps] * max(args.warmup, 1))
        s.reset_timing()
        s.step_replay([args.phase_sweeps] * args.steps)
        t = s.timing()
        n = t["steps"]
        out = {"mode": "phase-timing", "precision": prec, "box": [args.size] * 3,
               "sweeps_per_step": args.phase_sweeps, "steps": n, "peak_gbs": peak, "peak_kind": kind}
        for k, b in PHASE_BYTES.items():
            ms = t[k] / n
            out[k] = ms
            out[k.replace("_ms", "_frac")] = b[prec] * cells / (ms / 1e3) / 1e9 / peak
        out["prep_ms"] = t["prep_ms"] / n
        out["sweep_ms"] = t["poisson_ms"] / max(t["sweep_kernels"], 1)
        print(json.dumps(out), flush=True)
        s.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--precision", choices=("both", "fp64", "mixed"), default="both",
                    help="both: FP64 (the drop-in) is the headline value, mixed is reported beside it")
    ap.add_argument("--size", type=int, default=N_SIDE)
    ap.add_argument("--dual", action="store_true",
                    help="also require the kinetic fixed-point residual (GPU production switch)")
    ap.add_argument("--max-sweeps", type=int, default=500000,
                    help="per-step sweep cap (a multiple of 100); reported if reached")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the mixed-vs-FP64 error and mass-drift probe")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the reference-GPU, adjoint and batch samples of the default line")
    ap.add_argument("--sample-sweeps", type=int, default=3)
    ap.add_argument("--sweeps-per-step", type=float, default=DEFAULT_SWEEPS_PER_STEP)
    ap.add_argument("--phase-timing", action="store_true",
                    help="time the non-Poisson kernels per step with --phase-sweeps sweeps per step")
    ap.add_argument("--phase-sweeps", type=int, default=100)
    ap.add_argument("--krylov-tol", type=float, default=1e-10, help="tolerance of the krylov workload")
    ap.add_argument("--kinetic-tol", type=float, default=0.0,
                    help="krylov workload: the kinetic sweeps' relative-change tolerance (0: --krylov-tol)")
    ap.add_argument("--krylov-truth-tol", type=float, default=0.0,
                    help="krylov workload: also solve to this residual and report each form's error against it")
    ap.add_argument("--krylov-boundary", choices=("slip", "periodic"), default="slip",
                    help="krylov workload: x boundary (slip: the reference's walls)")
    ap.add_argument("--krylov-degrees", default="1,4,8",
                    help="krylov workload: polynomial preconditioner degrees to time (1: plain BiCGSTAB)")
    ap.add_argument("--workload", choices=("headon", "batch", "adjoint", "poisson-forms", "krylov",
                                           "coalescence-adjoint"), default="headon",
                    help="batch: the batched droplet oscillation (64 uneven boxes, mixed precision); "
                         "adjoint: the adjoint calibration run (FP64, 64^3), --steps forward steps")
    ap.add_argument("--adjoint-size", type=int, default=64)
    ap.add_argument("--adjoint-forward-tol", type=float, default=1e-10,
                    help="forward Poisson exit (relative change) of the adjoint workload")
    ap.add_argument("--adjoint-tol", type=float, default=1e-13, help="adjoint Poisson exit of the adjoint workload")
    ap.add_argument("--adjoint-krylov", action="store_true",
                    help="adjoint workload: solve the adjoint Poisson problems by BiCGSTAB")
    ap.add_argument("--adjoint-krylov-tol", type=float, default=1e-11)
    ap.add_argument("--adjoint-directions", type=int, default=2,
                    help="seeded random phi_0 directions checked by finite differences")
    ap.add_argument("--coalescence-samples", type=int, default=8,
                    help="coalescence-adjoint workload: kappa_f samples (uniform in [0.04, 0.08])")
    ap.add_argument("--binomial-slots", type=int, default=25,
                    help="coalescence-adjoint workload: binomial checkpoint slots")
    ap.add_argument("--coalescence-ratio", type=float, default=1000.0,
                    help="coalescence-adjoint workload: rho_L / rho_G")
    ap.add_argument("--coalescence-cap", type=int, default=0,
                    help="coalescence-adjoint workload: sweep cap per forward step (0: converge or fail)")
    ap.add_argument("--coalescence-fd", action="store_true",
                    help="coalescence-adjoint workload: finite-difference check of dJ/dk_f (FP64 forward)")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--batch-seed", type=int, default=2024)
    args = ap.parse_args(argv)
    if args.warmup < 0 or args.steps < 1:
        ap.error("steps >= 1, warmup >= 0")
    if args.phase_timing:
        return run_phase_timing(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "coalescence-adjoint":
        return run_coalescence_adjoint(args)
    if args.workload == "poisson-forms":
        return run_poisson_forms(args)
    if args.workload == "krylov":
        return run_krylov(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

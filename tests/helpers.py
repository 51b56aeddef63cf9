"""Shared helpers of the test suite (fixtures, params, comparisons)."""
from __future__ import annotations

import hashlib
import os
import tempfile

import numpy as np

import lbm_b200 as L

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(name: str):
    return np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)


def params_from_text(text: str) -> L.Params:
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write(str(text))
        path = f.name
    try:
        return L.params_load(path)
    finally:
        os.unlink(path)


def oracle_params(p: L.Params) -> dict:
    return {k: getattr(p, k) for k in ("rho_L", "rho_G", "mu_L", "mu_G", "tauf", "taug", "k_f",
                                       "k_g", "T", "a", "b", "fei_L", "fei_G")}


def fields_dict(arr6) -> dict:
    return {k: np.ascontiguousarray(arr6[i]) for i, k in enumerate(L.FIELDS)}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Norm-wise relative error max|a-b| / max|b| (0 when both are zero)."""
    scale = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(a - b)))
    if scale == 0.0:
        return d
    return d / scale


def laplace_case(shape, DD, noise=1e-4, seed=1, rho=(50.0, 1.0), kappa=(0.06, 6e-6)):
    """Laplace-test physics (single tanh drop, W = 4 <-> interface_width 2)."""
    p = L.make_params(lx=shape[0], ly=shape[1], lz=shape[2], rho_L=rho[0], rho_G=rho[1],
                      mu_L=0.1 * rho[0], mu_G=0.1 * rho[1], k_f=kappa[0], k_g=kappa[1],
                      DD=DD, init_single_droplet=1, init_tanh=1, init_velocity=0.0,
                      interface_width=2.0)
    f = L.init_droplets(p)
    if noise:
        f["phi"] = f["phi"] + np.random.default_rng(seed).uniform(-noise, noise, f["phi"].shape)
    return p, f

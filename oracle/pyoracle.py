"""ctypes wrapper of the FP64 C restatement (oracle/lbm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the lbm_b200 package.

Fields are numpy float64 arrays of shape (lz, ly, lx) (x fastest), the same
memory order as the CUDA library's physical-domain fields.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblbm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

PARAM_KEYS = ("rho_L", "rho_G", "mu_L", "mu_G", "tauf", "taug", "k_f", "k_g",
              "T", "a", "b", "fei_L", "fei_G")


class OrcParams(C.Structure):
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int)] + \
        [(k, C.c_double) for k in PARAM_KEYS] + \
        [("check_interval", C.c_int), ("tol", C.c_double), ("dual", C.c_int),
         ("max_sweeps", C.c_uint64), ("periodic_x", C.c_int), ("poisson_form", C.c_int),
         ("scalar_source_scale", C.c_double), ("pressure_relax_scale", C.c_double),
         ("fixed_point_relax", C.c_double), ("anderson_m1", C.c_int), ("anderson_beta_max", C.c_double),
         ("two_grid", C.c_int), ("two_grid_strength", C.c_double), ("source_aware_init", C.c_int),
         ("source_aware_scale", C.c_double)]


class OrcStepInfo(C.Structure):
    _fields_ = [("sweeps", C.c_uint64)] + [(k, C.c_double) for k in (
        "relative_error", "pressure_l1_delta", "pressure_l1_norm",
        "fp_h_l1", "fp_h_scale", "fp_h_rel", "fp_p_l1", "fp_p_scale", "fp_p_rel",
        "fp_rel", "divergence_mean", "gauge_target", "gauge_max_shift", "mass")]


_lib = None


# Where the reference checkout is read from when LBM_REFERENCE_DIR is unset
# (the build container's read-only copy; absent on machines without it).
DEFAULT_REFERENCE_DIR = "/root/reference"


def build() -> None:
    """Compiles the restatement (and, where the reference checkout exists, the
    reference harnesses) with oracle/Makefile."""
    env = dict(os.environ)
    env["CC"] = "gcc"   # the system gcc ships libgomp
    env["CXX"] = "g++"
    env.setdefault("LBM_REFERENCE_DIR", DEFAULT_REFERENCE_DIR)
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True, env=env)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams)] + [dp] * 6
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.restype = C.c_int
        L.orc_step.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(OrcStepInfo)]
        L.orc_get_fields.argtypes = [C.c_void_p] + [dp] * 6
        L.orc_get_populations.argtypes = [C.c_void_p] + [dp] * 3
        L.orc_get_derivatives.argtypes = [C.c_void_p, dp]
        L.orc_init_droplets.argtypes = [C.c_int] * 3 + [C.c_double] * 5 + [C.c_int] * 2 + \
            [C.c_double] * 7 + [dp] * 3
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    def __init__(self, code: int):
        super().__init__(f"oracle step failed with status {code}")
        self.code = code


class Oracle:
    """One FP64 reference-order solver instance."""

    def __init__(self, shape, params: Dict[str, float], fields: Dict[str, np.ndarray],
                 check_interval: int = 100, tol: float = 1e-3, dual: bool = False,
                 max_sweeps: int = 0, periodic_x: bool = False, poisson_form: int = 0,
                 scalar_source_scale: float = 2.0, accel: Dict[str, float] = None):
        lx, ly, lz = shape
        self.shape = (lz, ly, lx)
        prm = OrcParams(lx=lx, ly=ly, lz=lz, check_interval=check_interval, tol=tol,
                        dual=int(dual), max_sweeps=max_sweeps, periodic_x=int(periodic_x),
                        poisson_form=int(poisson_form), scalar_source_scale=float(scalar_source_scale),
                        **dict({"pressure_relax_scale": 1.0, "fixed_point_relax": 1.0, "anderson_beta_max": 1.0,
                                "two_grid_strength": 0.5, "source_aware_scale": 1.0}, **(accel or {})),
                        **{k: float(params[k]) for k in PARAM_KEYS})
        arrs = [np.ascontiguousarray(fields[k], dtype=np.float64).reshape(self.shape)
                for k in ("phi", "rho", "u", "v", "w")]
        p = fields.get("p")
        p = None if p is None else np.ascontiguousarray(p, dtype=np.float64).reshape(self.shape)
        self._h = lib().orc_create(C.byref(prm), *[_ptr(a) for a in arrs], _ptr(p))
        if not self._h:
            raise ValueError("orc_create rejected the parameters")

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, replay: int = 0) -> Dict[str, float]:
        info = OrcStepInfo()
        st = lib().orc_step(self._h, replay, C.byref(info))
        if st != 0:
            raise OracleError(st)
        return {k: getattr(info, k) for k, _ in OrcStepInfo._fields_}

    def fields(self) -> Dict[str, np.ndarray]:
        out = {k: np.empty(self.shape) for k in ("phi", "rho", "u", "v", "w", "p")}
        lib().orc_get_fields(self._h, *[_ptr(out[k]) for k in ("phi", "rho", "u", "v", "w", "p")])
        return out

    def populations(self):
        f, g, h = (np.empty((15,) + self.shape) for _ in range(3))
        lib().orc_get_populations(self._h, _ptr(f), _ptr(g), _ptr(h))
        return f, g, h

    def derivatives(self) -> np.ndarray:
        d = np.empty((19,) + self.shape)
        lib().orc_get_derivatives(self._h, _ptr(d))
        return d


def init_droplets(shape, DD, fei_max, fei_min, rho_L, rho_G, single=False, tanh=False,
                  velocity=0.035, width=2.0, center=(-1.0, -1.0, -1.0), separation=-1.0,
                  offset_x=0.0) -> Dict[str, np.ndarray]:
    """GPU/Inamuro.cpp:491-566 restated (see lbm_oracle.c).  Returns the five
    macro fields plus p = 0."""
    lx, ly, lz = shape
    phi = np.full((lz, ly, lx), fei_min)
    rho = np.full((lz, ly, lx), rho_G)
    w = np.zeros((lz, ly, lx))
    lib().orc_init_droplets(lx, ly, lz, DD, fei_max, fei_min, rho_L, rho_G, int(single),
                            int(tanh), velocity, width, center[0], center[1], center[2],
                            separation, offset_x, _ptr(phi), _ptr(rho), _ptr(w))
    z = np.zeros((lz, ly, lx))
    return {"phi": phi, "rho": rho, "u": z.copy(), "v": z.copy(), "w": w, "p": z.copy()}

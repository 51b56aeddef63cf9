"""lbm_b200 -- B200 (sm_100a) Inamuro two-phase D3Q15 droplet step.

Python view of the C ABI in include/lbm_b200.h (ctypes over the in-tree
liblbm_b200.so).  The class `InamuroCUDA` mirrors the reference's C++ class of
the same name (GPU/InamuroCUDA.hpp:16-91): construct from parameters and
initial fields, `perform_time_step_gpu()`, `download_fields()`,
`download_hh()`, `synchronize()`, `last_poisson_diagnostics`, and the Poisson
convergence setters.  Failures raise `LBMError` (the reference throws
std::runtime_error / std::invalid_argument).

There is no CPU fallback: without the CUDA library or an sm_100 GPU every
solver call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "lbm_b200.h")

FIELDS = ("phi", "rho", "u", "v", "w", "p")
FIELD_ID = {k: i for i, k in enumerate(FIELDS)}

STATUS = {0: "LBM_OK", 1: "LBM_ERR_CUDA", 2: "LBM_ERR_NONFINITE", 3: "LBM_ERR_POISSON_BUDGET",
          4: "LBM_ERR_BAD_ARG", 5: "LBM_ERR_OOM", 6: "LBM_ERR_IO", 7: "LBM_ERR_NO_DEVICE",
          8: "LBM_ERR_OVERFLOW"}


class Params(C.Structure):
    """lbm_params: the params.in contents (GPU/Inamuro.hpp:36-76)."""
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int), ("period", C.c_int),
                ("t_max", C.c_int), ("nwri", C.c_int)] + \
        [(k, C.c_double) for k in ("rho_L", "rho_G", "tauf", "taug", "mu_L", "mu_G", "k_f", "k_g",
                                    "T", "a", "b", "fei_max", "fei_min", "fei_L", "fei_G", "DD")] + \
        [("init_single_droplet", C.c_int), ("init_tanh", C.c_int)] + \
        [(k, C.c_double) for k in ("init_velocity", "interface_width", "init_center_x",
                                    "init_center_y", "init_center_z", "init_separation",
                                    "init_offset_x")] + \
        [("periodic_x", C.c_int)]

    @property
    def shape(self):
        return (self.lx, self.ly, self.lz)

    def as_dict(self) -> Dict[str, float]:
        return {k: getattr(self, k) for k, _ in self._fields_}


class PoissonCfg(C.Structure):
    _fields_ = [("check_interval", C.c_int), ("tolerance", C.c_double), ("dual_residual", C.c_int),
                ("max_sweeps", C.c_uint64), ("fail_on_limit", C.c_int)]


class StepStats(C.Structure):
    """lbm_step_stats: InamuroCUDA::PoissonStepDiagnostics + mass + device time."""
    _fields_ = [("iterations", C.c_uint64)] + \
        [(k, C.c_double) for k in (
            "relative_error", "pressure_l1_delta", "pressure_l1_norm",
            "fixed_point_h_l1", "fixed_point_h_scale", "fixed_point_h_relative",
            "fixed_point_p_l1", "fixed_point_p_scale", "fixed_point_p_relative",
            "fixed_point_relative", "source_mean", "source_abs_mean", "projected_source_mean",
            "pressure_gauge_target", "pressure_gauge_max_shift", "mass")] + \
        [(k, C.c_int) for k in ("fixed_point_evaluated", "pressure_converged",
                                 "fixed_point_converged", "dual_residual_enabled", "converged",
                                 "reserved")] + [("device_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timing(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("collide_ms", "moments_ms", "prep_ms", "poisson_ms",
                                           "correct_ms")] + \
        [(k, C.c_uint64) for k in ("steps", "sweeps", "sweep_kernels", "kernel_launches", "fused_sweeps")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchTuning(C.Structure):
    """lbm_batch_tuning: launch shape of the batched kernels."""
    _fields_ = [("tile_x", C.c_int), ("tile_y", C.c_int), ("zrun", C.c_int), ("ctas_per_sm", C.c_int),
                ("sweep2_zrun", C.c_int), ("reserved", C.c_int), ("sweep_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FieldStats(C.Structure):
    """lbm_field_stats: Inamuro::FieldStatistics (CPU/Inamuro.hpp:91-99) + sum."""
    _fields_ = [(k, C.c_double) for k in ("min", "max", "mean", "abs_max")] + \
        [("nan_count", C.c_uint64), ("inf_count", C.c_uint64), ("sum", C.c_double),
         ("valid_count", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Diagnostics(C.Structure):
    """lbm_diagnostics: Inamuro::DiagnosticsSnapshot (CPU/Inamuro.cpp:412-507)."""
    NAMES = ("rho", "fei", "u", "v", "w", "velocity_magnitude", "p")
    _fields_ = [(k, FieldStats) for k in NAMES]

    def as_dict(self):
        return {k: getattr(self, k).as_dict() for k in self.NAMES}


class PoissonAccel(C.Structure):
    """lbm_poisson_accel: the reference's Poisson accelerator settings."""
    _fields_ = [("pressure_relax_scale", C.c_double), ("fixed_point_relax", C.c_double),
                ("anderson_m1", C.c_int), ("anderson_beta_max", C.c_double), ("two_grid", C.c_int),
                ("two_grid_strength", C.c_double), ("source_aware_init", C.c_int),
                ("source_aware_scale", C.c_double), ("spatial_diagnostics", C.c_int), ("krylov_degree", C.c_int)]


class AdjointCfg(C.Structure):
    """lbm_adjoint_cfg: checkpoint interval and the adjoint Poisson solve's exit."""
    _fields_ = [("checkpoint_interval", C.c_int), ("check_interval", C.c_int), ("tolerance", C.c_double),
                ("max_sweeps", C.c_uint64), ("binomial_checkpoints", C.c_int), ("krylov", C.c_int),
                ("krylov_tolerance", C.c_double), ("precision", C.c_int)]


class AdjointStats(C.Structure):
    """lbm_adjoint_stats."""
    _fields_ = [("grad_kappa_f", C.c_double)] + \
        [(k, C.c_uint64) for k in ("forward_steps", "forward_sweeps", "recompute_steps", "adjoint_sweeps")] + \
        [("forward_ms", C.c_double), ("backward_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LBMError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        name = STATUS.get(status, str(status))
        super().__init__(f"{name}: {message}" if message else name)
        self.status = status
        self.name = name


_lib = None
# LBM_B200_ABI_VERSION of include/lbm_b200.h that the structures above mirror.
ABI_VERSION = 6


def load_library(path: str = LIB_PATH):
    """Loads liblbm_b200.so (raises if it was not built: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LBMError(7, f"CUDA library missing at {path}; run lbm_b200.build.build()")
    L = C.CDLL(path)
    dp = C.POINTER(C.c_double)
    H = C.c_void_p
    L.lbm_params_default.argtypes = [C.POINTER(Params)]
    L.lbm_params_default.restype = None
    L.lbm_params_load.argtypes = [C.c_char_p, C.POINTER(Params)]
    L.lbm_init_droplets.argtypes = [C.POINTER(Params)] + [dp] * 6
    L.lbm_create.argtypes = [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(H)]
    L.lbm_destroy.argtypes = [H]
    L.lbm_destroy.restype = None
    for name in ("lbm_load_fields", "lbm_load_fields_ghosted", "lbm_load_fields_device"):
        getattr(L, name).argtypes = [H] + [C.c_void_p] * 6
    L.lbm_set_poisson.argtypes = [H, C.POINTER(PoissonCfg)]
    L.lbm_get_poisson.argtypes = [H, C.POINTER(PoissonCfg)]
    L.lbm_set_poisson_form.argtypes = [H, C.c_int, C.c_double, C.c_double]
    L.lbm_get_poisson_form.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.lbm_set_poisson_accel.argtypes = [H, C.POINTER(PoissonAccel)]
    L.lbm_get_poisson_accel.argtypes = [H, C.POINTER(PoissonAccel)]
    L.lbm_step.argtypes = [H, C.c_int, C.POINTER(StepStats)]
    L.lbm_step_replay.argtypes = [H, C.c_int, C.POINTER(C.c_uint64), C.POINTER(StepStats)]
    L.lbm_download.argtypes = [H, C.c_int, dp]
    L.lbm_download_ghosted.argtypes = [H, C.c_int, dp]
    L.lbm_download_h.argtypes = [H, dp]
    L.lbm_field_device_ptr.argtypes = [H, C.c_int, C.POINTER(C.c_void_p)]
    L.lbm_synchronize.argtypes = [H]
    L.lbm_field_statistics.argtypes = [H, C.c_int, C.POINTER(FieldStats)]
    L.lbm_field_statistics_noalloc.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p,
                                               C.POINTER(FieldStats)]
    L.lbm_diagnostics_snapshot.argtypes = [H, C.POINTER(Diagnostics)]
    L.lbm_get_timing.argtypes = [H, C.POINTER(Timing)]
    L.lbm_reset_timing.argtypes = [H]
    L.lbm_set_timing.argtypes = [H, C.c_int]
    L.lbm_last_error.argtypes = [H]
    L.lbm_last_error.restype = C.c_char_p
    L.lbm_status_string.argtypes = [C.c_int]
    L.lbm_status_string.restype = C.c_char_p
    L.lbm_abi_version.restype = C.c_int
    L.lbm_selftest_division.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
    B = C.c_void_p
    L.lbm_batch_create.argtypes = [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(B)]
    L.lbm_batch_destroy.argtypes = [B]
    L.lbm_batch_destroy.restype = None
    L.lbm_batch_size.argtypes = [B]
    L.lbm_batch_load_fields.argtypes = [B, C.c_int] + [C.c_void_p] * 6
    L.lbm_batch_set_poisson.argtypes = [B, C.POINTER(PoissonCfg)]
    L.lbm_batch_step.argtypes = [B, C.c_int, C.POINTER(StepStats)]
    L.lbm_batch_step_replay.argtypes = [B, C.c_int, C.POINTER(C.c_uint64), C.POINTER(StepStats)]
    L.lbm_batch_download.argtypes = [B, C.c_int, C.c_int, dp]
    L.lbm_batch_tune.argtypes = [B, C.POINTER(BatchTuning)]
    L.lbm_batch_set_tuning.argtypes = [B, C.POINTER(BatchTuning)]
    L.lbm_batch_get_tuning.argtypes = [B, C.POINTER(BatchTuning)]
    L.lbm_batch_get_timing.argtypes = [B, C.POINTER(Timing)]
    L.lbm_batch_reset_timing.argtypes = [B]
    L.lbm_batch_last_error.argtypes = [B]
    L.lbm_batch_last_error.restype = C.c_char_p
    for name, n_ptr in (("lbm_collide_forward", 12), ("lbm_collide_backward", 19), ("lbm_moments_forward", 7),
                        ("lbm_moments_backward", 8), ("lbm_correct_forward", 5), ("lbm_correct_backward", 7)):
        getattr(L, name).argtypes = [C.POINTER(Params)] + [C.c_void_p] * n_ptr
    A = C.c_void_p
    L.lbm_adjoint_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(AdjointCfg), C.POINTER(A)]
    L.lbm_adjoint_destroy.argtypes = [A]
    L.lbm_adjoint_destroy.restype = None
    L.lbm_adjoint_set_poisson.argtypes = [A, C.POINTER(PoissonCfg)]
    L.lbm_adjoint_forward.argtypes = [A] + [C.c_void_p] * 6 + [C.c_int, C.POINTER(C.c_uint64)]
    L.lbm_adjoint_sweeps.argtypes = [A, C.POINTER(C.c_uint64)]
    L.lbm_adjoint_download.argtypes = [A, C.c_int, dp]
    L.lbm_adjoint_backward.argtypes = [A] + [C.c_void_p] * 12 + [C.POINTER(AdjointStats)]
    L.lbm_adjoint_last_error.argtypes = [A]
    L.lbm_adjoint_last_error.restype = C.c_char_p
    L.lbm_adjoint_schedule.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
    if L.lbm_abi_version() != ABI_VERSION:
        raise LBMError(7, f"{path} has ABI {L.lbm_abi_version()}, these bindings expect {ABI_VERSION}; "
                          "rebuild with lbm_b200.build.build()")
    _lib = L
    return L


def header_functions(path: str = HEADER_PATH) -> List[str]:
    """Names of the functions declared in include/lbm_b200.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def params_default() -> Params:
    p = Params()
    load_library().lbm_params_default(C.byref(p))
    return p


def params_load(path: str) -> Params:
    """Parses a params.in file (Inamuro::Parameters(const std::string&))."""
    p = Params()
    st = load_library().lbm_params_load(str(path).encode(), C.byref(p))
    if st != 0:
        raise LBMError(st, f"cannot parse {path}")
    return p


def make_params(**kw) -> Params:
    p = params_default()
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def init_droplets(p: Params) -> Dict[str, np.ndarray]:
    """Inamuro::initializeDroplets (GPU/Inamuro.cpp:491-566) on the host.
    Returns phi, rho, u, v, w, p of shape (lz, ly, lx)."""
    shape = (p.lz, p.ly, p.lx)
    out = {k: np.empty(shape) for k in FIELDS}
    st = load_library().lbm_init_droplets(C.byref(p), *[_dp(out[k]) for k in FIELDS])
    if st != 0:
        raise LBMError(st, "init_droplets")
    return out


NOALLOC_MAX_CELLS = 33554432  # LBM_NOALLOC_MAX_CELLS


def field_statistics_noalloc(dev_ptr: int, n_cells: int, stream: Optional[int] = None) -> Dict[str, float]:
    """lbm_field_statistics_noalloc: statistics of a caller-owned device field
    (doubles on the current device) computed without any device allocation.
    For callers that must not allocate (pre-reserved memory pools, loops where
    cudaMalloc's device-wide synchronisation is not allowed, plugins without an
    allocator).  The library's static scratch is shared by all calls on a
    device, so calls must not overlap on the GPU; the first call on a device
    should come before any stream capture."""
    if n_cells > NOALLOC_MAX_CELLS:
        raise LBMError(4, f"{n_cells} cells exceed the no-alloc maximum of {NOALLOC_MAX_CELLS}")
    st = FieldStats()
    code = load_library().lbm_field_statistics_noalloc(dev_ptr, n_cells, stream, C.byref(st))
    if code != 0:
        raise LBMError(code, "field_statistics_noalloc")
    return st.as_dict()


PRECISION = {"fp64": 0, "mixed": 1}


class InamuroCUDA:
    """One box on one GPU (GPU/InamuroCUDA.hpp:16-91)."""

    def __init__(self, params: Params, fields: Optional[Dict[str, np.ndarray]] = None,
                 precision: str = "fp64", device: int = 0):
        self._lib = load_library()
        self.params = params
        self.shape = (params.lz, params.ly, params.lx)
        self.precision = precision
        h = C.c_void_p()
        st = self._lib.lbm_create(C.byref(params), PRECISION[precision], device, C.byref(h))
        if st != 0:
            why = self._lib.lbm_last_error(None)
            raise LBMError(st, "lbm_create: " + (why.decode() if why else ""))
        self._h = h
        self.last_poisson_diagnostics: Dict[str, float] = {}
        if fields is not None:
            self.load_fields(fields)

    # -- errors ----------------------------------------------------------
    def _check(self, st: int, what: str):
        if st != 0:
            msg = self._lib.lbm_last_error(self._h)
            raise LBMError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state transfer ---------------------------------------------------
    def _arrs(self, fields, ghosted=False):
        shape = (self.shape[0] + 2,) + self.shape[1:] if ghosted else self.shape
        out = []
        for k in FIELDS:
            a = fields.get(k)
            if a is None:
                out.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(shape)
            out.append(a)
        return out

    def load_fields(self, fields: Dict[str, np.ndarray]):
        """InamuroCUDA::initFromCPU: uploads phi, rho, u, v, w (and p)."""
        arrs = self._arrs(fields)
        self._keep = arrs
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self._check(self._lib.lbm_load_fields(self._h, *ptrs), "load_fields")

    def load_fields_ghosted(self, fields: Dict[str, np.ndarray]):
        arrs = self._arrs(fields, ghosted=True)
        self._check(self._lib.lbm_load_fields_ghosted(self._h, *[a.ctypes.data for a in arrs]),
                    "load_fields_ghosted")

    def load_fields_device(self, ptrs: Sequence[int]):
        """Device pointers (ints) of phi, rho, u, v, w, p on this handle's GPU."""
        self._check(self._lib.lbm_load_fields_device(self._h, *ptrs), "load_fields_device")

    def download(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape)
        self._check(self._lib.lbm_download(self._h, FIELD_ID[name], _dp(out)), "download")
        return out

    def download_fields(self) -> Dict[str, np.ndarray]:
        """InamuroCUDA::downloadFieldsToCPU (physical layout)."""
        return {k: self.download(k) for k in FIELDS}

    def download_ghosted(self, name: str) -> np.ndarray:
        out = np.empty((self.shape[0] + 2,) + self.shape[1:])
        self._check(self._lib.lbm_download_ghosted(self._h, FIELD_ID[name], _dp(out)), "download_ghosted")
        return out

    def download_hh(self) -> np.ndarray:
        """InamuroCUDA::downloadHH: AoS cell*15+q."""
        out = np.empty(15 * int(np.prod(self.shape)))
        self._check(self._lib.lbm_download_h(self._h, _dp(out)), "download_hh")
        return out

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        self._check(self._lib.lbm_field_device_ptr(self._h, FIELD_ID[name], C.byref(p)), "device_ptr")
        return p.value

    def synchronize(self):
        self._check(self._lib.lbm_synchronize(self._h), "synchronize")

    def field_statistics(self, name: str) -> Dict[str, float]:
        """Device-side Inamuro::collectDiagnostics statistics of one field."""
        st = FieldStats()
        self._check(self._lib.lbm_field_statistics(self._h, FIELD_ID[name], C.byref(st)),
                    "field_statistics")
        return st.as_dict()

    def diagnostics(self) -> Dict[str, Dict[str, float]]:
        """Inamuro::collectDiagnostics on the device (lbm_diagnostics_snapshot)."""
        d = Diagnostics()
        self._check(self._lib.lbm_diagnostics_snapshot(self._h, C.byref(d)), "diagnostics_snapshot")
        return d.as_dict()

    # -- Poisson configuration --------------------------------------------
    def set_poisson(self, check_interval: int = 100, tolerance: float = 1e-3, dual: bool = False,
                    max_sweeps: int = 0, fail_on_limit: bool = False):
        cfg = PoissonCfg(check_interval, tolerance, int(dual), max_sweeps, int(fail_on_limit))
        self._check(self._lib.lbm_set_poisson(self._h, C.byref(cfg)), "set_poisson")

    POISSON_FORMS = {"kinetic": 0, "scalar": 1, "scalar-rb": 2, "onepass": 3, "krylov": 4, "varcoef-rb": 5, "refine": 6}

    def set_poisson_form(self, form: str = "kinetic", source_scale: float = 2.0, omega: float = 0.0):
        """lbm_set_poisson_form: "kinetic" (the production solve), "scalar"
        (the reference's scalar Jacobi form), "scalar-rb" (red-black SOR of
        the same scalar equation; omega 0 = the optimum for the box),
        "onepass" (the reference's one-pass form), "krylov" (BiCGSTAB on the
        kinetic fixed point), "varcoef-rb" (red-black SOR of
        div((1/rho) grad p) = s) or, on the mixed box, "refine" (the kinetic
        form by iterative refinement: FP64 residual, FP32 correction sweeps)."""
        self._check(self._lib.lbm_set_poisson_form(self._h, self.POISSON_FORMS[form], source_scale, omega),
                    "set_poisson_form")

    def set_poisson_accel(self, **kw):
        """lbm_set_poisson_accel: the reference's accelerators (pressure_relax_scale,
        fixed_point_relax, anderson_m1, anderson_beta_max, two_grid,
        two_grid_strength, source_aware_init, source_aware_scale), plus
        krylov_degree (the Neumann polynomial degree of the BiCGSTAB form, 0/1
        = plain, at most 16); unnamed settings keep their current values."""
        a = PoissonAccel()
        self._check(self._lib.lbm_get_poisson_accel(self._h, C.byref(a)), "get_poisson_accel")
        for k, v in kw.items():
            if not any(k == f for f, _ in PoissonAccel._fields_):
                raise KeyError(k)
            setattr(a, k, v)
        self._check(self._lib.lbm_set_poisson_accel(self._h, C.byref(a)), "set_poisson_accel")

    def poisson_form(self) -> Dict[str, float]:
        f, sc, om = C.c_int(), C.c_double(), C.c_double()
        self._check(self._lib.lbm_get_poisson_form(self._h, C.byref(f), C.byref(sc), C.byref(om)),
                    "get_poisson_form")
        names = {v: k for k, v in self.POISSON_FORMS.items()}
        return {"form": names[f.value], "source_scale": sc.value, "omega": om.value}

    # reference setter names (GPU/InamuroCUDA.hpp:83-86)
    def set_poisson_convergence(self, check_interval: int, tolerance: float):
        cfg = self.poisson_config()
        self.set_poisson(check_interval, tolerance, cfg["dual_residual"], cfg["max_sweeps"],
                         cfg["fail_on_limit"])

    def set_use_poisson_dual_residual(self, enabled: bool):
        cfg = self.poisson_config()
        self.set_poisson(cfg["check_interval"], cfg["tolerance"], enabled, cfg["max_sweeps"],
                         cfg["fail_on_limit"])

    def set_poisson_iteration_limit(self, max_iterations: int):
        cfg = self.poisson_config()
        self.set_poisson(cfg["check_interval"], cfg["tolerance"], cfg["dual_residual"],
                         max_iterations, cfg["fail_on_limit"])

    def poisson_config(self) -> Dict[str, float]:
        cfg = PoissonCfg()
        self._check(self._lib.lbm_get_poisson(self._h, C.byref(cfg)), "get_poisson")
        return {k: getattr(cfg, k) for k, _ in cfg._fields_}

    # -- stepping ---------------------------------------------------------
    def step(self, n: int = 1) -> List[Dict[str, float]]:
        stats = (StepStats * max(n, 1))()
        self._check(self._lib.lbm_step(self._h, n, stats), "step")
        out = [s.as_dict() for s in stats[:n]]
        if out:
            self.last_poisson_diagnostics = out[-1]
        return out

    def perform_time_step_gpu(self) -> Dict[str, float]:
        """InamuroCUDA::performTimeStepGPU."""
        return self.step(1)[0]

    def step_replay(self, sweeps: Sequence[int]) -> List[Dict[str, float]]:
        n = len(sweeps)
        arr = (C.c_uint64 * n)(*sweeps)
        stats = (StepStats * max(n, 1))()
        self._check(self._lib.lbm_step_replay(self._h, n, arr, stats), "step_replay")
        return [s.as_dict() for s in stats[:n]]

    # -- timing -----------------------------------------------------------
    def timing(self) -> Dict[str, float]:
        t = Timing()
        self._check(self._lib.lbm_get_timing(self._h, C.byref(t)), "timing")
        return t.as_dict()

    def reset_timing(self):
        self._check(self._lib.lbm_reset_timing(self._h), "reset_timing")

    def set_timing(self, enabled: bool):
        self._check(self._lib.lbm_set_timing(self._h, int(enabled)), "set_timing")


class Batch:
    """Many independent mixed-precision boxes advanced together (lbm_batch_*):
    one entry of `params` per instance, each with its own box and physics."""

    def __init__(self, params: Sequence[Params], fields: Optional[Sequence[Dict[str, np.ndarray]]] = None,
                 device: int = 0):
        self._lib = load_library()
        self.params = list(params)
        arr = (Params * len(self.params))(*self.params)
        h = C.c_void_p()
        st = self._lib.lbm_batch_create(arr, len(self.params), device, C.byref(h))
        if st != 0:
            why = self._lib.lbm_batch_last_error(None)
            raise LBMError(st, "lbm_batch_create: " + (why.decode() if why else ""))
        self._h = h
        if fields is not None:
            for i, f in enumerate(fields):
                self.load_fields(i, f)

    def _check(self, st: int, what: str):
        if st != 0:
            msg = self._lib.lbm_batch_last_error(self._h)
            raise LBMError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.params)

    def shape(self, i: int):
        p = self.params[i]
        return (p.lz, p.ly, p.lx)

    def load_fields(self, i: int, fields: Dict[str, np.ndarray]):
        arrs = []
        for k in FIELDS:
            a = fields.get(k)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.size != np.prod(self.shape(i)):
                    raise LBMError(4, f"field {k} of instance {i} has {a.size} values, box has {np.prod(self.shape(i))}")
            arrs.append(a)
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        self._check(self._lib.lbm_batch_load_fields(self._h, i, *ptrs), "batch_load_fields")

    def set_poisson(self, check_interval: int = 100, tolerance: float = 1e-3, max_sweeps: int = 0,
                    fail_on_limit: bool = False):
        cfg = PoissonCfg(check_interval, tolerance, 0, max_sweeps, int(fail_on_limit))
        self._check(self._lib.lbm_batch_set_poisson(self._h, C.byref(cfg)), "batch_set_poisson")

    def step(self, n: int = 1) -> List[List[Dict[str, float]]]:
        """n steps; returns [step][instance] diagnostics."""
        m = len(self)
        stats = (StepStats * max(n * m, 1))()
        self._check(self._lib.lbm_batch_step(self._h, n, stats), "batch_step")
        return [[stats[s * m + i].as_dict() for i in range(m)] for s in range(n)]

    def step_replay(self, sweeps: Sequence[Sequence[int]]) -> List[List[Dict[str, float]]]:
        """One step per row of `sweeps` (one count per instance)."""
        m = len(self)
        n = len(sweeps)
        flat = [int(c) for row in sweeps for c in row]
        if len(flat) != n * m:
            raise LBMError(4, "one sweep count per step and instance")
        arr = (C.c_uint64 * len(flat))(*flat)
        stats = (StepStats * max(n * m, 1))()
        self._check(self._lib.lbm_batch_step_replay(self._h, n, arr, stats), "batch_step_replay")
        return [[stats[s * m + i].as_dict() for i in range(m)] for s in range(n)]

    def download(self, i: int, name: str) -> np.ndarray:
        out = np.empty(self.shape(i), dtype=np.float64)
        self._check(self._lib.lbm_batch_download(self._h, i, FIELD_ID[name], _dp(out)), "batch_download")
        return out

    def download_fields(self, i: int) -> Dict[str, np.ndarray]:
        return {k: self.download(i, k) for k in FIELDS}

    def tune(self) -> Dict[str, float]:
        t = BatchTuning()
        self._check(self._lib.lbm_batch_tune(self._h, C.byref(t)), "batch_tune")
        return t.as_dict()

    def set_tuning(self, tile_x: int, tile_y: int, zrun: int, ctas_per_sm: int, sweep2_zrun: int = 0):
        t = BatchTuning(tile_x, tile_y, zrun, ctas_per_sm, sweep2_zrun, 0, 0.0)
        self._check(self._lib.lbm_batch_set_tuning(self._h, C.byref(t)), "batch_set_tuning")

    def tuning(self) -> Dict[str, float]:
        t = BatchTuning()
        self._check(self._lib.lbm_batch_get_tuning(self._h, C.byref(t)), "batch_get_tuning")
        return t.as_dict()

    def timing(self) -> Dict[str, float]:
        t = Timing()
        self._check(self._lib.lbm_batch_get_timing(self._h, C.byref(t)), "batch_timing")
        return t.as_dict()

    def reset_timing(self):
        self._check(self._lib.lbm_batch_reset_timing(self._h), "batch_reset_timing")


def selftest_division(samples: int = 1 << 30, seed: int = 12345) -> int:
    """lbm_selftest_division: number of pseudo-random operand pairs for which
    the FP64 kernels' division from a reciprocal differs from IEEE a/b."""
    lib = load_library()
    out = C.c_uint64(0)
    st = lib.lbm_selftest_division(samples, seed, C.byref(out))
    if st != 0:
        raise LBMError(st, "lbm_selftest_division")
    return int(out.value)


# ---- adjoints of the explicit FP64 kernels ---------------------------------
# Thin calls over caller-owned device buffers (integer device pointers, e.g.
# torch.Tensor.data_ptr()); argument order and meaning as in lbm_b200.h.
def _device_call(name: str, p: Params, ptrs) -> None:
    lib = load_library()
    st = getattr(lib, name)(C.byref(p), *[C.c_void_p(int(x)) if x else None for x in ptrs])
    if st != 0:
        raise LBMError(st, name)


def collide_forward(p, fin, gin, phi, rho, u, v, w, fout, gout, dux, dvy, dwz) -> None:
    _device_call("lbm_collide_forward", p, (fin, gin, phi, rho, u, v, w, fout, gout, dux, dvy, dwz))


def collide_backward(p, fin, gin, phi, rho, u, v, w, lam_fout, lam_gout, lam_dux, lam_dvy, lam_dwz,
                     lam_fin, lam_gin, lam_phi, lam_rho, lam_u, lam_v, lam_w) -> None:
    _device_call("lbm_collide_backward", p, (fin, gin, phi, rho, u, v, w, lam_fout, lam_gout, lam_dux, lam_dvy,
                                             lam_dwz, lam_fin, lam_gin, lam_phi, lam_rho, lam_u, lam_v, lam_w))


def moments_forward(p, f, g, phi, rho, u, v, w) -> None:
    _device_call("lbm_moments_forward", p, (f, g, phi, rho, u, v, w))


def moments_backward(p, phi, lam_phi, lam_rho, lam_u, lam_v, lam_w, lam_f, lam_g) -> None:
    _device_call("lbm_moments_backward", p, (phi, lam_phi, lam_rho, lam_u, lam_v, lam_w, lam_f, lam_g))


def correct_forward(p, u, v, w, press, rho) -> None:
    _device_call("lbm_correct_forward", p, (u, v, w, press, rho))


def correct_backward(p, press, rho, lam_u, lam_v, lam_w, lam_p, lam_rho) -> None:
    _device_call("lbm_correct_backward", p, (press, rho, lam_u, lam_v, lam_w, lam_p, lam_rho))


class Adjoint:
    """Gradients through whole FP64 steps of one box, slip walls or periodic x
    (lbm_adjoint_*):
    forward(fields, n_steps) runs and checkpoints, backward(lam) returns
    dJ/d(loaded fields) and dJ/dk_f for the adjoint lam of the final fields."""

    def __init__(self, params: Params, checkpoint_interval: int = 100, check_interval: int = 100,
                 tolerance: float = 1e-12, max_sweeps: int = 0, binomial_checkpoints: int = 0, krylov: bool = False,
                 krylov_tolerance: float = 0.0, device: int = 0, precision: str = "fp64"):
        self._lib = load_library()
        self.params = params
        self.cfg = AdjointCfg(checkpoint_interval, check_interval, tolerance, max_sweeps, binomial_checkpoints,
                              int(krylov), krylov_tolerance, {"fp64": 0, "mixed": 1}[precision])
        h = C.c_void_p()
        st = self._lib.lbm_adjoint_create(C.byref(params), device, C.byref(self.cfg), C.byref(h))
        if st != 0:
            why = self._lib.lbm_adjoint_last_error(None)
            raise LBMError(st, "lbm_adjoint_create: " + (why.decode() if why else ""))
        self._h = h
        self.n_steps = 0
        self.shape = (params.lz, params.ly, params.lx)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lbm_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, st, what):
        if st != 0:
            msg = self._lib.lbm_adjoint_last_error(self._h)
            raise LBMError(st, f"{what}: {msg.decode() if msg else ''}")

    def set_poisson(self, **kw):
        cfg = PoissonCfg(100, 1e-3, 0, 0, 0)
        for k, v in kw.items():
            setattr(cfg, k, v)
        self._check(self._lib.lbm_adjoint_set_poisson(self._h, C.byref(cfg)), "adjoint_set_poisson")

    def forward(self, fields: Dict[str, np.ndarray], n_steps: int, sweeps: Optional[Sequence[int]] = None):
        arrs = [np.ascontiguousarray(fields[k], dtype=np.float64) if fields.get(k) is not None else None
                for k in FIELDS]
        ptrs = [a.ctypes.data_as(C.c_void_p) if a is not None else None for a in arrs]
        sw = (C.c_uint64 * n_steps)(*sweeps) if sweeps is not None else None
        self._check(self._lib.lbm_adjoint_forward(self._h, *ptrs, n_steps, sw), "adjoint_forward")
        self.n_steps = n_steps

    def sweeps(self) -> List[int]:
        out = (C.c_uint64 * self.n_steps)()
        self._check(self._lib.lbm_adjoint_sweeps(self._h, out), "adjoint_sweeps")
        return [int(x) for x in out]

    def download(self, which: str) -> np.ndarray:
        out = np.empty(self.shape)
        self._check(self._lib.lbm_adjoint_download(self._h, FIELDS.index(which), _dp(out)), "adjoint_download")
        return out

    def backward(self, lam: Dict[str, np.ndarray]):
        """lam: adjoints of the final fields (missing = 0).  Returns (grads, stats):
        grads[k] = dJ/d(loaded field k); stats['grad_kappa_f'] = dJ/dk_f."""
        lams = [np.ascontiguousarray(lam[k], dtype=np.float64) if lam.get(k) is not None else None for k in FIELDS]
        grads = {k: np.empty(self.shape) for k in FIELDS}
        st = AdjointStats()
        args = [a.ctypes.data_as(C.c_void_p) if a is not None else None for a in lams] + \
            [grads[k].ctypes.data_as(C.c_void_p) for k in FIELDS]
        self._check(self._lib.lbm_adjoint_backward(self._h, *args, C.byref(st)), "adjoint_backward")
        return grads, st.as_dict()


def adjoint_schedule(n_steps: int, checkpoints: int) -> Dict[str, int]:
    """lbm_adjoint_schedule: forward steps a binomial reverse pass recomputes
    and the most checkpoints it holds at once (no device work)."""
    steps, peak = C.c_uint64(), C.c_int()
    st = load_library().lbm_adjoint_schedule(n_steps, checkpoints, C.byref(steps), C.byref(peak))
    if st != 0:
        raise LBMError(st, "lbm_adjoint_schedule")
    return {"recompute_steps": int(steps.value), "peak_checkpoints": int(peak.value)}

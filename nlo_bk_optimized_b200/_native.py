"""ctypes binding of ``libnlo_b200.so`` (include/nlo_b200.h).

The library is the only compute path: there is no CPU or eager-PyTorch fallback.
Loading fails loudly when the shared object is missing, and every call raises
``RuntimeError`` with the library's message when it returns an error code
(the reference raises ``RuntimeError`` from TORCH_CHECK in the same situations).
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch

from nlo_bk_optimized_b200 import build as _build

LIBRARY_PATH = _build.LIBRARY

PRECISION_MIXED = 0
PRECISION_FP64 = 1
STEPPERS = {"euler": 0, "rk3": 1, "rk4": 2}


class BKParams(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_double),
        ("nf", ctypes.c_double),
        ("lambda_qcd", ctypes.c_double),
        ("c2", ctypes.c_double),
        ("minr", ctypes.c_double),
        ("ksub", ctypes.c_double),
        ("fixed_alpha_s", ctypes.c_double),
        ("alpha_cap", ctypes.c_double),
        ("symmetrize", ctypes.c_int32),
        ("fixed_coupling", ctypes.c_int32),
        ("force_positive", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("rc_lo", ctypes.c_int32),
        ("resum_rc", ctypes.c_int32),
        ("rc_nlo", ctypes.c_int32),
        ("kinematical_constraint", ctypes.c_int32),
    ]


class SobolDirs(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int32),
        ("state", (ctypes.c_uint32 * 30) * 8),
        ("shift", ctypes.c_uint32 * 8),
    ]


class Box(ctypes.Structure):
    _fields_ = [("lower", ctypes.c_double * 4), ("width", ctypes.c_double * 4)]


MAX_QUARKS = 8

DIS_TERMS = {"LO": 0, "DIP0": 1, "DIP1": 2, "DIP2": 3, "I1": 4, "I2": 5, "I3": 6, "I2N": 7, "I3N": 8}
DIS_DIMS = {0: 2, 1: 2, 2: 3, 3: 4, 4: 5, 5: 6, 6: 7, 7: 5, 8: 5}
DIPOLE_GBW = 0
DIPOLE_TABLE = 1
VEGAS_VALUE, VEGAS_ERROR, VEGAS_EVALS, VEGAS_ITERATIONS, VEGAS_CONVERGED = 2, 3, 4, 5, 6


class DisKinematics(ctypes.Structure):
    _fields_ = [
        ("Q2", ctypes.c_double),
        ("xbj", ctypes.c_double),
        ("mf", ctypes.c_double),
        ("n_quarks", ctypes.c_int32),
        ("lo_mass", ctypes.c_double * MAX_QUARKS),
        ("lo_charge2", ctypes.c_double * MAX_QUARKS),
        ("maxr", ctypes.c_double),
        ("transverse", ctypes.c_int32),
        ("finite_nc", ctypes.c_int32),
        ("parent_coupling", ctypes.c_int32),
        ("smooth_coupling", ctypes.c_int32),
        ("mass_dependent_x", ctypes.c_int32),
        ("c2_alpha", ctypes.c_double),
        ("active_flavors", ctypes.c_double),
        ("max_alpha", ctypes.c_double),
    ]


class Dipole(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("qs0sqr", ctypes.c_double),
        ("lambda_", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("x0", ctypes.c_double),
        ("table", ctypes.c_void_p),
        ("nr", ctypes.c_int32),
        ("ny", ctypes.c_int32),
    ]


class VegasOptions(ctypes.Structure):
    _fields_ = [
        ("bins", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("min_iterations", ctypes.c_int32),
        ("samples_per_iteration", ctypes.c_int64),
        ("warmup_samples", ctypes.c_int64),
        ("epsrel", ctypes.c_double),
        ("epsabs", ctypes.c_double),
        ("inner_points", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("keep_edges", ctypes.c_int32),
    ]


class BKVegasOptions(ctypes.Structure):
    """nlo_bk_vegas_options: Vegas of the K2+Kf integral (IntegrationMethod.VEGAS)."""

    _fields_ = [
        ("samples_per_iteration", ctypes.c_int64),
        ("warmup_samples", ctypes.c_int64),
        ("max_iterations", ctypes.c_int32),
        ("min_iterations", ctypes.c_int32),
        ("bins", ctypes.c_int32),
        ("reuse_grid", ctypes.c_int32),
        ("reuse_warmup_fraction", ctypes.c_double),
        ("epsrel", ctypes.c_double),
        ("epsabs", ctypes.c_double),
        ("replicas", ctypes.c_int32),
    ]


class FixedSobolOptions(ctypes.Structure):
    _fields_ = [
        ("training_samples", ctypes.c_int64),
        ("training_rounds", ctypes.c_int32),
        ("samples_per_replicate", ctypes.c_int64),
        ("replicates", ctypes.c_int32),
        ("bins", ctypes.c_int32),
        ("fold_angle", ctypes.c_int32),
        ("i1_weight", ctypes.c_double),
        ("inner_points", ctypes.c_int32),
        ("precision", ctypes.c_int32),
    ]


EXPORTED = (
    "nlo_last_error",
    "nlo_abi_version",
    "nlo_sobol_draw",
    "nlo_bk_spline_doubles",
    "nlo_bk_splines",
    "nlo_bk_active",
    "nlo_bk_k1",
    "nlo_bk_k2kf_workspace_bytes",
    "nlo_bk_k2kf",
    "nlo_bk_k2kf_static",
    "nlo_bk_rhs_workspace_bytes",
    "nlo_bk_rhs",
    "nlo_bk_evolve",
    "nlo_bk_evolve_history",
    "nlo_bk_sets_workspace_bytes",
    "nlo_bk_evolve_sets",
    "nlo_bk_rhs_history",
    "nlo_ic_spline_doubles",
    "nlo_ic_spline",
    "nlo_ic_evaluate",
    "nlo_bk_rhs_shard",
    "nlo_bk_stage",
    "nlo_bk_vegas_state_doubles",
    "nlo_bk_vegas_workspace_bytes",
    "nlo_bk_rhs_vegas",
    "nlo_bk_evolve_vegas",
    "nlo_vegas_state_doubles",
    "nlo_vegas_workspace_bytes",
    "nlo_vegas_begin",
    "nlo_vegas_sample",
    "nlo_vegas_accumulate",
    "nlo_vegas_end_round",
    "nlo_dis_table_doubles",
    "nlo_dis_table_prepare",
    "nlo_dis_table_prepare_interpolated",
    "nlo_dis_table_initialize",
    "nlo_dis_dipole_amplitude",
    "nlo_dis_integrand",
    "nlo_dis_gauss_legendre_workspace_bytes",
    "nlo_dis_gauss_legendre",
    "nlo_dis_gauss_legendre_dipoles",
    "nlo_dis_vegas_state_doubles",
    "nlo_dis_vegas_workspace_bytes",
    "nlo_dis_vegas",
    "nlo_dis_vegas_dipoles",
    "nlo_dis_fixed_sobol_grid_doubles",
    "nlo_dis_fixed_sobol_workspace_bytes",
    "nlo_dis_fixed_sobol",
)

_lock = threading.Lock()
_handle: ctypes.CDLL | None = None


def _declare(lib: ctypes.CDLL) -> None:
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    i32, i64, sz, d = ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t, ctypes.c_double
    lib.nlo_last_error.restype = ctypes.c_char_p
    lib.nlo_last_error.argtypes = []
    lib.nlo_abi_version.restype = ctypes.c_int
    lib.nlo_sobol_draw.restype = ctypes.c_int
    lib.nlo_sobol_draw.argtypes = [P(SobolDirs), i64, i64, i32, vp, vp]
    lib.nlo_bk_spline_doubles.restype = sz
    lib.nlo_bk_spline_doubles.argtypes = [i32]
    lib.nlo_bk_splines.restype = ctypes.c_int
    lib.nlo_bk_splines.argtypes = [vp, vp, i32, i32, vp, vp]
    lib.nlo_bk_active.restype = ctypes.c_int
    lib.nlo_bk_active.argtypes = [vp, i32, vp, vp, vp]
    lib.nlo_bk_k1.restype = ctypes.c_int
    lib.nlo_bk_k1.argtypes = [P(BKParams), vp, i32, vp, vp, vp, vp, vp]
    lib.nlo_bk_k2kf_workspace_bytes.restype = sz
    lib.nlo_bk_k2kf_workspace_bytes.argtypes = [i32]
    lib.nlo_bk_k2kf.restype = ctypes.c_int
    lib.nlo_bk_k2kf.argtypes = [P(BKParams), vp, i32, vp, vp, vp, P(SobolDirs), i64, i64, P(Box), vp, vp, sz, vp]
    lib.nlo_bk_k2kf_static.restype = ctypes.c_int
    lib.nlo_bk_k2kf_static.argtypes = [P(BKParams), vp, i32, vp, vp, vp, P(SobolDirs), i64, i64, P(Box), vp, vp]
    lib.nlo_bk_rhs_workspace_bytes.restype = sz
    lib.nlo_bk_rhs_workspace_bytes.argtypes = [i32]
    lib.nlo_bk_rhs.restype = ctypes.c_int
    lib.nlo_bk_rhs.argtypes = [P(BKParams), vp, vp, i32, P(SobolDirs), i64, P(Box), vp, vp, vp, vp, sz, vp]
    lib.nlo_bk_evolve.restype = ctypes.c_int
    lib.nlo_bk_evolve.argtypes = [P(BKParams), vp, i32, i32, d, i32, P(SobolDirs), i64, P(Box), vp, vp, vp, sz, vp]
    lib.nlo_bk_evolve_history.restype = ctypes.c_int
    lib.nlo_bk_evolve_history.argtypes = [P(BKParams), vp, i32, vp, i32, i32, d, i32, P(SobolDirs), i64, P(Box), vp,
                                          vp, vp, sz, vp]
    lib.nlo_bk_sets_workspace_bytes.restype = sz
    lib.nlo_bk_sets_workspace_bytes.argtypes = [i32, i32, i32]
    lib.nlo_bk_evolve_sets.restype = ctypes.c_int
    lib.nlo_bk_evolve_sets.argtypes = [P(BKParams), vp, i32, i32, P(vp), i32, d, i32, P(SobolDirs), P(i64), P(Box),
                                       i32, vp, vp, sz, vp]
    lib.nlo_ic_spline_doubles.restype = sz
    lib.nlo_ic_spline_doubles.argtypes = [i32]
    lib.nlo_ic_spline.restype = ctypes.c_int
    lib.nlo_ic_spline.argtypes = [vp, vp, i32, vp, vp]
    lib.nlo_ic_evaluate.restype = ctypes.c_int
    lib.nlo_ic_evaluate.argtypes = [vp, i32, vp, i64, vp, vp]
    lib.nlo_bk_rhs_history.restype = ctypes.c_int
    lib.nlo_bk_rhs_history.argtypes = [P(BKParams), vp, i32, vp, vp, i32, P(SobolDirs), i64, P(Box), vp, vp, vp, vp,
                                       sz, vp]
    lib.nlo_bk_rhs_shard.restype = ctypes.c_int
    lib.nlo_bk_rhs_shard.argtypes = [P(BKParams), vp, vp, i32, i32, i32, P(SobolDirs), i64, P(Box), vp, vp, sz, vp]
    lib.nlo_bk_stage.restype = ctypes.c_int
    lib.nlo_bk_stage.argtypes = [vp, P(vp), P(d), i32, i32, i32, vp, vp, vp]
    lib.nlo_bk_vegas_state_doubles.restype = sz
    lib.nlo_bk_vegas_state_doubles.argtypes = [i32, i32]
    lib.nlo_bk_vegas_workspace_bytes.restype = sz
    lib.nlo_bk_vegas_workspace_bytes.argtypes = [i32, P(BKVegasOptions)]
    lib.nlo_bk_rhs_vegas.restype = ctypes.c_int
    lib.nlo_bk_rhs_vegas.argtypes = [P(BKParams), vp, i32, vp, vp, i32, i32, i32, P(BKVegasOptions), P(SobolDirs),
                                     P(Box), vp, vp, vp, vp, vp, sz, vp]
    lib.nlo_bk_evolve_vegas.restype = ctypes.c_int
    lib.nlo_bk_evolve_vegas.argtypes = [P(BKParams), vp, i32, vp, i32, i32, d, i32, P(BKVegasOptions), P(SobolDirs),
                                        P(Box), vp, vp, vp, vp, sz, vp]
    lib.nlo_vegas_state_doubles.restype = sz
    lib.nlo_vegas_state_doubles.argtypes = [i32, i32]
    lib.nlo_vegas_workspace_bytes.restype = sz
    lib.nlo_vegas_workspace_bytes.argtypes = [i32, i32]
    lib.nlo_vegas_begin.restype = ctypes.c_int
    lib.nlo_vegas_begin.argtypes = [i32, i32, i32, vp, vp, sz, vp]
    lib.nlo_vegas_sample.restype = ctypes.c_int
    lib.nlo_vegas_sample.argtypes = [P(SobolDirs), i64, i64, i32, i32, vp, P(d), P(d), vp, vp, vp, vp]
    lib.nlo_vegas_accumulate.restype = ctypes.c_int
    lib.nlo_vegas_accumulate.argtypes = [vp, vp, vp, i64, i32, i32, vp, sz, vp]
    lib.nlo_vegas_end_round.restype = ctypes.c_int
    lib.nlo_vegas_end_round.argtypes = [i32, i32, vp, i64, i32, i32, d, d, vp, sz, vp]
    lib.nlo_dis_table_doubles.restype = sz
    lib.nlo_dis_table_doubles.argtypes = [i32, i32]
    lib.nlo_dis_table_prepare.restype = ctypes.c_int
    lib.nlo_dis_table_prepare.argtypes = [vp, vp, vp, i32, i32, d, vp, vp]
    lib.nlo_dis_table_prepare_interpolated.restype = ctypes.c_int
    lib.nlo_dis_table_prepare_interpolated.argtypes = [vp, vp, vp, i32, i32, d, i32, vp, vp]
    lib.nlo_dis_table_initialize.restype = ctypes.c_int
    lib.nlo_dis_table_initialize.argtypes = [vp, i32, i32, d, vp]
    lib.nlo_dis_dipole_amplitude.restype = ctypes.c_int
    lib.nlo_dis_dipole_amplitude.argtypes = [P(Dipole), vp, vp, i64, i32, vp, vp]
    lib.nlo_dis_integrand.restype = ctypes.c_int
    lib.nlo_dis_integrand.argtypes = [P(DisKinematics), i32, P(Dipole), i32, i32, vp, i64, vp, vp]
    lib.nlo_dis_gauss_legendre_workspace_bytes.restype = sz
    lib.nlo_dis_gauss_legendre_workspace_bytes.argtypes = [i32]
    lib.nlo_dis_gauss_legendre.restype = ctypes.c_int
    lib.nlo_dis_gauss_legendre.argtypes = [P(DisKinematics), i32, i32, P(Dipole), i32, i32, vp, vp, sz, vp]
    lib.nlo_dis_gauss_legendre_dipoles.restype = ctypes.c_int
    lib.nlo_dis_gauss_legendre_dipoles.argtypes = [P(DisKinematics), i32, i32, P(Dipole), i32, i32, vp, vp, sz, vp]
    lib.nlo_dis_vegas_dipoles.restype = ctypes.c_int
    lib.nlo_dis_vegas_dipoles.argtypes = [P(DisKinematics), i32, i32, P(Dipole), P(VegasOptions), P(SobolDirs), vp,
                                          vp, sz, vp]
    lib.nlo_dis_vegas_state_doubles.restype = sz
    lib.nlo_dis_vegas_state_doubles.argtypes = [i32, i32]
    lib.nlo_dis_vegas_workspace_bytes.restype = sz
    lib.nlo_dis_vegas_workspace_bytes.argtypes = [i32, i32, P(VegasOptions)]
    lib.nlo_dis_vegas.restype = ctypes.c_int
    lib.nlo_dis_vegas.argtypes = [P(DisKinematics), i32, i32, P(Dipole), P(VegasOptions), P(SobolDirs), vp, vp, sz, vp]
    lib.nlo_dis_fixed_sobol_grid_doubles.restype = sz
    lib.nlo_dis_fixed_sobol_grid_doubles.argtypes = [i32]
    lib.nlo_dis_fixed_sobol_workspace_bytes.restype = sz
    lib.nlo_dis_fixed_sobol_workspace_bytes.argtypes = [P(FixedSobolOptions)]
    lib.nlo_dis_fixed_sobol.restype = ctypes.c_int
    lib.nlo_dis_fixed_sobol.argtypes = [P(DisKinematics), P(Dipole), P(FixedSobolOptions), P(SobolDirs), vp, vp, vp,
                                        sz, vp]


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load (once) and return the C-ABI library; raises if it is absent."""

    global _handle
    with _lock:
        if _handle is None:
            target = Path(path) if path is not None else LIBRARY_PATH
            if not target.exists():
                raise RuntimeError(
                    f"{target} is missing: build it with `python -m nlo_bk_optimized_b200.build` "
                    "(the B200 kernels have no CPU fallback)"
                )
            lib = ctypes.CDLL(str(target))
            _declare(lib)
            _handle = lib
        return _handle


def check(code: int) -> None:
    if code != 0:
        message = load().nlo_last_error().decode("utf-8", "replace")
        raise RuntimeError(f"nlo_b200 error {code}: {message}")


def require_cuda(tensor: torch.Tensor, name: str) -> None:
    if not tensor.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor: the B200 path has no CPU fallback")
    if not tensor.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def sobol_dirs(dims: int, seed: int) -> SobolDirs:
    """Direction numbers of SobolEngine(dims, scramble=True, seed)."""

    engine = torch.quasirandom.SobolEngine(dims, scramble=True, seed=seed)
    state = engine.sobolstate.tolist()
    shift = engine.shift.tolist()
    dirs = SobolDirs()
    dirs.dims = dims
    for d in range(dims):
        for j in range(30):
            dirs.state[d][j] = int(state[d][j])
        dirs.shift[d] = int(shift[d])
    return dirs


def box(lower, width) -> Box:
    b = Box()
    for d in range(4):
        b.lower[d] = float(lower[d])
        b.width[d] = float(width[d])
    return b

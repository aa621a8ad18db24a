"""ctypes binding of libstokesflow_b200.so (the C ABI in include/stokesflow_b200.h).

The library is built in-tree by ``stokesflow.jl_b200/csrc/Makefile`` into
``stokesflow.jl_b200/lib/``.  There is no fallback: if the shared library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_ROOT, "lib", "libstokesflow_b200.so")
CSRC = os.path.join(_PKG_ROOT, "csrc")

SF_OK = 0
SF_ERR_INVALID_ARG = 1
SF_ERR_CUDA = 2
SF_ERR_OOM = 3
SF_ERR_NO_DEVICE = 4
SF_ERR_NONFINITE = 5
SF_ERR_TOO_LARGE = 6
SF_ERR_BUSY = 7

# sf_engine_stats.tune_state
TUNE_STATES = {0: "fixed", 1: "measuring", 2: "measured", 3: "cached"}
# sf_mixed_options.tile_schedule / sf_engine_stats.tile_schedule
SCHEDULES = {1: "strided", 2: "chunked"}

# limits of the allocation-free deposit (include/stokesflow_b200.h)
SF_NOALLOC_MAX_MARKERS = 1048576
SF_NOALLOC_MAX_CELLS = 262144

_d = C.c_double
_i64 = C.c_int64
_i32 = C.c_int32
_vp = C.c_void_p
_pd = C.c_void_p  # device pointers are passed as integers


class SolveInfo(C.Structure):
    """sf_solve_info."""
    _fields_ = [("dt", _d), ("T_eff", _d), ("runtime", _d), ("iters", _i64), ("err", _d), ("n_checks", _i64),
                ("converged", _i32), ("reserved", _i32), ("loop_ms", _d), ("bytes_per_iter", _d),
                ("T_eff_essential", _d), ("fused_launches", _i64), ("fused_ms", _d)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Warnings(C.Structure):
    """sf_warnings."""
    _fields_ = [("bad_markers", _i64), ("empty_nodes", _i64), ("interp_failsafe", _i64), ("markers_outside", _i64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchInstance(C.Structure):
    """sf_batch_instance."""
    _fields_ = [("P", _vp), ("Vx_pad", _vp), ("Vy_pad", _vp), ("rho_vy", _vp), ("mu_b", _vp), ("mu_p", _vp),
                ("Vx_s", _vp), ("Vy_s", _vp), ("Nx", _i64), ("Ny", _i64), ("g_y", _d), ("dx", _d), ("dy", _d),
                ("dt", _d), ("maxdisp", _d), ("eps", _d), ("rel_tol", _d),
                ("use_free_surface_stabilization", _i32), ("retried", _i32), ("dt_out", _d), ("err", _d),
                ("eps_used", _d), ("inner_iters", _i64), ("outer_iters", _i64), ("converged", _i32),
                ("status", _i32), ("batch_ms", _d), ("dVxdt", _vp), ("dVydt", _vp)]

    RESULTS = ("dt_out", "err", "eps_used", "inner_iters", "outer_iters", "converged", "status", "batch_ms",
               "retried")

    def results(self):
        return {k: getattr(self, k) for k in self.RESULTS}


class MixedOptions(C.Structure):
    """sf_mixed_options."""
    _fields_ = [("max_sweeps", _i64), ("fold_every", _i32), ("use_graphs", _i32), ("dtau_local_max", _i32),
                ("retry_local_max", _i32), ("tile_rows", _i32), ("tile_schedule", _i32), ("overlap_launches", _i32),
                ("reserved", _i32)]


class EngineStats(C.Structure):
    """sf_engine_stats."""
    _fields_ = [("arena_bytes", _i64), ("arena_used", _i64), ("arena_peak", _i64), ("submitted", _i64),
                ("finished", _i64), ("rounds", _i64), ("sweeps", _i64), ("active", _i32), ("pending_results", _i32),
                ("tile_rows", _i32), ("tile_schedule", _i32), ("overlap_launches", _i32), ("tune_state", _i32),
                ("tune_classes", _i32), ("reserved", _i32), ("tune_rounds", _i64), ("tune_hits", _i64),
                ("tune_ns", _d * 12)]

    # rows/schedule/launch, in the library's candidate order
    CANDIDATES = tuple(f"{r}/{c}/{o}" for r in (8, 16, 32) for c in ("strided", "chunked")
                       for o in ("serial", "overlapped"))

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["tune_ns"] = dict(zip(self.CANDIDATES, list(self.tune_ns)))
        d["tile_schedule"] = SCHEDULES.get(self.tile_schedule, self.tile_schedule)
        d["tune_state"] = TUNE_STATES.get(self.tune_state, self.tune_state)
        return d


class DepositGrid(C.Structure):
    """sf_deposit_grid."""
    _fields_ = [("x_grid_min", _d), ("y_grid_min", _d), ("val_grid", _vp), ("nx", _i64), ("ny", _i64),
                ("val_m", _vp)]


class Domain(C.Structure):
    """sf_domain."""
    _fields_ = [(n, _vp) for n in ("ctx", "P", "Vx_pad", "Vy_pad", "rho_vy", "mu_b", "mu_p", "dVxdt", "dVydt",
                                    "Vx_s", "Vy_s")] + [("coord_x", _i32), ("coord_y", _i32)]


class RankArray(C.Structure):
    """sf_rank_array."""
    _fields_ = [("ctx", _vp), ("a", _vp), ("coord_x", _i32), ("coord_y", _i32)]


class MarkerRank(C.Structure):
    """sf_marker_rank."""
    _fields_ = [("ctx", _vp), ("x", _vp), ("y", _vp), ("rho", _vp), ("mu", _vp), ("n", _i64), ("x_out", _vp),
                ("y_out", _vp), ("rho_out", _vp), ("mu_out", _vp), ("capacity", _i64), ("n_out", _i64),
                ("coord_x", _i32), ("coord_y", _i32)]


class PlumeModelC(C.Structure):
    """sf_plume_model."""
    _fields_ = [(n, _d) for n in ("air_height", "plume_x", "plume_y", "plume_r", "rho_air", "rho_matrix",
                                  "rho_plume", "mu_air", "mu_matrix", "mu_plume")]


# name -> (restype, argtypes); mirrors include/stokesflow_b200.h
PROTOTYPES = {
    "sf_version": (C.c_int, []),
    "sf_status_string": (C.c_char_p, [C.c_int]),
    "sf_last_error": (C.c_char_p, []),
    "sf_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "sf_ctx_destroy": (C.c_int, [_vp]),
    "sf_ctx_scratch_bytes": (C.c_int, [_vp, C.POINTER(_i64)]),
    "sf_ctx_launch_count": (C.c_int, [_vp, C.POINTER(_i64)]),
    "sf_get_warnings": (C.c_int, [_vp, C.POINTER(Warnings), C.c_int]),
    "sf_selftest_bounded_wait": (C.c_int, [_vp, C.c_int, _i64, C.POINTER(_i32)]),
    "sf_bilinear_marker_to_grid": (C.c_int, [_vp, _d, _d, _pd, _i64, _i64, _pd, _pd, _pd, _i64, _d, _d, _pd, _pd,
                                             _i64, _i64, _vp]),
    "sf_bilinear_marker_to_grid_noalloc": (C.c_int, [_d, _d, _pd, _i64, _i64, _pd, _pd, _pd, _i64, _d, _d, _vp]),
    "sf_bilinear_marker_to_grids": (C.c_int, [_vp, C.POINTER(DepositGrid), C.c_int, _pd, _pd, _i64, _d, _d, _pd,
                                              _pd, _i64, _i64, _vp]),
    "sf_solve_stokes": (C.c_int, [_vp] + [_pd] * 19 + [_d, _d, _d, _i64, _i64, _d, _d, C.c_int, _d, C.c_int, _i64,
                                                       _vp, C.POINTER(SolveInfo)]),
    "sf_stokes_residual_scale": (C.c_int, [_vp, _pd, _i64, _i64, _d, _vp, C.POINTER(_d)]),
    "sf_solve_stokes_decomposed": (C.c_int, [C.POINTER(Domain), _i32, _i32, _i64, _i64, _d, _d, _d, _d, _d, C.c_int,
                                             _d, _i64, C.POINTER(SolveInfo)]),
    "sf_sum_overlapping_values": (C.c_int, [C.POINTER(RankArray), _i32, _i32, _i64, _i64, _i64, _i64]),
    "sf_safe_division": (C.c_int, [_vp, _pd, _i64, _i64, _pd, _pd, _i64, _vp]),
    "sf_exchange_markers": (C.c_int, [C.POINTER(MarkerRank), _i32, _i32, _d, _d, _d, _d]),
    "sf_solve_stokes_batch_mixed": (C.c_int, [_vp, C.POINTER(BatchInstance), C.c_int, C.POINTER(MixedOptions), _vp]),
    "sf_solve_stokes_mixed": (C.c_int, [_vp, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _d, _d, _d, _i64, _i64,
                                        _d, _d,
                                        C.c_int, _d, _d, C.POINTER(MixedOptions), _vp, C.POINTER(BatchInstance)]),
    "sf_engine_instance_bytes": (C.c_int, [_i64, _i64, C.POINTER(_i64)]),
    "sf_engine_create": (C.c_int, [_vp, _i64, _i32, C.POINTER(MixedOptions), C.POINTER(_vp)]),
    "sf_engine_destroy": (C.c_int, [_vp]),
    "sf_engine_submit": (C.c_int, [_vp, C.POINTER(BatchInstance), _vp, C.POINTER(_i64)]),
    "sf_engine_step": (C.c_int, [_vp, _vp, C.POINTER(_i64), _i32, C.POINTER(_i32), C.POINTER(_i32)]),
    "sf_engine_get_stats": (C.c_int, [_vp, C.POINTER(EngineStats)]),
    "sf_ctx_batch_stats": (C.c_int, [_vp, C.POINTER(EngineStats)]),
    "sf_move_markers_rk4": (C.c_int, [_vp, _pd, _pd, _i64, _pd, _i64, _i64, _pd, _i64, _i64, _d, _d, _d, _d, _d, _d,
                                      _d, _d, _d, _vp]),
    "sf_rebin_markers": (C.c_int, [_vp, _pd, _pd, _i64, _d, _d, _d, _d, _i64, _i64, _pd, _pd, _pd, _vp]),
    "sf_marker_count": (C.c_int, [_i64, _i64, _i64, C.POINTER(_i64), C.POINTER(_i64)]),
    "sf_init_markers_host": (C.c_int, [_i64, _d, _d, _d, _d, _i64, _i64, _d, C.c_uint64, _vp, _vp]),
    "sf_init_markers": (C.c_int, [_vp, _i64, _d, _d, _d, _d, _i64, _i64, _d, C.c_uint64, _pd, _pd, _vp]),
    "sf_uniform": (_d, [C.c_uint64, C.c_uint64]),
    "sf_marker_count_rank": (C.c_int, [_i64, _i64, _i64, _i32, _i32, _i32, _i32, C.POINTER(_i64), C.POINTER(_i64)]),
    "sf_init_markers_rank": (C.c_int, [_vp, _i64, _d, _d, _d, _d, _i64, _i64, _i32, _i32, _i32, _i32, _d, C.c_uint64,
                                       _pd, _pd, _vp]),
    "sf_set_marker_properties_host": (C.c_int, [C.POINTER(PlumeModelC), _vp, _vp, _i64, _d, _d, _vp, _vp]),
    "sf_set_marker_properties": (C.c_int, [_vp, C.POINTER(PlumeModelC), _pd, _pd, _i64, _d, _d, _pd, _pd, _vp]),
}

_lib = None


class StokesFlowError(RuntimeError):
    """A non-zero sf_status from the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def build(force: bool = False) -> str:
    """Compile the shared library with csrc/Makefile (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", CSRC, "-j4"], check=True)
    return LIB_PATH


def lib():
    """Load libstokesflow_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libstokesflow_b200.so not built: {LIB_PATH} missing "
                               "(run `make -C stokesflow.jl_b200/csrc` or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = ""):
    if status != SF_OK:
        msg = lib().sf_last_error().decode(errors="replace")
        raise StokesFlowError(status, f"{what}: {msg}" if what else msg)

"""stokesflow_b200 -- B200 (sm_100a) implementation of the StokesFlow.jl hot path.

Marker->grid deposit, pseudo-transient Stokes solve and RK4 marker advection
with rebinning, as hand-written CUDA behind the C ABI of
``include/stokesflow_b200.h`` (libstokesflow_b200.so).  This package is the
Python host side: a ctypes binding (``_lib``), mirrors of the reference's
Julia functions on CUDA tensors (``api``) and the timestep driver
(``driver``).  There is no CPU fallback.
"""
from ._lib import LIB_PATH, StokesFlowError, build, lib  # noqa: F401
from .api import (Context, Engine, MixedProblem, PlumeModel, batch_stats, bilinear_marker_to_grid,  # noqa: F401
                  bilinear_marker_to_grid_noalloc, bilinear_marker_to_grids, default_context, get_warnings,
                  initialize_markers, initialize_markers_host, marker_count, mixed_options, move_markers_rk4, rebin_markers,
                  residual_scale, selftest_bounded_wait, set_initial_marker_properties, solve_stokes,
                  solve_stokes_batch_mixed, solve_stokes_info, zeros)
from .driver import (StokesFlow2D, node_origins, plume_model_test_flow, plume_model_unit_square,  # noqa: F401
                     stokes_flow_2d)

__version__ = "0.1.0"

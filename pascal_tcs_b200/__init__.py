"""pascal_tcs_b200 -- the PaScaL_TCS per-timestep hot path (energy and momentum
ADI sweeps, FFT pressure Poisson solve, projection and diagnostics) as CUDA
kernels for one B200, behind the C ABI of include/tcs.h."""
from .tcs import (EXPORTS, Ensemble, FIELDS, HISTORY, LIB_PATH, SCALARS, Solver, TcsConfig,  # noqa: F401
                  TcsError, TdmaPlan, TdmaPlanSingle, default_config, kernel_names, timer_of_kernel, timer_names, bounds_checked, launch_count, load, measure_fp64_peak, check_reciprocal,
                  tdma_many_solve_noalloc, TDMA_NOALLOC_MAX_ELEMS, PREC_FP64, PREC_FP32_MIXED)

__all__ = ["Solver", "Ensemble", "TdmaPlan", "TdmaPlanSingle", "TcsError", "TcsConfig", "default_config", "kernel_names", "timer_of_kernel", "timer_names", "bounds_checked", "launch_count", "load", "measure_fp64_peak", "check_reciprocal",
           "FIELDS", "SCALARS", "HISTORY", "EXPORTS", "LIB_PATH", "PREC_FP64", "PREC_FP32_MIXED"]

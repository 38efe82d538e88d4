"""Python host binding of libtcs (include/tcs.h).

The reference's host side is the Fortran driver main.f90; this module mirrors
its call sequence and the module interfaces it uses (mpi_thermal,
mpi_momentum, mpi_pressure, mpi_subdomain, mpi_Post, PaScaL_TDMA) one call per
C-ABI entry point.  There is no CPU path: every method calls the CUDA library,
and loading fails loudly if libtcs.so has not been built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TCS_LIBRARY selects another build of the library (the bounds-check build
# libtcs_bc.so in its test); the default is the in-tree libtcs.so.
LIB_PATH = os.environ.get("TCS_LIBRARY") or os.path.join(_HERE, "libtcs.so")

FIELDS = {"T": 0, "U": 1, "V": 2, "W": 3, "P": 4, "dPhat": 5, "dP0": 6,
          "dU": 7, "dV": 8, "dW": 9, "dP": 10, "Mu": 11, "invRho": 12}
SCALARS = ["dt", "time", "CFL", "maxDivU", "Nu_bot", "Nu_top", "KE", "blowup",
           "aver", "step", "fixed_dt"]
HISTORY = ["dt", "time", "maxDivU", "CFL", "Nu_bot", "Nu_top", "KE"]
METRICS = ["x1", "dx1", "dmx1", "x2", "dx2", "dmx2", "x3", "dx3", "dmx3"]
TUNING = ["tl_strided", "tl_contig", "tl_modal", "fft_lines_x", "fft_lines_z", "lanes", "long_lines", "y_solver", "ifft_lines_x", "mixed_rows", "z_staging"]
ERRORS = {1: "bad argument", 2: "CUDA error", 3: "unsupported", 4: "BLOW UP",
          5: "out of device memory", 6: "non-finite scalar"}

# Every symbol include/tcs.h declares (checked by the CPU test suite).
EXPORTS = [
    "tcs_create", "tcs_destroy", "tcs_set_stream", "tcs_get_stream", "tcs_dims",
    "tcs_upload_field", "tcs_download_field", "tcs_upload_field_async",
    "tcs_download_field_async", "tcs_field_device_ptr", "tcs_synchronize", "tcs_set_dt",
    "tcs_get_metric", "tcs_thermal_coeffi", "tcs_thermal_solver", "tcs_thermal_coeffi_clean",
    "tcs_subdomain_ghostcell_update", "tcs_momentum_coeffi", "tcs_momentum_solvedU",
    "tcs_momentum_solvedV", "tcs_momentum_solvedW", "tcs_momentum_blockLdV",
    "tcs_momentum_blockLdU", "tcs_momentum_pseudoupdateUVW", "tcs_momentum_coeffi_clean",
    "tcs_pressure_RHS", "tcs_pressure_Poisson_FFT2", "tcs_pressure_Poisson_FFT1", "tcs_pressure_Projection",
    "tcs_post_div", "tcs_post_cfl", "tcs_step", "tcs_get_scalars", "tcs_get_history",
    "tcs_snapshot", "tcs_restore",
    "tcs_tdma_plan_many_create", "tcs_tdma_plan_many_destroy", "tcs_tdma_many_solve",
    "tcs_tdma_many_solve_cycle", "tcs_tdma_many_solve_noalloc", "tcs_kernel_count", "tcs_launch_count", "tcs_measure_fp64_peak", "tcs_check_reciprocal", "tcs_kernel_name", "tcs_timer_of_kernel", "tcs_timer_name", "tcs_bounds_checked",
    "tcs_bounds_violations", "tcs_probe_enable",
    "tcs_probe_read", "tcs_probe_reset", "tcs_set_use_graph", "tcs_set_tuning", "tcs_get_tuning",
    "tcs_last_error", "tcs_precision", "tcs_ensemble_create", "tcs_ensemble_destroy", "tcs_ensemble_step",
    "tcs_ensemble_size", "tcs_ensemble_set_batched", "tcs_ensemble_form", "tcs_autotune", "tcs_write_continue", "tcs_read_continue", "tcs_extract_plane",
    "tcs_tdma_plan_single_create", "tcs_tdma_plan_single_destroy", "tcs_tdma_single_solve",
    "tcs_tdma_single_solve_cycle", "tcs_tdma_many_solve_nonblocking", "tcs_tdma_many_solve_cycle_nonblocking",
]


class TcsError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


class TcsConfig(ctypes.Structure):
    _fields_ = [("n1m", ctypes.c_int), ("n2m", ctypes.c_int), ("n3m", ctypes.c_int),
                ("uniform1", ctypes.c_int), ("uniform2", ctypes.c_int), ("uniform3", ctypes.c_int),
                ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("gamma3", ctypes.c_double),
                ("aspect1", ctypes.c_double), ("H", ctypes.c_double), ("aspect3", ctypes.c_double),
                ("Ra", ctypes.c_double), ("Pr", ctypes.c_double), ("DeltaT", ctypes.c_double),
                ("MaxCFL", ctypes.c_double), ("dtStart", ctypes.c_double), ("tStart", ctypes.c_double),
                ("property_set", ctypes.c_int), ("fixed_dt", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("noise_amp", ctypes.c_double),
                ("init_mode", ctypes.c_int), ("top_wall_mode", ctypes.c_int), ("device", ctypes.c_int),
                ("precision", ctypes.c_int)]


PREC_FP64 = 0          # the reference's arithmetic
PREC_FP32_MIXED = 1    # FP32 fields/stencils/sweeps/FFTs, FP64 refinement, modal solves, projection, reductions


def default_config(**kw) -> dict:
    """The 64^3 constant-property Boussinesq case: Lx = Lz = 2, Ly = 1,
    tanh-stretched y (gamma 1.5), Ra = 1e5, Pr = 0.71, dt = 1e-3."""
    c = dict(n1m=64, n2m=64, n3m=64, uniform1=1, uniform2=0, uniform3=1,
             gamma1=3.0, gamma2=1.5, gamma3=3.0, aspect1=2.0, H=1.0, aspect3=2.0,
             Ra=1e5, Pr=0.71, DeltaT=10.0, MaxCFL=1.0, dtStart=1e-3, tStart=0.0,
             property_set=0, fixed_dt=1, seed=0, noise_amp=0.01, init_mode=0,
             top_wall_mode=0, device=0, precision=PREC_FP64)
    c.update(kw)
    return c


_lib = None


def load() -> ctypes.CDLL:
    """Load libtcs.so (built in-tree by pascal_tcs_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m pascal_tcs_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    sig = {
        "tcs_create": ([ctypes.POINTER(TcsConfig), ctypes.POINTER(vp)], ip),
        "tcs_destroy": ([vp], ip),
        "tcs_set_stream": ([vp, vp], ip),
        "tcs_get_stream": ([vp], vp),
        "tcs_dims": ([vp, ctypes.POINTER(ip)], ip),
        "tcs_upload_field": ([vp, ip, vp], ip),
        "tcs_download_field": ([vp, ip, vp], ip),
        "tcs_upload_field_async": ([vp, ip, vp], ip),
        "tcs_download_field_async": ([vp, ip, vp], ip),
        "tcs_field_device_ptr": ([vp, ip, ctypes.POINTER(vp)], ip),
        "tcs_synchronize": ([vp], ip),
        "tcs_set_dt": ([vp, ctypes.c_double], ip),
        "tcs_get_metric": ([vp, ip, dp], ip),
        "tcs_subdomain_ghostcell_update": ([vp, ip], ip),
        "tcs_post_div": ([vp, dp], ip),
        "tcs_post_cfl": ([vp, dp, dp], ip),
        "tcs_step": ([vp, ip, ctypes.POINTER(ip)], ip),
        "tcs_get_scalars": ([vp, dp], ip),
        "tcs_get_history": ([vp, ip, ip, dp], ip),
        "tcs_tdma_plan_many_create": ([ctypes.POINTER(vp), ip, ip, ip], ip),
        "tcs_tdma_plan_many_destroy": ([vp], ip),
        "tcs_tdma_many_solve": ([vp, vp, vp, vp, vp, ip, ip], ip),
        "tcs_tdma_many_solve_cycle": ([vp, vp, vp, vp, vp, ip, ip], ip),
        "tcs_tdma_many_solve_noalloc": ([vp, vp, vp, vp, ip, ip, ip], ip),
        "tcs_kernel_count": ([], ip),
        "tcs_launch_count": ([], ctypes.c_ulonglong),
        "tcs_kernel_name": ([ip], ctypes.c_char_p),
        "tcs_timer_of_kernel": ([ip], ip),
        "tcs_timer_name": ([ip], ctypes.c_char_p),
        "tcs_bounds_checked": ([], ip),
        "tcs_bounds_violations": ([vp, dp], ip),
        "tcs_probe_enable": ([vp, ctypes.c_uint64], ip),
        "tcs_probe_read": ([vp, ip, dp, ctypes.POINTER(ip)], ip),
        "tcs_probe_reset": ([vp], ip),
        "tcs_set_use_graph": ([vp, ip], ip),
        "tcs_set_tuning": ([vp, ip, ip], ip),
        "tcs_get_tuning": ([vp, ip, ctypes.POINTER(ip)], ip),
        "tcs_last_error": ([], ctypes.c_char_p),
        "tcs_precision": ([vp], ip),
        "tcs_ensemble_create": ([ctypes.POINTER(vp), ip, ctypes.POINTER(vp)], ip),
        "tcs_ensemble_destroy": ([vp], ip),
        "tcs_ensemble_step": ([vp, ip, ctypes.POINTER(ip)], ip),
        "tcs_measure_fp64_peak": ([ip, ctypes.POINTER(ctypes.c_double)], ip),
        "tcs_check_reciprocal": ([ip, ip, ctypes.POINTER(ctypes.c_double)], ip),
        "tcs_ensemble_size": ([vp], ip),
        "tcs_ensemble_set_batched": ([vp, ip], ip),
        "tcs_ensemble_form": ([vp, ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)], ip),
        "tcs_autotune": ([vp, ip, ctypes.c_char_p, ctypes.POINTER(ip)], ip),
        "tcs_write_continue": ([vp, ctypes.c_char_p], ip),
        "tcs_read_continue": ([vp, ctypes.c_char_p, ctypes.POINTER(ip)], ip),
        "tcs_extract_plane": ([vp, ip, ip, ip, ctypes.POINTER(ip), dp], ip),
        "tcs_tdma_plan_single_create": ([ctypes.POINTER(vp), ip, ip, ip], ip),
        "tcs_tdma_plan_single_destroy": ([vp], ip),
        "tcs_tdma_single_solve": ([vp, vp, vp, vp, vp, ip], ip),
        "tcs_tdma_single_solve_cycle": ([vp, vp, vp, vp, vp, ip], ip),
        "tcs_tdma_many_solve_nonblocking": ([vp, vp, vp, vp, vp, ip, ip], ip),
        "tcs_tdma_many_solve_cycle_nonblocking": ([vp, vp, vp, vp, vp, ip, ip], ip),
    }
    for name in ("tcs_thermal_coeffi", "tcs_thermal_solver", "tcs_thermal_coeffi_clean",
                 "tcs_momentum_coeffi", "tcs_momentum_solvedU", "tcs_momentum_solvedV",
                 "tcs_momentum_solvedW", "tcs_momentum_blockLdV", "tcs_momentum_blockLdU",
                 "tcs_momentum_pseudoupdateUVW", "tcs_momentum_coeffi_clean", "tcs_pressure_RHS",
                 "tcs_pressure_Poisson_FFT2", "tcs_pressure_Poisson_FFT1", "tcs_pressure_Projection", "tcs_snapshot",
                 "tcs_restore"):
        sig[name] = ([vp], ip)
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _check(r: int, where: str) -> None:
    if r != 0:
        raise TcsError(r, where, load().tcs_last_error().decode())


def launch_count() -> int:
    """Kernels launched by libtcs in this process (CUDA-graph replays included)."""
    return int(load().tcs_launch_count())


def timer_of_kernel() -> dict:
    """kernel name -> the reference's stage timer label (main.f90:55-72) its
    work falls under (None for kernels outside the time loop)."""
    L = load()
    out = {}
    for k, name in enumerate(kernel_names()):
        t = L.tcs_timer_of_kernel(k)
        out[name] = L.tcs_timer_name(t).decode() if t > 0 else None
    return out


def bounds_checked() -> bool:
    """Whether the loaded library is the bounds-check build (libtcs_bc.so)."""
    return bool(load().tcs_bounds_checked())


def timer_names() -> list[str]:
    """The reference's 18 stage-timer labels, in order (main.f90:55-72)."""
    L = load()
    return [L.tcs_timer_name(t).decode() for t in range(1, 19)]


def kernel_names() -> list[str]:
    L = load()
    return [L.tcs_kernel_name(i).decode() for i in range(L.tcs_kernel_count())]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One case resident on one GPU, driven with the reference's call sequence."""

    def __init__(self, **cfg):
        self.config = default_config(**cfg)
        L = load()
        h = ctypes.c_void_p()
        _check(L.tcs_create(ctypes.byref(TcsConfig(**self.config)), ctypes.byref(h)), "tcs_create")
        self._h = h
        d = (ctypes.c_int * 3)()
        _check(L.tcs_dims(h, d), "tcs_dims")
        self.shape = (d[2], d[1], d[0])
        self.n1m, self.n2m, self.n3m = (self.config[k] for k in ("n1m", "n2m", "n3m"))
        self._since_restore = 0

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tcs_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data -----------------------------------------------------------------
    def get(self, name: str) -> np.ndarray:
        a = np.empty(self.shape, dtype=np.float64)
        _check(load().tcs_download_field(self._h, FIELDS[name], a.ctypes.data), f"download {name}")
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
        _check(load().tcs_upload_field(self._h, FIELDS[name], a.ctypes.data), f"upload {name}")

    def upload_async(self, name: str, pinned_ptr: int) -> None:
        _check(load().tcs_upload_field_async(self._h, FIELDS[name], pinned_ptr), f"upload {name}")

    def download_async(self, name: str, pinned_ptr: int) -> None:
        _check(load().tcs_download_field_async(self._h, FIELDS[name], pinned_ptr), f"download {name}")

    def write_continue(self, directory: str) -> None:
        """cont_time/U/V/W/P/THETA.bin (the reference's continue files) plus cont_dPhat/dP0.bin."""
        _check(load().tcs_write_continue(self._h, directory.encode()), "write_continue")

    def read_continue(self, directory: str) -> bool:
        """Read continue files; True when dPhat and dP0 were there too."""
        h = ctypes.c_int(0)
        _check(load().tcs_read_continue(self._h, directory.encode(), ctypes.byref(h)), "read_continue")
        return bool(h.value)

    def plane(self, axis: int, index: int, fields=("U", "V", "W", "P", "T")) -> np.ndarray:
        """Padded planes (axis 1: i=index, 2: j=index, 3: k=index) of the fields, shape (nfields, nb, na)."""
        P3, P2, P1 = self.shape
        na = P2 if axis == 1 else P1
        nb = P2 if axis == 3 else P3
        ids = (ctypes.c_int * len(fields))(*[FIELDS[f] for f in fields])
        out = np.empty((len(fields), nb, na))
        _check(load().tcs_extract_plane(self._h, int(axis), int(index), len(fields), ids, _dptr(out)), "extract_plane")
        return out

    def bounds_violations(self) -> int:
        """Out-of-range indices the kernels met so far (bounds-check build; 0 otherwise)."""
        v = ctypes.c_double()
        _check(load().tcs_bounds_violations(self._h, ctypes.byref(v)), "tcs_bounds_violations")
        return int(v.value)

    @property
    def precision(self) -> int:
        """PREC_FP64 or PREC_FP32_MIXED; device buffers hold doubles or floats accordingly."""
        return int(load().tcs_precision(self._h))

    def device_ptr(self, name: str) -> int:
        p = ctypes.c_void_p()
        _check(load().tcs_field_device_ptr(self._h, FIELDS[name], ctypes.byref(p)), "device_ptr")
        return p.value

    def metric(self, name: str) -> np.ndarray:
        n = {"1": self.shape[2], "2": self.shape[1], "3": self.shape[0]}[name[-1]]
        a = np.empty(n, dtype=np.float64)
        _check(load().tcs_get_metric(self._h, METRICS.index(name), _dptr(a)), "metric")
        return a

    def set_stream(self, stream_handle: int | None) -> None:
        _check(load().tcs_set_stream(self._h, stream_handle or None), "set_stream")

    @property
    def stream(self) -> int:
        return load().tcs_get_stream(self._h) or 0

    def synchronize(self) -> None:
        _check(load().tcs_synchronize(self._h), "synchronize")

    def set_dt(self, dt: float) -> None:
        _check(load().tcs_set_dt(self._h, float(dt)), "set_dt")

    def scalars(self) -> dict:
        a = np.zeros(len(SCALARS))
        _check(load().tcs_get_scalars(self._h, _dptr(a)), "scalars")
        return dict(zip(SCALARS, a.tolist()))

    def history(self, first: int, count: int) -> np.ndarray:
        a = np.zeros((count, len(HISTORY)))
        _check(load().tcs_get_history(self._h, int(first), int(count), _dptr(a)), "history")
        return a

    # -- the reference's step, one call per routine (main.f90:133-221) ---------
    def _call(self, name: str) -> None:
        _check(getattr(load(), name)(self._h), name)

    def thermal_coeffi(self): self._call("tcs_thermal_coeffi")
    def thermal_solver(self): self._call("tcs_thermal_solver")
    def thermal_coeffi_clean(self): self._call("tcs_thermal_coeffi_clean")
    def momentum_coeffi(self): self._call("tcs_momentum_coeffi")
    def momentum_solvedU(self): self._call("tcs_momentum_solvedU")
    def momentum_solvedV(self): self._call("tcs_momentum_solvedV")
    def momentum_solvedW(self): self._call("tcs_momentum_solvedW")
    def momentum_blockLdV(self): self._call("tcs_momentum_blockLdV")
    def momentum_blockLdU(self): self._call("tcs_momentum_blockLdU")
    def momentum_pseudoupdateUVW(self): self._call("tcs_momentum_pseudoupdateUVW")
    def momentum_coeffi_clean(self): self._call("tcs_momentum_coeffi_clean")
    def pressure_RHS(self): self._call("tcs_pressure_RHS")
    def pressure_Poisson_FFT2(self): self._call("tcs_pressure_Poisson_FFT2")
    def pressure_Poisson_FFT1(self): self._call("tcs_pressure_Poisson_FFT1")
    def pressure_Projection(self): self._call("tcs_pressure_Projection")

    def ghostcell_update(self, name: str) -> None:
        _check(load().tcs_subdomain_ghostcell_update(self._h, FIELDS[name]), "ghostcell_update")

    def post_div(self) -> float:
        v = ctypes.c_double()
        _check(load().tcs_post_div(self._h, ctypes.byref(v)), "post_div")
        return v.value

    def post_cfl(self) -> tuple[float, float]:
        c, d = ctypes.c_double(), ctypes.c_double()
        _check(load().tcs_post_cfl(self._h, ctypes.byref(c), ctypes.byref(d)), "post_cfl")
        return c.value, d.value

    def driver_step(self) -> float:
        """One iteration of main.f90:129-223 through the stage entry points."""
        self.thermal_coeffi(); self.thermal_solver(); self.thermal_coeffi_clean()
        self.ghostcell_update("T")
        self.momentum_coeffi()
        self.momentum_solvedU(); self.ghostcell_update("dU")
        self.momentum_solvedV(); self.ghostcell_update("dV")
        self.momentum_solvedW(); self.ghostcell_update("dW")
        self.momentum_blockLdV(); self.ghostcell_update("dV")
        self.momentum_blockLdU()
        self.momentum_pseudoupdateUVW()
        for f in ("U", "V", "W"):
            self.ghostcell_update(f)
        self.pressure_RHS()
        self.pressure_Poisson_FFT2()
        self.ghostcell_update("dP")
        self.pressure_Projection()
        for f in ("U", "V", "W", "P", "dPhat"):
            self.ghostcell_update(f)
        self.momentum_coeffi_clean()
        div = self.post_div()
        self.post_cfl()
        self._since_restore += 1
        return div

    def step(self, n: int = 1) -> int:
        done = ctypes.c_int()
        _check(load().tcs_step(self._h, int(n), ctypes.byref(done)), "tcs_step")
        self._since_restore += done.value
        return done.value

    def scalars_step_mod(self, m: int) -> int:
        """Completed steps since the last restore, modulo m (host-side counter)."""
        return self._since_restore % m if m else 0

    def snapshot(self) -> None:
        """Keep an on-device copy of the step state (fields read by a step + scalars)."""
        self._call("tcs_snapshot")
        self._since_restore = 0

    def restore(self) -> None:
        """Return to the last snapshot (device-to-device copies on the solver stream)."""
        self._call("tcs_restore")
        self._since_restore = 0

    def set_tuning(self, knob: str, value: int) -> None:
        _check(load().tcs_set_tuning(self._h, TUNING.index(knob), int(value)), f"set_tuning {knob}")

    def autotune(self, trial_steps: int = 3, cache_path: str | None = None) -> tuple[dict, bool]:
        """Pick every launch-shape knob by timing (tcs_autotune); the case's state
        is left as it was.  Returns the knobs and whether they came from the cache."""
        hit = ctypes.c_int(0)
        _check(load().tcs_autotune(self._h, int(trial_steps), cache_path.encode() if cache_path else None,
                                   ctypes.byref(hit)), "autotune")
        return self.tuning(), bool(hit.value)

    def tuning(self) -> dict:
        out = {}
        for i, k in enumerate(TUNING):
            v = ctypes.c_int()
            _check(load().tcs_get_tuning(self._h, i, ctypes.byref(v)), "get_tuning")
            out[k] = v.value
        return out

    def use_graph(self, on: bool) -> None:
        _check(load().tcs_set_use_graph(self._h, int(bool(on))), "use_graph")

    # -- measurement ----------------------------------------------------------
    def probe(self, kernels) -> None:
        names = kernel_names()
        mask = 0
        for k in kernels:
            mask |= 1 << (names.index(k) if isinstance(k, str) else int(k))
        _check(load().tcs_probe_enable(self._h, ctypes.c_uint64(mask)), "probe_enable")

    def probe_read(self, kernel) -> tuple[float, int]:
        kid = kernel_names().index(kernel) if isinstance(kernel, str) else int(kernel)
        t, n = ctypes.c_double(), ctypes.c_int()
        _check(load().tcs_probe_read(self._h, kid, ctypes.byref(t), ctypes.byref(n)), "probe_read")
        return t.value, n.value

    def probe_reset(self) -> None:
        _check(load().tcs_probe_reset(self._h), "probe_reset")


def measure_fp64_peak(device: int = 0) -> float:
    """FP64 FMA throughput of the device in TFLOP/s (tcs_measure_fp64_peak)."""
    v = ctypes.c_double(0.0)
    _check(load().tcs_measure_fp64_peak(int(device), ctypes.byref(v)), "tcs_measure_fp64_peak")
    return v.value


def check_reciprocal(n: int = 1 << 16, fp32: bool = False) -> float:
    """Largest error (ulps) of the line solver's reciprocal (FP64, or FP32)
    against the correctly rounded 1/b (tcs_check_reciprocal)."""
    v = ctypes.c_double(0.0)
    _check(load().tcs_check_reciprocal(int(n), 1 if fp32 else 0, ctypes.byref(v)), "tcs_check_reciprocal")
    return v.value


class Ensemble:
    """Independent cases on one GPU advanced together by one CUDA-graph launch
    per step (tcs_ensemble_*).  batched: True = each line sweep is one launch
    over all cases (blocks pull (case, block) work items); False = every
    case's step is its own graph branch; None (default) = auto: the first 8
    steps measure both forms, then the faster one is kept."""

    def __init__(self, solvers, batched=None):
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = ctypes.c_void_p()
        _check(load().tcs_ensemble_create(arr, len(self.solvers), ctypes.byref(h)), "tcs_ensemble_create")
        self._h = h
        self.set_batched(batched)

    def set_batched(self, on) -> None:
        mode = -1 if on is None else (1 if on else 0)
        _check(load().tcs_ensemble_set_batched(self._h, mode), "tcs_ensemble_set_batched")

    def form(self):
        """(form in use: 1 batched, 0 branch per case, -1 still measuring;
        measured ms per step of the branch and batched forms, -1 if not measured)."""
        f, a, b = ctypes.c_int(0), ctypes.c_float(0), ctypes.c_float(0)
        _check(load().tcs_ensemble_form(self._h, ctypes.byref(f), ctypes.byref(a), ctypes.byref(b)), "tcs_ensemble_form")
        return f.value, a.value, b.value

    def step(self, n: int = 1) -> int:
        """n steps of every case; returns how many cases have blown up."""
        blown = ctypes.c_int(0)
        _check(load().tcs_ensemble_step(self._h, int(n), ctypes.byref(blown)), "tcs_ensemble_step")
        for s in self.solvers:
            s._since_restore += n
        return blown.value

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tcs_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __len__(self):
        return len(self.solvers)


class TdmaPlan:
    """PaScaL_TDMA_plan_many_create / many_solve / many_solve_cycle / destroy
    (pascal_tdma.f90:185-290, 487-578, 715-806) on one GPU."""

    def __init__(self, n_sys: int, myrank: int = 0, nprocs: int = 1):
        h = ctypes.c_void_p()
        _check(load().tcs_tdma_plan_many_create(ctypes.byref(h), int(n_sys), int(myrank), int(nprocs)),
               "PaScaL_TDMA_plan_many_create")
        self._h, self.n_sys = h, int(n_sys)

    def destroy(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tcs_tdma_plan_many_destroy(self._h)
            self._h = None

    def __del__(self):
        self.destroy()

    def _solve(self, fn: str, A, B, C, D, n_sys: int, n_row: int) -> None:
        ptrs = []
        for x in (A, B, C, D):
            if isinstance(x, np.ndarray):
                assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]
                ptrs.append(x.ctypes.data)
            else:                           # device tensor (data_ptr) or raw pointer
                ptrs.append(int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x))
        _check(getattr(load(), fn)(self._h, *ptrs, int(n_sys), int(n_row)), fn)

    def many_solve(self, A, B, C, D, n_sys: int, n_row: int) -> None:
        self._solve("tcs_tdma_many_solve", A, B, C, D, n_sys, n_row)

    def many_solve_cycle(self, A, B, C, D, n_sys: int, n_row: int) -> None:
        self._solve("tcs_tdma_many_solve_cycle", A, B, C, D, n_sys, n_row)

    def many_solve_nonblocking(self, A, B, C, D, n_sys: int, n_row: int) -> None:
        self._solve("tcs_tdma_many_solve_nonblocking", A, B, C, D, n_sys, n_row)

    def many_solve_cycle_nonblocking(self, A, B, C, D, n_sys: int, n_row: int) -> None:
        self._solve("tcs_tdma_many_solve_cycle_nonblocking", A, B, C, D, n_sys, n_row)


class TdmaPlanSingle(TdmaPlan):
    """PaScaL_TDMA_plan_single_create / single_solve(_cycle) / destroy
    (pascal_tdma.f90:139-175, 301-475): one system of n_row rows."""

    def __init__(self, myrank: int = 0, nprocs: int = 1, gather_rank: int = 0):
        h = ctypes.c_void_p()
        _check(load().tcs_tdma_plan_single_create(ctypes.byref(h), int(myrank), int(nprocs), int(gather_rank)),
               "PaScaL_TDMA_plan_single_create")
        self._h, self.n_sys = h, 1

    def destroy(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tcs_tdma_plan_single_destroy(self._h)
            self._h = None

    def _single(self, fn: str, A, B, C, D, n_row: int) -> None:
        ptrs = []
        for x in (A, B, C, D):
            assert isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]
            ptrs.append(x.ctypes.data)
        _check(getattr(load(), fn)(self._h, *ptrs, int(n_row)), fn)

    def single_solve(self, A, B, C, D, n_row: int) -> None:
        self._single("tcs_tdma_single_solve", A, B, C, D, n_row)

    def single_solve_cycle(self, A, B, C, D, n_row: int) -> None:
        self._single("tcs_tdma_single_solve_cycle", A, B, C, D, n_row)


# Largest n_sys * n_row accepted by tdma_many_solve_noalloc (TCS_TDMA_NOALLOC_MAX_ELEMS).
TDMA_NOALLOC_MAX_ELEMS = 1 << 18


def tdma_many_solve_noalloc(A: np.ndarray, B: np.ndarray, C: np.ndarray, D: np.ndarray,
                            n_sys: int, n_row: int, cyclic: bool = False) -> None:
    """PaScaL_TDMA many-systems solve for callers that cannot allocate device
    memory: host arrays are staged through a fixed device array inside the
    library (no plan, no cudaMalloc).  D receives the solution, A and C are
    clobbered.  Calls that overlap on the GPU share the array and race."""
    for x in (A, B, C, D):
        assert isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]
    _check(load().tcs_tdma_many_solve_noalloc(A.ctypes.data, B.ctypes.data, C.ctypes.data, D.ctypes.data,
                                              int(n_sys), int(n_row), int(bool(cyclic))),
           "tcs_tdma_many_solve_noalloc")

"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a C restatement of the PaScaL_TCS time step on one MPI rank
(see tcs_oracle.c).  Only the test suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` load it; the CUDA library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtcs_oracle.so")

FIELDS = {"T": 0, "U": 1, "V": 2, "W": 3, "P": 4, "dPhat": 5, "dP0": 6,
          "dU": 7, "dV": 8, "dW": 9, "dP": 10, "Mu": 11, "invRho": 12}
METRICS = {"x1": 0, "dx1": 1, "dmx1": 2, "x2": 3, "dx2": 4, "dmx2": 5,
           "x3": 6, "dx3": 7, "dmx3": 8}
STAGES = ["thermal", "ghost_T", "mom_coeffi", "dU", "dV", "dW", "blockLdV",
          "blockLdU", "pseudo", "prhs", "poisson", "project", "post"]
DIAG = ["dt", "time", "maxDivU", "CFL", "Nu_bot", "Nu_top", "KE"]


class OracleParams(ctypes.Structure):
    _fields_ = [("n1m", ctypes.c_int), ("n2m", ctypes.c_int), ("n3m", ctypes.c_int),
                ("uniform1", ctypes.c_int), ("uniform2", ctypes.c_int), ("uniform3", ctypes.c_int),
                ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("gamma3", ctypes.c_double),
                ("aspect1", ctypes.c_double), ("H", ctypes.c_double), ("aspect3", ctypes.c_double),
                ("Ra", ctypes.c_double), ("Pr", ctypes.c_double), ("DeltaT", ctypes.c_double),
                ("MaxCFL", ctypes.c_double), ("dtStart", ctypes.c_double), ("tStart", ctypes.c_double),
                ("property_set", ctypes.c_int), ("fixed_dt", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("noise_amp", ctypes.c_double),
                ("init_mode", ctypes.c_int), ("top_wall_mode", ctypes.c_int)]


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.tcs_oracle_create.restype = ctypes.c_void_p
        L.tcs_oracle_create.argtypes = [ctypes.POINTER(OracleParams)]
        L.tcs_oracle_destroy.argtypes = [ctypes.c_void_p]
        L.tcs_oracle_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        for fn in ("tcs_oracle_get_field", "tcs_oracle_set_field", "tcs_oracle_get_metric"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
            getattr(L, fn).restype = ctypes.c_int
        L.tcs_oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.tcs_oracle_step.restype = ctypes.c_int
        L.tcs_oracle_run_stage.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.tcs_oracle_run_stage.restype = ctypes.c_int
        L.tcs_oracle_scalars.argtypes = [ctypes.c_void_p, dp]
        L.tcs_oracle_diagnostics.argtypes = [ctypes.c_void_p, dp]
        L.tcs_oracle_set_threads.argtypes = [ctypes.c_int]
        L.tcs_oracle_set_threads.restype = ctypes.c_int
        L.tcs_oracle_get_prhs.argtypes = [ctypes.c_void_p, dp]
        L.tcs_oracle_set_prhs.argtypes = [ctypes.c_void_p, dp]
        L.tcs_oracle_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.tcs_oracle_tdma_many.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.tcs_oracle_tdma_many_cycle.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.tcs_oracle_fft_c2c.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        L.tcs_oracle_fft_c2c.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def default_params(**kw) -> dict:
    """The 64^3 constant-property case: Lx = Lz = 2, Ly = 1, tanh-stretched y."""
    p = dict(n1m=64, n2m=64, n3m=64, uniform1=1, uniform2=0, uniform3=1,
             gamma1=3.0, gamma2=1.5, gamma3=3.0, aspect1=2.0, H=1.0, aspect3=2.0,
             Ra=1e5, Pr=0.71, DeltaT=10.0, MaxCFL=1.0, dtStart=1e-3, tStart=0.0,
             property_set=0, fixed_dt=1, seed=0, noise_amp=0.01, init_mode=0,
             top_wall_mode=0)
    p.update(kw)
    return p


def set_threads(n: int) -> int:
    return lib().tcs_oracle_set_threads(int(n))


class Oracle:
    """One simulation case held by the C oracle.  Fields are numpy arrays of
    shape (N3+2, N2+2, N1+2) -- C order, so i is the fastest index as in the
    reference's Fortran arrays (0:n1sub, 0:n2sub, 0:n3sub)."""

    def __init__(self, **params):
        self.params = default_params(**params)
        cp = OracleParams(**self.params)
        self._h = lib().tcs_oracle_create(ctypes.byref(cp))
        if not self._h:
            raise ValueError("oracle rejected the parameters")
        d = (ctypes.c_int * 3)()
        lib().tcs_oracle_dims(self._h, d)
        self.shape = (d[2], d[1], d[0])
        self.n1m, self.n2m, self.n3m = self.params["n1m"], self.params["n2m"], self.params["n3m"]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.tcs_oracle_destroy(h)
            self._h = None

    def get(self, name: str) -> np.ndarray:
        a = np.empty(self.shape, dtype=np.float64)
        if lib().tcs_oracle_get_field(self._h, FIELDS[name], _ptr(a)) != 0:
            raise KeyError(name)
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
        if lib().tcs_oracle_set_field(self._h, FIELDS[name], _ptr(a)) != 0:
            raise KeyError(name)

    def metric(self, name: str) -> np.ndarray:
        n = {"1": self.shape[2], "2": self.shape[1], "3": self.shape[0]}[name[-1]]
        a = np.empty(n, dtype=np.float64)
        lib().tcs_oracle_get_metric(self._h, METRICS[name], _ptr(a))
        return a

    def step(self, n: int = 1) -> np.ndarray:
        diag = np.zeros((n, len(DIAG)), dtype=np.float64)
        r = lib().tcs_oracle_step(self._h, int(n), _ptr(diag))
        if r < 0:
            raise FloatingPointError(f"oracle BLOW UP at step {-r}")
        return diag

    def stage(self, name: str) -> None:
        if lib().tcs_oracle_run_stage(self._h, STAGES.index(name)) != 0:
            raise ValueError(name)

    def scalars(self) -> dict:
        a = np.zeros(7)
        lib().tcs_oracle_scalars(self._h, _ptr(a))
        return dict(zip(["time", "dt", "CFL", "maxDivU", "Cmu", "Ct", "dtMax"], a.tolist()))

    def diagnostics(self) -> dict:
        a = np.zeros(3)
        lib().tcs_oracle_diagnostics(self._h, _ptr(a))
        return dict(zip(["Nu_bot", "Nu_top", "KE"], a.tolist()))

    def get_prhs(self) -> np.ndarray:
        a = np.empty((self.n3m, self.n2m, self.n1m), dtype=np.float64)
        lib().tcs_oracle_get_prhs(self._h, _ptr(a))
        return a

    def set_prhs(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.n3m, self.n2m, self.n1m)
        lib().tcs_oracle_set_prhs(self._h, _ptr(a))

    def set_dt(self, dt: float) -> None:
        lib().tcs_oracle_set_dt(self._h, float(dt))


def tdma_many(A, B, C, D, cyclic: bool = False) -> np.ndarray:
    """PaScaL_TDMA_many_solve(_cycle) on one rank.  Inputs are (n_row, n_sys)
    numpy arrays (C order = system index fastest, as the Fortran (n_sys, n_row));
    returns the solution, leaving the inputs untouched."""
    A, B, C, D = (np.ascontiguousarray(x, dtype=np.float64).copy() for x in (A, B, C, D))
    n_row, n_sys = D.shape
    fn = lib().tcs_oracle_tdma_many_cycle if cyclic else lib().tcs_oracle_tdma_many
    fn(_ptr(A), _ptr(B), _ptr(C), _ptr(D), n_sys, n_row)
    return D


def fft_c2c(x: np.ndarray, sign: int = -1) -> np.ndarray:
    """Unnormalised complex DFT along the last axis (sign -1 forward)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    n = x.shape[-1]
    buf = x.reshape(-1, n).view(np.float64).copy()
    lib().tcs_oracle_fft_c2c(n, buf.shape[0], _ptr(buf), int(sign))
    return buf.view(np.complex128).reshape(x.shape)

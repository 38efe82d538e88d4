"""Make the golden fixtures of tests/golden (run from the repository root:
`python tests/golden/make_golden.py`).  Test infrastructure.

The reference (Fortran, MPI, FFTW/MKL) has no toolchain on this machine and
ships no stored answers, so the fixtures come from two sources, each named
in the file:
  * tdma_dense.npz: tridiagonal and cyclic-tridiagonal systems in the
    PaScaL_TDMA layout (n_row, n_sys), system index fastest, with solutions
    from a dense LU solve of each system (numpy.linalg.solve); independent of
    both the oracle and the library;
  * rb16_*_oracle.npz: short runs of the test oracle (the one-rank C
    restatement of main.f90's time step) on small seeded cases: the
    configuration, the padded fields T, U, V, W, P after the run and the
    per-step series dt, time, maxDivU, CFL, Nu_bot, Nu_top, KE.  They pin the
    oracle against later changes and give the GPU tests a fixed answer.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# systems of the dense fixture: odd row count, a few systems
TDMA_ROWS, TDMA_SYS, TDMA_SEED = 33, 6, 20260

# the oracle runs: (file, steps, configuration over the oracle's defaults)
RUNS = [
    ("rb16_water_oracle.npz", 6, dict(n1m=16, n2m=12, n3m=10, property_set=1, Pr=7.0, Ra=1e6, DeltaT=10.0,
                                      dtStart=5e-4, fixed_dt=1, seed=5)),
    ("rb16_glycerol_oracle.npz", 6, dict(n1m=12, n2m=16, n3m=10, property_set=2, Pr=7.0, Ra=1e5,
                                         dtStart=5e-4, fixed_dt=1, seed=6, uniform1=0, gamma1=1.2,
                                         top_wall_mode=1)),
]
FIELDS = ("T", "U", "V", "W", "P")


def dense_solution(A, B, C, D, cyclic):
    n_row, n_sys = D.shape
    X = np.empty_like(D)
    for s in range(n_sys):
        M = np.zeros((n_row, n_row))
        M[np.arange(n_row), np.arange(n_row)] = B[:, s]
        M[np.arange(1, n_row), np.arange(n_row - 1)] = A[1:, s]
        M[np.arange(n_row - 1), np.arange(1, n_row)] = C[:-1, s]
        if cyclic:
            M[0, n_row - 1] = A[0, s]
            M[n_row - 1, 0] = C[n_row - 1, s]
        X[:, s] = np.linalg.solve(M, D[:, s])
    return X


def make_tdma():
    rng = np.random.default_rng(TDMA_SEED)
    out = {}
    for cyclic in (0, 1):
        shape = (TDMA_ROWS, TDMA_SYS)
        A = rng.uniform(-0.4, 0.4, shape)
        C = rng.uniform(-0.4, 0.4, shape)
        B = 1.0 + rng.uniform(0.0, 1.0, shape)
        D = rng.uniform(-1.0, 1.0, shape)
        out.update({f"A{cyclic}": A, f"B{cyclic}": B, f"C{cyclic}": C, f"D{cyclic}": D,
                    f"X{cyclic}": dense_solution(A, B, C, D, cyclic)})
    np.savez_compressed(os.path.join(HERE, "tdma_dense.npz"), **out)


def make_runs():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    O.build()
    for name, steps, cfg in RUNS:
        params = O.default_params(**cfg)
        o = O.Oracle(**params)
        diag = o.step(steps)
        arrays = {f: o.get(f) for f in FIELDS}
        np.savez_compressed(os.path.join(HERE, name), config=json.dumps(params), steps=steps,
                            series=diag, **arrays)


if __name__ == "__main__":
    make_tdma()
    make_runs()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))

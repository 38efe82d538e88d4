"""Fill the launch-shape cache that tcs_autotune reads (one line per grid
shape and precision): python -m pascal_tcs_b200.tune --out FILE [--trial-steps K]
SHAPE... where SHAPE is N1xN2xN3:PREC (PREC 0 = FP64 plain, 1 = FP32-mixed).
Tuning runs on the current GPU; every shape starts from its seeded state."""
from __future__ import annotations

import argparse
import sys

from .tcs import Solver

CACHE = __file__.replace("tune.py", "tune_cache.txt")


def parse(shape: str) -> dict:
    dims, _, prec = shape.partition(":")
    n1, n2, n3 = (int(x) for x in dims.split("x"))
    return dict(n1m=n1, n2m=n2, n3m=n3, precision=int(prec or 0))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("shapes", nargs="+")
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--trial-steps", type=int, default=3)
    args = ap.parse_args(argv)
    for sh in args.shapes:
        cfg = dict(parse(sh), gamma2=1.5, property_set=1, Pr=7.0, Ra=1e8, DeltaT=10.0, dtStart=2e-4, fixed_dt=1,
                   seed=1, noise_amp=0.01)
        s = Solver(**cfg)
        knobs, hit = s.autotune(trial_steps=args.trial_steps, cache_path=args.out)
        print(sh, "cached" if hit else "tuned", knobs, flush=True)
        s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

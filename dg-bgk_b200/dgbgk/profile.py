"""Per-kernel device times of a few pseudo-time steps of a generated case.

    python -m dgbgk.profile --config channel --precision 32 --steps 3

Builds the case, starts it from its initial condition, runs two untimed
steps and then `--steps` steps launch by launch (dgbgk_profile_steps), and
prints the mean device milliseconds per step of the moment, wall-flux,
sweep and residual kernels.  It is the command the ncu captures of single
kernels are taken under (a short run, so that a capture stays small).
"""
import argparse
import json

from .cases import config1, config2, config5
from .solver import Solver

CONFIGS = {"cavity": config1, "channel": config2, "large": config5}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="channel", choices=sorted(CONFIGS))
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--tile-elems", type=int, default=0)
    ap.add_argument("--moment-rows", type=int, default=0, help="moment rows per warp step (1-4; 0: the library's)")
    ap.add_argument("--lib", default=None, help="a library build to time instead of lib/libdgbgk.so "
                    "(e.g. an earlier build kept for an A/B timing)")
    a = ap.parse_args(argv)
    if a.lib:
        from . import _lib
        _lib.use_library(a.lib)
    case = CONFIGS[a.config]()
    s = Solver.from_case(case, precision=a.precision, tile_elems=a.tile_elems, moment_rows=a.moment_rows)
    s.init_case()
    s.advance(2)
    ms = s.profile(a.steps)
    info = s.info()
    print(json.dumps({"case": case.name, "precision": a.precision, "tile_elems": info["tile_elems"],
                      "steps": a.steps, "kernel_ms": dict(zip(["k_moments", "k_wall", "k_sweep", "k_resid"],
                                                              [float(x) for x in ms]))}))


if __name__ == "__main__":
    main()

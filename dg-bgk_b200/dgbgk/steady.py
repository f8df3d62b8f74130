"""Marching a case to steady state, and the time it takes.

    python -m dgbgk.steady --config cavity --precision 64 --tol 1e-8

`march` runs pseudo-time steps on the device until the L2 residual falls to
`tol` times the reference residual, in chunks (the device stops by itself
inside a chunk; the host only decides whether to launch the next one).  The
reference is the first step's residual of a cold start; a warm start is
judged against the cold start's reference (`ref`), so both runs stop at the
same absolute residual.  Device time comes from the library's CUDA events
around each advance call.
"""
import argparse
import json
import time

import numpy as np

from .cases import config1, config2, config5, cavity_case
from .solver import Solver

CONFIGS = {"cavity": config1, "channel": config2, "large": config5,
           "cavity16": lambda: cavity_case(16, 16, 32, mach=0.3, kn=0.1)}


def march(solver, tol, max_steps, chunk=200000, ref=None):
    """Steps `solver` until its L2 residual <= tol * reference or max_steps.
    Returns steps, device seconds, wall seconds, the last relative residual
    and the reference used."""
    if ref is not None:
        solver.set_residual_reference(ref)
    steps, dev_ms, last = 0, 0.0, np.nan
    t0 = time.perf_counter()
    while steps < max_steps:
        n = min(chunk, max_steps - steps)
        r = solver.advance(n, tol=tol)
        steps += r["steps"]
        dev_ms += solver.last_ms()
        if r["steps"]:
            last = float(r["res_l2"][-1])
        ref_used = solver.residual_reference()
        if r["steps"] < n or (ref_used > 0 and last <= tol * ref_used):
            break
    ref_used = solver.residual_reference()
    return {"steps": steps, "device_s": dev_ms * 1e-3, "wall_s": time.perf_counter() - t0,
            "res_rel": last / ref_used if ref_used > 0 else np.nan, "ref": ref_used,
            "converged": bool(ref_used > 0 and last <= tol * ref_used)}


def cold_march(case, precision, tol, max_steps, **kw):
    s = Solver.from_case(case, precision=precision, **kw)
    s.init_case()
    out = march(s, tol, max_steps)
    out.update({"case": case.name, "precision": precision, "dofs": case.dofs})
    return out, s


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="cavity", choices=sorted(CONFIGS))
    ap.add_argument("--precision", type=int, default=64, choices=[32, 64])
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-steps", type=int, default=2000000)
    a = ap.parse_args(argv)
    out, _ = cold_march(CONFIGS[a.config](), a.precision, a.tol, a.max_steps)
    print(json.dumps(out))


if __name__ == "__main__":
    main()

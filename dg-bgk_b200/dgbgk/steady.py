"""Marching a case to steady state, and the time it takes.

    python -m dgbgk.steady --config cavity --precision 64 --tol 1e-8
    python -m dgbgk.steady --config batch64 --precision 32 --budget-s 600 --out r.json

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


def batch_march(cases, precision, tol, budget_s, chunk=2000, window=4000):
    """The batched workload: every case in one Batch (autotuned shape),
    marched in chunks until all reach tol or `budget_s` seconds of device
    time have run.  Per case: steps, the relative residual reached, its
    decay over the last `window` steps (decades per 1000 steps) and, for a
    case short of tol, the steps still needed at that rate."""
    from .solver import Batch
    ss = [Solver.from_case(c, precision=precision) for c in cases]
    for s in ss:
        s.init_case()
    b = Batch(ss)
    n = len(ss)
    steps = np.zeros(n, dtype=np.int64)
    rel = np.full(n, np.nan)
    hist = [[] for _ in range(n)]  # (step, rel) per chunk
    status = np.zeros(n, dtype=np.int32)
    dev = 0.0
    while dev < budget_s:
        live = (status == 0) & ~(rel <= tol)
        if not live.any():
            break
        b.set_active(live)
        r = b.advance(chunk, tol=tol, raise_on_error=False)
        dev += b.last_ms() * 1e-3
        for i in np.flatnonzero(live):
            steps[i] += r["steps"][i]
            status[i] = r["status"][i]
            ref = ss[i].residual_reference()
            if r["steps"][i] and ref > 0:
                rel[i] = r["res_l2_last"][i] / ref
                hist[i].append((int(steps[i]), float(rel[i])))
    per = []
    for i, c in enumerate(cases):
        h = [x for x in hist[i] if x[0] >= steps[i] - window] or hist[i][-1:]
        rate = None
        if len(h) >= 2 and h[0][1] > 0 and h[-1][1] > 0 and h[-1][0] > h[0][0]:
            rate = (np.log10(h[0][1]) - np.log10(h[-1][1])) / ((h[-1][0] - h[0][0]) / 1000.0)
        more = None
        if not rel[i] <= tol and rate and rate > 0:
            more = int(np.ceil((np.log10(rel[i]) - np.log10(tol)) / rate * 1000.0))
        per.append({"case": c.name, "dofs": c.dofs, "mach": c.info.get("mach"), "kn": c.info.get("kn"),
                    "steps": int(steps[i]), "res_rel": float(rel[i]), "status": int(status[i]),
                    "converged": bool(rel[i] <= tol), "decades_per_1000_steps": rate, "steps_still_needed": more})
    info = b.shape_record()
    out = {"ncases": n, "precision": precision, "tol": tol, "device_s": dev, "budget_s": budget_s,
           "batch_shape": info, "tuning_ms_per_step": {str(k): v for k, v in b.tuning().items()},
           "converged": int(sum(p["converged"] for p in per)), "cases": per}
    b.close()
    for s in ss:
        s.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="cavity", choices=sorted(CONFIGS) + ["batch64"])
    ap.add_argument("--precision", type=int, default=64, choices=[32, 64])
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-steps", type=int, default=2000000)
    ap.add_argument("--budget-s", type=float, default=600.0, help="device seconds for --config batch64")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.config == "batch64":
        from .cases import config3
        out = batch_march(config3(), a.precision, a.tol, a.budget_s)
    else:
        out, _ = cold_march(CONFIGS[a.config](), a.precision, a.tol, a.max_steps)
    print(json.dumps(out))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()

"""The learned warm start, end to end: data, training, and the time to
steady state with and without it.

    python -m dgbgk.study --train 384 --test 32 --out study.json
    torchrun --nproc-per-node 8 --master-addr 127.0.0.1 -m dgbgk.study ...

Under torchrun the training set is generated by every rank, each on its own
GPU, as a round-robin share of the cases (independent steady states: no
data crosses GPUs), and gathered once by rank 0, which trains and evaluates.

A family of supersonic channel cases (square obstacle; Mach, Kn and the
obstacle side drawn per case) is marched to steady state by the batch API
in FP32; the nodal density, velocity and temperature are resampled to a
64 x 128 grid and an MLP (3 -> 512 x 4 -> 32768, BF16 tensor-core kernels)
learns the map from the case parameters to those grids.  Held-out cases are
then brought to the L2 residual 1e-8 (relative to the first step of a cold
start) four ways:

  plain        FP64, cold start, one case at a time (the reference method)
  batch64      FP64, cold start, all cases in one batch
  batch64_warm FP64, started from the network's prediction, one batch
  fast         started from the prediction, FP32 in one batch until the
               residual reaches `switch_tol` (or the FP32 rounding plateau),
               then the state is handed to FP64 handles (dgbgk_copy_state)
               and the batch finishes to 1e-8
  fast_cold    as fast, from the cold start (no network)
  *_rre        the same with reduced-rank extrapolation of the iterates
               (march_batch_rre: the same fixed point in fewer steps)

A stored FP32 state stops changing once every update is below half an ulp,
so an FP32 march settles anywhere within about tau * ulp / 2 of its fixed
point (tau = the slowest mode's decay time in steps, ~600 on these
channels): ~1e-5 in the fields, far above the FP64 solution's own
tolerance.  The FP64 finish removes that offset; the fast path's final
fields are compared with the plain path's.  A warm-started march confirms
that it has converged: a residual at tol must still be falling WARM_CONFIRM
steps later (a warm start can set off a slow transient whose residual dips
below tol on its way).
"""
import argparse
import json
import math
import os
import time

import numpy as np

from .cases import channel_case
from .resample import GridResampler
from .solver import Batch, Solver

# The case family: the channel of the Mach 2 workload widened to
# [-5,15]x[-10,10] with free-stream top and bottom sides, 100 x 100 quads
# (h = 0.2), 16 x 32 velocities, Mach U[2,3], Kn logU[0.04,0.12], obstacle
# side U[0.6,1.4] (snapped to whole cells).
#  * The steady state must not depend on the starting state, or a warm start
#    converges to another answer.  With zero-gradient top and bottom sides
#    (the [-5,5] channel) it does: a transverse disturbance there is neither
#    damped nor fixed, and restarts from perturbed or neighbouring steady
#    fields settled 5-20% away from the cold start's answer.  Free-stream
#    sides at y = +-5 are crossed by the bow shock, and the reset against the
#    post-shock flow left two steady states (1e-3 apart, at the outflow
#    corner).  At y = +-10 the shock leaves through the outflow for every
#    Mach number in the family, and restarts from perturbed (T +-5-10%,
#    n +-10%, u -5%, v +5%) and neighbouring fields all land within 4e-7 of
#    the cold start's fields at residual 1e-8.
#  * The explicit scheme diverges for M <= 1.5 and for the most rarefied
#    cases (Kn >= 0.14 at obstacle side >= 1.4); the study drops any case the
#    cold FP64 march does not bring to 1e-8.
FAMILY = {"box": (-5.0, 15.0, -10.0, 10.0), "nx": 100, "ny": 100, "nr": 16, "nt": 32,
          "mach": (2.0, 3.0), "kn": (0.04, 0.12), "side": (0.6, 1.4), "sides": "freestream"}
GRID = (64, 128)  # ny, nx of the resampled fields
NF = 4            # n, u, v, T


def draw_cases(n, seed, family=FAMILY):
    """n cases with parameters drawn by numpy PCG64(seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    f = family
    out = []
    for _ in range(n):
        m = float(rng.uniform(*f["mach"]))
        kn = float(10.0 ** rng.uniform(math.log10(f["kn"][0]), math.log10(f["kn"][1])))
        side = float(rng.uniform(*f["side"]))
        x0, x1, y0, y1 = f["box"]
        c = channel_case(x0, x1, y0, y1, f["nx"], f["ny"], f["nr"], f["nt"], mach=m, kn=kn, obstacle_side=side,
                         sides=f["sides"])
        c.info["side_drawn"] = side
        out.append(c)
    return out


def params_vector(case, family=FAMILY):
    """Network input in [-1, 1]^3: Mach, log10 Kn, snapped obstacle side."""
    f = family
    lk = [math.log10(k) for k in f["kn"]]

    def sc(x, lo, hi):
        return 2.0 * (x - lo) / (hi - lo) - 1.0
    return np.array([sc(case.info["mach"], *f["mach"]), sc(math.log10(case.info["kn"]), *lk),
                     sc(case.info["obstacle_side"], *f["side"])], dtype=np.float32)


def _freestream(case):
    T1, P1, U0 = case.init["T1"], case.init["P1"], case.init["U0"]
    mm = case.molar_mass / 6.022e26
    n1 = (P1 * 1e5) / (case.rgas * T1) / mm
    return n1, U0, T1, mm


def nodal_fields(solver, case):
    """(4, NELEM, 3): n / n_inf, u / U_inf, v / U_inf, T / T_inf per DG node
    (T = DISPS / (DISND m R), the pressure moment over n m R)."""
    nf = solver.node_fields()
    n1, U, T1, mm = _freestream(case)
    nd = nf["disnd"]
    t = np.where(nd > 0, nf["disps"] / np.maximum(nd * mm * case.rgas, 1e-300), 0.0)
    return np.stack([nd / n1, nf["disux"] / U, nf["disuy"] / U, t / T1])


def init_from_fields(solver, case, q):
    """Maxwellian per DG node from normalised fields q (4, NELEM, 3)."""
    n1, U, T1, _ = _freestream(case)
    n = np.maximum(q[0], 1e-3) * n1
    t = np.maximum(q[3], 1e-2) * T1
    solver.init_maxwellian(n, q[1] * U, q[2] * U, t)


def resampler(case):
    m = case.mesh
    return GridResampler(m.intma, m.coord, GRID[1], GRID[0], box=FAMILY["box"])


# The batch autotuner's choice per (precision, the cases' sizes): a family's
# later batches take it instead of tuning again (the tuning is a per-family
# cost, as a production host would cache it).
_TUNED = {}


def _family_key(solvers):
    return (solvers[0].precision, tuple(sorted((s.E, s.V) for s in solvers)))


def tuned_batch(solvers):
    """A Batch over `solvers` with the shape tuned once per family."""
    key = _family_key(solvers)
    if key in _TUNED:
        sh = _TUNED[key]
        return Batch(solvers, tile_elems=sh["tile_elems"], units_per_cta=sh["units_per_cta"],
                     moment_rows=sh["moment_rows"], tune_steps=1)
    b = Batch(solvers)
    _TUNED[key] = b.shape_record()
    return b


def pretune(cases, precision, device=0):
    """Tunes the batch shape of `cases` at `precision` (outside any timing)."""
    ss = [Solver.from_case(c, precision=precision, device=device) for c in cases]
    for s in ss:
        s.init_case()
    b = tuned_batch(ss)
    shape = b.shape_record()
    b.close()
    for s in ss:
        s.close()
    return shape


def march_batch(b, solvers, tol, max_steps, chunk=1000, stall=0.8, stall_below=1e-3):
    """Advances batch `b` until every case has reached tol (relative to its
    reference), has stalled (below stall_below, its residual fell by less
    than the factor `stall` over the last chunk: an FP32 march at its
    rounding plateau; the transient's residual may rise for a while above
    that), has diverged, or max_steps have run.  A finished case is left
    out of the following chunks (dgbgk_batch_set_active).  Returns steps per
    case, the last relative residuals, the statuses and the device
    seconds."""
    n = len(solvers)
    steps = np.zeros(n, dtype=np.int64)
    status = np.zeros(n, dtype=np.int32)
    prev = np.full(n, np.inf)
    rel = np.full(n, np.inf)
    done = np.zeros(n, dtype=bool)
    dev = 0.0
    while steps.max() < max_steps:
        r = b.advance(min(chunk, max_steps - int(steps.max())), tol=tol, raise_on_error=False)
        dev += b.last_ms() * 1e-3
        live = (status == 0) & ~done
        steps[live] += r["steps"][live]
        status[live] = r["status"][live]
        refs = np.array([s.residual_reference() for s in solvers])
        now = r["res_l2_last"] / np.maximum(refs, 1e-300)
        rel = np.where(live & (r["steps"] > 0), now, rel)
        done |= (rel <= tol * (1 + 1e-9)) | (status != 0) | ((rel > stall * prev) & (rel < stall_below))
        prev = np.where(live, rel, prev)
        if done.all():
            break
        b.set_active(~done)
    b.set_active(np.ones(n, dtype=bool))
    return steps, rel, status, dev


def march_batch_rre(b, solvers, tol, max_steps, start=1e-2, every=100, m=8, stall=0.8, stall_below=1e-3,
                    confirm=0):
    """march_batch with reduced-rank extrapolation (dgbgk_extrapolate):
    once a case's relative residual is below `start`, each cycle of `every`
    steps ends with m + 1 single steps whose m + 2 states the case
    snapshots and extrapolates from.  A case whose residual grew tenfold
    over the cycle after an extrapolation extrapolates no more.  The fixed
    point and the convergence test are the march's own; only the path to it
    changes.

    confirm > 0: a case that reaches tol extrapolates no more, marches
    `confirm` more steps without the test and counts as converged only if
    its residual then is still at or below both tol and its value at the
    hit; otherwise it marches on (plainly) to the next hit.  A warm start can
    put a case on a transient whose residual grows for thousands of steps
    before it decays (a transport operator far from normal), and each
    extrapolation pulls such a residual down for a while: measured on a
    channel of the bench's set, the extrapolated march reached 1e-8 2e-3 (T)
    from the plain march's answer; marched on plainly its residual rose to
    4e-5 and then fell to the plain answer.  A case on its way to the fixed
    point keeps falling."""
    n = len(solvers)
    steps = np.zeros(n, dtype=np.int64)
    status = np.zeros(n, dtype=np.int32)
    prev = np.full(n, np.inf)
    rel = np.full(n, np.inf)
    done = np.zeros(n, dtype=bool)
    use = np.ones(n, dtype=bool)
    dev = [0.0]
    refs = np.array([s.residual_reference() for s in solvers])

    jumped = np.zeros(n, dtype=bool)  # marched a confirmation window this cycle

    def adv(k):
        run = ~done
        b.set_active(run)
        r = b.advance(k, tol=tol, raise_on_error=False)
        dev[0] += b.last_ms() * 1e-3
        live = (status == 0) & run
        steps[live] += r["steps"][live]
        status[live] = r["status"][live]
        now = r["res_l2_last"] / np.maximum(refs, 1e-300)
        rel[:] = np.where(live & (r["steps"] > 0), now, rel)
        reached = (status == 0) & run & (rel <= tol * (1 + 1e-9))
        done[:] |= status != 0
        if confirm <= 0:
            done[:] |= reached
            return
        # the cases that reached tol extrapolate no more and march `confirm`
        # steps more, all together and without the test; those still falling
        # are done
        if reached.any():
            use[:] &= ~reached
            hit = rel.copy()
            adv_confirm = reached & ~done
            b.set_active(adv_confirm)
            r = b.advance(confirm, tol=0.0, raise_on_error=False)
            dev[0] += b.last_ms() * 1e-3
            live = (status == 0) & adv_confirm
            steps[live] += r["steps"][live]
            status[live] = r["status"][live]
            now = r["res_l2_last"] / np.maximum(refs, 1e-300)
            rel[:] = np.where(live & (r["steps"] > 0), now, rel)
            done[:] |= (status != 0) | (live & (rel <= tol * (1 + 1e-9)) & (rel <= hit))
            jumped[:] |= adv_confirm

    cyc_before = np.full(n, np.inf)
    win_start = 0  # the stall test compares residuals 1000 steps apart
    while steps.max() < max_steps and not done.all():
        adv(every - (m + 1))
        grew = use & np.isfinite(cyc_before) & (rel > 10 * cyc_before)
        use &= ~grew
        if steps.max() - win_start >= 1000:
            stalled = (rel > stall * prev) & (rel < stall_below) & ~done
            prev = rel.copy()
            win_start = int(steps.max())
            done |= stalled
        if done.all():
            break
        act = np.flatnonzero(~done & use & (rel < start))
        cyc_before[:] = np.inf
        jumped[:] = False
        if len(act) == 0:
            continue
        # the snapshots and the extrapolation of the whole set in batch calls
        # (copies queued without a wait, one wait for all Gram matrices)
        sel = np.zeros(n, dtype=bool)
        sel[act] = True
        b.snapshot(0, sel)
        for j in range(m + 1):
            adv(1)
            b.snapshot(j + 1, sel)
        ext = sel & ~done & ~jumped  # not finished, snapshots consecutive
        if ext.any():
            cyc_before[ext] = rel[ext]
            st, _ = b.extrapolate(m + 2, ext)
            use[ext & (st != 0)] = False
    for s in solvers:
        s.snapshot(-1)
    b.set_active(np.ones(n, dtype=bool))
    return steps, rel.copy(), status, dev[0]


def shard(n, rank, world):
    """The case indices one rank of `world` generates: rank, rank + world, ...
    (round robin, so every rank gets the same mix of mesh sizes and Mach
    numbers).  The cases are independent steady states: no data crosses
    ranks until the finished sets are gathered."""
    return list(range(rank, n, world))


def generate(cases, precision=32, tol=1e-5, accept=1e-4, group=64, max_steps=60000, log=None, rank=0, world=1,
             device=0):
    """Marches this rank's share of the cases (batches of `group`) to tol, or
    to their FP32 rounding plateau; keeps those whose relative residual is
    <= accept.  Returns X (n, 3), Y (n, 4 * 64 * 128) and the kept cases'
    indices into `cases`."""
    X, Y, keep = [], [], []
    idx = shard(len(cases), rank, world)
    for g0 in range(0, len(idx), group):
        part_idx = idx[g0:g0 + group]
        part = [cases[i] for i in part_idx]
        ss = [Solver.from_case(c, precision=precision, device=device) for c in part]
        for s in ss:
            s.init_case()
        b = tuned_batch(ss)
        t = time.perf_counter()
        steps, rel, status, dev = march_batch(b, ss, tol, max_steps)
        if log:
            log(f"generate rank {rank}/{world} {g0}..{g0 + len(part)}: steps {int(steps.min())}..{int(steps.max())} "
                f"diverged {int((status != 0).sum())} kept {int(((status == 0) & (rel <= accept)).sum())} "
                f"device {dev:.1f} s wall {time.perf_counter() - t:.1f} s shape {b.shape_record()}")
        for k, (c, s) in enumerate(zip(part, ss)):
            if status[k] == 0 and rel[k] <= accept:
                q = nodal_fields(s, c)
                X.append(params_vector(c))
                Y.append(resampler(c).to_grid(q).reshape(-1).astype(np.float32))
                keep.append(part_idx[k])
        b.close()
        for s in ss:
            s.close()
    return np.array(X, dtype=np.float32), np.array(Y, dtype=np.float32), keep


def merge_generated(parts):
    """The (X, Y, keep) sets of every rank as one set in case order."""
    parts = [p for p in parts if len(p[2])]
    if not parts:
        return np.zeros((0, 3), np.float32), np.zeros((0, NF * GRID[0] * GRID[1]), np.float32), []
    X = np.concatenate([p[0] for p in parts])
    Y = np.concatenate([p[1] for p in parts])
    keep = [i for p in parts for i in p[2]]
    order = np.argsort(keep, kind="stable")
    return X[order], Y[order], [keep[i] for i in order]


class WarmStart:
    """The network and its output standardisation."""

    def __init__(self, width=512, depth=4, batch=128, seed=0):
        from .warmstart import MLP
        self.mlp = MLP(3, width, depth, NF * GRID[0] * GRID[1], batch, seed=seed)
        self.mean = None
        self.std = None
        self.train_s = 0.0

    def fit(self, X, Y, schedule=((3000, 1e-3), (1500, 3e-4), (1500, 1e-4)), seed=0):
        self.mean = Y.mean(axis=0)
        self.std = np.maximum(Y.std(axis=0), 1e-3)
        Z = ((Y - self.mean) / self.std).astype(np.float32)
        self.mlp.set_data(X, Z)
        hist = []
        t = time.perf_counter()
        for i, (iters, lr) in enumerate(schedule):
            hist.append(self.mlp.train(iters, lr=lr, seed=seed + i))
        self.train_s = time.perf_counter() - t
        return np.concatenate(hist)

    def predict_grids(self, X):
        z = self.mlp.forward(np.asarray(X, dtype=np.float32))
        return (z * self.std + self.mean).reshape(-1, NF, GRID[0], GRID[1])

    def warm(self, solvers, cases):
        """Initialises each solver from the prediction for its case."""
        grids = self.predict_grids(np.stack([params_vector(c) for c in cases]))
        for s, c, g in zip(solvers, cases, grids):
            init_from_fields(s, c, resampler(c).to_nodes(g))
        return grids


def cold_reference(case, device=0):
    """The L2 residual of the first FP64 step from the cold start."""
    s = Solver.from_case(case, precision=64, device=device)
    s.init_case()
    s.advance(1)
    r = s.residual_reference()
    s.close()
    return r


def rel_fields(a, b):
    """Relative L2 differences of n, u, v, T (normalised fields)."""
    return {k: float(np.linalg.norm(a[i] - b[i]) / max(np.linalg.norm(b[i]), 1e-300))
            for i, k in enumerate(("n", "u", "v", "T"))}


# steps a warm-started case marches past its first residual <= tol before it
# counts as converged (march_batch_rre's confirm)
WARM_CONFIRM = 200


def evaluate(cases, ws, tol=1e-8, switch_tol=1e-5, max_steps=200000,
             ways=("plain", "batch64", "batch64_warm", "fast"), log=None, device=0):
    """Time to tol for each way (see the module docstring); returns the
    results, the final normalised nodal fields per way and the cases kept."""
    from ._lib import DgbgkError
    refs = [cold_reference(c, device) for c in cases]
    out = {"ncases": len(cases), "tol": tol, "switch_tol": switch_tol}
    final = {}

    if "plain" in ways:
        # cases the reference method does not bring to tol are left out of
        # every comparison
        steps, dev, wall, fields, kept = [], 0.0, 0.0, [], []
        for i, (c, ref) in enumerate(zip(cases, refs)):
            s = Solver.from_case(c, precision=64, device=device)
            s.init_case()
            s.set_residual_reference(ref)
            t = time.perf_counter()
            try:
                r = s.advance(max_steps, tol=tol)
            except DgbgkError:
                s.close()
                continue
            if r["steps"] >= max_steps:
                s.close()
                continue
            wall += time.perf_counter() - t
            dev += s.last_ms() * 1e-3
            steps.append(r["steps"])
            fields.append(nodal_fields(s, c))
            kept.append(i)
            s.close()
        out["plain"] = {"wall_s": wall, "device_s": dev, "steps": [int(x) for x in steps]}
        out["ncases"] = len(kept)
        out["dropped"] = len(cases) - len(kept)
        cases = [cases[i] for i in kept]
        refs = [refs[i] for i in kept]
        final["plain"] = fields
        if log:
            log(f"plain: {wall:.2f} s, steps {min(steps)}..{max(steps)}, dropped {out['dropped']}")

    # the batch shapes of this set, tuned once per precision outside the
    # timed marches (the plain arm has no tuning either)
    if any(w != "plain" for w in ways):
        out["batch_shapes"] = {f"fp{p}": pretune(cases, p, device) for p in (32, 64)}

    def batched(name, warm, precision_first, switch, rre=False):
        t0 = time.perf_counter()
        first = [Solver.from_case(c, precision=precision_first, device=device) for c in cases]
        fin = [Solver.from_case(c, precision=64, device=device) for c in cases] if switch else first
        t_setup = time.perf_counter() - t0
        t = time.perf_counter()
        if warm:
            ws.warm(first, cases)
        else:
            for s in first:
                s.init_case()
        for s, ref in zip(first, refs):
            s.set_residual_reference(ref)
        t_init = time.perf_counter() - t
        b = tuned_batch(first)
        t_tune = time.perf_counter() - t
        # a warm-started march to tol confirms its convergence (march_batch_rre)
        confirm = WARM_CONFIRM if warm else 0
        if rre:
            steps1, _, st1, dev = march_batch_rre(b, first, switch or tol, max_steps,
                                                  stall_below=1e-3 if switch else 0.0,
                                                  confirm=0 if switch else confirm)
        elif switch:
            steps1, _, st1, dev = march_batch(b, first, switch, max_steps)
        else:
            steps1, _, st1, dev = march_batch(b, first, tol, max_steps, chunk=max_steps, stall_below=0.0)
        # the cold start is the fallback: a warm-started case that diverged
        # starts again from the free stream
        fell_back = np.flatnonzero(st1 != 0)
        if len(fell_back):
            b.close()
            again = [first[i] for i in fell_back]
            for i in fell_back:
                first[i].init_case()
                first[i].set_residual_reference(refs[i])
            b = tuned_batch(again)
            s_again, _, st_again, d_again = march_batch(b, again, switch or tol, max_steps,
                                                        stall_below=1e-3 if switch else 0.0)
            if (st_again != 0).any():
                raise RuntimeError(f"{name}: a case diverged from the cold start too")
            steps1[fell_back] += s_again
            dev += d_again
        steps2 = np.zeros_like(steps1)
        if switch:
            for a, s in zip(fin, first):
                a.copy_state_from(s)
            b2 = tuned_batch(fin)
            if rre:
                steps2, _, _, d2 = march_batch_rre(b2, fin, tol, max_steps, stall_below=0.0, confirm=confirm)
                dev += d2
            else:
                r2 = b2.advance(max_steps, tol=tol)
                dev += b2.last_ms() * 1e-3
                steps2 = r2["steps"]
            b2.close()
        wall = time.perf_counter() - t
        fields = [nodal_fields(s, c) for s, c in zip(fin, cases)]
        res = {"wall_s": wall, "device_s": dev, "init_s": t_init, "init_and_tune_s": t_tune, "setup_s": t_setup,
               "steps": [int(x) for x in steps1], "steps_fp64_finish": [int(x) for x in steps2],
               "fell_back_to_cold": [int(i) for i in fell_back]}
        b.close()
        for s in first + (fin if switch else []):
            s.close()
        final[name] = fields
        if log:
            log(f"{name}: {wall:.2f} s (device {dev:.2f} s), steps {int(steps1.min())}..{int(steps1.max())}"
                + (f" + fp64 {int(steps2.min())}..{int(steps2.max())}" if switch else ""))
        return res

    if "batch64" in ways:
        out["batch64"] = batched("batch64", False, 64, None)
    if "batch64_warm" in ways:
        out["batch64_warm"] = batched("batch64_warm", True, 64, None)
    if "fast" in ways:
        out["fast"] = batched("fast", True, 32, switch_tol)
    if "fast_cold" in ways:
        out["fast_cold"] = batched("fast_cold", False, 32, switch_tol)
    if "batch64_rre" in ways:
        out["batch64_rre"] = batched("batch64_rre", False, 64, None, rre=True)
    if "fast_rre" in ways:
        out["fast_rre"] = batched("fast_rre", True, 32, switch_tol, rre=True)
    if "fast_cold_rre" in ways:
        out["fast_cold_rre"] = batched("fast_cold_rre", False, 32, switch_tol, rre=True)
    if "plain" in final:
        for k in final:
            if k == "plain":
                continue
            errs = [rel_fields(a, b) for a, b in zip(final[k], final["plain"])]
            out[k]["max_rel_l2_vs_plain"] = {f: max(e[f] for e in errs) for f in ("n", "u", "v", "T")}
            out[k]["rel_l2_vs_plain"] = [{f: float(f"{e[f]:.3e}") for f in e} for e in errs]
            out[k]["speedup_vs_plain"] = out["plain"]["wall_s"] / out[k]["wall_s"]
    return out, final, cases


def warm_quality(ws, cases, truth_fields):
    """Median relative L2 of the predicted nodal fields against steady ones."""
    grids = ws.predict_grids(np.stack([params_vector(c) for c in cases]))
    errs = [rel_fields(resampler(c).to_nodes(g), q) for c, g, q in zip(cases, grids, truth_fields)]
    return {f: float(np.median([e[f] for e in errs])) for f in ("n", "u", "v", "T")}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--train", type=int, default=384)
    ap.add_argument("--test", type=int, default=32)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--data-tol", type=float, default=1e-5)
    ap.add_argument("--switch-tol", type=float, default=1e-5)
    ap.add_argument("--ways", default="plain,batch64,batch64_warm,fast")
    ap.add_argument("--out", default=None)
    ap.add_argument("--gather-timeout", type=float, default=7200.0,
                    help="seconds a rank may wait for the others' training sets (torchrun)")
    a = ap.parse_args(argv)

    def log(m):
        print(m, flush=True)

    # torchrun: every rank generates its share of the training set on its own
    # GPU; rank 0 gathers the sets (host objects over gloo, once, with a
    # timeout above a share's generation time), trains and evaluates
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=a.gather_timeout))
    t = time.perf_counter()
    train_cases = draw_cases(a.train, a.seed)
    X, Y, keep = generate(train_cases, tol=a.data_tol, log=log, rank=rank, world=world, device=local)
    if dist is not None:
        parts = [None] * world if rank == 0 else None
        dist.gather_object((X, Y, keep), parts, dst=0)
        dist.destroy_process_group()
        if rank != 0:
            return
        X, Y, keep = merge_generated(parts)
    gen_s = time.perf_counter() - t
    log(f"training set: {len(keep)} of {a.train} cases kept ({gen_s:.1f} s)")
    ws = WarmStart()
    hist = ws.fit(X, Y)
    log(f"trained: loss {hist[:10].mean():.3e} -> {hist[-50:].mean():.3e} in {ws.train_s:.1f} s")
    test_cases = draw_cases(a.test, a.seed + 1000)
    res, final, kept = evaluate(test_cases, ws, switch_tol=a.switch_tol, ways=tuple(a.ways.split(",")), log=log)
    if "plain" in final:
        res["warm_start_rel_l2_median"] = warm_quality(ws, kept, final["plain"])
    res.update({"family": FAMILY, "grid": GRID, "train_requested": a.train, "train_kept": len(keep),
                "generate_s": gen_s, "train_s": ws.train_s, "loss_first": float(hist[:10].mean()),
                "loss_last": float(hist[-50:].mean())})
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()

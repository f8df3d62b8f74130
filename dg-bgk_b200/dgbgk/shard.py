"""Velocity-space sharding: a case's speed rings split over GPUs.

The reference splits velocity space into NVSPACEPART contiguous blocks of
whole speed rings (src/spectralbgk.f90:163-199), each rank holding every
element for its velocities, and adds up the velocity sums of MACROS,
COMPMU and FLUCON2 with MPI_ALLREDUCE over the V-communicator
(src/macros.f90:114-119, 153-154; src/compmu.f90:80-81;
src/flucon2.f90:215-216).  Here each rank's GPU holds one block as a shard
handle (dgbgk_params.shard) and a step is four library phases with three
exchanges between them:

    phase 1 -> sums1 (pass-1 sums)                         all-reduce SUM
    phase 2 -> sums2 (pass-2 sums, wall sums)              all-reduce SUM
    phase 3 -> moments, dt, sweep; res (residual partials) all-reduce MAX/SUM
    phase 4    bookkeeping (history, convergence)

The exchange buffers are device tensors owned here; the all-reduces are
enqueued on the library's stream (torch.cuda.ExternalStream), so a step
never waits on the host.  Whole rings keep the sweep local (ALPHA = 1: the
wall's specular part, which reads mirrored velocities, is not sharded).

`advance_distributed` runs one shard per rank over torch.distributed (NCCL
on GPUs); `advance_local` runs several shards of one case on one GPU with
the sums added in the process (for tests and for a single GPU).
"""
import ctypes
from ctypes import c_double, c_int, c_void_p

import numpy as np

from ._lib import check, lib, ptr
from .solver import Solver, setup_mesh, vspace


def ring_split(rorder, world):
    """(first ring, ring count) of each of `world` shards: contiguous whole
    rings, counts as equal as possible (the reference's blocks need
    NVSPACEPART | RORDER; here any split works)."""
    if world < 1 or world > rorder:
        raise ValueError(f"cannot split {rorder} rings over {world} shards")
    base, extra = divmod(rorder, world)
    out, r0 = [], 0
    for k in range(world):
        n = base + (1 if k < extra else 0)
        out.append((r0, n))
        r0 += n
    return out


class ShardedSolver:
    """Shard `rank` of `world` of a case on `device` (velocities of rings
    ring_split(...)[rank]); the state is DISNF(3, local VNPNT, NELEM)."""

    def __init__(self, case, rank, world, precision=64, device=0):
        import torch
        from .cases import gll
        self.rank, self.world = rank, world
        self.r0, self.nr = ring_split(case.rorder, world)[rank]
        m = case.mesh
        st = setup_mesh(m.intma, m.coord, m.bsido)
        eta, w = gll(case.rorder)
        vc, sw = vspace(case.rorder, case.torder, eta, w)  # the full grid's SUMWEIGHT
        to = case.torder
        self.v0, self.vn = self.r0 * to, self.nr * to
        self.solver = Solver(m.intma, m.coord, m.bsido, st, vc[self.v0:self.v0 + self.vn], sw, self.nr, to, case.rv,
                             immat=case.immat, csafm=case.csafm, alpha=case.alpha, rgas=case.rgas,
                             molar_mass=case.molar_mass, diameter=case.diameter, cinf=case.cinf,
                             precision=precision, wall_velocity=m.wall_velocity, device=device, shard=1)
        self.solver.case = case
        self.case = case
        h = self.solver.h
        n1, n2 = ctypes.c_longlong(0), ctypes.c_longlong(0)
        check(lib().dgbgk_shard_sizes(h, ctypes.byref(n1), ctypes.byref(n2)))
        dev = torch.device("cuda", device)
        self.sums1 = torch.zeros(n1.value, dtype=torch.float64, device=dev)
        self.sums2 = torch.zeros(n2.value, dtype=torch.float64, device=dev)
        self.res = torch.zeros(2, dtype=torch.float64, device=dev)
        sp = c_void_p()
        check(lib().dgbgk_shard_stream(h, ctypes.byref(sp)))
        self.stream = torch.cuda.ExternalStream(sp.value or 0, device=dev)

    # -- the library's phases ------------------------------------------
    def phase(self, k):
        check(lib().dgbgk_shard_phase(self.solver.h, k, c_void_p(self.sums1.data_ptr()),
                                      c_void_p(self.sums2.data_ptr()), c_void_p(self.res.data_ptr())))

    def begin(self, max_steps, tol):
        check(lib().dgbgk_shard_begin(self.solver.h, max_steps, tol))

    def poll(self):
        d = c_int(0)
        check(lib().dgbgk_shard_poll(self.solver.h, ctypes.byref(d)))
        return bool(d.value)

    def end(self, max_steps):
        n = max(max_steps, 1)
        linf, l2, dte = np.zeros(n), np.zeros(n), np.zeros(n)
        steps, done = c_int(0), c_int(0)
        rc = lib().dgbgk_shard_end(self.solver.h, ctypes.byref(steps), ptr(linf), ptr(l2), ptr(dte),
                                   ctypes.byref(done))
        k = steps.value
        out = {"steps": k, "res_linf": linf[:k], "res_l2": l2[:k], "dte": dte[:k], "rc": rc}
        check(rc)
        return out

    # -- state of the shard's velocities -------------------------------
    def set_state(self, disnf_local):
        self.solver.set_state(disnf_local)

    def get_state(self):
        return self.solver.get_state()

    def init_case(self):
        self.solver.init_case()

    def close(self):
        self.solver.close()


class TorchGroup:
    """The exchanges of one shard per rank: torch.distributed all-reduces
    (NCCL between GPUs) enqueued on the shard's stream."""

    def __init__(self, dist=None):
        if dist is None:
            import torch.distributed as dist
        self.dist = dist

    @staticmethod
    def _on(shard):
        import contextlib
        import torch
        return torch.cuda.stream(shard.stream) if shard.stream is not None else contextlib.nullcontext()

    def sum(self, shard, t):
        with self._on(shard):
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)

    def res(self, shard):
        with self._on(shard):
            self.dist.all_reduce(shard.res[0:1], op=self.dist.ReduceOp.MAX)
            self.dist.all_reduce(shard.res[1:2], op=self.dist.ReduceOp.SUM)


def _steps(shards, exchange_sum, exchange_res, n, tol, poll_every):
    """n steps of the shards (one per rank, or all of one case in this
    process), with the exchanges between the phases; stops early once the
    (global) convergence test has stopped them."""
    for s in shards:
        s.begin(n, tol)
    for k in range(n):
        for ph, ex in ((1, "sums1"), (2, "sums2"), (3, "res")):
            for s in shards:
                s.phase(ph)
            if ex == "res":
                exchange_res()
            else:
                exchange_sum(ex)
        for s in shards:
            s.phase(4)
        if poll_every and (k + 1) % poll_every == 0 and k + 1 < n and shards[0].poll():
            break
    return [s.end(n) for s in shards]


def advance_distributed(shard, n, tol=0.0, group=None, poll_every=64):
    """This rank's shard for n steps (to tol), the others running the same
    call; returns the step count and histories (the same on every rank)."""
    g = group or TorchGroup()
    return _steps([shard], lambda name: g.sum(shard, getattr(shard, name)), lambda: g.res(shard), n, tol,
                  poll_every)[0]


def _local_exchanges(shards):
    import torch

    def sync():
        torch.cuda.synchronize(shards[0].sums1.device)

    def ex_sum(name):
        sync()
        tot = sum(getattr(s, name) for s in shards)
        for s in shards:
            getattr(s, name).copy_(tot)
        sync()

    def ex_res():
        sync()
        mx = torch.stack([s.res[0] for s in shards]).max()
        sq = sum(s.res[1] for s in shards)
        for s in shards:
            s.res[0] = mx
            s.res[1] = sq
        sync()
    return ex_sum, ex_res


def advance_local(shards, n, tol=0.0, poll_every=64):
    """All the shards of one case in this process (one GPU): the phases of
    one shard after another, the sums added on the device between them."""
    ex_sum, ex_res = _local_exchanges(shards)
    return _steps(shards, ex_sum, ex_res, n, tol, poll_every)


def local_moments(shards):
    """The moments of the current state on every shard (phases 0, 1, 2, 5):
    then each shard's macros(), node_fields() and forces() are the case's."""
    ex_sum, _ = _local_exchanges(shards)
    for ph, ex in ((0, None), (1, "sums1"), (2, "sums2"), (5, None)):
        for s in shards:
            s.phase(ph)
        if ex:
            ex_sum(ex)
    import torch
    torch.cuda.synchronize(shards[0].sums1.device)


def distributed_moments(shard, group=None):
    g = group or TorchGroup()
    for ph, ex in ((0, None), (1, "sums1"), (2, "sums2"), (5, None)):
        shard.phase(ph)
        if ex:
            g.sum(shard, getattr(shard, ex))

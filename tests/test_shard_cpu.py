"""The velocity-shard step's exchanges as two gloo ranks on CPU.

Each rank holds a fake shard: the library's phases replaced by numpy sums of
a synthetic distribution over the rank's speed rings (the same velocity
sums the kernels form: MACROS pass 1, then pass 2 with the bulk velocity of
the summed pass-1 sums).  After the exchanges of dgbgk.shard's step driver
every rank holds the sums of the whole grid, the max of the residual
partials and their sum; the ring split covers the grid.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dgbgk.shard import TorchGroup, _steps, ring_split

RO, TO, NODES = 6, 8, 5


def grid():
    rng = np.random.default_rng(3)
    f = rng.uniform(0.1, 1.0, (NODES, RO * TO))
    r = np.repeat(np.linspace(0.2, 3.0, RO), TO)
    th = np.tile(np.linspace(0, 2 * np.pi, TO, endpoint=False), RO)
    w = rng.uniform(0.5, 1.5, RO * TO)
    return f, r * np.cos(th), r * np.sin(th), w


def pass1(f, cx, cy, w):
    return np.concatenate([(f * w).sum(1), (f * w * cx).sum(1), (f * w * cy).sum(1)])


def pass2(f, cx, cy, w, s1):
    n = s1[:NODES]
    ux, uy = s1[NODES:2 * NODES] / n, s1[2 * NODES:] / n
    q = (cx[None] - ux[:, None]) ** 2 + (cy[None] - uy[:, None]) ** 2
    return np.concatenate([0.5 * (f * w * q).sum(1), (f * w * np.sqrt(q)).sum(1)])


class FakeShard:
    """A shard's phases on the CPU (no GPU, no library)."""

    def __init__(self, rank, world):
        f, cx, cy, w = grid()
        r0, nr = ring_split(RO, world)[rank]
        sl = slice(r0 * TO, (r0 + nr) * TO)
        self.f, self.cx, self.cy, self.w = f[:, sl], cx[sl], cy[sl], w[sl]
        self.sums1 = torch.zeros(3 * NODES, dtype=torch.float64)
        self.sums2 = torch.zeros(2 * NODES, dtype=torch.float64)
        self.res = torch.zeros(2, dtype=torch.float64)
        self.stream = None
        self.rank = rank
        self.seen = []

    def begin(self, n, tol):
        self.seen.append(("begin", n))

    def phase(self, k):
        self.seen.append(k)
        if k == 1:
            self.sums1[:] = torch.from_numpy(pass1(self.f, self.cx, self.cy, self.w))
        elif k == 2:
            self.sums2[:] = torch.from_numpy(pass2(self.f, self.cx, self.cy, self.w, self.sums1.numpy()))
        elif k == 3:
            self.res[:] = torch.tensor([float(self.f.max()), float((self.f ** 2).sum())], dtype=torch.float64)
        elif k == 4:
            self.got = (self.sums1.clone(), self.sums2.clone(), self.res.clone())

    def poll(self):
        return False

    def end(self, n):
        return {"steps": n}


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = FakeShard(rank, world)
        g = TorchGroup(dist)
        out = _steps([s], lambda name: g.sum(s, getattr(s, name)), lambda: g.res(s), 2, 0.0, 0)
        q.put((rank, [t.numpy().tolist() for t in s.got], s.seen, out[0]["steps"]))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_shard_exchanges_give_the_whole_grid_sums(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    f, cx, cy, w = grid()
    s1 = pass1(f, cx, cy, w)
    s2 = pass2(f, cx, cy, w, s1)
    for rank, (g1, g2, res), seen, steps in got:
        np.testing.assert_allclose(g1, s1, rtol=1e-13)
        np.testing.assert_allclose(g2, s2, rtol=1e-13)
        np.testing.assert_allclose(res, [f.max(), (f ** 2).sum()], rtol=1e-13)
        assert seen == [("begin", 2), 1, 2, 3, 4, 1, 2, 3, 4] and steps == 2


def test_ring_split_covers_the_grid():
    for ro in (1, 5, 12, 24, 40):
        for world in range(1, ro + 1):
            sp = ring_split(ro, world)
            assert sp[0][0] == 0 and sum(n for _, n in sp) == ro
            assert all(a + n == b for (a, n), (b, _) in zip(sp, sp[1:]))
            assert max(n for _, n in sp) - min(n for _, n in sp) <= 1
    with pytest.raises(ValueError):
        ring_split(4, 5)

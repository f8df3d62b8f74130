"""The training-set generation sharded over ranks (CPU, gloo, two ranks):
each rank marches a round-robin share of the cases and rank 0's merged set
equals the one-rank set, case by case.  The solver, batch and march are
replaced by fakes (the sharding and the merge are host logic)."""
import json
import os
import socket

import numpy as np

from conftest import PKG


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Fake:
    """Stands in for Solver and Batch: records the case it was made for."""

    def __init__(self, case=None, **kw):
        self.case = case
        self.kw = kw

    @classmethod
    def from_case(cls, case, precision=32, device=0):
        return cls(case, precision=precision, device=device)

    def init_case(self):
        pass

    def close(self):
        pass


def _patch(study):
    from dgbgk.study import NF, GRID

    def march(b, ss, tol, max_steps):
        n = len(ss)
        # a case "diverges" above Mach 2.5; the others reach a residual that
        # grows with Kn (cases with Kn > 0.2 miss the acceptance bound)
        status = np.array([1 if s.case.info["mach"] > 2.5 else 0 for s in ss])
        rel = np.array([5e-4 * s.case.info["kn"] for s in ss])
        return np.full(n, 100), rel, status, 0.0

    class Res:
        def __init__(self, case):
            self.case = case

        def to_grid(self, q):
            return np.full((NF, GRID[0], GRID[1]), q, np.float32)

    study.Solver = _Fake
    study.Batch = lambda ss: _Fake()
    study.tuned_batch = lambda ss: _Fake()
    study.march_batch = march
    study.nodal_fields = lambda s, c: float(c.info["mach"] * 10 + c.info["kn"])
    study.resampler = Res


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, PKG)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank)})
    import torch.distributed as dist
    from dgbgk import study
    _patch(study)
    cases = study.draw_cases(11, 5)
    X, Y, keep = study.generate(cases, group=3, rank=rank, world=world, device=rank)
    dist.init_process_group("gloo")
    parts = [None] * world if rank == 0 else None
    dist.gather_object((X, Y, keep), parts, dst=0)
    dist.destroy_process_group()
    if rank == 0:
        X, Y, keep = study.merge_generated(parts)
        np.savez(out, X=X, Y=Y, keep=np.array(keep))


def test_shard_round_robin():
    import sys
    sys.path.insert(0, PKG)
    from dgbgk.study import shard
    assert shard(7, 0, 3) == [0, 3, 6] and shard(7, 2, 3) == [2, 5] and shard(2, 3, 4) == []
    assert sorted(i for r in range(4) for i in shard(10, r, 4)) == list(range(10))


def test_generate_two_ranks_matches_one(tmp_path):
    import sys
    sys.path.insert(0, PKG)
    import torch.multiprocessing as mp
    from dgbgk import study
    port = free_port()
    out = str(tmp_path / "merged.npz")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert [p.exitcode for p in procs] == [0, 0]
    got = np.load(out)
    # one rank, the same fakes
    _patch(study)
    cases = study.draw_cases(11, 5)
    ref = study.generate(cases, group=3)
    assert 0 < len(ref[2]) < len(cases)  # the fakes keep some cases and drop others
    assert list(got["keep"]) == ref[2]
    np.testing.assert_array_equal(got["X"], ref[0])
    np.testing.assert_array_equal(got["Y"], ref[1])
    # every kept case's row carries its own value
    for row, i in zip(got["Y"], got["keep"]):
        c = cases[i]
        assert row[0] == np.float32(c.info["mach"] * 10 + c.info["kn"])

"""Velocity-space shards (GPU): the case split into whole speed rings, its
steps run as the library's phases with the partial sums added between
them, equals the case on one handle -- states, residual histories, step
counts, nodal fields and forces.  The shards run in one process on one GPU
(the sums added on the device between the phases), the same library calls
a rank makes with one shard per GPU.
"""
import numpy as np
import pytest

from dgbgk import Solver, cavity_case, channel_case
from dgbgk.shard import ShardedSolver, advance_local, local_moments
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def channel():
    return channel_case(-2.0, 4.0, -3.0, 3.0, 30, 30, 12, 24, mach=2.5, kn=0.07, obstacle_side=1.0,
                        sides="freestream")


def pair(case, world, prec):
    full = Solver.from_case(case, precision=prec)
    full.init_case()
    shards = [ShardedSolver(case, k, world, precision=prec) for k in range(world)]
    for s in shards:
        s.init_case()
    return full, shards


def state_of(shards):
    return np.concatenate([s.get_state() for s in shards], axis=1)


@pytest.mark.parametrize("mk,world", [(channel, 1), (channel, 2), (channel, 3), (lambda: cavity_case(8, 8, 16), 2)])
@pytest.mark.parametrize("prec", [64, 32])
def test_shards_equal_the_whole_grid(mk, world, prec):
    c = mk()
    full, shards = pair(c, world, prec)
    tol = 1e-12 if prec == 64 else 1e-6
    assert rel_l2(state_of(shards), full.get_state()) == 0.0
    r = full.advance(20)
    q = advance_local(shards, 20)
    for x in q:
        assert x["steps"] == 20
        assert rel_l2(x["res_l2"], r["res_l2"]) <= tol
        assert rel_l2(x["dte"], r["dte"]) <= tol
    assert rel_l2(state_of(shards), full.get_state()) <= tol
    local_moments(shards)
    a, b = shards[-1].solver.macros(), full.macros()
    for k in ("rho", "u", "v", "temp", "ps"):
        assert rel_l2(a[k], b[k], 1.0 if k in "uv" else 0.0) <= tol, k
    if c.mesh.bsido[:, 3].tolist().count(4):
        # lift is a small difference of pressure terms of drag's size: the
        # tolerance is on the forces' scale
        fb = np.array(full.forces())
        np.testing.assert_allclose(shards[0].solver.forces(), fb, rtol=tol, atol=tol * np.abs(fb).max())
    for s in shards + [full]:
        s.close()


def test_shards_stop_on_the_global_tolerance():
    c = channel()
    full, shards = pair(c, 2, 64)
    n = full.advance(2000, tol=0.05)["steps"]
    assert n < 2000
    q = advance_local(shards, 2000, tol=0.05, poll_every=16)
    assert [x["steps"] for x in q] == [n, n]
    assert rel_l2(state_of(shards), full.get_state()) <= 1e-12
    for s in shards + [full]:
        s.close()


def test_a_shard_refuses_the_whole_grid_calls():
    from dgbgk._lib import DGBGK_EINVAL, DgbgkError
    s = ShardedSolver(channel(), 0, 2)
    with pytest.raises(DgbgkError) as e:
        s.solver.advance(1)
    assert e.value.code == DGBGK_EINVAL
    s.close()

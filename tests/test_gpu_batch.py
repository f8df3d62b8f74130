"""Batched cases (dgbgk_batch_*) against the same cases run alone and
against the oracle (GPU).

A batch advances cases of different meshes and velocity grids with one
launch per kernel and step; each case's arithmetic is the one a single
handle does (the element blocking may differ, which does not change any
value), so a case's state after n batch steps equals its state after n
steps alone, and the FP64 batch matches the FP64 oracle at the parity bar.
"""
import numpy as np
import pytest

from dgbgk import Batch, Solver, cavity_case, channel_case
from helpers import rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def mixed_cases():
    return [
        cavity_case(8, 8, 16, mach=0.3, kn=0.1),
        channel_case(-2.0, 4.0, -2.0, 2.0, 24, 16, 5, 7, mach=2.0, kn=0.05, obstacle_side=1.0),
        cavity_case(12, 6, 20, mach=0.8, kn=0.02, seed=3),
    ]


def started(case, prec):
    s = Solver.from_case(case, precision=prec)
    s.init_case()
    return s


@pytest.mark.parametrize("prec", [64, 32])
def test_batch_equals_cases_alone(prec):
    cases = mixed_cases()
    alone = [started(c, prec) for c in cases]
    for s in alone:
        s.advance(6)
    batched = [started(c, prec) for c in cases]
    b = Batch(batched, tune_steps=1)
    r = b.advance(6)
    assert list(r["steps"]) == [6, 6, 6]
    tol = 1e-13 if prec == 64 else 1e-6
    for s, t in zip(batched, alone):
        assert rel_l2(s.get_state(), t.get_state()) <= tol
    info = b.info()
    assert info["ncases"] == 3 and info["tile_elems"] in (64, 128)
    assert len(b.tuning()) >= 1


def test_batch_fp64_matches_oracle():
    cases = mixed_cases()
    ss = [started(c, 64) for c in cases]
    os_ = []
    for c in cases:
        o = Oracle.from_case(c, prec=64)
        i = c.init
        o.inicon2(i["T1"], i["P1"], i["U0"], i["V0"])
        from dgbgk import node_scale
        sc = node_scale(c)
        if sc is not None:
            o.set_state(o.get_state() * sc[:, None, :])
        os_.append(o)
    b = Batch(ss, tile_elems=64, units_per_cta=4, tune_steps=1)
    b.advance(4)
    for s, o in zip(ss, os_):
        o.advance(4)
        assert rel_l2(s.get_state(), o.get_state()) <= 1e-10


def test_batch_cases_stop_on_their_own_tolerance():
    # two cavities whose residuals fall at different rates: each stops when
    # its own L2 residual reaches tol times its first step's, the other
    # goes on
    cases = [cavity_case(8, 8, 16, mach=0.3, kn=0.1), cavity_case(12, 6, 20, mach=0.8, kn=0.02, seed=3)]
    ss = [started(c, 64) for c in cases]
    b = Batch(ss, tune_steps=1)
    r = b.advance(3000, tol=0.2)
    steps = r["steps"]
    assert (steps < 3000).all() and steps[0] != steps[1]
    for s, n, l2 in zip(ss, steps, r["res_l2_last"]):
        assert l2 <= 0.2 * s.residual_reference() * (1 + 1e-12)
    # each case alone stops at the same step
    for c, n in zip(cases, steps):
        t = started(c, 64)
        assert t.advance(3000, tol=0.2)["steps"] == n


def test_batch_with_partial_accommodation_equals_cases_alone():
    # ALPHA = 0.9 cases (the specular part runs per case after the sweep)
    # beside an ALPHA = 1 case
    a = cavity_case(8, 12, 12, mach=0.3, kn=0.1)
    a.alpha = 0.9
    b = channel_case(-2.0, 4.0, -2.0, 2.0, 30, 20, 12, 12, mach=2.0, kn=0.05, obstacle_side=1.0)
    b.alpha = 0.9
    cases = [a, b, cavity_case(8, 8, 16, mach=0.3, kn=0.1)]
    alone = [started(c, 64) for c in cases]
    for s in alone:
        s.advance(5)
    batched = [started(c, 64) for c in cases]
    Batch(batched, tune_steps=1).advance(5)
    for s, t in zip(batched, alone):
        assert rel_l2(s.get_state(), t.get_state()) <= 1e-13

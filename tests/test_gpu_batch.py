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


def stopping_cases():
    """Eight cases of different meshes and velocity grids; the first (the
    zero-gradient-sided channel at Kn = 1) diverges within a few hundred
    steps, the scheme's stability limit, and stops while the others run."""
    # the other seven stay finite for at least 1000 steps (checked with the
    # FP32 oracle)
    return [
        channel_case(-5, 15, -5, 5, 40, 20, 8, 16, mach=2.0, kn=1.0, obstacle_side=1.0),
        cavity_case(8, 8, 16, mach=0.3, kn=0.1),
        channel_case(-2.0, 4.0, -3.0, 3.0, 30, 30, 12, 24, mach=2.5, kn=0.07, obstacle_side=1.0, sides="freestream"),
        cavity_case(12, 6, 20, mach=0.8, kn=0.02, seed=3),
        cavity_case(16, 8, 24, mach=0.5, kn=0.05, seed=5),
        cavity_case(12, 8, 16, mach=0.6, kn=0.05, seed=5),
        cavity_case(10, 10, 10, mach=0.2, kn=0.3, seed=7),
        cavity_case(20, 4, 36, mach=0.9, kn=0.5, seed=9),
    ]


SHAPES = [(eb, upc, rows) for eb in (64, 128) for upc in (2, 4, 8, 16) for rows in (1, 2, 3, 4)]


def test_every_batch_shape_with_a_case_stopping_early():
    # every candidate tile shape (elements per CTA x units per CTA x moment
    # rows), forced, on eight FP32 cases of which one diverges and stops
    # while the others go on: each case's state (and the diverging case's
    # step count) equals the case run alone.  This is the long heterogeneous
    # march in which finished cases' work units are skipped.
    from dgbgk._lib import DGBGK_ENONFINITE
    cases = stopping_cases()
    n = 700  # the first case's state turns non-finite near step 480 (oracle: between 450 and 500)
    alone = [started(c, 32) for c in cases]
    bad_steps = None
    for k, s in enumerate(alone):
        if k == 0:
            r = s.advance(n, raise_on_error=False)
            assert r["rc"] == DGBGK_ENONFINITE and r["steps"] < n
            bad_steps = r["steps"]
        else:
            assert s.advance(n)["steps"] == n
    states = [s.get_state() for s in alone[1:]]
    for s in alone:
        s.close()
    for eb, upc, rows in SHAPES:
        batched = [started(c, 32) for c in cases]
        b = Batch(batched, tile_elems=eb, units_per_cta=upc, moment_rows=rows, tune_steps=1)
        assert b.shape_record() == {"tile_elems": eb, "units_per_cta": upc, "moment_rows": rows}
        r = b.advance(n, raise_on_error=False)
        # the blow-up's step moves with the FP32 summation order of the
        # moment shape (a step either way was seen)
        assert r["status"][0] == DGBGK_ENONFINITE and abs(int(r["steps"][0]) - bad_steps) <= 5, \
            (eb, upc, rows, int(r["steps"][0]), bad_steps)
        assert (r["status"][1:] == 0).all() and (r["steps"][1:] == n).all(), (eb, upc, rows)
        for s, ref in zip(batched[1:], states):
            assert rel_l2(s.get_state(), ref) <= 1e-5, (eb, upc, rows)
        b.close()
        for s in batched:
            s.close()


def test_batch_leaves_inactive_and_diverged_cases_alone():
    # dgbgk_batch_set_active: an inactive case runs no step and keeps its
    # state; a diverged case stays stopped, with its status, until its state
    # is set again, and then runs like a fresh case
    from dgbgk._lib import DgbgkError, DGBGK_ENONFINITE
    cases = stopping_cases()[:3]
    ss = [started(c, 32) for c in cases]
    b = Batch(ss, tune_steps=1)
    r = b.advance(700, raise_on_error=False)
    assert r["status"][0] == DGBGK_ENONFINITE
    kept = ss[2].get_state()
    b.set_active([True, True, False])
    with pytest.raises(DgbgkError) as e:
        b.advance(10)
    assert e.value.code == DGBGK_ENONFINITE
    st = b.advance(10, raise_on_error=False)
    assert list(st["steps"]) == [0, 10, 0] and list(st["status"]) == [DGBGK_ENONFINITE, 0, 0]
    assert np.array_equal(ss[2].get_state(), kept)
    # a new state lets the diverged case run again, like a fresh handle
    ss[0].init_case()
    b.set_active([True, False, False])
    r0 = b.advance(5)
    assert list(r0["steps"]) == [5, 0, 0] and list(r0["status"]) == [0, 0, 0]
    fresh = started(cases[0], 32)
    fresh.advance(5)
    assert rel_l2(ss[0].get_state(), fresh.get_state()) <= 1e-6
    b.close()
    for s in ss + [fresh]:
        s.close()


def test_batch_rebuilds_its_table_after_a_case_moves_its_buffers():
    # a case advanced alone for more steps than its history holds gets new
    # device buffers; the batch must notice before its next launch
    cases = stopping_cases()[1:4]
    ss = [started(c, 64) for c in cases]
    b = Batch(ss, tune_steps=1)
    b.advance(3)
    ss[1].advance(3000)              # grows that handle's history buffers
    alone = [started(c, 64) for c in cases]
    for s, n in zip(alone, (3, 3003, 3)):
        s.advance(n)
    b.advance(4)
    for s in alone:
        s.advance(4)
    for s, t in zip(ss, alone):
        assert rel_l2(s.get_state(), t.get_state()) <= 1e-12
    b.close()
    for s in ss + alone:
        s.close()

"""The warm-start path on the GPU: precision handoff, per-case batch status,
and what the trained network gains over a cold start.

The cases are the warm-start family's channel (free-stream sides, 100 x 100
quads) on a 12 x 24 velocity grid, drawn from the middle of the family's
ranges, so that a test marches in seconds (an 8 x 16 grid is too coarse: the
explicit scheme diverges on it).  The cold FP64 march is the yardstick: a
warm-started (or FP32-started) march must end, at the same residual, on the
same fields.
"""
import numpy as np
import pytest

from dgbgk import Batch, Solver, channel_case
from dgbgk._lib import DGBGK_ENONFINITE, DgbgkError
from dgbgk.study import FAMILY, WarmStart, cold_reference, draw_cases, generate, nodal_fields, rel_fields
from helpers import rel_l2

pytestmark = pytest.mark.gpu

SMALL = dict(FAMILY, nr=12, nt=24, mach=(2.2, 2.8), kn=(0.06, 0.12))


def family_case(m, kn, side=1.0):
    x0, x1, y0, y1 = FAMILY["box"]
    return channel_case(x0, x1, y0, y1, FAMILY["nx"], FAMILY["ny"], 12, 24, mach=m, kn=kn, obstacle_side=side,
                        sides="freestream")


def cold(case, prec, tol, ref=None, max_steps=60000):
    s = Solver.from_case(case, precision=prec)
    s.init_case()
    if ref is not None:
        s.set_residual_reference(ref)
    r = s.advance(max_steps, tol=tol)
    return s, r


def test_copy_state_converts_precision_and_keeps_the_reference():
    c = family_case(2.5, 0.07)
    s64, _ = cold(c, 64, 0.0, max_steps=30)
    s32 = Solver.from_case(c, precision=32)
    s32.copy_state_from(s64)
    assert s32.residual_reference() == s64.residual_reference()
    a = s64.get_state()
    assert np.array_equal(s32.get_state(np.float32), a.astype(np.float32))
    back = Solver.from_case(c, precision=64)
    back.copy_state_from(s32)
    assert np.array_equal(back.get_state(), a.astype(np.float32).astype(np.float64))
    # same precision: an exact copy
    twin = Solver.from_case(c, precision=64)
    twin.copy_state_from(s64)
    assert np.array_equal(twin.get_state(), a)
    for s in (s64, s32, back, twin):
        s.close()


def test_fp32_transient_fp64_finish_matches_fp64():
    c = family_case(2.5, 0.07)
    ref = cold_reference(c)
    plain, r = cold(c, 64, 1e-8, ref)
    assert r["steps"] < 60000
    s32, r32 = cold(c, 32, 1e-4, ref)
    s64 = Solver.from_case(c, precision=64)
    s64.copy_state_from(s32)
    r64 = s64.advance(60000, tol=1e-8)
    assert r64["res_l2"][-1] <= 1e-8 * ref * (1 + 1e-9)
    e = rel_fields(nodal_fields(s64, c), nodal_fields(plain, c))
    assert max(e["n"], e["u"], e["T"]) <= 1e-6
    for s in (plain, s32, s64):
        s.close()


def test_batch_reports_a_diverging_case_and_finishes_the_rest():
    # the zero-gradient-sided channel at Kn = 1 diverges within a few hundred
    # steps (the explicit scheme's stability limit; the oracle diverges on
    # it too); the cavity next to it must run on untouched
    from dgbgk import cavity_case
    bad = channel_case(-5, 15, -5, 5, 40, 20, 8, 16, mach=2.0, kn=1.0, obstacle_side=1.0)
    good = cavity_case(8, 8, 16, mach=0.3, kn=0.1)
    ss = [Solver.from_case(x, precision=32) for x in (bad, good)]
    for s in ss:
        s.init_case()
    b = Batch(ss, tune_steps=1)
    r = b.advance(1500, raise_on_error=False)
    assert r["status"][0] == DGBGK_ENONFINITE and r["steps"][0] < 1500
    assert r["status"][1] == 0 and r["steps"][1] == 1500
    alone = Solver.from_case(good, precision=32)
    alone.init_case()
    alone.advance(1500)
    assert rel_l2(ss[1].get_state(), alone.get_state()) <= 1e-6
    # the diverged case stays stopped with its status; the advance reports
    # it and runs the cavity on
    with pytest.raises(DgbgkError) as e:
        b.advance(10)
    assert e.value.code == DGBGK_ENONFINITE
    assert list(b.advance(10, raise_on_error=False)["steps"]) == [0, 10]
    b.close()
    for s in ss + [alone]:
        s.close()
    # the context is healthy: a fresh handle steps and matches the oracle
    from pyoracle import Oracle
    from dgbgk import node_scale
    s = Solver.from_case(good, precision=64)
    s.init_case()
    s.advance(3)
    o = Oracle.from_case(good, prec=64)
    i = good.init
    o.inicon2(i["T1"], i["P1"], i["U0"], i["V0"])
    o.set_state(o.get_state() * node_scale(good)[:, None, :])
    o.advance(3)
    assert rel_l2(s.get_state(), o.get_state()) <= 1e-10
    s.close()


def test_trained_network_gains_over_the_cold_start():
    train = draw_cases(24, 11, family=SMALL)
    X, Y, keep = generate(train, tol=1e-4, accept=1e-3)
    assert len(keep) >= 20
    ws = WarmStart(width=256, depth=3, batch=128, seed=1)
    hist = ws.fit(X, Y, schedule=((1500, 1e-3), (500, 3e-4)))
    assert hist[-20:].mean() < 0.1 * hist[:5].mean()
    test = draw_cases(1, 12, family=SMALL)[0]
    ref = cold_reference(test)
    plain, r_cold = cold(test, 64, 1e-8, ref)
    warm = Solver.from_case(test, precision=64)
    ws.warm([warm], [test])
    warm.set_residual_reference(ref)
    r_warm = warm.advance(60000, tol=1e-8)
    assert r_warm["steps"] < 0.9 * r_cold["steps"], (r_warm["steps"], r_cold["steps"])
    e = rel_fields(nodal_fields(warm, test), nodal_fields(plain, test))
    assert max(e["n"], e["u"], e["T"]) <= 1e-6
    plain.close()
    warm.close()


def test_extrapolation_matches_numpy_rre():
    # dgbgk_extrapolate on five consecutive iterates: the coefficients and
    # the extrapolated state equal a float64 restatement of reduced-rank
    # extrapolation on the same snapshots
    c = family_case(2.5, 0.07)
    s, _ = cold(c, 64, 0.0, max_steps=40)
    xs = []
    for j in range(5):
        s.snapshot(j)
        xs.append(s.get_state())
        if j < 4:
            s.advance(1)
    g = s.extrapolate(5)
    U = np.stack([(xs[j + 1] - xs[j]).ravel() for j in range(4)])
    G = U @ U.T
    G += 1e-14 * np.trace(G) * np.eye(4)
    gr = np.linalg.solve(G, np.ones(4))
    gr /= gr.sum()
    # the difference system is ill-conditioned (coefficients of opposite
    # signs and |gamma| >> 1): summation order moves gamma at ~1e-7
    np.testing.assert_allclose(g, gr, rtol=1e-4)
    x = np.maximum(sum(gj * xj for gj, xj in zip(g, xs[:4])), 0.0)
    assert rel_l2(s.get_state(), x) <= 1e-12
    s.snapshot(-1)
    s.close()


def numpy_rre(xs):
    """Reduced-rank extrapolation of consecutive iterates xs in float64 (the
    library's ridge and normalisation): the coefficients."""
    U = np.stack([(xs[j + 1] - xs[j]).ravel() for j in range(len(xs) - 1)])
    G = U @ U.T
    G += 1e-14 * np.trace(G) * np.eye(len(xs) - 1)
    g = np.linalg.solve(G, np.ones(len(xs) - 1))
    return g / g.sum()


@pytest.mark.parametrize("prec", [32, 64])
def test_batch_snapshot_and_extrapolation_match_numpy_rre(prec):
    # dgbgk_batch_snapshot / _extrapolate on two of three cases (the copies
    # queued on the batch's stream, each case then stepping on its own
    # stream): per selected case the coefficients and the new state equal a
    # float64 restatement on the same iterates, as dgbgk_extrapolate's do;
    # the case left out is untouched; a case with too few snapshots reports
    # its error and keeps its state
    cs = [family_case(2.5, 0.07), family_case(2.2, 0.09), family_case(2.8, 0.06)]
    b = [cold(c, prec, 0.0, max_steps=30)[0] for c in cs]
    batch = Batch(b, tune_steps=1)
    which = np.array([True, False, True])
    xs = {0: [], 2: []}
    for j in range(5):
        for i in xs:
            xs[i].append(b[i].get_state())
        batch.snapshot(j, which)
        if j < 4:
            for s in b:
                s.advance(1)
    kept = b[1].get_state()
    st, gb = batch.extrapolate(5, which)
    assert (st == 0).all()
    for i in xs:
        # an ill-conditioned system: summation order moves gamma at ~1e-7
        np.testing.assert_allclose(gb[i], numpy_rre(xs[i]), rtol=1e-4)
        x = np.maximum(sum(gj * xj for gj, xj in zip(gb[i], xs[i][:4])), 0.0)
        assert rel_l2(b[i].get_state(), x) <= (1e-12 if prec == 64 else 1e-7), i
    assert np.array_equal(b[1].get_state(), kept)
    st, _ = batch.extrapolate(5, [False, True, False])  # case 1 took no snapshot
    assert st[1] != 0 and st[0] == 0 and st[2] == 0
    assert np.array_equal(b[1].get_state(), kept)
    batch.close()
    for s in b:
        s.snapshot(-1)
        s.close()


def test_extrapolated_march_reaches_the_same_fixed_point_sooner():
    from dgbgk.study import march_batch_rre
    c = family_case(2.5, 0.07)
    ref = cold_reference(c)
    plain, r = cold(c, 64, 1e-8, ref)
    s = Solver.from_case(c, precision=64)
    s.init_case()
    s.set_residual_reference(ref)
    b = Batch([s], tune_steps=1)
    steps, rel, status, _ = march_batch_rre(b, [s], 1e-8, 60000, stall_below=0.0)
    assert status[0] == 0 and rel[0] <= 1e-8 * (1 + 1e-9)
    assert steps[0] < 0.8 * r["steps"], (steps[0], r["steps"])
    e = rel_fields(nodal_fields(s, c), nodal_fields(plain, c))
    assert max(e["n"], e["u"], e["T"]) <= 1e-6
    b.close()
    plain.close()
    s.close()


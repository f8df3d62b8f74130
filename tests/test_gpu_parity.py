"""Parity of the sm_100a path with the oracle, through the C ABI (GPU).

Tolerances: the FP64 path must match the FP64 oracle (the reference promoted
to double) to relative L2 <= 1e-10 on the nodal rho, u, v, T and on f; it
differs only by summation order and the refactored (algebraically equal)
flux expressions, so the observed error is ~1e-14 and the bound has margin
for roundoff growth over the step counts used here.  The FP32-storage path
is compared with the FP64 oracle at <= 1e-5 after a few steps.
"""
import numpy as np
import pytest

from dgbgk import Solver, cavity_case, channel_case, node_scale
from helpers import load_plt, reference_case, rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def pair(case, prec=64, oracle_prec=64, tile_elems=0, lobatto=None, moment_rows=0):
    if lobatto is not None:
        from dgbgk.solver import setup_mesh, vspace
        eta, w = lobatto
        m = case.mesh
        st = setup_mesh(m.intma, m.coord, m.bsido)
        vc, sw = vspace(case.rorder, case.torder, eta, w)
        s = Solver(m.intma, m.coord, m.bsido, st, vc, sw, case.rorder, case.torder, case.rv, immat=case.immat,
                   csafm=case.csafm, alpha=case.alpha, rgas=case.rgas, molar_mass=case.molar_mass,
                   diameter=case.diameter, cinf=case.cinf, precision=prec, wall_velocity=m.wall_velocity,
                   tile_elems=tile_elems)
        s.case = case
        o = Oracle(m.intma, m.coord, m.bsido, case.rorder, case.torder, eta, w, rv=case.rv, csafm=case.csafm,
                   alpha=case.alpha, rgas=case.rgas, molar_mass=case.molar_mass, diameter=case.diameter,
                   cinf=case.cinf, immat=case.immat, prec=oracle_prec, wall_velocity=m.wall_velocity)
    else:
        s = Solver.from_case(case, precision=prec, tile_elems=tile_elems, moment_rows=moment_rows)
        o = Oracle.from_case(case, prec=oracle_prec)
    # identical initial state: the oracle's INICON2 times the per-node scale
    i = case.init
    o.inicon2(i["T1"], i["P1"], i["U0"], i["V0"])
    f0 = o.get_state()
    sc = node_scale(case)
    if sc is not None:
        f0 = f0 * sc[:, None, :]
        o.set_state(f0)
    s.set_state(f0)
    return s, o, f0


def vscale(s):
    """Thermal-speed scale sqrt(R T) of the case, the floor for velocity
    errors (the bulk velocity is ~0 in a gas at rest)."""
    c = s.case
    return float(np.sqrt(c.rgas * c.init["T1"]))


def compare_macros(s, o, tol):
    a, b = s.macros(), o.macros()
    for k in ("rho", "u", "v", "temp", "ps", "nd"):
        sc = vscale(s) if k in ("u", "v") else 0.0
        assert rel_l2(a[k], b[k], sc) <= tol, (k, rel_l2(a[k], b[k], sc))


def small_cavity():
    return cavity_case(8, 8, 16, mach=0.3, kn=0.1)


def small_channel():
    return channel_case(-2.0, 4.0, -2.0, 2.0, 30, 20, 8, 16, mach=2.0, kn=0.05, obstacle_side=1.0)


def test_state_round_trip_exact():
    s, o, f0 = pair(small_cavity())
    np.testing.assert_array_equal(s.get_state(), f0)
    s.set_state(f0.astype(np.float32))
    np.testing.assert_array_equal(s.get_state(np.float32), f0.astype(np.float32))


def test_inicon2_on_device_matches_oracle():
    c = small_channel()
    s, o, f0 = pair(c)
    s.inicon2(c.init["T1"], c.init["P1"], c.init["U0"], c.init["V0"])
    assert rel_l2(s.get_state(), f0) <= 1e-15


@pytest.mark.parametrize("mk", [small_cavity, small_channel])
def test_moments_and_wall_flux(mk):
    s, o, f0 = pair(mk())
    ref = o.compmu()
    got = s.node_fields()
    assert rel_l2(got["disnd"].ravel(), ref["DISND"]) <= 1e-13
    assert rel_l2(got["disux"].ravel(), ref["DISUX"], vscale(s)) <= 1e-13
    assert rel_l2(got["disuy"].ravel(), ref["DISUY"], vscale(s)) <= 1e-13
    assert rel_l2(got["disps"].ravel(), ref["DISPS"]) <= 1e-13
    assert rel_l2(got["mu"].ravel(), ref["MU"]) <= 1e-13
    eta = s.wall_eta()
    assert rel_l2(eta, ref["ETA"]) <= 1e-13
    compare_macros(s, o, 1e-13)


@pytest.mark.parametrize("mk,steps", [(small_cavity, 1), (small_cavity, 20), (small_channel, 1), (small_channel, 20)])
def test_fp64_steps_match_oracle(mk, steps):
    s, o, f0 = pair(mk())
    r = s.advance(steps)
    q = o.advance(steps)
    assert r["steps"] == steps
    assert rel_l2(r["dte"], q["dte"]) <= 1e-13
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64
    compare_macros(s, o, TOL64)


@pytest.mark.parametrize("tile", [64, 128])
@pytest.mark.parametrize("prec", [64, 32])
def test_tile_shapes_agree(tile, prec):
    s, o, f0 = pair(small_channel(), prec=prec, tile_elems=tile)
    s.advance(3)
    o.advance(3)
    assert rel_l2(s.get_state(), o.get_state()) <= (TOL64 if prec == 64 else 1e-5)


@pytest.mark.parametrize("rows", [1, 2, 3, 4])
@pytest.mark.parametrize("prec", [64, 32])
def test_moment_modes_agree(rows, prec):
    # every moment-kernel mode (1, 2 or 4 rows of any elements per warp
    # step, or the three rows of one element) on a ragged velocity count:
    # the moments, MU and three steps match the oracle
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 30, 20, 6, 11, mach=2.0, kn=0.05, obstacle_side=1.0)
    s, o, f0 = pair(c, prec=prec, moment_rows=rows)
    tol = 1e-13 if prec == 64 else 1e-6
    ref = o.compmu()
    got = s.node_fields()
    assert rel_l2(got["disnd"].ravel(), ref["DISND"]) <= tol
    assert rel_l2(got["disux"].ravel(), ref["DISUX"], vscale(s)) <= tol
    assert rel_l2(got["disps"].ravel(), ref["DISPS"]) <= tol
    assert rel_l2(got["mu"].ravel(), ref["MU"]) <= tol
    s.advance(3)
    o.advance(3)
    assert rel_l2(s.get_state(), o.get_state()) <= (TOL64 if prec == 64 else 1e-5)


@pytest.mark.parametrize("prec", [64, 32])
def test_ragged_velocity_count(prec):
    # V = 5 x 7 = 35: the last velocity segment is partly past V and the
    # padding rows of f must stay zero
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 24, 16, 5, 7, mach=2.0, kn=0.05, obstacle_side=1.0)
    s, o, f0 = pair(c, prec=prec)
    s.advance(4)
    o.advance(4)
    assert rel_l2(s.get_state(), o.get_state()) <= (TOL64 if prec == 64 else 1e-5)
    compare_macros(s, o, TOL64 if prec == 64 else 1e-5)


@pytest.mark.parametrize("mesh,immat", [("tc3_nanotubesphere.plt.gz", 1), ("tc1_reentry.plt.gz", 0)])
def test_reference_meshes(mesh, immat):
    # real reference meshes (tc3: inflow + type-3 and type-4 walls; tc1:
    # inflow, outflow and walls) with the tc1 gas, Lobatto10 x 10 angles,
    # fully diffuse walls
    c = reference_case(load_plt(mesh), 10, 10, alpha=1.0, immat=immat)
    s, o, f0 = pair(c, lobatto=c.lobatto)
    r = s.advance(2)
    q = o.advance(2)
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64
    compare_macros(s, o, TOL64)


def test_fp32_path_against_fp64_oracle():
    s, o, f0 = pair(small_channel(), prec=32)
    s.advance(5)
    o.advance(5)
    assert rel_l2(s.get_state(), o.get_state()) <= 1e-5
    a, b = s.macros(), o.macros()
    for k in ("rho", "u", "v", "temp"):
        assert rel_l2(a[k], b[k], vscale(s) if k in ("u", "v") else 0.0) <= 1e-5, k


def test_early_stop_on_tolerance():
    s, o, f0 = pair(small_cavity())
    r = s.advance(1)
    ref = r["res_l2"][0]
    assert s.residual_reference() == ref
    tol = 0.5
    r2 = s.advance(500, tol)
    n = r2["steps"]
    assert 0 < n < 500
    assert r2["res_l2"][-1] <= tol * ref
    assert (r2["res_l2"][:-1] > tol * ref).all()
    # the state after the early stop equals an uninterrupted run of 1 + n steps
    s2, o2, _ = pair(small_cavity())
    s2.advance(1 + n)
    np.testing.assert_array_equal(s.get_state(), s2.get_state())


def test_odd_and_even_step_counts_continue_identically():
    s, o, f0 = pair(small_channel())
    s.advance(3)
    s.advance(4)
    t, _, _ = pair(small_channel())
    t.advance(7)
    np.testing.assert_array_equal(s.get_state(), t.get_state())


# ---- partial wall accommodation (ALPHA < 1, the reference cases' 0.9) ----
# GETBOU's specular part reads the element's own f at the mirrored velocity
# in the reference's velocity order (new values for earlier velocities);
# RORDER = TORDER, the grids the reference's ring lookup serves.  The cavity
# has corner elements with two wall sides (chains of mirrored velocities).

def cavity_alpha():
    c = cavity_case(8, 12, 12, mach=0.3, kn=0.1)
    c.alpha = 0.9
    return c


def channel_alpha():
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 30, 20, 12, 12, mach=2.0, kn=0.05, obstacle_side=1.0)
    c.alpha = 0.9
    return c


@pytest.mark.parametrize("mk,steps", [(cavity_alpha, 1), (cavity_alpha, 10), (channel_alpha, 1), (channel_alpha, 10)])
def test_partial_accommodation_matches_oracle(mk, steps):
    s, o, f0 = pair(mk())
    r = s.advance(steps)
    q = o.advance(steps)
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64
    compare_macros(s, o, TOL64)


@pytest.mark.parametrize("mesh", ["tc3_nanotubesphere.plt.gz", "tc1_reentry.plt.gz"])
def test_reference_meshes_partial_accommodation(mesh):
    # the reference cases' own accommodation (ALPHA = 0.9, IMMAT = 1)
    c = reference_case(load_plt(mesh), 10, 10, alpha=0.9, immat=1)
    s, o, f0 = pair(c, lobatto=c.lobatto)
    r = s.advance(2)
    q = o.advance(2)
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64
    compare_macros(s, o, TOL64)


def test_partial_accommodation_fp32_against_fp64_oracle():
    s, o, f0 = pair(channel_alpha(), prec=32)
    s.advance(5)
    o.advance(5)
    assert rel_l2(s.get_state(), o.get_state()) <= 1e-5


@pytest.mark.parametrize("mk,steps", [(cavity_alpha, 10), (channel_alpha, 10)])
def test_partial_accommodation_consistent_mass(mk, steps):
    # ALPHA < 1 with CMMINC (IMMAT = 0): the deferred wall nodes keep RHS*DTE
    # and COLL*DTE apart for CMMINC's residual
    c = mk()
    c.immat = 0
    s, o, f0 = pair(c)
    r = s.advance(steps)
    q = o.advance(steps)
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64
    compare_macros(s, o, TOL64)
    # FP32 f against the same FP64 oracle
    s32, o32, _ = pair(c, prec=32)
    s32.advance(steps)
    o32.advance(steps)
    assert rel_l2(s32.get_state(), o32.get_state()) <= 1e-5


def test_reference_mesh_partial_accommodation_consistent_mass():
    c = reference_case(load_plt("tc1_reentry.plt.gz"), 10, 10, alpha=0.9, immat=0)
    s, o, f0 = pair(c, lobatto=c.lobatto)
    r = s.advance(2)
    q = o.advance(2)
    assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    assert rel_l2(s.get_state(), o.get_state()) <= TOL64

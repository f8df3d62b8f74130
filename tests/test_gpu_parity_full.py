"""Parity at the benchmark workloads' full sizes (GPU).

The small-case parity tests pin the arithmetic; these run the benchmark
workloads themselves against the oracle:
  * the 32 x 32 lid-driven cavity with 16 x 32 velocities (3.1e6 DOFs),
    20 steps;
  * the 200 x 100 supersonic channel with 24 x 48 velocities (1.4e8 DOFs),
    2 steps (the oracle takes about a second per FP64 step on all the host's
    cores);
in FP64 against the FP64 oracle at the parity bar (relative L2 <= 1e-10 on
rho, u, v, T and on f), and with f stored in FP32 against the same FP64
oracle, at the bound written in each test (FP32 storage rounds every value
to 2^-24 relative each step; moments and the Maxwellian parameters stay in
FP64).  The oracle runs with one OpenMP thread per host core.

A test that reaches steady state closes the file: a small free-stream
channel marched by both sides for 3000 steps (its residual falls below 1e-4
of the first step's) still agrees at the parity bar.
"""
import os

import numpy as np
import pytest

from dgbgk import Solver, channel_case, config1, config2, node_scale
from helpers import rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
THREADS = os.cpu_count() or 1


def pair(case, prec):
    s = Solver.from_case(case, precision=prec)
    o = Oracle.from_case(case, prec=64, threads=THREADS)
    i = case.init
    o.inicon2(i["T1"], i["P1"], i["U0"], i["V0"])
    f0 = o.get_state()
    sc = node_scale(case)
    if sc is not None:
        f0 *= sc[:, None, :]
        o.set_state(f0)
    s.set_state(f0)
    return s, o


def errors(s, o):
    """Relative L2 differences of the nodal rho, u, v, T (velocities on the
    thermal-speed scale sqrt(R T)) and of f."""
    a, b = s.macros(), o.macros()
    vs = float(np.sqrt(s.case.rgas * s.case.init["T1"]))
    e = {k: rel_l2(a[k], b[k], vs if k in ("u", "v") else 0.0) for k in ("rho", "u", "v", "temp")}
    e["f"] = rel_l2(s.get_state(), o.get_state())
    return e


@pytest.mark.parametrize("prec,tol", [(64, TOL64), (32, 2e-6)])
def test_cavity_32x32_v16x32_20_steps(prec, tol):
    # FP32 bound: 20 steps of FP32 rounding (~6e-8 relative per value and
    # step) on a smooth rest state; measured ~1e-7
    s, o = pair(config1(), prec)
    r = s.advance(20)
    q = o.advance(20)
    assert r["steps"] == 20
    assert rel_l2(r["dte"], q["dte"]) <= (1e-13 if prec == 64 else 1e-6)
    e = errors(s, o)
    print(f"cavity32 FP{prec} vs FP64 oracle after 20 steps: {e}")
    assert max(e.values()) <= tol, e
    if prec == 64:
        assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-9
    s.close()
    o.close()


@pytest.mark.parametrize("prec,tol", [(64, TOL64), (32, 2e-6)])
def test_channel_200x100_v24x48_2_steps(prec, tol):
    # the benchmark's Mach 2 channel: inflow, outflow, diffuse obstacle
    # walls.  FP32 bound as above (2 steps; measured ~1e-7)
    s, o = pair(config2(), prec)
    r = s.advance(2)
    q = o.advance(2)
    assert r["steps"] == 2
    e = errors(s, o)
    print(f"channel200x100 FP{prec} vs FP64 oracle after 2 steps: {e}")
    assert max(e.values()) <= tol, e
    if prec == 64:
        assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-9
        assert rel_l2(r["res_linf"], q["res_linf"]) <= 1e-9
    s.close()
    o.close()


def test_small_channel_at_steady_state():
    # 3000 steps take the 30 x 30 free-stream channel (12 x 24 velocities,
    # Mach 2.5, Kn 0.07) to a residual near 3e-5 of its first step's (the
    # oracle: 3.3e-5); the FP64 path stays at the parity bar
    c = channel_case(-2.0, 4.0, -3.0, 3.0, 30, 30, 12, 24, mach=2.5, kn=0.07, obstacle_side=1.0, sides="freestream")
    s, o = pair(c, 64)
    n = 3000
    r = s.advance(n)
    q = o.advance(n)
    assert r["res_l2"][-1] <= 1e-4 * r["res_l2"][0]
    assert rel_l2(r["res_l2"], q["res_l2"]) <= 1e-8
    e = errors(s, o)
    print(f"channel30x30 FP64 vs FP64 oracle after {n} steps: {e}")
    assert max(e.values()) <= TOL64, e
    s.close()
    o.close()

"""Device-side observables (GPU): GETFOR's lift and drag reduced on the
device, and ADVNCE's periodic GETMAC/GETFOR output recorded into a device
ring during the time loop, against the host computation on the fields
gathered through dgbgk_get_macros.

The reference gathers the nodal fields at MOD(ITIME,1000) = 0 and computes
lift and drag from the gathered pressure (src/advnce.f90:403-435,
src/getfor.f90:29-49); the ring records the same fields at the same steps
(here every 50 steps) without a host round trip.
"""
import numpy as np
import pytest

from dgbgk import Solver, channel_case

pytestmark = pytest.mark.gpu

KEYS = ("nd", "rho", "u", "v", "ps", "temp")


def getfor(mesh, ps):
    """GETFOR on the host, in the reference's loop order (FP64)."""
    lift = drag = 0.0
    for b in range(mesh.nboun):
        if mesh.bsido[b, 3] != 4:
            continue
        p1, p2 = mesh.bsido[b, 0] - 1, mesh.bsido[b, 1] - 1
        (x1, y1), (x2, y2) = mesh.coord[p1], mesh.coord[p2]
        ln = np.hypot(x2 - x1, y2 - y1)
        px, py = -(y2 - y1), x2 - x1
        mg = np.hypot(px, py)
        pav = 0.5 * (ps[p1] + ps[p2])
        lift -= pav * ln * py / mg
        drag -= pav * ln * px / mg
    return lift, drag


def case():
    # the obstacle's four sides are diffuse walls (BSIDO type 4)
    return channel_case(-2.0, 4.0, -3.0, 3.0, 30, 30, 12, 24, mach=2.5, kn=0.07, obstacle_side=1.0,
                        sides="freestream")


def test_forces_on_device_match_the_host():
    c = case()
    s = Solver.from_case(c, precision=64)
    s.init_case()
    for n in (0, 7, 30):
        if n:
            s.advance(n)
        lift, drag = s.forces()
        ps = s.macros()["ps"]
        hl, hd = getfor(c.mesh, ps)
        if n:
            assert abs(drag) > 0  # the bow shock has formed
        # the scale of the sum's terms: pressure times the obstacle's perimeter
        np.testing.assert_allclose([lift, drag], [hl, hd], rtol=1e-12, atol=1e-13 * np.abs(ps).max() * 4.0)
    s.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_output_ring_records_getmac_and_getfor(prec):
    c = case()
    s = Solver.from_case(c, precision=prec)
    s.init_case()
    s.set_output(50, 4)
    s.advance(120)             # records at ITIME 50, 100
    s.advance(110)             # 150, 200 (ITIME counts across calls)
    recs = s.outputs()
    assert [r["itime"] for r in recs] == [50, 100, 150, 200]
    # the same case marched alone, gathered on the host at those steps
    t = Solver.from_case(c, precision=prec)
    t.init_case()
    done = 0
    for r in recs:
        t.advance(r["itime"] - done)
        done = r["itime"]
        m = t.macros()
        for k in KEYS:
            assert np.array_equal(r[k], m[k]), (r["itime"], k)
        hl, hd = getfor(c.mesh, m["ps"])
        np.testing.assert_allclose([r["lift"], r["drag"]], [hl, hd], rtol=1e-12,
                                   atol=1e-13 * np.abs(m["ps"]).max() * 4.0)
    # the ring keeps the last four; a call that ends on a multiple records
    # its last step
    s.advance(70)
    assert [r["itime"] for r in s.outputs()] == [150, 200, 250, 300]
    # a new state starts ITIME again; every = 0 stops recording
    s.init_case()
    s.set_output(20, 2)
    s.advance(45)
    assert [r["itime"] for r in s.outputs()] == [20, 40]
    s.set_output(0)
    s.advance(5)
    assert s.outputs() == []
    s.close()
    t.close()

"""The command-line driver (dgbgk_run) on the GPU against the library called
directly.

A channel case (the warm-start family's geometry: inflow, free-stream sides,
outflow, a diffuse-wall obstacle with ALPHA = 0.9, the reference cases'
accommodation; RORDER = TORDER = 20, fewer angles diverge over this many
steps) is written as the reference's input files and run for 1 200 steps.  The driver's RESULTS
blocks (steps 0 and 1000, and the repeat of the last gather after the loop)
must hold the library's nodal fields to the 6 digits of the 1PE12.5 format,
RESIDUAL.RES must hold log(max|DELUN| / the first step's) for every step,
and its lift and drag (GETFOR) must come from the last gathered pressure.
"""
import os
import subprocess

import numpy as np
import pytest

from cli_case import BIN, read_results, write_case
from dgbgk import Solver, channel_case
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def getfor(mesh, ps):
    lift = drag = 0.0
    for b in mesh.bsido:
        if b[3] != 4:
            continue
        p1, p2 = b[0] - 1, b[1] - 1
        (x1, y1), (x2, y2) = mesh.coord[p1], mesh.coord[p2]
        ln = np.hypot(x2 - x1, y2 - y1)
        px, py = -(y2 - y1), x2 - x1
        mg = np.hypot(px, py)
        pav = 0.5 * (ps[p1] + ps[p2])
        lift -= pav * ln * py / mg
        drag -= pav * ln * px / mg
    return lift, drag


def test_driver_matches_library(tmp_path):
    c = channel_case(-5.0, 15.0, -10.0, 10.0, 100, 100, 20, 20, mach=2.5, kn=0.07, obstacle_side=1.0,
                     sides="freestream")
    c.alpha = 0.9
    d = str(tmp_path)
    con = write_case(d, c, 1200, forceout=1)
    r = subprocess.run([BIN, con], capture_output=True, text=True, cwd=d, timeout=600)
    assert r.returncode == 0, r.stderr

    s = Solver.from_case(c, precision=64)
    s.init_case()
    m0 = s.macros()
    h = s.advance(1000)
    m1 = s.macros()
    h2 = s.advance(200)

    r1 = read_results(os.path.join(d, "RESULTS1.RES"))
    r2 = read_results(os.path.join(d, "RESULTS2.RES"))
    assert sorted(r1) == [0, 1000, 1201] and sorted(r2) == [0, 1000, 1201]
    for blk, m in ((0, m0), (1000, m1), (1201, m1)):
        a = r1[blk]
        b = r2[blk]
        assert rel_l2(a[:, 0], m["nd"]) <= 1e-5
        assert rel_l2(a[:, 1], m["u"], 1.0) <= 1e-5
        assert rel_l2(a[:, 2], m["v"], 1.0) <= 1e-5
        assert rel_l2(b[:, 0], m["rho"]) <= 1e-5
        assert rel_l2(b[:, 1], m["ps"]) <= 1e-5
        assert rel_l2(b[:, 2], m["temp"]) <= 1e-5

    res = np.loadtxt(os.path.join(d, "RESIDUAL.RES"))
    assert res.shape == (1200, 4)
    assert np.array_equal(res[:, 0], np.arange(1, 1201))
    linf = np.concatenate([h["res_linf"], h2["res_linf"]])
    np.testing.assert_allclose(res[:, 1], np.log(linf / linf[0]), rtol=1e-6, atol=1e-7)
    l0, d0 = getfor(c.mesh, m0["ps"])
    l1, d1 = getfor(c.mesh, m1["ps"])
    np.testing.assert_allclose(res[:999, 2], l0, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(res[:999, 3], d0, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(res[999:, 2], l1, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(res[999:, 3], d1, rtol=1e-6, atol=1e-12)

    out = open(os.path.join(d, "FILE.OUT")).read().splitlines()
    assert out[-1] == f"{20:6d}{20:6d}{400:6d}" and out[-3] == "V-SPACE STATS:"
    s.close()


def test_restart_round_trip_continues_exactly(tmp_path):
    # 10 steps, write the restart file, read it back (RS = 1) for 10 more:
    # the state equals 20 steps in one run (the file holds 17 digits)
    c = channel_case(-5.0, 15.0, -10.0, 10.0, 100, 100, 20, 20, mach=2.5, kn=0.07, obstacle_side=1.0,
                     sides="freestream")
    c.alpha = 0.9
    d1, d2 = str(tmp_path / "a"), str(tmp_path / "b")
    os.makedirs(d1)
    os.makedirs(d2)
    one = write_case(d1, c, 20)
    assert subprocess.run([BIN, one, "--restart-out"], capture_output=True, cwd=d1).returncode == 0
    first = write_case(d2, c, 10)
    assert subprocess.run([BIN, first, "--restart-out"], capture_output=True, cwd=d2).returncode == 0
    os.replace(os.path.join(d2, "RESTART.RES"), os.path.join(d2, "half.res"))
    text = open(first).read().replace("IVD%RS = 0,", 'IVD%RS = 1,\nIVD%RestartInFile = "half.res",')
    open(first, "w").write(text)
    r = subprocess.run([BIN, first, "--restart-out"], capture_output=True, text=True, cwd=d2)
    assert r.returncode == 0, r.stderr
    a = open(os.path.join(d1, "RESTART.RES")).read()
    b = open(os.path.join(d2, "RESTART.RES")).read()
    assert a == b

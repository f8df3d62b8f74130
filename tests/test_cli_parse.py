"""The command-line driver's namelist reader against the Python one (CPU).

dgbgk_run --parse-only reads the &Input namelist the way the reference's
driver does (quoted strings as gfortran writes them, bare ones as ifort
accepts them, '!' comments, D exponents, the reference's defaults for what
is left out) and prints it; no GPU is touched.
"""
import json
import subprocess

import pytest

from cli_case import BIN, write_case
from dgbgk import channel_case
from dgbgk.formats import read_namelist


@pytest.mark.parametrize("quoted", [True, False])
def test_parse_only_matches_python_reader(tmp_path, quoted):
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 12, 8, 6, 6, mach=2.0, kn=0.05, obstacle_side=1.0)
    c.alpha = 0.9
    con = write_case(str(tmp_path), c, 1200, forceout=1, quoted=quoted)
    got = json.loads(subprocess.run([BIN, con, "--parse-only"], capture_output=True, text=True, check=True).stdout)
    ref = read_namelist(con)
    for k, v in got.items():
        if isinstance(v, list):
            assert v == pytest.approx(ref[k], rel=1e-15)
        elif isinstance(v, str):
            assert v == ref[k]
        else:
            assert v == pytest.approx(ref[k], rel=1e-15), k
    # defaults of the reference for keys the file leaves out
    assert got["NVSPACEPART"] == 1 and got["W"] == 1.0


def test_incompatible_restart_file_is_refused(tmp_path):
    # the check of INICON2's restart branch: NPOIN and VNPNT must match (it
    # comes before any device work)
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 12, 8, 6, 6, mach=2.0, kn=0.05, obstacle_side=1.0)
    con = write_case(str(tmp_path), c, 10)
    text = open(con).read().replace("IVD%RS = 0,", 'IVD%RS = 1,\nIVD%RestartInFile = "old.res",')
    open(con, "w").write(text)
    open(str(tmp_path / "old.res"), "w").write("NPOIN     VNPNT\n 7 36\n")
    r = subprocess.run([BIN, con], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode != 0 and "NOT COMPATIBLE" in r.stderr


def test_lobatto_file_round_trip(tmp_path):
    from dgbgk.cases import gll
    from dgbgk.formats import read_lobatto, write_lobatto
    eta, w = gll(12)
    p = str(tmp_path / "lob.txt")
    write_lobatto(p, eta, w)
    n, e2, w2 = read_lobatto(p)
    assert n == 12 and (e2 == eta).all() and (w2 == w).all()


def test_plt_mesh_round_trip_is_exact(tmp_path):
    # the driver's inputs hold the generated mesh bit for bit (the march
    # amplifies last-digit changes of the geometry beyond the output format)
    import numpy as np
    from dgbgk.formats import read_plt, write_plt
    c = channel_case(-5.0, 15.0, -10.0, 10.0, 40, 40, 4, 4, mach=2.0, kn=0.05, sides="freestream")
    p = str(tmp_path / "m.plt")
    write_plt(p, c.mesh)
    m = read_plt(p)
    assert np.array_equal(m.coord, c.mesh.coord) and np.array_equal(m.intma, c.mesh.intma)
    assert np.array_equal(m.bsido, c.mesh.bsido)


@pytest.mark.parametrize("damage,message", [
    ("lobatto_count", "bad point count in the Lobatto file"),
    ("lobatto_short", "truncated Lobatto file"),
    ("mesh_counts", "bad element / point / boundary counts"),
    ("mesh_short", "truncated"),
])
def test_malformed_inputs_are_refused(tmp_path, damage, message):
    # broken input files end the driver with a message before any device
    # work (the velocity space and the mesh are read and set up on the host)
    c = channel_case(-2.0, 4.0, -2.0, 2.0, 12, 8, 6, 6, mach=2.0, kn=0.05, obstacle_side=1.0)
    con = write_case(str(tmp_path), c, 10)
    lob, mesh = tmp_path / "lob.txt", tmp_path / "mesh.plt"
    if damage == "lobatto_count":
        lines = lob.read_text().splitlines()
        lob.write_text("\n".join(["-3"] + lines[1:]) + "\n")
    elif damage == "lobatto_short":
        lob.write_text("\n".join(lob.read_text().splitlines()[:3]) + "\n")
    elif damage == "mesh_counts":
        text = mesh.read_text().splitlines()
        k = next(i for i, ln in enumerate(text) if ln.split()[:3] == [str(c.mesh.nelem), str(c.mesh.npoin),
                                                                      str(c.mesh.nboun)])
        text[k] = f"-{c.mesh.nelem} {c.mesh.npoin} {c.mesh.nboun}"
        mesh.write_text("\n".join(text) + "\n")
    else:
        mesh.write_text("\n".join(mesh.read_text().splitlines()[:40]) + "\n")
    r = subprocess.run([BIN, con], capture_output=True, text=True, cwd=str(tmp_path), timeout=60)
    assert r.returncode != 0 and message in r.stderr, (r.returncode, r.stderr[-500:])

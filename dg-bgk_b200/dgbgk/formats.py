"""Readers and writers of the reference's file formats.

  * Lobatto file: RORDER, then RORDER lines "eta weight" (src/vspace.f90:16-18,
    src/spectralbgk.f90:161).
  * .plt mesh: NLINES title lines, dimension, counts, then the sections
    "connectivities", "coordinates" and "boundary sides" (src/spectralbgk.f90
    :240-272, src/gtinpt.f90:24-50).
  * .con namelist &Input with IVD%... keys, quoted (gfortran) or unquoted
    (ifort) strings (src/spectralbgk.f90:116-148).
  * RESULTS1/2.RES blocks and RESIDUAL.RES lines (src/advnce.f90:164-169,
    410-432, 488-489).
"""
import re

import numpy as np

from .cases import RawMesh


def read_lobatto(path):
    with open(path) as fh:
        toks = fh.read().split()
    n = int(float(toks[0]))
    vals = np.array([float(t) for t in toks[1:1 + 2 * n]]).reshape(n, 2)
    return n, vals[:, 0].copy(), vals[:, 1].copy()


def write_lobatto(path, eta, w):
    with open(path, "w") as fh:
        fh.write(f"{len(eta)}\n")
        for a, b in zip(eta, w):
            fh.write(f"{float(a)!r}\t{float(b)!r}\n")


def read_plt(path):
    """The .plt mesh; a path ending in .gz is read through gzip."""
    if str(path).endswith(".gz"):
        import gzip
        with gzip.open(path, "rt") as fh:
            lines = fh.read().splitlines()
    else:
        with open(path) as fh:
            lines = fh.read().splitlines()
    pos = 0
    nlines = int(lines[pos].split()[0]); pos += 1
    pos += nlines          # title lines
    pos += 1               # "number of dimensions"
    ndimn = int(lines[pos].split()[0]); pos += 1
    if ndimn != 2:
        raise ValueError("only 2-D meshes are supported")
    pos += 1               # "nelem npoin nboun"
    nelem, npoin, nboun = (int(x) for x in lines[pos].split()[:3]); pos += 1
    pos += 1               # "connectivities"
    intma = np.array([[int(x) for x in lines[pos + i].split()[1:4]] for i in range(nelem)], dtype=np.int32)
    pos += nelem + 1       # + "coordinates"
    coord = np.array([[float(x) for x in lines[pos + i].split()[1:3]] for i in range(npoin)], dtype=np.float64)
    pos += npoin + 1       # + "boundary sides"
    bsido = np.array([[int(x) for x in lines[pos + i].split()[:6]] for i in range(nboun)], dtype=np.int32)
    return RawMesh(intma, coord, bsido.reshape(nboun, 6), None, {"kind": "plt", "path": str(path)})


def write_plt(path, mesh, title="title"):
    with open(path, "w") as fh:
        fh.write("           1\n")
        fh.write(f"{title}\n")
        fh.write("number of dimensions\n           2\n")
        fh.write("nelem   npoin   nboun\n")
        fh.write(f"{mesh.nelem:12d}{mesh.npoin:12d}{mesh.nboun:12d}\n")
        fh.write("  connectivities \n")
        for i, (a, b, c) in enumerate(mesh.intma, 1):
            fh.write(f"{i:10d}{a:15d}{b:10d}{c:10d}{0:10d}\n")
        fh.write("  coordinates \n")
        for i, (x, y) in enumerate(mesh.coord, 1):
            # 17 significant digits: the file holds the coordinates exactly
            fh.write(f"{i:10d}  {x: .16E}  {y: .16E}\n")
        fh.write("  boundary sides \n")
        for r in mesh.bsido:
            fh.write("".join(f"{int(x):10d}" for x in r) + "\n")


_NUM = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eEdD][+-]?\d+)?$")


def read_namelist(path):
    """Parses &Input ... / into {"TORDER": 40, "CINF": [..4..], "LobattoFile": "...", ...}
    with the reference defaults of src/spectralbgk.f90:116-147 filled in."""
    out = {"TORDER": 20, "NTIME": 10000, "FORCEOUT": 0, "IMMAT": 1, "INF": 1, "RS": 0, "CSAFM": 0.5,
           "rv": 2000.0, "T1": 293.0, "P1": 0.1, "U0": 100.0, "V0": 0.0, "W": 1.0, "ALPHA": 0.9, "R": 287.0,
           "d": 250e-12, "M": 32.0, "CINF": [294.0, 0.001473, 171.85, 0.0], "NVSPACEPART": 1,
           "LobattoFile": "Lobatto20.txt", "PSpaceFile": "AEROFOIL.RES", "OutFile": "FILE.OUT",
           "PartitionFile": "METIS3WAYPARTAEROFOIL13.RES", "RestartInFile": "RESTART.RES",
           "ResidualFile": "RESIDUAL.RES", "ResultsFile1": "RESULTS1.RES", "ResultsFile2": "RESULTS2.RES",
           "RestartOutFile": "RESTART.RES", "GIDMeshFile": "GIDMESH.RES"}
    canon = {k.lower(): k for k in out}
    text = open(path).read()
    m = re.search(r"&input(.*?)(^\s*/\s*$|\Z)", text, re.S | re.I | re.M)
    body = m.group(1) if m else text
    for raw in body.splitlines():
        line = raw.split("!")[0].strip().rstrip(",").strip()
        if "=" not in line:
            continue
        key, val = (s.strip() for s in line.split("=", 1))
        key = key.split("%")[-1]
        idx = None
        km = re.match(r"(\w+)\((\d+)\)", key)
        if km:
            key, idx = km.group(1), int(km.group(2))
        val = val.rstrip(",").strip().strip('"').strip("'")
        if _NUM.match(val):
            v = float(val.replace("d", "e").replace("D", "e"))
        else:
            v = val
        name = canon.get(key.lower(), key)
        if idx is not None:
            out.setdefault(name, [0.0] * 4)[idx - 1] = v
        else:
            out[name] = v
    for k in ("TORDER", "NTIME", "FORCEOUT", "IMMAT", "INF", "RS", "NVSPACEPART"):
        out[k] = int(out[k])
    return out


def write_results_block(fh1, fh2, itime, nd, u, v, rho, ps, temp):
    """One GiD results block per file (src/advnce.f90:164-169, 488-489)."""
    fh1.write(f"RESULTS        1   {itime:5d}    2      1      0\n")
    fh2.write(f"RESULTS        1   {itime:5d}    2      1      0\n")
    for ip in range(len(nd)):
        fh1.write(f"{ip + 1:5d}    {_e(nd[ip])} {_e(u[ip])} {_e(v[ip])} \n")
        fh2.write(f"{ip + 1:5d}    {_e(rho[ip])} {_e(ps[ip])} {_e(temp[ip])} \n")


def _e(x):
    """Fortran 1pe12.5."""
    s = f"{x:.5E}"
    mant, ex = s.split("E")
    e = int(ex)
    return f"{mant}E{'+' if e >= 0 else '-'}{abs(e):02d}".rjust(12)

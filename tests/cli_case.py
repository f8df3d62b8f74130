"""Writes a generated case as the reference's input files (.con namelist,
.plt mesh, Lobatto file) for the command-line driver's tests."""
import os

from dgbgk.cases import gll
from dgbgk.formats import write_lobatto, write_plt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dg-bgk_b200", "bin", "dgbgk_run")


def write_case(d, case, ntime, forceout=1, quoted=True):
    eta, w = gll(case.rorder)
    write_lobatto(os.path.join(d, "lob.txt"), eta, w)
    write_plt(os.path.join(d, "mesh.plt"), case.mesh)
    i = case.init
    q = (lambda s: f'"{s}"') if quoted else (lambda s: s)
    e = lambda x: repr(float(x)).replace("e", "D")  # Fortran double-precision exponents
    con = f"""&Input
IVD%TORDER = {case.torder},  !LOBATTO QUADRATURE ORDER FOR V-SPACE
IVD%rv = {e(case.rv)},  !RADIAL EXTENT OF THE V-SPACE
IVD%FORCEOUT = {forceout}, !OUTPUT FORCES IN RESIDUAL YES/NO?
IVD%NTIME = {ntime}, !NUMBER OF TIMESTEPS
IVD%IMMAT = {case.immat},
IVD%ALPHA = {case.alpha!r},  !MOLECULAR WALL REFLECTION PARAMETER
IVD%CSAFM = {case.csafm!r},
IVD%RS = 0,
IVD%T1 = {e(i["T1"])},
IVD%P1 = {e(i["P1"])},
IVD%U0 = {e(i["U0"])},
IVD%V0 = {e(i["V0"])},
IVD%INF = 1,
IVD%CINF(1) = {e(case.cinf[0])}, !INFLOW TEMP
IVD%CINF(2) = {e(case.cinf[1])},
IVD%CINF(3) = {e(case.cinf[2])},
IVD%CINF(4) = {e(case.cinf[3])},
IVD%R = {e(case.rgas)},
IVD%d = {e(case.diameter)},
IVD%M = {e(case.molar_mass)},
IVD%LobattoFile = {q("lob.txt")}, !Lobatto Quadrature File
IVD%PSpaceFile = {q("mesh.plt")}, !PSpace Mesh File
IVD%OutFile = {q("FILE.OUT")},
IVD%ResidualFile = {q("RESIDUAL.RES")} !RESIDUAL FILE
IVD%ResultsFile1 = {q("RESULTS1.RES")}
IVD%ResultsFile2 = {q("RESULTS2.RES")}
/
"""
    path = os.path.join(d, "case.con")
    with open(path, "w") as fh:
        fh.write(con)
    return path


def read_results(path):
    """{itime: array (NPOIN, 3)} of a RESULTS1/2.RES file."""
    import numpy as np
    out, cur, rows = {}, None, []
    for line in open(path):
        if line.startswith("RESULTS"):
            if cur is not None:
                out[cur] = np.array(rows)
            cur, rows = int(line.split()[2]), []
        elif line.strip():
            rows.append([float(x) for x in line.split()[1:4]])
    if cur is not None:
        out[cur] = np.array(rows)
    return out

"""Shared test helpers: meshes from the golden fixtures, product/oracle pairs
built on the same inputs, and error norms."""
import gzip
import os
import tempfile

import numpy as np

from conftest import GOLDEN


def rel_l2(a, b, scale=0.0):
    """||a - b|| / max(||b||, scale * sqrt(n)).  `scale` floors the
    denominator for fields that can be ~0 (a bulk velocity at rest is
    compared on the thermal-speed scale, not relative to its own size)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = max(np.linalg.norm(b), scale * np.sqrt(b.size))
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def load_plt(name):
    from dgbgk.formats import read_plt
    with gzip.open(os.path.join(GOLDEN, name), "rt") as fh, tempfile.NamedTemporaryFile("w", suffix=".plt",
                                                                                      delete=False) as tmp:
        tmp.write(fh.read())
        path = tmp.name
    try:
        return read_plt(path)
    finally:
        os.unlink(path)


def lobatto(n):
    from dgbgk.formats import read_lobatto
    return read_lobatto(os.path.join(GOLDEN, f"Lobatto{n}.txt"))


def reference_case(mesh, rorder_file=10, torder=10, alpha=1.0, immat=1, prec=64, scale_phys=True):
    """A CaseDef on a reference mesh (tc1/tc3) with the tc1 namelist's gas
    (T 300 K, p 7.5e-10 bar, U0 8680 m/s, R 287, M 32, d 250e-12, rv 13000),
    on the rorder_file-point Lobatto file."""
    from dgbgk.cases import CaseDef
    n, eta, w = lobatto(rorder_file)
    c = CaseDef(name="tc", mesh=mesh, rorder=n, torder=torder, rv=13000.0, immat=immat, csafm=0.5, alpha=alpha,
                rgas=287.0, molar_mass=32.0, diameter=250e-12, cinf=(300.0, 0.00000000075, 8680.0, 0.0),
                init={"T1": 300.0, "P1": 0.00000000075, "U0": 8680.0, "V0": 0.0, "perturb": 0.0, "seed": 0})
    c.lobatto = (eta, w)
    return c

"""The oracle against the reference's own known answers (CPU)."""
import json
import os

import numpy as np

from conftest import GOLDEN
from helpers import load_plt, lobatto
from pyoracle import Oracle


def _kat():
    return json.load(open(os.path.join(GOLDEN, "kat.json")))


def test_sumweight_lobatto40_fp32():
    # tc/tc1/output:24 prints SUMWEIGHT=   79.99974 for Lobatto40, TORDER = 40
    n, eta, w = lobatto(40)
    m = load_plt("tc1_reentry.plt.gz")
    o = Oracle(m.intma, m.coord, m.bsido, n, 40, eta, w, rv=13000.0, prec=32)
    sw = np.float32(o.get("SUMWEIGHT")[0])
    assert f"{sw:.7g}" == _kat()["sumweight_lobatto40_torder40_fp32"]


def test_tc1_counts():
    # tc/tc1/FILE.OUT:5,8
    k = _kat()
    m = load_plt("tc1_reentry.plt.gz")
    assert [m.nelem, m.npoin, m.nboun] == k["tc1_nelem_npoin_nboun"]
    n, eta, w = lobatto(40)
    assert [n, 40, n * 40] == k["tc1_rorder_torder_vnpnt"]


def test_gll_generator_matches_reference_lobatto_files():
    from dgbgk.cases import gll
    for n in (10, 40):
        _, eta, w = lobatto(n)
        x, ww = gll(n)
        assert np.max(np.abs(x - eta)) < 5e-10
        assert np.max(np.abs(ww - w)) < 5e-10


def test_tc1_mesh_is_counter_clockwise():
    m = load_plt("tc1_reentry.plt.gz")
    x = m.coord[m.intma - 1]
    rj = (x[:, 1, 0] - x[:, 0, 0]) * (x[:, 2, 1] - x[:, 0, 1]) - (x[:, 2, 0] - x[:, 0, 0]) * (x[:, 1, 1] - x[:, 0, 1])
    assert (rj > 0).all()

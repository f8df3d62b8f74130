"""The library's host setup (dgbgk_setup_mesh, dgbgk_vspace_build) against the
oracle's restatement of GETSID/NORMAL/GETGEO/GETLEN/GETMAT/CONMAT/GETNOR and
VSPACE, on generated and reference meshes (CPU)."""
import numpy as np
import pytest

from dgbgk import cavity_mesh, channel_mesh, setup_mesh, vspace
from helpers import load_plt, lobatto
from pyoracle import Oracle

MESHES = {
    "cavity8": lambda: cavity_mesh(8, 0.3),
    "channel": lambda: channel_mesh(-2.0, 4.0, -2.0, 2.0, 30, 20, 1.0),
    "tc1": lambda: load_plt("tc1_reentry.plt.gz"),
    "tc3": lambda: load_plt("tc3_nanotubesphere.plt.gz"),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_setup_arrays_match_oracle(name):
    m = MESHES[name]()
    n, eta, w = lobatto(10)
    o = Oracle(m.intma, m.coord, m.bsido, n, 10, eta, w, rv=1.0, prec=64)
    st = setup_mesh(m.intma, m.coord, m.bsido)
    assert st.nside == o.S
    np.testing.assert_array_equal(st.iside.ravel(), o.get("ISIDE").astype(np.int32))
    for key, arr in (("NX", st.nx), ("NY", st.ny), ("EL", st.el), ("GEOME", st.geome), ("RELEN", st.relen),
                     ("MMAT", st.mmat), ("RSIDO", st.rsido)):
        np.testing.assert_array_equal(arr.ravel(), o.get(key), err_msg=key)
    # the CONMAT branch runs only for IMMAT = 0
    o0 = Oracle(m.intma, m.coord, m.bsido, n, 10, eta, w, rv=1.0, prec=64, immat=0)
    np.testing.assert_array_equal(st.cmmat.ravel(), o0.get("CMMAT"))
    # every element has its three edges claimed by exactly one side
    E = m.nelem
    cnt = np.zeros((E, 3), dtype=int)
    for s in st.iside:
        cnt[s[2] - 1, s[4] - 1] += 1
        if s[3] > 0:
            cnt[s[3] - 1, s[7] - 1] += 1
    assert (cnt == 1).all()


@pytest.mark.parametrize("n,t", [(10, 10), (40, 40), (10, 7)])
def test_vspace_matches_oracle(n, t):
    nn, eta, w = lobatto(n)
    m = cavity_mesh(2)
    o = Oracle(m.intma, m.coord, m.bsido, nn, t, eta, w, rv=1.0, prec=64)
    vc, sw = vspace(nn, t, eta, w)
    np.testing.assert_array_equal(vc.ravel(), o.get("VCORD"))
    assert sw == o.get("SUMWEIGHT")[0]


def test_boundary_conventions_of_generated_meshes():
    # BSIDO IP1 -> IP2 follows the element's CCW order: the GETNOR normal
    # points out of the fluid (away from the element centroid)
    for m in (cavity_mesh(6), channel_mesh(-2.0, 4.0, -2.0, 2.0, 30, 20, 1.0)):
        st = setup_mesh(m.intma, m.coord, m.bsido)
        cen = m.coord[m.intma - 1].mean(axis=1)
        for b, row in enumerate(m.bsido):
            mid = 0.5 * (m.coord[row[0] - 1] + m.coord[row[1] - 1])
            assert np.dot(st.rsido[b, :2], mid - cen[row[2] - 1]) > 0


@pytest.mark.parametrize("damage,code,message", [
    ("node_index", -2, "INTMA references a node outside"),
    ("bside_index", -2, "BSIDO references a node outside"),
    ("zero_area", -2, "has zero or non-finite area"),
    ("zero_side", -2, "has zero or non-finite length"),
    ("no_elements", -1, "bad arguments"),
])
def test_setup_refuses_broken_meshes(damage, code, message):
    # broken meshes end with a status code and a message (the reference
    # would divide by zero or index out of bounds); host only, no GPU
    from dgbgk._lib import DgbgkError
    m = cavity_mesh(4, 0.3)
    intma, coord, bsido = m.intma.copy(), m.coord.copy(), m.bsido.copy()
    if damage == "node_index":
        intma[5, 1] = m.npoin + 1
    elif damage == "bside_index":
        bsido[2, 0] = 0
    elif damage == "zero_area":
        # element 1's three nodes on one line: its third node moved onto
        # the line through the first two
        a, b, c = intma[0] - 1
        coord[c] = 0.5 * (coord[a] + coord[b])
    elif damage == "zero_side":
        a, b, _ = intma[0] - 1
        coord[b] = coord[a]
    else:
        intma = intma[:0]
    with pytest.raises(DgbgkError) as ei:
        setup_mesh(intma, coord, bsido)
    assert ei.value.code == code and message in str(ei.value)

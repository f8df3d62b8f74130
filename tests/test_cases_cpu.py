"""The synthetic workloads' host logic (CPU): the (Mach, Kn) mapping to the
reference's physical inputs, the Gauss-Lobatto-Legendre velocity grid, the
seeded density perturbation, the mesh conventions and the batched draw."""
import math

import numpy as np
import pytest

from dgbgk import cavity_case, channel_case, config3, gll, node_scale, physical_params
from dgbgk.cases import GAMMA, PI_REF


@pytest.mark.parametrize("mach,kn", [(0.3, 0.1), (2.0, 0.05), (1.0, 0.01), (0.5, 1.0)])
def test_mach_kn_mapping_inverts(mach, kn):
    p = physical_params(mach, kn)
    n = 1.0 * 6.022e26 / p["molar_mass"]  # number density (M = NA: equal to rho)
    # hard-sphere mean free path with the reference's collision model
    lam = 1.0 / (math.sqrt(2.0) * PI_REF * n * p["diameter"] ** 2)
    assert lam / 1.0 == pytest.approx(kn, rel=1e-12)
    assert p["speed"] / math.sqrt(GAMMA * p["rgas"] * p["temp"]) == pytest.approx(mach, rel=1e-14)
    assert p["p_bar"] * 1e5 == pytest.approx(1.0 * p["rgas"] * p["temp"], rel=1e-14)


@pytest.mark.parametrize("n", [2, 3, 8, 16, 24, 40])
def test_gll_rule(n):
    x, w = gll(n)
    assert x[0] == -1.0 and x[-1] == 1.0 and np.all(np.diff(x) > 0)
    assert np.allclose(x, -x[::-1], atol=1e-15) and np.allclose(w, w[::-1], atol=1e-15)
    # exact for polynomials up to degree 2n - 3
    for k in range(2 * n - 2):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert np.dot(w, x ** k) == pytest.approx(exact, abs=1e-13)


def test_density_perturbation_is_seeded_and_bounded():
    c = cavity_case(8, 4, 8, perturb=1e-3, seed=3)
    a, b = node_scale(c), node_scale(cavity_case(8, 4, 8, perturb=1e-3, seed=3))
    assert a.shape == (c.mesh.nelem, 3) and np.array_equal(a, b)
    assert np.all(np.abs(a - 1.0) <= 1e-3) and np.abs(a - 1.0).max() > 9e-4
    assert not np.array_equal(a, node_scale(cavity_case(8, 4, 8, perturb=1e-3, seed=4)))
    assert node_scale(cavity_case(8, 4, 8, perturb=0.0)) is None


def test_generated_meshes_follow_the_reference_conventions():
    for c in (cavity_case(6, 4, 8), channel_case(-2.0, 4.0, -2.0, 2.0, 12, 8, 4, 8, mach=2.0, kn=0.05)):
        m = c.mesh
        xy = m.coord[m.intma - 1]  # (E, 3, 2)
        area2 = ((xy[:, 1, 0] - xy[:, 0, 0]) * (xy[:, 2, 1] - xy[:, 0, 1]) -
                 (xy[:, 2, 0] - xy[:, 0, 0]) * (xy[:, 1, 1] - xy[:, 0, 1]))
        assert np.all(area2 > 0)  # counter-clockwise, 1-based
        assert m.intma.min() == 1 and m.intma.max() == m.npoin
        # BSIDO: IP1 -> IP2 in the element's local order, so (dy, -dx) points
        # out of the fluid (away from the element's centroid)
        for ip1, ip2, iel, typ, tw, a10 in m.bsido:
            loc = list(m.intma[iel - 1])
            k = loc.index(ip1)
            assert loc[(k + 1) % 3] == ip2 and typ in (1, 2, 4)
            p1, p2 = m.coord[ip1 - 1], m.coord[ip2 - 1]
            nrm = np.array([p2[1] - p1[1], -(p2[0] - p1[0])])
            cen = m.coord[np.array(loc) - 1].mean(axis=0)
            assert np.dot(nrm, 0.5 * (p1 + p2) - cen) > 0


def test_batched_draw_is_within_its_ranges():
    cases = config3(ncases=16, seed=1)
    assert len(cases) == 16
    for k, c in enumerate(cases):
        n = int(round(math.sqrt(c.mesh.nelem / 2)))
        assert n in range(16, 97, 8) and c.mesh.nelem == 2 * n * n
        assert 8 <= c.rorder <= 24 and 16 <= c.torder <= 64
        assert 0.1 <= c.info["mach"] <= 1.0 and 0.01 <= c.info["kn"] <= 1.0
        assert c.init["seed"] == 1000 + k
    assert [c.name for c in cases] == [c.name for c in config3(ncases=16, seed=1)]

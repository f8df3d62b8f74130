"""Nodal fields <-> regular grid resampling of the warm start (CPU).

A P1 field that is linear in space is reproduced exactly by both maps
(barycentric evaluation inside the triangles, bilinear interpolation of a
linear grid field); a smooth field survives the round trip to within the
grid's interpolation error; grid points inside the obstacle are filled.
"""
import numpy as np

from dgbgk import channel_case
from dgbgk.resample import GridResampler


def mesh():
    return channel_case(-5, 15, -5, 5, 50, 25, 4, 8, mach=2.0, kn=0.05, obstacle_side=1.6).mesh


def test_linear_field_is_exact_both_ways():
    m = mesh()
    R = GridResampler(m.intma, m.coord, 128, 64, box=(-5, 15, -5, 5))
    xy = m.coord[m.intma - 1]
    lin = lambda x, y: 2.0 * x - 3.0 * y + 1.0
    G = R.to_grid(lin(xy[..., 0], xy[..., 1]))
    XX, YY = np.meshgrid(R.xc, R.yc)
    inside = R.inside.reshape(64, 128)
    assert np.abs(G - lin(XX, YY))[inside].max() < 1e-12
    # the obstacle's grid points were filled from their neighbours
    assert (~inside).sum() > 0 and np.isfinite(G).all()
    # a linear grid field interpolates exactly at nodes inside the
    # outermost cell centres
    q = R.to_nodes(lin(XX, YY))
    ex = lin(xy[..., 0], xy[..., 1])
    interior = (np.abs(xy[..., 0] - 5) < 10 - 20 / 256) & (np.abs(xy[..., 1]) < 5 - 10 / 128)
    assert np.abs(q - ex)[interior].max() < 1e-12


def test_smooth_round_trip_and_batched_shapes():
    m = mesh()
    R = GridResampler(m.intma, m.coord, 128, 64, box=(-5, 15, -5, 5))
    xy = m.coord[m.intma - 1]
    f = np.stack([np.sin(0.3 * xy[..., 0]) * np.cos(0.5 * xy[..., 1]) + k for k in range(4)])
    G = R.to_grid(f)
    assert G.shape == (4, 64, 128)
    q = R.to_nodes(G)
    assert q.shape == f.shape
    assert np.linalg.norm(q - f) / np.linalg.norm(f) < 1e-2

"""Resampling between DG nodal fields and a regular grid.

The warm-start network predicts macroscopic fields on a fixed ny x nx grid of
cell centres over the mesh's bounding box, independent of the mesh.  Fields
on the mesh are the discontinuous P1 values per DG node, (NELEM, 3) arrays
in the reference's (3, NELEM) order:

  * nodes -> grid evaluates, at each grid point, the P1 field of the
    triangle that contains it (barycentric weights of its three DG nodes);
    grid points outside every triangle (inside an obstacle) take the mean of
    their already-filled 4-neighbours, sweep by sweep from the obstacle's
    surface inwards;
  * grid -> nodes interpolates the filled grid bilinearly at each DG node's
    coordinates (clamped to the outermost cell centres).

Both maps are linear and precomputed once per mesh.
"""
import numpy as np


class GridResampler:
    def __init__(self, intma, coord, nx=128, ny=64, box=None):
        intma = np.asarray(intma)
        if intma.shape[0] == 3 and intma.shape[1] != 3:
            intma = intma.T
        coord = np.asarray(coord, dtype=np.float64)
        tri = coord[intma - 1]                                        # (E, 3, 2)
        if box is None:
            box = (coord[:, 0].min(), coord[:, 0].max(), coord[:, 1].min(), coord[:, 1].max())
        x0, x1, y0, y1 = map(float, box)
        self.nx, self.ny, self.box = nx, ny, (x0, x1, y0, y1)
        dx, dy = (x1 - x0) / nx, (y1 - y0) / ny
        self.E = tri.shape[0]
        self.xc = x0 + (np.arange(nx) + 0.5) * dx
        self.yc = y0 + (np.arange(ny) + 0.5) * dy

        # ---- point location: candidate grid points per triangle bounding box
        lo = tri.min(axis=1)
        hi = tri.max(axis=1)
        i_lo = np.clip(np.ceil((lo[:, 0] - x0) / dx - 0.5), 0, nx - 1).astype(np.int64)
        i_hi = np.clip(np.floor((hi[:, 0] - x0) / dx - 0.5), -1, nx - 1).astype(np.int64)
        j_lo = np.clip(np.ceil((lo[:, 1] - y0) / dy - 0.5), 0, ny - 1).astype(np.int64)
        j_hi = np.clip(np.floor((hi[:, 1] - y0) / dy - 0.5), -1, ny - 1).astype(np.int64)
        ki = int(max(1, (i_hi - i_lo + 1).max()))
        kj = int(max(1, (j_hi - j_lo + 1).max()))
        owner = np.full(nx * ny, -1, dtype=np.int64)
        bary = np.zeros((nx * ny, 3))
        p0, p1, p2 = tri[:, 0], tri[:, 1], tri[:, 2]
        det = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1])
        eidx = np.arange(self.E)
        eps = 1e-10
        for a in range(ki):
            for b in range(kj):
                i = i_lo + a
                j = j_lo + b
                ok = (i <= i_hi) & (j <= j_hi)
                if not ok.any():
                    continue
                e = eidx[ok]
                px, py = self.xc[i[ok]], self.yc[j[ok]]
                rx, ry = px - p0[ok, 0], py - p0[ok, 1]
                l1 = (rx * (p2[ok, 1] - p0[ok, 1]) - (p2[ok, 0] - p0[ok, 0]) * ry) / det[ok]
                l2 = ((p1[ok, 0] - p0[ok, 0]) * ry - rx * (p1[ok, 1] - p0[ok, 1])) / det[ok]
                l0 = 1.0 - l1 - l2
                inside = (l0 >= -eps) & (l1 >= -eps) & (l2 >= -eps)
                g = j[ok][inside] * nx + i[ok][inside]
                owner[g] = e[inside]
                bary[g] = np.stack([l0[inside], l1[inside], l2[inside]], axis=1)
        self.owner = owner
        self.bary = bary
        self.inside = owner >= 0

        # ---- fill order for the points no triangle covers
        known = self.inside.reshape(ny, nx).copy()
        steps = []
        while not known.all():
            cnt = np.zeros((ny, nx))
            for sl_to, sl_from in self._shifts():
                cnt[sl_to] += known[sl_from]
            new = (~known) & (cnt > 0)
            if not new.any():
                raise ValueError("grid points unreachable from the mesh")
            steps.append(np.flatnonzero(new))
            known |= new
        self.fill_steps = steps

        # ---- bilinear weights of every DG node
        xy = tri.reshape(-1, 2)
        fx = np.clip((xy[:, 0] - x0) / dx - 0.5, 0.0, nx - 1.0)
        fy = np.clip((xy[:, 1] - y0) / dy - 0.5, 0.0, ny - 1.0)
        i0 = np.minimum(np.floor(fx).astype(np.int64), nx - 2)
        j0 = np.minimum(np.floor(fy).astype(np.int64), ny - 2)
        tx, ty = fx - i0, fy - j0
        self.bl_idx = np.stack([j0 * nx + i0, j0 * nx + i0 + 1, (j0 + 1) * nx + i0, (j0 + 1) * nx + i0 + 1], axis=1)
        self.bl_w = np.stack([(1 - tx) * (1 - ty), tx * (1 - ty), (1 - tx) * ty, tx * ty], axis=1)

    @staticmethod
    def _shifts():
        # (destination slice, source slice) pairs of the 4-neighbourhood
        return [((slice(None), slice(1, None)), (slice(None), slice(None, -1))),
                ((slice(None), slice(None, -1)), (slice(None), slice(1, None))),
                ((slice(1, None), slice(None)), (slice(None, -1), slice(None))),
                ((slice(None, -1), slice(None)), (slice(1, None), slice(None)))]

    def to_grid(self, q):
        """(..., NELEM, 3) nodal fields -> (..., ny, nx)."""
        q = np.asarray(q, dtype=np.float64)
        lead = q.shape[:-2]
        q = q.reshape((-1, self.E, 3))
        out = np.zeros((q.shape[0], self.ny * self.nx))
        g = np.flatnonzero(self.inside)
        e = self.owner[g]
        out[:, g] = np.einsum("kgi,gi->kg", q[:, e, :], self.bary[g])
        known = self.inside.copy()
        for pts in self.fill_steps:
            grid = out.reshape(-1, self.ny, self.nx)
            kn = known.reshape(self.ny, self.nx)
            s = np.zeros_like(grid)
            c = np.zeros((self.ny, self.nx))
            for sl_to, sl_from in self._shifts():
                s[(slice(None),) + sl_to] += grid[(slice(None),) + sl_from] * kn[sl_from]
                c[sl_to] += kn[sl_from]
            out[:, pts] = s.reshape(out.shape[0], -1)[:, pts] / c.reshape(-1)[pts]
            known[pts] = True
        return out.reshape(lead + (self.ny, self.nx))

    def to_nodes(self, grid):
        """(..., ny, nx) grid fields -> (..., NELEM, 3) nodal values."""
        grid = np.asarray(grid, dtype=np.float64)
        lead = grid.shape[:-2]
        g = grid.reshape((-1, self.ny * self.nx))
        v = (g[:, self.bl_idx] * self.bl_w[None]).sum(axis=-1)
        return v.reshape(lead + (self.E, 3))

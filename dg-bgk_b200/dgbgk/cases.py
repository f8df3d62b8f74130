"""Synthetic cases: structured P1 triangle meshes, Gauss-Lobatto-Legendre
velocity grids and the mapping from (Mach, Kn) to the reference's physical
inputs.

Meshes follow the reference's mesh conventions (src/gtinpt.f90, the .plt
files of tc/): 1-based INTMA(3,NELEM) with counter-clockwise triangles,
COORD(2,NPOIN), and BSIDO(6,NBOUN) rows (IP1, IP2, IEL, TYPE, T_wall,
ALPHA*10) whose IP1 -> IP2 follows the element's local order, so that the
GETNOR normal (dy, -dx)/L points out of the fluid.  Boundary types: 1 inflow,
2 outflow (zero gradient), 4 diffuse wall.

Build choices (documented, not reference behaviour):
  * units R = 1, T = 1, rho = 1 and M = NA = 6.022e26 (so M/NA = 1 and the
    number density equals the density); P = rho R T, passed in bar (/1e5);
  * 2-D monatomic gas: gamma = 2, U = Ma * sqrt(gamma R T);
  * hard-sphere diameter from Kn = lambda / L with the reference's own
    collision model (MU = sqrt(2) CT PI d^2 n, PI = 3.1416):
    d = (sqrt(2) * PI * n * Kn * L) ** -0.5;
  * velocity radius rv = 4 sqrt(R T) (+ the bulk speed for channels), radial
    nodes at the Gauss-Lobatto-Legendre points (the reference's Lobatto
    files hold GLL nodes and weights, e.g. tc/tc1/Lobatto40.txt).
"""
import math
from dataclasses import dataclass, field

import numpy as np

PI_REF = 3.1416
GAMMA = 2.0


def gll(n):
    """Gauss-Lobatto-Legendre nodes (ascending) and weights on [-1, 1] by
    Newton iteration on the Legendre recurrence, started from the
    Chebyshev-Gauss-Lobatto points."""
    if n < 2:
        raise ValueError("GLL needs at least 2 points")
    N = n - 1
    x = -np.cos(np.pi * np.arange(n) / N)
    P = np.zeros((n, n))
    xold = np.full(n, 2.0)
    for _ in range(100):
        if np.max(np.abs(x - xold)) <= 1e-16:
            break
        xold = x.copy()
        P[:, 0] = 1.0
        P[:, 1] = x
        for k in range(2, n):
            P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
        x = xold - (x * P[:, N] - P[:, N - 1]) / (n * P[:, N])
    P[:, 0] = 1.0
    P[:, 1] = x
    for k in range(2, n):
        P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
    w = 2.0 / (N * n * P[:, N] ** 2)
    x[0], x[-1] = -1.0, 1.0
    return x, w


@dataclass
class RawMesh:
    intma: np.ndarray  # (E,3) int32, 1-based (== INTMA(3,E) column-major)
    coord: np.ndarray  # (NP,2) float64
    bsido: np.ndarray  # (B,6) int32
    wall_velocity: np.ndarray = None  # (B,2) float64 or None
    info: dict = field(default_factory=dict)

    @property
    def nelem(self):
        return self.intma.shape[0]

    @property
    def npoin(self):
        return self.coord.shape[0]

    @property
    def nboun(self):
        return self.bsido.shape[0]


def _grid_mesh(x0, x1, y0, y1, nx, ny, active, side_type, t_wall=1):
    """Quads (i, j) with active[j, i] split into (a,b,c) and (a,c,d); the
    boundary side of each quad edge facing a missing neighbour gets
    side_type(kind, i, j) with kind in {'bottom','right','top','left'} and
    whether the neighbour is outside the domain."""
    hx = (x1 - x0) / nx
    hy = (y1 - y0) / ny
    used = np.zeros((ny + 1, nx + 1), dtype=bool)
    for j in range(ny):
        for i in range(nx):
            if active[j, i]:
                used[j:j + 2, i:i + 2] = True
    nid = -np.ones((ny + 1, nx + 1), dtype=np.int64)
    jj, ii = np.nonzero(used)
    order = np.lexsort((ii, jj))
    jj, ii = jj[order], ii[order]
    nid[jj, ii] = np.arange(1, len(jj) + 1)
    coord = np.stack([x0 + ii * hx, y0 + jj * hy], axis=1).astype(np.float64)
    intma, bsido = [], []

    def act(i, j):
        return 0 <= i < nx and 0 <= j < ny and active[j, i]

    for j in range(ny):
        for i in range(nx):
            if not active[j, i]:
                continue
            a, b, c, d = nid[j, i], nid[j, i + 1], nid[j + 1, i + 1], nid[j + 1, i]
            intma.append((a, b, c))
            e1 = len(intma)
            intma.append((a, c, d))
            e2 = len(intma)
            for kind, (p, q, e, ni, nj) in (("bottom", (a, b, e1, i, j - 1)), ("right", (b, c, e1, i + 1, j)),
                                           ("top", (c, d, e2, i, j + 1)), ("left", (d, a, e2, i - 1, j))):
                if not act(ni, nj):
                    outside = not (0 <= ni < nx and 0 <= nj < ny)
                    bsido.append((p, q, e, side_type(kind, outside, i, j), t_wall, 10))
    return (np.asarray(intma, dtype=np.int32), coord, np.asarray(bsido, dtype=np.int32))


def cavity_mesh(n, lid_speed=0.0):
    """[0,1]^2 cavity of n x n quads split into 2n^2 triangles; all four
    sides are diffuse walls (type 4, T_wall = 1); the top wall moves with
    lid_speed in +x (moving-wall extension)."""
    active = np.ones((n, n), dtype=bool)
    intma, coord, bsido = _grid_mesh(0.0, 1.0, 0.0, 1.0, n, n, active, lambda k, o, i, j: 4)
    wv = np.zeros((bsido.shape[0], 2))
    ytop = np.isclose(coord[bsido[:, 0] - 1, 1], 1.0) & np.isclose(coord[bsido[:, 1] - 1, 1], 1.0)
    wv[ytop, 0] = lid_speed
    return RawMesh(intma, coord, bsido, wv, {"kind": "cavity", "n": n, "lid_speed": lid_speed})


def channel_mesh(x0, x1, y0, y1, nx, ny, obstacle_side=1.0, center=(0.0, 0.0), sides="outflow"):
    """Channel [x0,x1]x[y0,y1] of nx x ny quads; quads whose centres lie in
    the square obstacle (side obstacle_side, snapped to whole cells) are
    removed.  Left: inflow (type 1); right: outflow (type 2); top and
    bottom: outflow (sides="outflow"), free stream (sides="freestream",
    type 1: the INFLOW reset holds them at the inflow Maxwellian) or diffuse
    walls (sides="wall", type 4); obstacle surface: diffuse wall (type 4).

    A zero-gradient side parallel to the stream neither damps nor fixes a
    transverse disturbance, so with outflow sides the steady state the march
    reaches depends on where it started; free-stream sides pin it."""
    if sides not in ("outflow", "freestream", "wall"):
        raise ValueError("sides: 'outflow', 'freestream' or 'wall'")
    hx = (x1 - x0) / nx
    hy = (y1 - y0) / ny
    xc = x0 + (np.arange(nx) + 0.5) * hx
    yc = y0 + (np.arange(ny) + 0.5) * hy
    half = 0.5 * obstacle_side + 1e-9
    inside = (np.abs(yc[:, None] - center[1]) < half) & (np.abs(xc[None, :] - center[0]) < half)
    active = ~inside

    def st(kind, outside, i, j):
        if not outside:
            return 4
        if kind in ("top", "bottom") and sides != "outflow":
            return 1 if sides == "freestream" else 4
        return 1 if kind == "left" else 2

    intma, coord, bsido = _grid_mesh(x0, x1, y0, y1, nx, ny, active, st)
    side = float(inside.any(axis=0).sum() * hx)
    return RawMesh(intma, coord, bsido, None,
                   {"kind": "channel", "nx": nx, "ny": ny, "obstacle_cells": int(inside.sum()),
                    "obstacle_side": side, "sides": sides})


def physical_params(mach, kn, length=1.0, rho=1.0, temp=1.0, rgas=1.0):
    """(Mach, Kn) -> reference inputs; see the module docstring."""
    M = 6.022e26  # M/NA = 1
    n = rho * 6.022e26 / M
    d = (math.sqrt(2.0) * PI_REF * n * kn * length) ** -0.5
    U = mach * math.sqrt(GAMMA * rgas * temp)
    p_bar = rho * rgas * temp / 1e5
    return {"rgas": rgas, "molar_mass": M, "diameter": d, "speed": U, "p_bar": p_bar, "temp": temp}


@dataclass
class CaseDef:
    """One benchmark workload: mesh, velocity grid, parameters, initial state."""
    name: str
    mesh: RawMesh
    rorder: int
    torder: int
    rv: float
    immat: int = 1
    csafm: float = 0.5
    alpha: float = 1.0
    rgas: float = 1.0
    molar_mass: float = 6.022e26
    diameter: float = 1.0
    cinf: tuple = (0.0, 0.0, 0.0, 0.0)
    init: dict = field(default_factory=dict)  # T1, P1, U0, V0, perturb, seed
    info: dict = field(default_factory=dict)

    @property
    def dofs(self):
        return 3 * self.mesh.nelem * self.rorder * self.torder


def cavity_case(n=32, nr=16, nt=32, mach=0.3, kn=0.1, perturb=1e-3, seed=0):
    """Lid-driven cavity: n x n quads, nr x nt velocities, lid Mach, Kn; rest
    Maxwellian (rho = 1, T = 1) times (1 + U(-perturb, perturb)) per DG node
    (numpy PCG64 seeded with `seed`)."""
    ph = physical_params(mach, kn)
    mesh = cavity_mesh(n, lid_speed=ph["speed"])
    rv = 4.0 * math.sqrt(ph["rgas"] * ph["temp"])
    return CaseDef(name=f"cavity{n}_v{nr}x{nt}", mesh=mesh, rorder=nr, torder=nt, rv=rv, rgas=ph["rgas"],
                   molar_mass=ph["molar_mass"], diameter=ph["diameter"], cinf=(0.0, 0.0, 0.0, 0.0),
                   init={"T1": 1.0, "P1": ph["p_bar"], "U0": 0.0, "V0": 0.0, "perturb": perturb, "seed": seed},
                   info={"mach": mach, "kn": kn, "lid_speed": ph["speed"]})


def channel_case(x0=-5.0, x1=15.0, y0=-5.0, y1=5.0, nx=200, ny=100, nr=24, nt=48, mach=2.0, kn=0.05,
                 obstacle_side=1.0, sides="outflow"):
    """Supersonic channel flow past a square obstacle; the domain starts at
    the free-stream Maxwellian (INICON2 with U0 = U).  `sides`: the top and
    bottom boundary type (channel_mesh)."""
    ph = physical_params(mach, kn, length=obstacle_side)
    mesh = channel_mesh(x0, x1, y0, y1, nx, ny, obstacle_side, sides=sides)
    rv = 4.0 * math.sqrt(ph["rgas"] * ph["temp"]) + ph["speed"]
    cinf = (ph["temp"], ph["p_bar"], ph["speed"], 0.0)
    return CaseDef(name=f"channel{nx}x{ny}_v{nr}x{nt}", mesh=mesh, rorder=nr, torder=nt, rv=rv, rgas=ph["rgas"],
                   molar_mass=ph["molar_mass"], diameter=ph["diameter"], cinf=cinf,
                   init={"T1": 1.0, "P1": ph["p_bar"], "U0": ph["speed"], "V0": 0.0, "perturb": 0.0, "seed": 0},
                   info={"mach": mach, "kn": kn, "obstacle_side": mesh.info["obstacle_side"]})


# The benchmark workloads: the 32 x 32 lid-driven cavity, the 200 x 100
# supersonic channel, the 400 x 200 large channel
def config1():
    return cavity_case(32, 16, 32, mach=0.3, kn=0.1)


def config2():
    return channel_case(-5.0, 15.0, -5.0, 5.0, 200, 100, 24, 48, mach=2.0, kn=0.05)


def config5():
    return channel_case(-10.0, 30.0, -10.0, 10.0, 400, 200, 32, 64, mach=1.5, kn=0.02)


def config3(ncases=64, seed=1, n_choices=tuple(range(16, 97, 8))):
    """The batched workload: `ncases` lid-driven cavities, each with its own
    draw (numpy PCG64, `seed`) of the mesh size N from `n_choices`, radial
    velocities from 8..24, angles from 16..64, lid Mach from U[0.1, 1] and
    Kn from logU[0.01, 1]; case k's density perturbation uses seed 1000 + k."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(ncases):
        n = int(rng.choice(n_choices))
        nr = int(rng.integers(8, 25))
        nt = int(rng.integers(16, 65))
        mach = float(rng.uniform(0.1, 1.0))
        kn = float(10.0 ** rng.uniform(-2.0, 0.0))
        out.append(cavity_case(n, nr, nt, mach=mach, kn=kn, seed=1000 + k))
    return out


def node_scale(case):
    """Per-DG-node density factor (3,NELEM) of the seeded perturbation, or
    None without one."""
    p = case.init.get("perturb", 0.0)
    if not p:
        return None
    rng = np.random.Generator(np.random.PCG64(case.init.get("seed", 0)))
    return 1.0 + rng.uniform(-p, p, size=(case.mesh.nelem, 3))

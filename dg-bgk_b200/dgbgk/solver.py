"""Python host side of the drop-in: the same steps DG_LIN_CONVEC takes around
ADVNCE (src/dg_lin_convec.f90:96-206) -- setup arrays, initial condition,
time loop, nodal output -- with every compute call going through the C ABI
of lib/libdgbgk.so.
"""
import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib, ptr


@dataclass
class Setup:
    """The reference's setup arrays (src/dg_lin_convec.f90:96-125)."""
    nside: int
    iside: np.ndarray  # (S,8) int32
    nx: np.ndarray
    ny: np.ndarray
    el: np.ndarray
    geome: np.ndarray  # (E,7)
    relen: np.ndarray
    mmat: np.ndarray   # (E,3)
    cmmat: np.ndarray  # (E,3,3) as CMMAT(3,3,E): [e, j, i]
    rsido: np.ndarray  # (B,3)


def setup_mesh(intma, coord, bsido):
    """GETSID, NORMAL, GETGEO, GETLEN, GETMAT/CONMAT, GETNOR on the host."""
    intma = np.ascontiguousarray(intma, dtype=np.int32)
    coord = np.ascontiguousarray(coord, dtype=np.float64)
    bsido = np.ascontiguousarray(bsido, dtype=np.int32)
    E, NP, B = intma.shape[0], coord.shape[0], bsido.shape[0]
    mx = 2 * (E + B)
    iside = np.zeros((mx, 8), dtype=np.int32)
    nx = np.zeros(mx)
    ny = np.zeros(mx)
    el = np.zeros(mx)
    geome = np.zeros((E, 7))
    relen = np.zeros(E)
    mmat = np.zeros((E, 3))
    cmmat = np.zeros((E, 3, 3))
    rsido = np.zeros((max(B, 1), 3))
    ns = c_int(0)
    check(lib().dgbgk_setup_mesh(E, NP, B, ptr(intma, c_int), ptr(coord), ptr(bsido, c_int), ctypes.byref(ns),
                                 ptr(iside, c_int), ptr(nx), ptr(ny), ptr(el), ptr(geome), ptr(relen), ptr(mmat),
                                 ptr(cmmat), ptr(rsido)))
    S = ns.value
    return Setup(S, iside[:S].copy(), nx[:S].copy(), ny[:S].copy(), el[:S].copy(), geome, relen, mmat, cmmat,
                 rsido[:B].copy())


def vspace(rorder, torder, eta, w):
    """VSPACE: VCORD(3,V) and SUMWEIGHT."""
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    vc = np.zeros((rorder * torder, 3))
    sw = c_double(0)
    check(lib().dgbgk_vspace_build(rorder, torder, ptr(eta), ptr(w), ptr(vc), ctypes.byref(sw)))
    return vc, sw.value


class Solver:
    """One case on one GPU.  Arrays use the reference layouts: DISNF is
    (NELEM, VNPNT, 3) C-order == DISNF(3,VNPNT,NELEM) column-major."""

    def __init__(self, intma, coord, bsido, setup, vcord, sumweight, rorder, torder, rv, *, immat=1, csafm=0.5,
                 alpha=1.0, rgas=1.0, molar_mass=6.022e26, diameter=1.0, cinf=(0, 0, 0, 0), precision=64,
                 wall_velocity=None, tile_elems=0, moment_rows=0, device=0, shard=0):
        L = lib()
        self._keep = []

        def keep(a, dt=np.float64):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        intma = keep(intma, np.int32)
        coord = keep(coord)
        bsido = keep(bsido, np.int32)
        self.E, self.NP, self.B = intma.shape[0], coord.shape[0], bsido.shape[0]
        self.V = rorder * torder
        m = _lib.Mesh()
        m.nelem, m.npoin, m.nboun, m.nside = self.E, self.NP, self.B, setup.nside
        m.intma = ptr(intma, c_int)
        m.coord = ptr(coord)
        m.bsido = ptr(bsido, c_int) if self.B else None
        m.iside = ptr(keep(setup.iside, np.int32), c_int)
        m.nx = ptr(keep(setup.nx))
        m.ny = ptr(keep(setup.ny))
        m.el = ptr(keep(setup.el))
        m.geome = ptr(keep(setup.geome))
        m.relen = ptr(keep(setup.relen))
        m.mmat = ptr(keep(setup.mmat))
        m.cmmat = ptr(keep(setup.cmmat))
        m.rsido = ptr(keep(setup.rsido)) if self.B else None
        vs = _lib.VSpace()
        vs.rorder, vs.torder = rorder, torder
        vs.vcord = ptr(keep(vcord))
        vs.sumweight = sumweight
        vs.rv = rv
        p = _lib.Params()
        L.dgbgk_default_params(ctypes.byref(p))
        p.immat, p.csafm, p.alpha, p.rgas = immat, csafm, alpha, rgas
        p.molar_mass, p.diameter = molar_mass, diameter
        for i in range(4):
            p.cinf[i] = cinf[i]
        p.precision = precision
        p.wall_velocity = ptr(keep(wall_velocity)) if wall_velocity is not None else None
        p.tile_elems = tile_elems
        p.moment_rows = moment_rows
        p.device = device
        p.shard = shard
        h = c_void_p()
        check(L.dgbgk_create(ctypes.byref(m), ctypes.byref(vs), ctypes.byref(p), ctypes.byref(h)))
        self.h = h
        self.precision = precision

    @classmethod
    def from_case(cls, case, precision=64, tile_elems=0, moment_rows=0, device=0):
        from .cases import gll
        m = case.mesh
        st = setup_mesh(m.intma, m.coord, m.bsido)
        eta, w = gll(case.rorder)
        vc, sw = vspace(case.rorder, case.torder, eta, w)
        s = cls(m.intma, m.coord, m.bsido, st, vc, sw, case.rorder, case.torder, case.rv, immat=case.immat,
                csafm=case.csafm, alpha=case.alpha, rgas=case.rgas, molar_mass=case.molar_mass,
                diameter=case.diameter, cinf=case.cinf, precision=precision, wall_velocity=m.wall_velocity,
                tile_elems=tile_elems, moment_rows=moment_rows, device=device)
        s.case = case
        s.setup = st
        s.vcord = vc
        s.sumweight = sw
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().dgbgk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state --------------------------------------------------------
    def set_state(self, disnf):
        if disnf.dtype == np.float32:
            a = np.ascontiguousarray(disnf)
            assert a.size == 3 * self.E * self.V
            check(lib().dgbgk_set_state_f32(self.h, ptr(a, c_float)))
        else:
            a = np.ascontiguousarray(disnf, dtype=np.float64)
            assert a.size == 3 * self.E * self.V
            check(lib().dgbgk_set_state(self.h, ptr(a)))

    def get_state(self, dtype=np.float64, out=None):
        """DISNF as (NELEM, VNPNT, 3); into `out` when given (a C-contiguous
        array of that shape and dtype, e.g. a pinned host buffer: the device
        copy lands in it directly)."""
        if out is None:
            out = np.empty((self.E, self.V, 3), dtype=dtype)
        else:
            dtype = out.dtype.type
            assert out.shape == (self.E, self.V, 3) and out.flags["C_CONTIGUOUS"]
        if dtype == np.float32:
            check(lib().dgbgk_get_state_f32(self.h, ptr(out, c_float)))
        else:
            check(lib().dgbgk_get_state(self.h, ptr(out)))
        return out

    def inicon2(self, T1, P1, U0, V0, node_scale=None):
        sc = None if node_scale is None else np.ascontiguousarray(node_scale, dtype=np.float64)
        check(lib().dgbgk_init_uniform(self.h, T1, P1, U0, V0, ptr(sc)))

    def init_case(self):
        from .cases import node_scale
        c = self.case
        i = c.init
        self.inicon2(i["T1"], i["P1"], i["U0"], i["V0"], node_scale(c))

    def init_maxwellian(self, n, u, v, t):
        a = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (n, u, v, t)]
        check(lib().dgbgk_init_maxwellian(self.h, *(ptr(x) for x in a)))

    # -- time loop ----------------------------------------------------
    def advance(self, nsteps, tol=0.0, raise_on_error=True):
        """Runs up to nsteps steps (to tol relative to the residual
        reference when tol > 0).  With raise_on_error=False a failed advance
        returns its status in "rc" (the steps run before it, and their
        residuals, are kept)."""
        linf = np.zeros(max(nsteps, 1))
        l2 = np.zeros(max(nsteps, 1))
        dte = np.zeros(max(nsteps, 1))
        done = c_int(0)
        rc = lib().dgbgk_advance(self.h, nsteps, tol, ctypes.byref(done), ptr(linf), ptr(l2), ptr(dte))
        n = done.value
        res = {"steps": n, "res_linf": linf[:n], "res_l2": l2[:n], "dte": dte[:n], "rc": rc}
        if raise_on_error:
            check(rc)
        return res

    def last_ms(self):
        t = c_double(0)
        check(lib().dgbgk_last_timing(self.h, ctypes.byref(t)))
        return t.value

    def profile(self, nsteps):
        """Mean device ms per step of [moments, wall, sweep, residual]."""
        ms = np.zeros(4)
        check(lib().dgbgk_profile_steps(self.h, nsteps, ptr(ms)))
        return ms

    def set_residual_reference(self, r):
        check(lib().dgbgk_set_residual_reference(self.h, r))

    def residual_reference(self):
        r = c_double(0)
        check(lib().dgbgk_get_residual_reference(self.h, ctypes.byref(r)))
        return r.value

    def snapshot(self, slot):
        """Copies the state into extrapolation slot `slot` (< 0: frees them)."""
        check(lib().dgbgk_snapshot(self.h, slot))

    def extrapolate(self, n):
        """Reduced-rank extrapolation from slots 0 .. n-1; returns gamma."""
        g = np.zeros(max(n - 1, 1))
        check(lib().dgbgk_extrapolate(self.h, n, ptr(g)))
        return g[:n - 1]

    def copy_state_from(self, other):
        """Takes `other`'s state (converted to this handle's precision on the
        device) and residual reference; same mesh and velocity grid."""
        check(lib().dgbgk_copy_state(self.h, other.h))

    # -- observables ----------------------------------------------------
    def macros(self):
        out = {k: np.zeros(self.NP) for k in ("nd", "rho", "u", "v", "ps", "temp")}
        check(lib().dgbgk_get_macros(self.h, *(ptr(out[k]) for k in ("nd", "rho", "u", "v", "ps", "temp"))))
        return out

    def forces(self):
        """GETFOR's (lift, drag) of the current state, reduced on the device."""
        lift, drag = c_double(0), c_double(0)
        check(lib().dgbgk_get_forces(self.h, ctypes.byref(lift), ctypes.byref(drag)))
        return lift.value, drag.value

    def set_output(self, every, capacity=16):
        """Record GETMAC's nodal fields and GETFOR's forces every `every`
        steps of advance() into a device ring (every = 0: stop)."""
        check(lib().dgbgk_set_output(self.h, every, capacity))
        self._out_cap = capacity if every > 0 else 0

    def outputs(self):
        """The records held by the ring, oldest first: dicts of itime, lift,
        drag and the six nodal fields."""
        n = c_int(0)
        check(lib().dgbgk_output_count(self.h, ctypes.byref(n)))
        out = []
        keys = ("nd", "rho", "u", "v", "ps", "temp")
        for k in range(min(n.value, getattr(self, "_out_cap", 0))):
            f = {key: np.zeros(self.NP) for key in keys}
            it, lift, drag = c_int(0), c_double(0), c_double(0)
            check(lib().dgbgk_get_output(self.h, k, ctypes.byref(it), *(ptr(f[key]) for key in keys),
                                         ctypes.byref(lift), ctypes.byref(drag)))
            f.update(itime=it.value, lift=lift.value, drag=drag.value)
            out.append(f)
        return out

    def node_fields(self):
        out = {k: np.zeros((self.E, 3)) for k in ("disnd", "disux", "disuy", "disps", "mu")}
        check(lib().dgbgk_get_node_fields(self.h, *(ptr(out[k]) for k in ("disnd", "disux", "disuy", "disps", "mu"))))
        return out

    def wall_eta(self):
        out = np.zeros(max(self.B, 1))
        check(lib().dgbgk_get_wall_eta(self.h, ptr(out)))
        return out[:self.B]

    def info(self):
        o = np.zeros(10, dtype=np.int32)
        check(lib().dgbgk_info(self.h, ptr(o, c_int)))
        keys = ["nelem", "npoin", "nboun", "nside", "vnpnt", "precision", "tile_elems", "tile_vels", "n_blocks",
                "max_halo"]
        return dict(zip(keys, (int(x) for x in o)))


class Batch:
    """Many Solver cases advanced together (dgbgk_batch_*): one persistent
    launch per kernel and step over all the cases, steps replayed from one
    CUDA graph, tile shape chosen by the library's autotuner.  The solvers
    must share precision, IMMAT and device; they stay usable on their own
    between batch calls."""

    TUNE_KEYS = [(eb, upc) for eb in (64, 128) for upc in (2, 4, 8, 16)] + [("rows", r) for r in (1, 2, 3, 4)]

    def __init__(self, solvers, tile_elems=0, units_per_cta=0, tune_steps=4, moment_rows=0):
        from ._lib import BatchParams
        self.solvers = list(solvers)
        p = BatchParams()
        lib().dgbgk_batch_default_params(ctypes.byref(p))
        p.tile_elems = tile_elems
        p.units_per_cta = units_per_cta
        p.tune_steps = tune_steps
        p.moment_rows = moment_rows
        hs = (c_void_p * len(self.solvers))(*[s.h for s in self.solvers])
        b = c_void_p()
        check(lib().dgbgk_batch_create(hs, len(self.solvers), ctypes.byref(p), ctypes.byref(b)))
        self.h = b
        # the autotuner's choice, kept for the record
        self.shape = self.info()

    def advance(self, max_steps, tol=0.0, raise_on_error=True):
        """Steps every case to tol (relative to its reference) or max_steps.
        With raise_on_error=False a case that diverges only stops: its
        status (0, or the error code) is in the result."""
        n = len(self.solvers)
        steps = np.zeros(n, dtype=np.int32)
        l2 = np.zeros(n)
        rc = lib().dgbgk_batch_advance(self.h, max_steps, tol, ptr(steps, c_int), ptr(l2))
        status = np.zeros(n, dtype=np.int32)
        check(lib().dgbgk_batch_status(self.h, ptr(status, c_int)))
        diverged_only = bool(np.isin(status, (0, _lib.DGBGK_ENONFINITE)).all() and (status != 0).any())
        if rc != 0 and (raise_on_error or not diverged_only):
            check(rc)
        return {"steps": steps, "res_l2_last": l2, "status": status}

    def set_active(self, active):
        """Leaves the cases with active[i] false out of the following
        advances (0 steps, state untouched)."""
        a = np.ascontiguousarray(np.asarray(active, dtype=bool).astype(np.int32))
        assert a.size == len(self.solvers)
        check(lib().dgbgk_batch_set_active(self.h, ptr(a, c_int)))

    def _mask(self, which):
        if which is None:
            return None
        a = np.ascontiguousarray(np.asarray(which, dtype=bool).astype(np.int32))
        assert a.size == len(self.solvers)
        return a

    def snapshot(self, slot, which=None):
        """Solver.snapshot(slot) of the cases with which[i] true (None: all),
        queued on the batch's stream without a wait."""
        a = self._mask(which)
        check(lib().dgbgk_batch_snapshot(self.h, slot, None if a is None else ptr(a, c_int)))

    def extrapolate(self, n, which=None):
        """Solver.extrapolate(n) of the cases with which[i] true (None: all),
        their Gram matrices formed before one wait.  Returns (status, gamma):
        per case 0 or the error code Solver.extrapolate would raise (the
        case then keeps its state), and its n-1 coefficients (zeros where
        not extrapolated)."""
        a = self._mask(which)
        k = len(self.solvers)
        status = np.zeros(k, dtype=np.int32)
        gamma = np.zeros((k, max(n - 1, 1)))
        rc = lib().dgbgk_batch_extrapolate(self.h, n, None if a is None else ptr(a, c_int), ptr(status, c_int),
                                           ptr(gamma))
        if rc not in (0, _lib.DGBGK_EINVAL, _lib.DGBGK_ENONFINITE):
            check(rc)  # not a case's own result (a CUDA error)
        return status, gamma[:, :n - 1]

    def shape_record(self):
        """The tile shape in use: elements per CTA, units per CTA and moment
        rows per warp step."""
        return {k: self.shape[k] for k in ("tile_elems", "units_per_cta", "moment_rows")}

    def info(self):
        o = np.zeros(7, dtype=np.int32)
        check(lib().dgbgk_batch_info(self.h, ptr(o, c_int)))
        return dict(zip(["ncases", "tile_elems", "units_per_cta", "sweep_units", "sweep_ctas", "moment_ctas",
                         "moment_rows"], (int(x) for x in o)))

    def tuning(self):
        ms = np.zeros(12)
        check(lib().dgbgk_batch_tuning(self.h, 12, ptr(ms)))
        return {k: float(v) for k, v in zip(self.TUNE_KEYS, ms) if v > 0}

    def last_ms(self):
        t = c_double(0)
        check(lib().dgbgk_batch_last_timing(self.h, ctypes.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "h", None):
            lib().dgbgk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

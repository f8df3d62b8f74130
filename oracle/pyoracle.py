"""ctypes wrapper of the parity oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.  See the header of
oracle/dgbgk_oracle.cpp for what it restates and its parity status.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_create.restype = c_void_p
        L.orc_create.argtypes = [c_int, c_int, c_int, c_int, POINTER(c_int), POINTER(c_double), POINTER(c_int), c_int,
                                 c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double), c_int, c_int,
                                 POINTER(c_double)]
        L.orc_destroy.argtypes = [c_void_p]
        L.orc_set_threads.argtypes = [c_void_p, c_int]
        L.orc_sizes.argtypes = [c_void_p, POINTER(c_int)]
        L.orc_get.argtypes = [c_void_p, c_char_p, POINTER(c_double)]
        L.orc_get.restype = c_int
        L.orc_set_state.argtypes = [c_void_p, POINTER(c_double)]
        L.orc_get_state.argtypes = [c_void_p, POINTER(c_double)]
        L.orc_inicon2.argtypes = [c_void_p, c_double, c_double, c_double, c_double]
        L.orc_advance.argtypes = [c_void_p, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double)]
        L.orc_advance.restype = c_int
        L.orc_macros.argtypes = [c_void_p] + [POINTER(c_double)] * 6
        L.orc_compmu.argtypes = [c_void_p]
        L.orc_last_error.restype = c_char_p
        _L = L
    return _L


def _p(a, t=c_double):
    return None if a is None else a.ctypes.data_as(POINTER(t))


class Oracle:
    """The reference algorithm on the CPU, in float (prec=32) or double (64)."""

    def __init__(self, intma, coord, bsido, rorder, torder, eta, w, *, rv, csafm=0.5, alpha=1.0, rgas=1.0,
                 molar_mass=6.022e26, diameter=1.0, cinf=(0, 0, 0, 0), immat=1, prec=64, ring_fix=False,
                 wall_velocity=None, threads=1):
        L = _lib()
        self._a = [np.ascontiguousarray(intma, dtype=np.int32), np.ascontiguousarray(coord, dtype=np.float64),
                   np.ascontiguousarray(bsido, dtype=np.int32), np.ascontiguousarray(eta, dtype=np.float64),
                   np.ascontiguousarray(w, dtype=np.float64)]
        intma, coord, bsido, eta, w = self._a
        scal = np.array([rv, csafm, alpha, rgas, molar_mass, diameter, *cinf], dtype=np.float64)
        wv = None if wall_velocity is None else np.ascontiguousarray(wall_velocity, dtype=np.float64)
        self._a += [scal, wv]
        self.h = L.orc_create(prec, intma.shape[0], coord.shape[0], bsido.shape[0], _p(intma, c_int), _p(coord),
                              _p(bsido, c_int), rorder, torder, _p(eta), _p(w), _p(scal), immat, 1 if ring_fix else 0,
                              _p(wv))
        if not self.h:
            raise RuntimeError("oracle: " + L.orc_last_error().decode())
        sz = np.zeros(6, dtype=np.int32)
        L.orc_sizes(self.h, _p(sz, c_int))
        self.E, self.NP, self.B, self.S, self.V, self.MXSID = (int(x) for x in sz)
        L.orc_set_threads(self.h, threads)

    @classmethod
    def from_case(cls, case, prec=64, threads=1, **kw):
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(HERE), "dg-bgk_b200"))
        from dgbgk.cases import gll
        eta, w = gll(case.rorder)
        m = case.mesh
        return cls(m.intma, m.coord, m.bsido, case.rorder, case.torder, eta, w, rv=case.rv, csafm=case.csafm,
                   alpha=case.alpha, rgas=case.rgas, molar_mass=case.molar_mass, diameter=case.diameter,
                   cinf=case.cinf, immat=case.immat, prec=prec, wall_velocity=m.wall_velocity, threads=threads, **kw)

    def close(self):
        if self.h:
            _lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n):
        _lib().orc_set_threads(self.h, n)

    def get(self, name):
        sizes = {"ISIDE": 8 * self.S, "NX": self.S, "NY": self.S, "EL": self.S, "GEOME": 7 * self.E,
                 "RELEN": self.E, "MMAT": 3 * self.E, "CMMAT": 9 * self.E, "RSIDO": 3 * self.B, "VCORD": 3 * self.V,
                 "SUMWEIGHT": 1, "DTEC": 1, "DTE": 1, "DISND": 3 * self.E, "DISUX": 3 * self.E, "DISUY": 3 * self.E,
                 "DISPS": 3 * self.E, "MU": 3 * self.E, "ETA": self.B}
        out = np.zeros(max(sizes[name], 1))
        rc = _lib().orc_get(self.h, name.encode(), _p(out))
        assert rc == 0
        return out[:sizes[name]]

    def set_state(self, disnf):
        a = np.ascontiguousarray(disnf, dtype=np.float64)
        assert a.size == 3 * self.V * self.E
        _lib().orc_set_state(self.h, _p(a))

    def get_state(self):
        out = np.empty((self.E, self.V, 3))
        _lib().orc_get_state(self.h, _p(out))
        return out

    def inicon2(self, T1, P1, U0, V0):
        _lib().orc_inicon2(self.h, T1, P1, U0, V0)

    def advance(self, n):
        a, b, c = np.zeros(n), np.zeros(n), np.zeros(n)
        rc = _lib().orc_advance(self.h, n, _p(a), _p(b), _p(c))
        if rc != 0:
            raise RuntimeError("oracle: " + _lib().orc_last_error().decode())
        return {"res_linf": a, "res_l2": b, "dte": c}

    def macros(self):
        out = {k: np.zeros(self.NP) for k in ("nd", "rho", "u", "v", "ps", "temp")}
        _lib().orc_macros(self.h, *(_p(out[k]) for k in ("nd", "rho", "u", "v", "ps", "temp")))
        return out

    def compmu(self):
        _lib().orc_compmu(self.h)
        return {k: self.get(k) for k in ("DISND", "DISUX", "DISUY", "DISPS", "MU", "ETA", "DTE")}

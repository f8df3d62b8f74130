"""dgbgk_get_macros_noalloc against dgbgk_get_macros, through the C ABI (GPU).

The no-allocation entry point serves callers that cannot allocate device
memory at call time (their GPU memory belongs to another allocator or pool,
or their time loop must not pay cudaMalloc/cudaFree's device-wide
synchronisation).  It stages the nodal fields in the library's static device
array instead of a per-call cudaMalloc, so its results must equal those of
the allocating entry point; meshes with more than DGBGK_NOALLOC_MAX_NPOIN
nodes are refused.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from dgbgk import Solver, cavity_case
from dgbgk._lib import DGBGK_EINVAL, check, lib, ptr

pytestmark = pytest.mark.gpu

KEYS = ("nd", "rho", "u", "v", "ps", "temp")
MAX_NPOIN = 131072  # DGBGK_NOALLOC_MAX_NPOIN in include/dgbgk.h


def noalloc_macros(s):
    out = {k: np.zeros(s.NP) for k in KEYS}
    rc = lib().dgbgk_get_macros_noalloc(s.h, *(ptr(out[k]) for k in KEYS))
    check(rc)
    return out


def test_noalloc_macros_match_allocating_entry_point_twice():
    s = Solver.from_case(cavity_case(8, 8, 16, mach=0.3, kn=0.1))
    s.init_case()
    s.advance(3)
    # both entry points run the same moment and nodal-gather kernels on the
    # same state, so their fields agree bit for bit (a stale or half-written
    # scratch array would show here)
    for call in range(2):  # two calls in a row share the static array
        a = noalloc_macros(s)
        b = s.macros()
        for k in KEYS:
            assert np.array_equal(a[k], b[k]), (call, k)
    s.advance(2)
    a = noalloc_macros(s)
    b = s.macros()
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_noalloc_rejects_meshes_above_the_limit():
    case = cavity_case(363, 2, 4, mach=0.3, kn=0.1)  # 364^2 = 132496 nodes
    assert case.mesh.npoin > MAX_NPOIN
    s = Solver.from_case(case)
    s.init_case()
    out = [np.zeros(s.NP) for _ in KEYS]
    rc = lib().dgbgk_get_macros_noalloc(s.h, *(ptr(x) for x in out))
    assert rc == DGBGK_EINVAL
    assert b"DGBGK_NOALLOC_MAX_NPOIN" in lib().dgbgk_last_error()

"""The C-ABI library loads and exports every entry point include/dgbgk.h
declares; without a GPU it refuses to run instead of falling back (CPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared():
    src = open(os.path.join(ROOT, "include", "dgbgk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dgbgk_\w+)\s*\(", src)))


def test_header_declares_the_abi():
    names = declared()
    for n in ("dgbgk_create", "dgbgk_advance", "dgbgk_set_state", "dgbgk_get_state", "dgbgk_get_macros",
              "dgbgk_destroy", "dgbgk_last_error", "dgbgk_setup_mesh"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from dgbgk import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(declared()) <= set(_lib.SIGNATURES)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_create_without_gpu_fails_loudly():
    from dgbgk import cavity_case, Solver
    from dgbgk._lib import DgbgkError, DGBGK_ECUDA
    with pytest.raises(DgbgkError) as ei:
        Solver.from_case(cavity_case(4, 4, 8))
    assert ei.value.code == DGBGK_ECUDA
    assert "no CPU fallback" in str(ei.value) or "CUDA" in str(ei.value)


def test_another_build_of_the_abi_can_be_chosen_before_loading():
    # `python -m dgbgk.profile --lib ...` times another build of the
    # library (e.g. one compiled with other flags); the choice is refused
    # once a library is loaded
    import subprocess
    import sys
    code = ("import dgbgk._lib as L, os; L.use_library('variant.so'); print(L.LIB_PATH); "
            "L.use_library(os.path.join(os.path.dirname(L.__file__), '..', 'lib', 'libdgbgk.so')); L.lib()\n"
            "try:\n    L.use_library('other.so')\nexcept RuntimeError as e:\n    print('refused')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT,
                       env=dict(os.environ, PYTHONPATH=os.path.join(ROOT, "dg-bgk_b200")))
    assert r.returncode == 0, r.stderr
    out = r.stdout.split()
    assert out[0] == os.path.join(ROOT, "variant.so") and out[1] == "refused"


def test_batch_extrapolation_calls_refuse_a_null_batch():
    # argument checks before any device work (no GPU needed)
    from dgbgk._lib import lib, DGBGK_EINVAL
    L = lib()
    assert L.dgbgk_batch_snapshot(None, 0, None) == DGBGK_EINVAL
    st = (ctypes.c_int * 2)()
    assert L.dgbgk_batch_extrapolate(None, 5, None, st, None) == DGBGK_EINVAL
    assert b"NULL" in L.dgbgk_last_error()


def declared_arity():
    """Parameter count of every dgbgk_* function the header declares."""
    src = open(os.path.join(ROOT, "include", "dgbgk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(dgbgk_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        args = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_python_binding_takes_the_header_arguments():
    # the ctypes argument lists match the C declarations one for one
    from dgbgk import _lib
    ar = declared_arity()
    assert set(ar) == set(declared())
    wrong = {n: (k, len(_lib.SIGNATURES[n][1])) for n, k in ar.items() if len(_lib.SIGNATURES[n][1]) != k}
    assert not wrong, wrong

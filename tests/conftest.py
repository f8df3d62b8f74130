import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dg-bgk_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; runs the CUDA path")


def _make(d, target):
    if not os.path.exists(target):
        subprocess.run(["make", "-s", "-C", d], check=True)


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    _make(ORACLE, os.path.join(ORACLE, "_build", "liboracle.so"))
    _make(PKG, os.path.join(PKG, "lib", "libdgbgk.so"))
    _make(PKG, os.path.join(PKG, "bin", "dgbgk_run"))
    yield

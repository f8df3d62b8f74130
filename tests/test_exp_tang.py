"""The FP64 sweep's exp (Tang's table-driven method, csrc/exp_tang.h) against
long-double exp on the host: the same header compiled by g++ with the
table filled from exp2l."""
import os
import subprocess
import tempfile

import pytest

from conftest import PKG

PROG = r"""
#include <cmath>
#include <cstdio>
#include <random>
#include "exp_tang.h"
int main() {
  double tab[dgbgk::EXP_TAB];
  for (int j = 0; j < dgbgk::EXP_TAB; ++j) tab[j] = (double)exp2l((long double)j / dgbgk::EXP_TAB);
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> wide(-706.9, 700.0), near(-1.0, 0.0), small(-1e-6, 1e-6);
  double worst = 0.0, worst_x = 0.0;
  auto check = [&](double x) {
    const long double ref = expl((long double)x);
    const double got = dgbgk::exp_tang(x, tab);
    const double rel = (double)fabsl(((long double)got - ref) / ref);
    if (rel > worst) { worst = rel; worst_x = x; }
  };
  for (int i = 0; i < 2000000; ++i) { check(wide(g)); check(near(g)); check(small(g)); }
  // every table boundary and half-way point over [-706, 0]
  const double step = 0.6931471805599453 / 64;
  for (int k = -65200; k <= 0; ++k) { check(k * step); check((k + 0.5) * step); }
  check(0.0); check(-0.0); check(-706.99);
  const double flushed = dgbgk::exp_tang(-707.5, tab), nan_in = dgbgk::exp_tang(NAN, tab);
  const double neg_inf = dgbgk::exp_tang(-INFINITY, tab);
  printf("%.3e %.17g %d %d %d\n", worst, worst_x, flushed == 0.0, nan_in != nan_in, neg_inf == 0.0);
  return 0;
}
"""


def test_exp_tang_accuracy():
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        exe = os.path.join(d, "t")
        open(src, "w").write(PROG)
        r = subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(PKG, "csrc"), src,
                            "-o", exe], capture_output=True, text=True)
        if r.returncode != 0:
            pytest.fail("g++ failed:\n" + r.stderr)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=120).stdout.split()
    worst, worst_x = float(out[0]), float(out[1])
    # about one unit in the last place (2^-52 = 2.2e-16)
    assert worst < 3.5e-16, (worst, worst_x)
    assert out[2:] == ["1", "1", "1"]

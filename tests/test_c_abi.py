"""include/dgbgk.h as a C99 header (gcc -std=c99 -pedantic -Werror), linked
from C against lib/libdgbgk.so: the host setup entry points run from C and,
without a GPU, dgbgk_create returns DGBGK_ECUDA with a message (CPU)."""
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT

PROG = r"""
#include <stdio.h>
#include <string.h>
#include "dgbgk.h"

int main(void) {
  /* the unit square as two P1 triangles, four diffuse walls (type 4) */
  const int intma[6] = {1, 2, 3, 1, 3, 4};
  const double coord[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 1.0, 0.0, 1.0};
  const int bsido[24] = {1, 2, 1, 4, 1, 10, 2, 3, 1, 4, 1, 10, 3, 4, 2, 4, 1, 10, 4, 1, 2, 4, 1, 10};
  int nside = 0, iside[8 * 12];
  double nx[12], ny[12], el[12], geome[14], relen[2], mmat[6], cmmat[18], rsido[12];
  int rc = dgbgk_setup_mesh(2, 4, 4, intma, coord, bsido, &nside, iside, nx, ny, el, geome, relen, mmat, cmmat,
                            rsido);
  if (rc != DGBGK_OK) { printf("setup %d %s\n", rc, dgbgk_last_error()); return 1; }
  /* velocity space: 2 radial Lobatto points x 4 angles */
  const double eta[2] = {-1.0, 1.0}, w[2] = {1.0, 1.0};
  double vcord[3 * 8], sumweight = 0.0;
  rc = dgbgk_vspace_build(2, 4, eta, w, vcord, &sumweight);
  if (rc != DGBGK_OK) { printf("vspace %d %s\n", rc, dgbgk_last_error()); return 1; }
  dgbgk_mesh m;
  memset(&m, 0, sizeof m);
  m.nelem = 2; m.npoin = 4; m.nboun = 4; m.nside = nside;
  m.intma = intma; m.coord = coord; m.bsido = bsido; m.iside = iside; m.nx = nx; m.ny = ny; m.el = el;
  m.geome = geome; m.relen = relen; m.mmat = mmat; m.cmmat = cmmat; m.rsido = rsido;
  dgbgk_vspace vs;
  vs.rorder = 2; vs.torder = 4; vs.vcord = vcord; vs.sumweight = sumweight; vs.rv = 4.0;
  dgbgk_params p;
  dgbgk_default_params(&p);
  p.rgas = 1.0; p.molar_mass = 6.022e26; p.diameter = 1e-10;
  dgbgk_handle* h = NULL;
  rc = dgbgk_create(&m, &vs, &p, &h);
  printf("%d %d %.6f %d %s\n", nside, rc, geome[6], h == NULL, rc ? dgbgk_last_error() : "");
  if (h) dgbgk_destroy(h);
  return 0;
}
"""


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU path of dgbgk_create")
def test_header_is_c99_and_host_setup_runs_from_c():
    from dgbgk._lib import DGBGK_ECUDA, LIB_PATH
    gcc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    libdir = os.path.dirname(LIB_PATH)
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(src, "w").write(PROG)
        r = subprocess.run([gcc, "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-I",
                            os.path.join(ROOT, "include"), src, "-o", exe, "-L", libdir, "-ldgbgk",
                            f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    f = out.stdout.split(maxsplit=4)
    # 5 sides (4 boundary + the diagonal); twice the area of each triangle
    assert int(f[0]) == 5 and float(f[2]) == pytest.approx(1.0)
    assert int(f[1]) == DGBGK_ECUDA and f[3] == "1" and len(f) == 5 and f[4].strip()

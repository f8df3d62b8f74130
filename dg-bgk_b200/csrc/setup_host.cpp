// Host-side setup of the geometric arrays that the reference computes once
// before the time loop (src/dg_lin_convec.f90:96-125) and of the velocity
// grid (src/vspace.f90).  The side table keeps the reference's side order and
// local-node conventions exactly, so a Fortran host and this library agree on
// every array.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dgbgk.h"

namespace dgbgk {
void set_error(const std::string& m);
}

extern "C" void dgbgk_default_params(dgbgk_params* p) {
  // src/spectralbgk.f90:116-147
  std::memset(p, 0, sizeof(*p));
  p->immat = 1;
  p->csafm = 0.5;
  p->alpha = 0.9;
  p->rgas = 287;
  p->molar_mass = 32;
  p->diameter = 250e-12;
  p->cinf[0] = 294;
  p->cinf[1] = 0.001473;
  p->cinf[2] = 171.85;
  p->cinf[3] = 0.0;
  p->precision = 64;
  p->wall_velocity = nullptr;
  p->tile_elems = 0;
  p->moment_rows = 0;
  p->shard = 0;
  p->device = 0;
}

// VSPACE: eta-major, zeta-minor; zeta_i = -1 + i*2/TORDER, weight 1
// (src/vspace.f90:27-49).
extern "C" int dgbgk_vspace_build(int rorder, int torder, const double* eta, const double* w,
                                  double* vcord, double* sumweight) {
  if (rorder < 1 || torder < 1 || !eta || !w || !vcord || !sumweight) {
    dgbgk::set_error("dgbgk_vspace_build: bad arguments");
    return DGBGK_EINVAL;
  }
  const double gap = 2.0 / (double)torder;
  double s = 0.0;
  size_t k = 0;
  for (int r = 0; r < rorder; ++r)
    for (int t = 1; t <= torder; ++t) {
      vcord[3 * k + 0] = eta[r];
      vcord[3 * k + 1] = -1.0 + (double)t * gap;
      vcord[3 * k + 2] = w[r] * 1.0;
      s += vcord[3 * k + 2];
      ++k;
    }
  *sumweight = s;
  return DGBGK_OK;
}

namespace {

struct SideRec {
  int a, b;     // ISIDE(1), ISIDE(2)
  int left, right;
};

// The reference side table (src/getsid.f90:1-216): sides are created while
// scanning points in ascending order; a side (P, Q) with Q > P is created by
// the first element around P (ascending element order) that contains it.
// The element in which Q follows P in local order goes to ISIDE(3), the
// other to ISIDE(4); sides with only an ISIDE(4) element are boundary sides
// and are flipped so that ISIDE(4) = 0.
int build_sides(int nelem, int npoin, const int* intma, std::vector<SideRec>& sides) {
  std::vector<std::vector<int>> around(npoin + 1);
  for (int e = 1; e <= nelem; ++e)
    for (int k = 0; k < 3; ++k) {
      int p = intma[3 * (e - 1) + k];
      if (p < 1 || p > npoin) return -1;
      around[p].push_back(e);
    }
  sides.clear();
  std::vector<int> mine;  // indices of sides created for the current point
  for (int P = 1; P <= npoin; ++P) {
    if (around[P].empty()) continue;
    mine.clear();
    for (int e : around[P]) {
      const int* n = &intma[3 * (e - 1)];
      int k = (n[0] == P) ? 0 : (n[1] == P) ? 1 : 2;
      for (int J = 1; J <= 2; ++J) {
        int Q = n[(k + J) % 3];
        if (Q < P) continue;
        int found = -1;
        for (int s : mine)
          if (sides[s].b == Q) {
            found = s;
            break;
          }
        if (found < 0) {
          sides.push_back(SideRec{P, Q, 0, 0});
          found = (int)sides.size() - 1;
          mine.push_back(found);
        }
        if (J == 1)
          sides[found].left = e;
        else
          sides[found].right = e;
      }
    }
    for (int s : mine)
      if (sides[s].left == 0) {
        sides[s].left = sides[s].right;
        sides[s].right = 0;
        std::swap(sides[s].a, sides[s].b);
      }
  }
  return 0;
}

inline int local_of(const int* intma, int e, int p) {
  for (int k = 0; k < 3; ++k)
    if (intma[3 * (e - 1) + k] == p) return k + 1;
  return -2;
}

}  // namespace

extern "C" int dgbgk_setup_mesh(int nelem, int npoin, int nboun, const int* intma,
                                const double* coord, const int* bsido, int* nside, int* iside,
                                double* nx, double* ny, double* el, double* geome, double* relen,
                                double* mmat, double* cmmat, double* rsido) {
  if (nelem < 1 || npoin < 3 || nboun < 0 || !intma || !coord || (nboun && !bsido) || !nside ||
      !iside || !nx || !ny || !el || !geome || !relen || !mmat || !cmmat || (nboun && !rsido)) {
    dgbgk::set_error("dgbgk_setup_mesh: bad arguments");
    return DGBGK_EINVAL;
  }
  std::vector<SideRec> sides;
  if (build_sides(nelem, npoin, intma, sides) != 0) {
    dgbgk::set_error("dgbgk_setup_mesh: INTMA references a node outside 1..NPOIN");
    return DGBGK_EMESH;
  }
  const int mxsid = 2 * (nelem + nboun);
  if ((int)sides.size() > mxsid) {
    dgbgk::set_error("dgbgk_setup_mesh: more sides than MXSID = 2*(NELEM+NBOUN)");
    return DGBGK_EMESH;
  }
  *nside = (int)sides.size();
  for (size_t s = 0; s < sides.size(); ++s) {
    const SideRec& r = sides[s];
    int* I = &iside[8 * s];
    I[0] = r.a;
    I[1] = r.b;
    I[2] = r.left;
    I[3] = r.right;
    int il = local_of(intma, r.left, r.a);
    I[4] = il;
    I[5] = (il == 3) ? 1 : il + 1;
    if (r.right == 0) {
      I[6] = 0;
      I[7] = 0;
    } else {
      int ir = local_of(intma, r.right, r.b);
      if (ir < 0) ir = il;
      I[6] = (ir == 3) ? 1 : ir + 1;
      I[7] = ir;
    }
    // NORMAL (src/normal.f90:24-33)
    double dx = coord[2 * (r.b - 1)] - coord[2 * (r.a - 1)];
    double dy = coord[2 * (r.b - 1) + 1] - coord[2 * (r.a - 1) + 1];
    double L = std::sqrt((dx * dx) + (dy * dy));
    if (!(L > 0.0) || !std::isfinite(L)) {  // the reference would divide by zero here
      dgbgk::set_error("dgbgk_setup_mesh: side between nodes " + std::to_string(r.a) + " and " +
                       std::to_string(r.b) + " has zero or non-finite length");
      return DGBGK_EMESH;
    }
    el[s] = L;
    nx[s] = dy / L;
    ny[s] = -dx / L;
  }
  // GETGEO (src/getgeo.f90:22-59), GETLEN, GETMAT / CONMAT
  static const double NXI[3] = {-1.0, 1.0, 0.0}, NET[3] = {-1.0, 0.0, 1.0};
  for (int e = 0; e < nelem; ++e) {
    double X[3], Y[3];
    for (int k = 0; k < 3; ++k) {
      int p = intma[3 * e + k];
      X[k] = coord[2 * (p - 1)];
      Y[k] = coord[2 * (p - 1) + 1];
    }
    double x21 = X[1] - X[0], x31 = X[2] - X[0], y21 = Y[1] - Y[0], y31 = Y[2] - Y[0];
    double rj = x21 * y31 - x31 * y21;
    if (!(rj != 0.0) || !std::isfinite(rj)) {
      dgbgk::set_error("dgbgk_setup_mesh: element " + std::to_string(e + 1) + " has zero or non-finite area");
      return DGBGK_EMESH;
    }
    double rj1 = 1. / rj;
    double xix = y31 * rj1, xiy = -x31 * rj1, etx = -y21 * rj1, ety = x21 * rj1;
    double* G = &geome[7 * e];
    for (int k = 0; k < 3; ++k) {
      G[k] = xix * NXI[k] + etx * NET[k];
      G[k + 3] = xiy * NXI[k] + ety * NET[k];
    }
    G[6] = rj;
    double dmin = 0;
    for (int k = 0; k < 3; ++k) {
      double d = 1.0 / std::sqrt(G[k] * G[k] + G[k + 3] * G[k + 3]);
      dmin = (k == 0) ? d : std::fmin(dmin, d);
    }
    relen[e] = dmin;
    double rj24 = rj * (1. / 24.);
    for (int k = 0; k < 3; ++k) mmat[3 * e + k] = 1. / (0.0 + 4.0 * rj24);
    double r1 = 1 / rj24, r11 = 0.75 * r1, r12 = -0.25 * r1;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) cmmat[9 * e + i + 3 * j] = (i == j) ? r11 : r12;
  }
  // GETNOR (src/getnor.f90:21-31): RSIDO(3) is the side length
  for (int b = 0; b < nboun; ++b) {
    int p0 = bsido[6 * b], p1 = bsido[6 * b + 1];
    if (p0 < 1 || p0 > npoin || p1 < 1 || p1 > npoin) {
      dgbgk::set_error("dgbgk_setup_mesh: BSIDO references a node outside 1..NPOIN");
      return DGBGK_EMESH;
    }
    double dx = coord[2 * (p1 - 1)] - coord[2 * (p0 - 1)];
    double dy = coord[2 * (p1 - 1) + 1] - coord[2 * (p0 - 1) + 1];
    double rl = std::sqrt(dx * dx + dy * dy);
    if (!(rl > 0.0)) {
      dgbgk::set_error("dgbgk_setup_mesh: boundary side " + std::to_string(b + 1) + " has zero length");
      return DGBGK_EMESH;
    }
    double rt = 1.0 / rl;
    rsido[3 * b] = dy * rt;
    rsido[3 * b + 1] = -dx * rt;
    rsido[3 * b + 2] = rl;
  }
  return DGBGK_OK;
}

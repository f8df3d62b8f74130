// Plan builder: turns the reference's setup arrays into the element-centric,
// locality-ordered tables of the sm_100a kernels.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <numeric>
#include <set>
#include <unordered_map>

namespace dgbgk {

static const double PI_REF = 3.1416;  // the reference's PI (src/advnce.f90:94)

// Position along a Hilbert curve of order 16 (the rotate-and-flip
// construction), used to order elements so that a block of consecutive
// elements is spatially compact.
static uint64_t hilbert16(uint32_t x, uint32_t y) {
  uint64_t d = 0;
  const uint32_t n = 1u << 16;
  for (uint32_t s = n / 2; s > 0; s /= 2) {
    uint32_t rx = (x & s) ? 1 : 0, ry = (y & s) ? 1 : 0;
    d += (uint64_t)s * (uint64_t)s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      std::swap(x, y);
    }
  }
  return d;
}

void build_blocks(Plan& pl, int EB) {
  const int E = pl.E;
  pl.EB = EB;
  pl.nblocks = (E + EB - 1) / EB;
  pl.halo_off.assign(pl.nblocks + 1, 0);
  pl.halo_list.clear();
  pl.eslot.assign(3 * (size_t)E, -1);
  pl.max_halo = 0;
  for (int b = 0; b < pl.nblocks; ++b) {
    const int e0 = b * EB, e1 = std::min(E, e0 + EB);
    std::vector<int> halo;
    for (int e = e0; e < e1; ++e)
      for (int k = 0; k < 3; ++k) {
        int n = pl.edge[3 * (size_t)e + k].nbr;
        if (n >= 0 && (n < e0 || n >= e1)) halo.push_back(n);
      }
    std::sort(halo.begin(), halo.end());
    halo.erase(std::unique(halo.begin(), halo.end()), halo.end());
    for (int e = e0; e < e1; ++e)
      for (int k = 0; k < 3; ++k) {
        int n = pl.edge[3 * (size_t)e + k].nbr;
        if (n < 0) continue;
        if (n >= e0 && n < e1)
          pl.eslot[3 * (size_t)e + k] = n - e0;
        else
          pl.eslot[3 * (size_t)e + k] =
              EB + (int)(std::lower_bound(halo.begin(), halo.end(), n) - halo.begin());
      }
    pl.halo_off[b + 1] = pl.halo_off[b] + (int)halo.size();
    pl.halo_list.insert(pl.halo_list.end(), halo.begin(), halo.end());
    pl.max_halo = std::max(pl.max_halo, (int)halo.size());
  }
}

// GETBOU's mirrored-velocity lookup (src/getbou.f90:198-242) for every wall
// side and outgoing velocity, in FP64 as the oracle evaluates it, and the
// item lists of the specular update (see Plan::spec).  The ring of the
// mirrored speed is found by the reference's own formula: it compares ETAref
// with VCORD(1, 1 + (IETA-1)*(RORDER-1)) and takes the angles of ring
// IETA-1, which selects the right ring when RORDER = TORDER; other grids
// follow the same formula and fail here where it leaves VCORD.
static int build_specular(const dgbgk_mesh& m, const dgbgk_vspace& vs, Plan& pl, std::string* err) {
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  const int E = pl.E, B = pl.B, V = pl.V, RO = pl.RORDER, TO = pl.TORDER;
  const double PI = PI_REF;
  auto VC = [&](int row, int idx1) { return vs.vcord[3 * (size_t)(idx1 - 1) + (row - 1)]; };  // VCORD(row, idx)
  pl.rside.assign(B, -1);
  int rows = 0;
  for (int b = 0; b < B; ++b) {
    const int t = m.bsido[6 * b + 3];
    if (t != 1 && t != 2) pl.rside[b] = rows++;
  }
  pl.rf_i.assign((size_t)rows * V * 2, -1);
  pl.rf_z.assign((size_t)rows * V * 2, 0.0);
  for (int b = 0; b < B; ++b) {
    const int row = pl.rside[b];
    if (row < 0) continue;
    const double ANX = m.rsido[3 * b], ANY = m.rsido[3 * b + 1];
    for (int v = 0; v < V; ++v) {
      const double UX = pl.cx[v], UY = pl.cy[v];
      const double TEST = UX * ANX + UY * ANY;
      if (!(TEST < 0.0)) continue;
      const double CXR = UX + std::fabs(2 * TEST) * ANX, CYR = UY + std::fabs(2 * TEST) * ANY;
      const double RT = std::sqrt(CXR * CXR + CYR * CYR);
      const double QUO = std::fabs(CXR / RT);
      double THETA = std::fabs(std::acos(QUO));
      if (CXR < 0.0) THETA = PI - THETA;
      if (CYR < 0.0) THETA = -THETA;
      double ETAref = ((2 * RT) / vs.rv) - 1;
      if (ETAref > 1.0) ETAref = 1.0;
      const double ZETAref = THETA / PI;
      int IETA;
      for (IETA = 1; IETA <= RO; ++IETA) {
        const int idx = 1 + (IETA - 1) * (RO - 1);
        if (idx < 1 || idx > V)
          return fail(DGBGK_EUNSUP, "dgbgk_create: ALPHA < 1: the mirrored-speed lookup leaves VCORD for this "
                                    "velocity grid (RORDER > TORDER + 1)");
        if (std::fabs(ETAref - VC(1, idx)) < 0.0001) break;
      }
      const int ring = IETA - 1;
      int IZETA, I1, I2;
      double ZD1 = 0, ZD2 = 0;
      bool found = false;
      for (IZETA = 1; IZETA <= TO - 1; ++IZETA) {
        const double Z1 = VC(2, IZETA), Z2 = VC(2, IZETA + 1);
        ZD1 = Z2 - Z1;
        ZD2 = ZETAref - Z1;
        if (ZETAref >= Z1 && ZETAref <= Z2) {
          found = true;
          break;
        }
      }
      if (found) {
        I1 = (ring - 1) * TO + IZETA;
        I2 = (ring - 1) * TO + IZETA + 1;
      } else {
        ZD1 = VC(2, 1) - (-1.0);
        ZD2 = ZETAref - (-1.0);
        I1 = ring * TO;
        I2 = (ring - 1) * TO + 1;
      }
      if (I1 < 1 || I1 > V || I2 < 1 || I2 > V)
        return fail(DGBGK_EUNSUP, "dgbgk_create: ALPHA < 1: the mirrored velocity falls outside the velocity grid "
                                  "(the reference's ring lookup needs RORDER = TORDER)");
      const size_t o = ((size_t)row * V + v) * 2;
      pl.rf_i[o] = I1 - 1;
      pl.rf_i[o + 1] = I2 - 1;
      pl.rf_z[o] = ZD1;
      pl.rf_z[o + 1] = ZD2;
    }
  }
  // wall elements and their items
  pl.wslot.assign(E, -1);
  pl.welem.clear();
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k)
      if ((pl.edge[3 * (size_t)e + k].low & 3) == 3 && pl.wslot[e] < 0) {
        pl.wslot[e] = (int)pl.welem.size();
        pl.welem.push_back(e);
      }
  const int ns = (int)pl.welem.size();
  std::vector<unsigned char> mask((size_t)ns * V, 0);
  for (int s = 0; s < ns; ++s) {
    const int e = pl.welem[s];
    for (int k = 0; k < 3; ++k) {
      const PlanEdge& ed = pl.edge[3 * (size_t)e + k];
      if ((ed.low & 3) != 3) continue;
      const int row = pl.rside[ed.bside];
      for (int v = 0; v < V; ++v)
        if (pl.rf_i[((size_t)row * V + v) * 2] >= 0) mask[(size_t)s * V + v] |= (1 << k) | (1 << ((k + 1) % 3));
    }
  }
  pl.spec_par.clear();
  pl.spec_seq.clear();
  pl.spec_seq_off.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s) {
    const int e = pl.welem[s];
    for (int v = 0; v < V; ++v) {
      if (!mask[(size_t)s * V + v]) continue;
      bool dep = false;
      for (int k = 0; k < 3 && !dep; ++k) {
        const PlanEdge& ed = pl.edge[3 * (size_t)e + k];
        if ((ed.low & 3) != 3) continue;
        const size_t o = ((size_t)pl.rside[ed.bside] * V + v) * 2;
        if (pl.rf_i[o] < 0) continue;
        for (int j = 0; j < 2 && !dep; ++j) {
          const int I = pl.rf_i[o + j];
          const unsigned char mI = mask[(size_t)s * V + I];
          if (I < v && (((mI >> k) & 1) || ((mI >> ((k + 1) % 3)) & 1))) dep = true;
        }
      }
      if (dep)
        pl.spec_seq.push_back(s * V + v);
      else
        pl.spec_par.push_back(s * V + v);
    }
    pl.spec_seq_off[s + 1] = (int)pl.spec_seq.size();
  }
  pl.spec = true;
  return 0;
}

int build_plan(const dgbgk_mesh& m, const dgbgk_vspace& vs, const dgbgk_params& p, int EB, Plan& pl,
               std::string* err) {
  auto fail = [&](int code, const std::string& msg) {
    if (err) *err = msg;
    return code;
  };
  const int E = m.nelem, NP = m.npoin, B = m.nboun, S = m.nside;
  if (E < 1 || NP < 3 || B < 0 || S < 1 || !m.intma || !m.coord || !m.iside || !m.nx || !m.ny ||
      !m.el || !m.geome || !m.relen || (B > 0 && (!m.bsido || !m.rsido)))
    return fail(DGBGK_EINVAL, "dgbgk_create: missing or empty mesh array");
  if (p.immat == 1 && !m.mmat) return fail(DGBGK_EINVAL, "dgbgk_create: IMMAT = 1 needs MMAT");
  if (p.immat == 0 && !m.cmmat) return fail(DGBGK_EINVAL, "dgbgk_create: IMMAT = 0 needs CMMAT");
  if (p.immat != 0 && p.immat != 1) return fail(DGBGK_EINVAL, "dgbgk_create: IMMAT must be 0 or 1");
  if (vs.rorder < 1 || vs.torder < 1 || !vs.vcord || !(vs.rv > 0) || !(vs.sumweight > 0))
    return fail(DGBGK_EINVAL, "dgbgk_create: bad velocity space");
  pl.E = E;
  pl.NP = NP;
  pl.B = B;
  pl.S = S;
  pl.RORDER = vs.rorder;
  pl.TORDER = vs.torder;
  pl.V = vs.rorder * vs.torder;
  pl.immat = p.immat;
  pl.alpha = p.alpha;
  pl.rgas = p.rgas;
  pl.M = p.molar_mass;
  pl.d = p.diameter;
  pl.rv = vs.rv;
  pl.sumweight = vs.sumweight;
  for (int i = 0; i < 4; ++i) pl.cinf[i] = p.cinf[i];
  const int V = pl.V;
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k) {
      int q = m.intma[3 * e + k];
      if (q < 1 || q > NP) return fail(DGBGK_EMESH, "dgbgk_create: INTMA entry outside 1..NPOIN");
    }

  // ---- element order along a Hilbert curve of the centroids
  std::vector<double> cxs(E), cys(E);
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
  for (int e = 0; e < E; ++e) {
    double sx = 0, sy = 0;
    for (int k = 0; k < 3; ++k) {
      int q = m.intma[3 * e + k] - 1;
      sx += m.coord[2 * q];
      sy += m.coord[2 * q + 1];
    }
    cxs[e] = sx / 3;
    cys[e] = sy / 3;
    xmin = std::min(xmin, cxs[e]);
    xmax = std::max(xmax, cxs[e]);
    ymin = std::min(ymin, cys[e]);
    ymax = std::max(ymax, cys[e]);
  }
  double span = std::max(xmax - xmin, ymax - ymin);
  if (!(span > 0)) span = 1;
  std::vector<uint64_t> key(E);
  for (int e = 0; e < E; ++e) {
    uint32_t ix = (uint32_t)std::min(65535.0, std::floor((cxs[e] - xmin) / span * 65535.0));
    uint32_t iy = (uint32_t)std::min(65535.0, std::floor((cys[e] - ymin) / span * 65535.0));
    key[e] = hilbert16(ix, iy);
  }
  pl.perm.resize(E);
  std::iota(pl.perm.begin(), pl.perm.end(), 0);
  std::stable_sort(pl.perm.begin(), pl.perm.end(), [&](int a, int b) { return key[a] < key[b]; });
  pl.inv.resize(E);
  for (int i = 0; i < E; ++i) pl.inv[pl.perm[i]] = i;

  // ---- per element geometry
  std::vector<int> inflow_pt(NP + 1, 0);
  for (int b = 0; b < B; ++b)
    if (m.bsido[6 * b + 3] == 1) {
      for (int j = 0; j < 2; ++j) {
        int q = m.bsido[6 * b + j];
        if (q < 1 || q > NP) return fail(DGBGK_EMESH, "dgbgk_create: BSIDO node outside 1..NPOIN");
        inflow_pt[q] = 1;
      }
    }
  pl.geo.assign(E, PlanGeo());
  pl.cmax.assign(3 * (size_t)E, 0);
  pl.cmin.assign(3 * (size_t)E, 0);
  for (int en = 0; en < E; ++en) {
    int eo = pl.perm[en];
    const double* G = &m.geome[7 * (size_t)eo];
    PlanGeo& g = pl.geo[en];
    for (int k = 0; k < 3; ++k) {
      g.gx[k] = G[k];
      g.gy[k] = G[k + 3];
    }
    g.area = 0.5 * G[6];
    g.inflow = 0;
    for (int k = 0; k < 3; ++k) {
      if (inflow_pt[m.intma[3 * eo + k]]) g.inflow |= 1 << k;
      if (p.immat == 1) {
        g.mm[k] = m.mmat[3 * (size_t)eo + k];
      } else {
        const double* C = &m.cmmat[9 * (size_t)eo];
        double c0 = C[k], c1 = C[k + 3], c2 = C[k + 6];  // CMMAT(k,1..3)
        g.mm[k] = c0 + c1 + c2;
        pl.cmax[3 * (size_t)en + k] = std::max(c0, std::max(c1, c2));
        pl.cmin[3 * (size_t)en + k] = std::min(c0, std::min(c1, c2));
      }
    }
  }

  // ---- element edges from the side table
  pl.edge.assign(3 * (size_t)E, PlanEdge{});
  std::vector<char> seen(3 * (size_t)E, 0);
  // GETBOU's boundary-side lookup: the first BSIDO entry with the side's
  // element and first node (src/getbou.f90:48-53)
  std::map<std::pair<int, int>, int> bfind;
  for (int b = B - 1; b >= 0; --b) bfind[{m.bsido[6 * b + 2], m.bsido[6 * b]}] = b;
  const double sixth = 1.0 / 6.0;
  for (int s = 0; s < S; ++s) {
    const int* I = &m.iside[8 * (size_t)s];
    int ip1 = I[0], iel = I[2], ier = I[3];
    if (iel < 1 || iel > E || ier < 0 || ier > E || I[4] < 1 || I[4] > 3 || I[5] < 1 || I[5] > 3)
      return fail(DGBGK_EMESH, "dgbgk_create: ISIDE entry out of range (partition edges are not supported)");
    int kl = I[4] - 1;  // left element's edge starts at its node INL1
    int enl = pl.inv[iel - 1];
    size_t il = 3 * (size_t)enl + kl;
    if (seen[il]) return fail(DGBGK_EMESH, "dgbgk_create: element edge claimed by two sides");
    seen[il] = 1;
    PlanEdge& L = pl.edge[il];
    if (ier > 0) {
      if (I[6] < 1 || I[6] > 3 || I[7] < 1 || I[7] > 3)
        return fail(DGBGK_EMESH, "dgbgk_create: ISIDE right local nodes out of range");
      int kr = I[7] - 1;  // right element's edge starts at its node INR2
      int enr = pl.inv[ier - 1];
      size_t ir = 3 * (size_t)enr + kr;
      if (seen[ir]) return fail(DGBGK_EMESH, "dgbgk_create: element edge claimed by two sides");
      seen[ir] = 1;
      PlanEdge& Rr = pl.edge[ir];
      double alen = sixth * m.el[s];
      L.nx = m.nx[s];
      L.ny = m.ny[s];
      L.alen = alen;
      L.nbr = enr;
      // my point k = IP1 <-> right's INR1; my point k+1 = IP2 <-> INR2
      L.low = 0 | 4 | ((I[6] - 1) << 3) | ((I[7] - 1) << 5);
      Rr.nx = -m.nx[s];
      Rr.ny = -m.ny[s];
      Rr.alen = alen;
      Rr.nbr = enl;
      // my point k = IP2 <-> left's INL2; my point k+1 = IP1 <-> INL1
      Rr.low = 0 | ((I[5] - 1) << 3) | ((I[4] - 1) << 5);
    } else {
      auto it = bfind.find({iel, ip1});
      if (it == bfind.end())
        return fail(DGBGK_EMESH, "dgbgk_create: boundary side without a BSIDO entry (GETBOU search fails)");
      int b = it->second;
      int type = m.bsido[6 * b + 3];
      int kind = (type == 1) ? 1 : (type == 2) ? 2 : 3;
      L.nx = m.rsido[3 * b];
      L.ny = m.rsido[3 * b + 1];
      L.alen = sixth * m.rsido[3 * b + 2];
      L.nbr = -1;
      L.low = kind;
      L.bside = b;
      if (kind == 3) pl.has_wall_incoming = true;
    }
  }
  for (size_t i = 0; i < seen.size(); ++i)
    if (!seen[i]) return fail(DGBGK_EMESH, "dgbgk_create: element edge without a side (inconsistent orientation?)");

  // ---- velocity tables (src/advnce.f90:286-292, src/macros.f90:94-103)
  pl.cx.resize(V);
  pl.cy.resize(V);
  pl.wjf.resize(V);
  pl.nfinf.resize(V);
  const double frac = 4.0 / vs.sumweight;
  // INFLOW (src/inflow.f90:28-39)
  const double Tin = p.cinf[0], Pin = p.cinf[1] * 100000.0, U0 = p.cinf[2], V0 = p.cinf[3];
  const double RHOin = Pin / (p.rgas * Tin);
  const double BETA = std::sqrt(RHOin / (2 * Pin));
  const double C0 = (RHOin * 6.022e26) / p.molar_mass, C1 = (BETA * BETA) / PI_REF;
  for (int v = 0; v < V; ++v) {
    double eta = vs.vcord[3 * v], zeta = vs.vcord[3 * v + 1], w = vs.vcord[3 * v + 2];
    double r = (vs.rv / 2) * (eta + 1);
    double th = zeta * PI_REF;
    pl.cx[v] = r * std::cos(th);
    pl.cy[v] = r * std::sin(th);
    double jac = PI_REF * vs.rv * vs.rv * 0.25 * (eta + 1);
    pl.wjf[v] = w * jac * frac;
    double ud = pl.cx[v] - U0, vd = pl.cy[v] - V0;
    pl.nfinf[v] = C0 * C1 * std::exp(-(BETA * BETA) * (ud * ud + vd * vd));
  }

  // ---- boundary sides
  pl.bTw.assign(B, 0);
  pl.bUw.assign(2 * (size_t)B, 0);
  for (int b = 0; b < B; ++b) {
    pl.bTw[b] = (double)m.bsido[6 * b + 4];
    if (p.wall_velocity) {
      pl.bUw[2 * b] = p.wall_velocity[2 * b];
      pl.bUw[2 * b + 1] = p.wall_velocity[2 * b + 1];
    }
  }
  // FLUCON2's wall sides (src/flucon2.f90:47-128, 218-233)
  std::map<std::pair<int, int>, int> sfind;
  for (int s = S - 1; s >= 0; --s) {
    sfind[{m.iside[8 * s], m.iside[8 * s + 1]}] = s;
  }
  // GETFOR's sides (src/getfor.f90:29-49): LEN and the rotated unit normal
  // PERP from the node coordinates, in FP64
  pl.fsides.clear();
  for (int b = 0; b < B; ++b) {
    if (m.bsido[6 * b + 3] != 4) continue;
    const int ip1 = m.bsido[6 * b] - 1, ip2 = m.bsido[6 * b + 1] - 1;
    if (ip1 < 0 || ip1 >= NP || ip2 < 0 || ip2 >= NP)
      return fail(DGBGK_EMESH, "dgbgk_create: BSIDO node outside 1..NPOIN");
    const double x1 = m.coord[2 * ip1], y1 = m.coord[2 * ip1 + 1], x2 = m.coord[2 * ip2], y2 = m.coord[2 * ip2 + 1];
    const double len = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    double px = -(y2 - y1), py = x2 - x1;  // ROTMAT * VEC
    const double mag = std::sqrt(px * px + py * py);
    if (!(mag > 0.0)) return fail(DGBGK_EMESH, "dgbgk_create: zero-length wall side (GETFOR)");
    px /= mag;
    py /= mag;
    pl.fsides.push_back(ForceSide{ip1, ip2, len * px, len * py});
  }
  pl.walls.clear();
  for (int b = 0; b < B; ++b) {
    if (m.bsido[6 * b + 3] != 4) continue;
    int ip1 = m.bsido[6 * b], ip2 = m.bsido[6 * b + 1], iel = m.bsido[6 * b + 2];
    if (iel < 1 || iel > E) return fail(DGBGK_EMESH, "dgbgk_create: BSIDO element outside 1..NELEM");
    // first side in ISIDE order matching (IP1,IP2) in either orientation
    int best = -1, in1 = 0, in2 = 0;
    auto a = sfind.find({ip1, ip2});
    auto c = sfind.find({ip2, ip1});
    if (a != sfind.end()) {
      best = a->second;
      in1 = m.iside[8 * best + 4];
      in2 = m.iside[8 * best + 5];
    }
    if (c != sfind.end() && (best < 0 || c->second < best)) {
      best = c->second;
      in1 = m.iside[8 * best + 5];
      in2 = m.iside[8 * best + 4];
    }
    if (best < 0) return fail(DGBGK_EMESH, "dgbgk_create: wall side not found in ISIDE (FLUCON2)");
    long long tw = m.bsido[6 * b + 4];
    double sb = std::sqrt(2 * PI_REF * (p.rgas * p.rgas * p.rgas) * (double)(tw * tw * tw));
    if (sb < 0.1)
      return fail(DGBGK_EINVAL, "dgbgk_create: flux conservation parameter denominator < 0.1 (FLUCON2)");
    WallSide w;
    w.elem = pl.inv[iel - 1];
    w.in1 = in1 - 1;
    w.in2 = in2 - 1;
    w.bside = b;
    w.anx = m.rsido[3 * b];
    w.any = m.rsido[3 * b + 1];
    w.sumbottom = sb;
    pl.walls.push_back(w);
  }

  // ---- the specular part of the wall flux for ALPHA < 1
  pl.spec = false;
  if (p.alpha != 1.0 && pl.has_wall_incoming) {
    int rc = build_specular(m, vs, pl, err);
    if (rc != 0) return rc;
  }

  // ---- Courant limit (src/alotim.f90:12-18, MXSPD = rv)
  double dtc = 0;
  for (int e = 0; e < E; ++e) {
    double dd = (p.csafm * m.relen[e]) / vs.rv;
    dtc = (e == 0) ? dd : std::min(dtc, dd);
  }
  pl.dtc = dtc;

  // ---- nodal gather in the reference's element order
  pl.node_off.assign(NP + 1, 0);
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k) pl.node_off[m.intma[3 * e + k]] += 1;
  for (int i = 0; i < NP; ++i) pl.node_off[i + 1] += pl.node_off[i];
  pl.node_dg.assign(3 * (size_t)E, 0);
  pl.node_ae.assign(3 * (size_t)E, 0);
  std::vector<int> fill(NP, 0);
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k) {
      int q = m.intma[3 * e + k] - 1;
      int pos = pl.node_off[q] + fill[q]++;
      pl.node_dg[pos] = 3 * pl.inv[e] + k;
      pl.node_ae[pos] = m.geome[7 * (size_t)e + 6];
    }

  build_blocks(pl, EB);
  return DGBGK_OK;
}

}  // namespace dgbgk

// sm_100a kernels of the DG-BGK pseudo-time step.
//
// One step (src/advnce.f90:220-400) is four launches on one stream:
//   k_moments : MACROS passes 1+2 (src/macros.f90:80-154) fused with COMPMU
//               (src/compmu.f90:242-290) and the GTEQNF parameters
//               (src/gteqnf.f90:315-326): one warp per DG node, the node's
//               velocity row staged in shared memory so f is read from HBM
//               once for both passes; FP64 accumulation for every precision.
//   k_wall    : FLUCON2 (src/flucon2.f90:134-233), one warp per wall side.
//   k_sweep   : the whole velocity loop body (GTEQNF, GETFLA, GETELC,
//               EDGFLXOPT/GETBOU, GETINC/CMMINC, ADTHEM, INFLOW; src/advnce.f90
//               :286-377) for a tile of (element block x velocity tile), with
//               the block's and its halo's f and UMEAN staged in shared memory.
//   k_resid   : GETRES + the residual bookkeeping (src/advnce.f90:385,422-429),
//               the convergence test and the step counter.
#pragma once
#include <cuda_runtime.h>

#include "types.h"

namespace dgbgk {

constexpr double PI_D = 3.1416;  // the reference's PI
constexpr double NA_D = 6.022e26;
constexpr double TINY_D = 1e-20;

template <class T> __device__ __forceinline__ T dexp(T x);
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float dexp<float>(float x) { return expf(x); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ------------------------------------------------------------ moments ----
template <class T> struct MomArgs {
  const T* __restrict__ f;
  const double* __restrict__ cx;
  const double* __restrict__ cy;
  const double* __restrict__ wjf;  // WEIGHT*JAC*FRAC
  NodeP<T>* __restrict__ np;
  double* __restrict__ nraw;   // INT (number density before the 1e-20 test)
  double* __restrict__ disux;
  double* __restrict__ disuy;
  double* __restrict__ disps;
  double* __restrict__ mu;
  Ctrl* ctrl;
  int ndg, V;
  double MM, sigt;  // M/NA, PI*d*d
};

template <class T, int WPB>
__global__ void __launch_bounds__(WPB * 32) k_moments(MomArgs<T> a) {
  if (a.ctrl->done) return;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* row = reinterpret_cast<T*>(sm_raw) + (threadIdx.x >> 5) * a.V;
  const int lane = threadIdx.x & 31;
  const int node = blockIdx.x * WPB + (threadIdx.x >> 5);
  if (node >= a.ndg) return;
  const T* fr = a.f + (size_t)node * a.V;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int v = lane; v < a.V; v += 32) {
    T x = __ldcs(fr + v);  // streamed: each value is read exactly once from HBM
    row[v] = x;
    double w = a.wjf[v] * (double)x;
    s0 += w;
    s1 += a.cx[v] * w;
    s2 += a.cy[v] * w;
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  double nd = 0, ux = 0, uy = 0;
  if (s0 >= TINY_D) {  // src/macros.f90:126-134
    nd = s0;
    ux = s1 / s0;
    uy = s2 / s0;
  }
  __syncwarp();
  double sp = 0, sc = 0;
  for (int v = lane; v < a.V; v += 32) {
    double x = (double)row[v];
    double dx = a.cx[v] - ux, dy = a.cy[v] - uy;
    double d2 = dx * dx + dy * dy;
    double w = a.wjf[v] * x;
    sp += 0.5 * d2 * w;   // src/macros.f90:144-148
    sc += sqrt(d2) * w;   // src/compmu.f90:264-267
  }
  sp = warp_sum(sp);
  sc = warp_sum(sc);
  if (lane == 0) {
    double ps = sp * a.MM;
    double ct = (nd >= TINY_D) ? sc / nd : 0.0;
    double mu = sqrt(2.0) * ct * a.sigt * nd;
    NodeP<T> p;
    if (ps >= TINY_D) {  // GTEQNF (src/gteqnf.f90:317-326)
      double rho = a.MM * nd;
      double b2 = rho / (2 * ps);
      p.A = (T)(nd * (b2 / PI_D));
      p.B = (T)b2;
    } else {
      p.A = (T)0;
      p.B = (T)0;
    }
    p.ux = (T)ux;
    p.uy = (T)uy;
    p.mu = (T)mu;
    a.np[node] = p;
    a.nraw[node] = s0;
    a.disux[node] = ux;
    a.disuy[node] = uy;
    a.disps[node] = ps;
    a.mu[node] = mu;
    atomicMax(reinterpret_cast<unsigned long long*>(&a.ctrl->maxmu),
              (unsigned long long)__double_as_longlong(mu));
  }
}

// --------------------------------------------------------- wall flux ----
template <class T> struct WallArgs {
  const T* __restrict__ f;
  const WallSide* __restrict__ walls;
  const double* __restrict__ cx;
  const double* __restrict__ cy;
  const double* __restrict__ wjf;
  T* __restrict__ beta_t;   // ETA per boundary side (sweep precision)
  double* __restrict__ beta_d;
  Ctrl* ctrl;
  int nwall, V;
};

template <class T> __global__ void __launch_bounds__(256) k_wall(WallArgs<T> a) {
  if (a.ctrl->done) return;
  const int w = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (w >= a.nwall) return;
  const WallSide ws = a.walls[w];
  const T* f1 = a.f + ((size_t)ws.elem * 3 + ws.in1) * a.V;
  const T* f2 = a.f + ((size_t)ws.elem * 3 + ws.in2) * a.V;
  double s = 0;
  for (int v = lane; v < a.V; v += 32) {
    double test = a.cx[v] * ws.anx + a.cy[v] * ws.any;
    if (test > 0.0) s += fabs(test) * (0.5 * ((double)f1[v] + (double)f2[v])) * a.wjf[v];
  }
  s = warp_sum(s);
  if (lane == 0) {
    double eta = s / ws.sumbottom;
    a.beta_d[ws.bside] = eta;
    a.beta_t[ws.bside] = (T)eta;
  }
}

// -------------------------------------------------------------- sweep ----
template <class T> struct SweepArgs {
  const T* __restrict__ fin;
  T* __restrict__ fout;
  const ElemGeo<T>* __restrict__ geo;
  const ElemEdge<T>* __restrict__ edge;
  const int* __restrict__ eslot;
  const NodeP<T>* __restrict__ np;
  const int* __restrict__ halo_off;
  const int* __restrict__ halo_list;
  const T* __restrict__ cx;
  const T* __restrict__ cy;
  const T* __restrict__ nfinf;
  const T* __restrict__ bTw;
  const T* __restrict__ bUw;
  const T* __restrict__ bEta;
  const T* __restrict__ cmax;  // IMMAT = 0 only
  const T* __restrict__ cmin;
  double* __restrict__ part_max;
  double* __restrict__ part_sq;
  Ctrl* ctrl;
  int E, V, EB, slots, immat;
  T alpha, rgas;
};

// DTE = min(CSAFE/maxMU, DTEc)  (src/alotim2.f90:10-15, src/advnce.f90:258-262)
__device__ __forceinline__ double step_dt(const Ctrl* c) {
  double mx = c->maxmu;
  double dtb = (mx > 0.0) ? 0.9 * (1.0 / mx) : 1000000.0;
  return fmin(dtb, c->dtc);
}

// UMEAN of one element at one velocity (src/getelc.f90:54-83):
// 0.5*DTE*(div F - 1/3 sum MU (NFO - f)), div F = sum (N_i,x cx + N_i,y cy) f_i.
template <class T>
__device__ __forceinline__ T umean_of(const T* f, const T* q, const ElemGeo<T>& g, const NodeP<T>* P,
                                      T cx, T cy, T dth) {
  T dive = (g.gx[0] * cx + g.gy[0] * cy) * f[0] + (g.gx[1] * cx + g.gy[1] * cy) * f[1] +
           (g.gx[2] * cx + g.gy[2] * cy) * f[2];
  T coll = P[0].mu * (q[0] - f[0]) + P[1].mu * (q[1] - f[1]) + P[2].mu * (q[2] - f[2]);
  return (dive - coll * (T)(1.0 / 3.0)) * dth;
}

template <class T>
__device__ __forceinline__ T feq_of(const NodeP<T>& p, T cx, T cy) {
  T dx = p.ux - cx, dy = p.uy - cy;
  return p.A * dexp<T>(-p.B * (dx * dx + dy * dy));
}

template <class T, int M>
__global__ void __launch_bounds__(256) k_sweep(SweepArgs<T> a) {
  if (a.ctrl->done) return;
  const int VT = blockDim.x, TY = blockDim.y;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int blk = blockIdx.x;
  const int v = blockIdx.y * VT + tx;
  const bool vok = v < a.V;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* fs = reinterpret_cast<T*>(sm_raw);  // [slots][3][VT]
  T* us = fs + (size_t)a.slots * 3 * VT;  // [slots][VT]
  const double dtd = step_dt(a.ctrl);
  const T dt = (T)dtd, dth = (T)(dtd * 0.5);
  const T cx = vok ? a.cx[v] : (T)0, cy = vok ? a.cy[v] : (T)0;
  const int e0 = blk * a.EB;
  const int nb = min(a.EB, a.E - e0);
  const size_t V = (size_t)a.V;
  const int vv = vok ? v : 0;

  // phase 1: f and UMEAN of the block (kept in registers + shared) ...
  T fr[M][3], qr[M][3], ur[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int j = ty + TY * m;
    if (j < nb) {
      const int e = e0 + j;
      const NodeP<T>* P = a.np + 3 * (size_t)e;
      const ElemGeo<T> g = a.geo[e];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        fr[m][i] = vok ? __ldcs(a.fin + ((size_t)e * 3 + i) * V + vv) : (T)0;
        qr[m][i] = feq_of(P[i], cx, cy);
      }
      ur[m] = umean_of(fr[m], qr[m], g, P, cx, cy, dth);
#pragma unroll
      for (int i = 0; i < 3; ++i) fs[((size_t)j * 3 + i) * VT + tx] = fr[m][i];
      us[(size_t)j * VT + tx] = ur[m];
    }
  }
  // ... and of the halo (neighbours outside the block)
  const int h0 = a.halo_off[blk], nh = a.halo_off[blk + 1] - h0;
  for (int h = ty; h < nh; h += TY) {
    const int e = a.halo_list[h0 + h];
    const NodeP<T>* P = a.np + 3 * (size_t)e;
    const ElemGeo<T> g = a.geo[e];
    T f[3], q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      f[i] = vok ? a.fin[((size_t)e * 3 + i) * V + vv] : (T)0;
      q[i] = feq_of(P[i], cx, cy);
    }
    const int j = a.EB + h;
#pragma unroll
    for (int i = 0; i < 3; ++i) fs[((size_t)j * 3 + i) * VT + tx] = f[i];
    us[(size_t)j * VT + tx] = umean_of(f, q, g, P, cx, cy, dth);
  }
  __syncthreads();

  // phase 2: volume + edge terms, increment, positivity, inflow reset
  double rmax = 0.0, rsq = 0.0;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int j = ty + TY * m;
    if (j < nb && vok) {
      const int e = e0 + j;
      const ElemGeo<T> g = a.geo[e];
      const NodeP<T>* P = a.np + 3 * (size_t)e;
      const T um = ur[m];
      // GETELC second half: RHS_i = AREA*(N_i,x FXME + N_i,y FYME)
      const T fm = ((fr[m][0] - um) + (fr[m][1] - um) + (fr[m][2] - um)) * (T)(1.0 / 3.0);
      T rhs[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) rhs[i] = g.area * ((g.gx[i] * cx) * fm + (g.gy[i] * cy) * fm);
      // EDGFLXOPT / GETBOU, gathered per element
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int p = k, q = (k + 1) % 3;
        const ElemEdge<T> ed = a.edge[3 * (size_t)e + k];
        const int kind = ed.info & 3;
        if (kind == 1) continue;  // inflow sides carry no flux
        const T sc = ed.nx * cx + ed.ny * cy;
        T up, uq;
        if (kind == 0) {
          const bool left = (ed.info & 4) != 0;
          const bool mine = left ? (sc > (T)0) : (sc >= (T)0);
          if (mine) {
            up = fr[m][p] - um;
            uq = fr[m][q] - um;
          } else {
            const int s = a.eslot[3 * (size_t)e + k];
            const int np_ = (ed.info >> 3) & 3, nq_ = (ed.info >> 5) & 3;
            const T un = us[(size_t)s * VT + tx];
            up = fs[((size_t)s * 3 + np_) * VT + tx] - un;
            uq = fs[((size_t)s * 3 + nq_) * VT + tx] - un;
          }
        } else if (kind == 2 || sc >= (T)0) {
          up = fr[m][p] - um;
          uq = fr[m][q] - um;
        } else {
          // wall, molecules leaving the wall (src/getbou.f90:189-255):
          // fully diffuse part ALPHA*ETA*Mw (the reflected part is handled
          // by the wall fix-up pass when ALPHA < 1)
          const int bs = ed.info >> 8;
          const T tw = a.bTw[bs];
          const T uwx = a.bUw[2 * bs], uwy = a.bUw[2 * bs + 1];
          T mw;
          if (uwx == (T)0 && uwy == (T)0) {
            const T spd = sqrt(cx * cx + cy * cy);
            mw = dexp<T>(-(spd * spd) / ((T)2 * a.rgas * tw));
          } else {
            const T dx = cx - uwx, dy = cy - uwy;
            mw = dexp<T>(-(dx * dx + dy * dy) / ((T)2 * a.rgas * tw));
          }
          up = uq = a.alpha * (mw * a.bEta[bs]);
        }
        const T fnp = sc * up, fnq = sc * uq;
        rhs[p] -= ed.alen * ((T)2 * fnp + fnq);
        rhs[q] -= ed.alen * (fnp + (T)2 * fnq);
      }
      // GETINC / CMMINC, ADTHEM, INFLOW
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const T x = rhs[i] * dt;
        const T cdt = P[i].mu * (qr[m][i] - fr[m][i]) * dt;
        const T d = g.mm[i] * x + cdt;
        double rr;
        if (a.immat == 1) {
          rr = fabs((double)d);
        } else {
          const T c = (x >= (T)0) ? a.cmax[3 * (size_t)e + i] : a.cmin[3 * (size_t)e + i];
          rr = fmax(0.0, (double)(c * x + cdt));
        }
        rmax = fmax(rmax, rr);
        rsq += (double)d * (double)d;
        T fn = fr[m][i] + d;
        if (fn < (T)0) fn = (T)0;
        if (g.inflow & (1 << i)) fn = a.nfinf[v];
        __stcs(a.fout + ((size_t)e * 3 + i) * V + v, fn);
      }
    }
  }
  // per-CTA residual partials (deterministic final reduction in k_resid)
  rmax = warp_max(rmax);
  rsq = warp_sum(rsq);
  __shared__ double red_m[32], red_s[32];
  const int wid = (ty * VT + tx) >> 5, nw = (VT * TY) >> 5;
  if (((ty * VT + tx) & 31) == 0) {
    red_m[wid] = rmax;
    red_s[wid] = rsq;
  }
  __syncthreads();
  if (ty == 0 && tx == 0) {
    double mm = 0, ss = 0;
    for (int w = 0; w < nw; ++w) {
      mm = fmax(mm, red_m[w]);
      ss += red_s[w];
    }
    const int cta = blockIdx.y * gridDim.x + blockIdx.x;
    a.part_max[cta] = mm;
    a.part_sq[cta] = ss;
  }
}

// ----------------------------------------------------------- residual ----
struct ResidArgs {
  const double* part_max;
  const double* part_sq;
  double* hist_linf;
  double* hist_l2;
  double* hist_dt;
  Ctrl* ctrl;
};

__global__ void __launch_bounds__(1024) k_resid(ResidArgs a) {
  Ctrl* c = a.ctrl;
  if (c->done) return;
  __shared__ double sm[32], ss[32];
  double m = 0, s = 0;
  for (int i = threadIdx.x; i < c->nparts; i += blockDim.x) {
    m = fmax(m, a.part_max[i]);
    s += a.part_sq[i];
  }
  // NaN must survive fmax: track it separately
  int bad = (isnan(m) || isnan(s)) ? 1 : 0;
  bad = __syncthreads_or(bad);
  m = warp_max(m);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) {
    sm[threadIdx.x >> 5] = m;
    ss[threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0, sq = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      mm = fmax(mm, sm[w]);
      sq += ss[w];
    }
    const int st = c->step;
    const double l2 = sqrt(sq);
    a.hist_linf[st] = mm;
    a.hist_l2[st] = l2;
    a.hist_dt[st] = step_dt(c);
    if (bad || !isfinite(l2) || !isfinite(mm)) {
      c->nonfinite = 1;
      c->done = 1;
    }
    if (c->ref == 0.0 && l2 > 0.0) c->ref = l2;
    c->step = st + 1;
    if (c->step >= c->max_steps) c->done = 1;
    if (c->tol > 0.0 && l2 <= c->tol * c->ref) c->done = 1;
  }
}

// -------------------------------------------------------------- nodal ----
// MACROS tail (src/macros.f90:156-188) and GETMAC with one partition.
struct NodalArgs {
  const int* node_off;
  const int* node_dg;
  const double* node_ae;
  const double* nraw;
  const double* disux;
  const double* disuy;
  const double* disps;
  double *nd, *rho, *u, *v, *ps, *temp;
  int NP;
  double MM, R;
};

__global__ void k_nodal(NodalArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.NP) return;
  double flag = 0, nd = 0, u = 0, v = 0, ps = 0;
  for (int k = a.node_off[q]; k < a.node_off[q + 1]; ++k) {
    const int dg = a.node_dg[k];
    const double ae = a.node_ae[k];
    flag += ae;
    nd += a.nraw[dg] * ae;
    if (a.nraw[dg] >= TINY_D) {
      u += ae * a.disux[dg];
      v += ae * a.disuy[dg];
    }
    ps += a.disps[dg] * ae;
  }
  double rho = 0, t = 0;
  if (nd < TINY_D) {
    u = v = ps = 0;
  } else {
    nd = nd / flag;
    rho = nd * a.MM;
    u = u / flag;
    v = v / flag;
    ps = ps / flag;
    t = ps / (a.R * rho);
  }
  a.nd[q] = nd;
  a.rho[q] = rho;
  a.u[q] = u;
  a.v[q] = v;
  a.ps[q] = ps;
  a.temp[q] = t;
}

// ----------------------------------------------------- layout changes ----
// reference DISNF(3,V,E) (old element order) <-> f[e][i][v] (plan order)
template <class S, class T>
__global__ void k_to_internal(const S* __restrict__ src, T* __restrict__ dst, const int* __restrict__ inv,
                              int V) {
  const int eo = blockIdx.x;
  const size_t en = (size_t)inv[eo];
  const S* s = src + (size_t)eo * 3 * V;
  for (int i = 0; i < 3; ++i)
    for (int v = threadIdx.x; v < V; v += blockDim.x) dst[(en * 3 + i) * V + v] = (T)s[(size_t)v * 3 + i];
}

template <class T, class S>
__global__ void k_from_internal(const T* __restrict__ src, S* __restrict__ dst, const int* __restrict__ inv,
                                int V) {
  const int eo = blockIdx.x;
  const size_t en = (size_t)inv[eo];
  S* d = dst + (size_t)eo * 3 * V;
  for (int i = 0; i < 3; ++i)
    for (int v = threadIdx.x; v < V; v += blockDim.x) d[(size_t)v * 3 + i] = (S)src[(en * 3 + i) * V + v];
}

// INICON2 (src/inicon2.f90:231-262) times an optional per-DG-node scale.
template <class T>
__global__ void k_init_uniform(T* __restrict__ f, const double* __restrict__ g, const double* __restrict__ scale,
                               double n1, int V, size_t total) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int v = (int)(idx % V);
  const size_t dg = idx / V;
  double val = n1 * g[v];
  if (scale) val = val * scale[dg];
  f[idx] = (T)val;
}

// Maxwellian from per-DG-node (n, u, v, T) (the warm start): the INICON2
// formula with RHO = n*M/NA, P = RHO*R*T, BETA^2 = RHO/(2P).
template <class T>
__global__ void k_init_maxwellian(T* __restrict__ f, const double* __restrict__ prm /* [dg][4] */,
                                  const double* __restrict__ cx, const double* __restrict__ cy, double MM,
                                  double R, int V, size_t total) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int v = (int)(idx % V);
  const size_t dg = idx / V;
  const double n = prm[4 * dg], u = prm[4 * dg + 1], w = prm[4 * dg + 2], t = prm[4 * dg + 3];
  double val = 0.0;
  if (n >= TINY_D && t > 0.0) {
    const double rho = n * MM, p = rho * R * t;
    const double b2 = rho / (2 * p);
    const double dx = cx[v] - u, dy = cy[v] - w;
    val = n * ((b2 / PI_D) * exp(-(b2 * (dx * dx + dy * dy))));
  }
  f[idx] = (T)val;
}

}  // namespace dgbgk

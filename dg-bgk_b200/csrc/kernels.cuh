// sm_100a kernels of the DG-BGK pseudo-time step.
//
// One step (src/advnce.f90:220-400) is four launches on one stream:
//   k_moments : MACROS passes 1+2 (src/macros.f90:80-154) fused with COMPMU
//               (src/compmu.f90:242-290) and the GTEQNF parameters
//               (src/gteqnf.f90:315-326).  Persistent warps stream whole
//               velocity rows of f into shared memory with 1-D bulk copies
//               (cp.async.bulk, a ring of stages per warp), so f is read from
//               HBM once for both passes; the velocity tables sit in shared
//               memory and every access is a 16-byte vector.
//   k_wall    : FLUCON2 (src/flucon2.f90:134-233), one warp per wall side.
//   k_sweep   : the whole velocity-loop body (GTEQNF, GETFLA, GETELC,
//               EDGFLXOPT/GETBOU, GETINC/CMMINC, ADTHEM, INFLOW;
//               src/advnce.f90:286-377) on tiles of (element block x 32
//               velocities).  Persistent CTAs; each tile's inputs -- the
//               block's f rows in one 2-D TMA box, each halo element's rows
//               in a 3-row box, the block's element records in one bulk copy
//               and the halo's record heads -- land in a two-stage
//               shared-memory ring while the previous tile is computed.
//   k_resid   : GETRES + the residual bookkeeping (src/advnce.f90:385,
//               422-429), the convergence test and the step counter.
// Every device-side wait is bounded: on expiry the kernel sets
// Ctrl::timeout, drains its own copies with a second bounded wait and
// returns; the host reports DGBGK_ECUDA.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "types.h"

namespace dgbgk {

constexpr double PI_D = 3.1416;  // the reference's PI
constexpr double TINY_D = 1e-20;
constexpr unsigned WAIT_TRIES = 1u << 22;  // x ~256 ns sleep: ~1 s

// e^x in FP32 for the FP32 sweep: t = x*log2(e) is formed with its rounding
// error recovered by an FMA (t_lo = fma(x, L, -t) + x*(log2(e) - L)), 2^t
// comes from the SFU's ex2.approx and the low part enters to first order,
// 2^t_lo ~ 1 + t_lo*ln2.  Relative error ~2.5e-7 (the SFU's 2^-22 bound).
// Arguments here are finite and <= 0 (x = -BETA2*|c-u|^2).
__device__ __forceinline__ float exp_sfu(float x) {
  const float L = 1.44269502163f, Llo = 1.92596303e-8f;
  const float t = x * L;
  const float tl = fmaf(x, L, -t) + x * Llo;
  float p;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p) : "f"(t));
  return fmaf(p, tl * 0.693147181f, p);
}
template <class T> __device__ __forceinline__ T dexp(T x);
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float dexp<float>(float x) { return exp_sfu(x); }

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

// ------------------------------------------------- TMA / mbarrier helpers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (unsigned i = 0; i < WAIT_TRIES; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 32) __nanosleep(256);
  }
  return false;
}
// 2-D tiled TMA load (no multicast) of box {x, y} into shared memory.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// 1-D bulk copy global -> shared (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// ------------------------------------------------------------ moments ----
template <class T> struct MomArgs {
  const T* __restrict__ f;
  const T* __restrict__ tabs;  // [3][Vp] cx, cy, WEIGHT*JAC*FRAC, zero past V
  ElemRec<T>* __restrict__ rec;
  double* __restrict__ nraw;   // INT (number density before the 1e-20 test)
  double* __restrict__ disux;
  double* __restrict__ disuy;
  double* __restrict__ disps;
  double* __restrict__ mu;
  Ctrl* ctrl;
  int ndg, V, Vp, nstage;
  unsigned rowbytes;  // V*sizeof(T) rounded up to 16
  double MM, sigt;    // M/NA, PI*d*d
};

// sqrt by a reciprocal-square-root seed and one Newton step for 1/sqrt(x),
// y <- y (3 - x y^2)/2, in FP64 (relative error ~1e-14 from a ~1e-7 seed).
__device__ __forceinline__ double sqrt_newton(double x) {
  const float xf = (float)x;
  if (!(xf > 0.f)) return 0.0;
  const double y0 = (double)rsqrtf(xf);
  const double y1 = y0 * (1.5 - 0.5 * x * y0 * y0);
  return x * y1;
}
__device__ __forceinline__ float sqrt_fast(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

// Pass sums over one velocity row in shared memory, one 16-byte vector per
// lane and iteration.  FP64 storage: FP64 arithmetic.  FP32 storage: FP32
// products and 4-value partial sums accumulated in FP64 (an FP64-accumulated
// FP32 kernel was FP64-pipe bound).
template <class T> struct RowMath;

template <> struct RowMath<double> {
  static __device__ __forceinline__ void pass1(const double* row, const double* tb, int Vp, int nq, int lane,
                                               double& s0, double& s1, double& s2) {
    const double2* r = reinterpret_cast<const double2*>(row);
    const double2* cx = reinterpret_cast<const double2*>(tb);
    const double2* cy = reinterpret_cast<const double2*>(tb + Vp);
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
    for (int q = lane; q < nq; q += 32) {
      const double2 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const double a0 = w.x * x.x, a1 = w.y * x.y;
      s0 += a0 + a1;
      s1 = fma(c.x, a0, fma(c.y, a1, s1));
      s2 = fma(d.x, a0, fma(d.y, a1, s2));
    }
  }
  static __device__ __forceinline__ void pass2(const double* row, const double* tb, int Vp, int nq, int lane,
                                               double ux, double uy, double& sp, double& sc) {
    const double2* r = reinterpret_cast<const double2*>(row);
    const double2* cx = reinterpret_cast<const double2*>(tb);
    const double2* cy = reinterpret_cast<const double2*>(tb + Vp);
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
    for (int q = lane; q < nq; q += 32) {
      const double2 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const double dx0 = c.x - ux, dy0 = d.x - uy, dx1 = c.y - ux, dy1 = d.y - uy;
      const double q0 = dx0 * dx0 + dy0 * dy0, q1 = dx1 * dx1 + dy1 * dy1;
      const double a0 = w.x * x.x, a1 = w.y * x.y;
      sp = fma(0.5 * q0, a0, fma(0.5 * q1, a1, sp));                // src/macros.f90:144-148
      sc = fma(sqrt_newton(q0), a0, fma(sqrt_newton(q1), a1, sc));  // src/compmu.f90:264-267
    }
  }
};

template <> struct RowMath<float> {
  static __device__ __forceinline__ void pass1(const float* row, const float* tb, int Vp, int nq, int lane,
                                               double& s0, double& s1, double& s2) {
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* cx = reinterpret_cast<const float4*>(tb);
    const float4* cy = reinterpret_cast<const float4*>(tb + Vp);
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    for (int q = lane; q < nq; q += 32) {
      const float4 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const float a0 = w.x * x.x, a1 = w.y * x.y, a2 = w.z * x.z, a3 = w.w * x.w;
      s0 += (double)((a0 + a1) + (a2 + a3));
      s1 += (double)fmaf(c.x, a0, fmaf(c.y, a1, fmaf(c.z, a2, c.w * a3)));
      s2 += (double)fmaf(d.x, a0, fmaf(d.y, a1, fmaf(d.z, a2, d.w * a3)));
    }
  }
  static __device__ __forceinline__ void pass2(const float* row, const float* tb, int Vp, int nq, int lane,
                                               double ux, double uy, double& sp, double& sc) {
    const float fx = (float)ux, fy = (float)uy;
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* cx = reinterpret_cast<const float4*>(tb);
    const float4* cy = reinterpret_cast<const float4*>(tb + Vp);
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    for (int q = lane; q < nq; q += 32) {
      const float4 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const float e0 = c.x - fx, e1 = c.y - fx, e2 = c.z - fx, e3 = c.w - fx;
      const float g0 = d.x - fy, g1 = d.y - fy, g2 = d.z - fy, g3 = d.w - fy;
      const float q0 = fmaf(e0, e0, g0 * g0), q1 = fmaf(e1, e1, g1 * g1), q2 = fmaf(e2, e2, g2 * g2),
                  q3 = fmaf(e3, e3, g3 * g3);
      const float a0 = w.x * x.x, a1 = w.y * x.y, a2 = w.z * x.z, a3 = w.w * x.w;
      sp += (double)(0.5f * fmaf(q0, a0, fmaf(q1, a1, fmaf(q2, a2, q3 * a3))));
      sc += (double)fmaf(sqrt_fast(q0), a0, fmaf(sqrt_fast(q1), a1, fmaf(sqrt_fast(q2), a2, sqrt_fast(q3) * a3)));
    }
  }
};

template <class T>
__global__ void __launch_bounds__(512) k_moments(MomArgs<T> a) {
  if (a.ctrl->done) return;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // layout: [barriers][tables 3*Vp][rings]
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm_raw) + warp * a.nstage;
  T* tb = reinterpret_cast<T*>(sm_raw + 128 * ((nwarp * a.nstage * 8 + 127) / 128));
  unsigned char* ring =
      reinterpret_cast<unsigned char*>(tb + 3 * (size_t)a.Vp) + (size_t)warp * a.nstage * a.rowbytes;
  for (int i = threadIdx.x; i < 3 * a.Vp; i += blockDim.x) tb[i] = a.tabs[i];
  const int gw = blockIdx.x * nwarp + warp, stride = gridDim.x * nwarp;
  if (lane == 0) {
    for (int s = 0; s < a.nstage; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // prologue: fill the ring
  if (lane == 0)
    for (int s = 0; s < a.nstage; ++s) {
      const int node = gw + s * stride;
      if (node < a.ndg) {
        mbar_expect_tx(&bars[s], a.rowbytes);
        bulk_load(ring + (size_t)s * a.rowbytes, a.f + (size_t)node * a.Vp, a.rowbytes, &bars[s]);
      }
    }
  const int nq = (int)(a.rowbytes / 16);
  uint32_t parity = 0;  // bit s: parity of stage s
  int s = 0;
  bool aborted = false;
  for (int node = gw; node < a.ndg; node += stride) {
    int ok = 1;
    if (lane == 0) ok = mbar_wait_bounded(&bars[s], (parity >> s) & 1) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) {
      aborted = true;
      break;
    }
    mbar_wait_bounded(&bars[s], (parity >> s) & 1);  // completed: returns at once
    parity ^= 1u << s;
    const T* row = reinterpret_cast<const T*>(ring + (size_t)s * a.rowbytes);
    double s0 = 0, s1 = 0, s2 = 0;
    RowMath<T>::pass1(row, tb, a.Vp, nq, lane, s0, s1, s2);
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    double nd = 0, ux = 0, uy = 0;
    if (s0 >= TINY_D) {  // src/macros.f90:126-134
      nd = s0;
      ux = s1 / s0;
      uy = s2 / s0;
    }
    double sp = 0, sc = 0;
    RowMath<T>::pass2(row, tb, a.Vp, nq, lane, ux, uy, sp, sc);
    sp = warp_sum(sp);
    sc = warp_sum(sc);
    __syncwarp();
    // the row is consumed: refill this stage with the row nstage ahead
    if (lane == 0) {
      const int nxt = node + a.nstage * stride;
      if (nxt < a.ndg) {
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[s], a.rowbytes);
        bulk_load(ring + (size_t)s * a.rowbytes, a.f + (size_t)nxt * a.Vp, a.rowbytes, &bars[s]);
      }
    }
    if (lane == 0) {
      const double ps = sp * a.MM;
      const double ct = (nd >= TINY_D) ? sc / nd : 0.0;
      const double mu = sqrt(2.0) * ct * a.sigt * nd;
      const int e = node / 3, i = node - 3 * (node / 3);
      ElemRec<T>& en = a.rec[e];
      if (ps >= TINY_D) {  // GTEQNF (src/gteqnf.f90:317-326)
        const double rho = a.MM * nd;
        const double b2 = rho / (2 * ps);
        en.A[i] = (T)(nd * (b2 / PI_D));
        en.B[i] = (T)b2;
      } else {
        en.A[i] = (T)0;
        en.B[i] = (T)0;
      }
      en.ux[i] = (T)ux;
      en.uy[i] = (T)uy;
      en.mu[i] = (T)mu;
      a.nraw[node] = s0;
      a.disux[node] = ux;
      a.disuy[node] = uy;
      a.disps[node] = ps;
      a.mu[node] = mu;
      atomicMax(reinterpret_cast<unsigned long long*>(&a.ctrl->maxmu), (unsigned long long)__double_as_longlong(mu));
    }
    s = (s + 1 == a.nstage) ? 0 : s + 1;
  }
  if (aborted && lane == 0) {
    a.ctrl->timeout = 1;
    for (int k = 0; k < a.nstage; ++k) mbar_wait_bounded(&bars[k], (parity >> k) & 1);
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
  int nwall, V, Vp;
};

template <class T> __global__ void __launch_bounds__(256) k_wall(WallArgs<T> a) {
  if (a.ctrl->done) return;
  const int w = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (w >= a.nwall) return;
  const WallSide ws = a.walls[w];
  const T* f1 = a.f + ((size_t)ws.elem * 3 + ws.in1) * a.Vp;
  const T* f2 = a.f + ((size_t)ws.elem * 3 + ws.in2) * a.Vp;
  double s = 0;
  for (int v = lane; v < a.V; v += 32) {
    const double test = a.cx[v] * ws.anx + a.cy[v] * ws.any;
    if (test > 0.0) s += fabs(test) * (0.5 * ((double)f1[v] + (double)f2[v])) * a.wjf[v];
  }
  s = warp_sum(s);
  if (lane == 0) {
    const double eta = s / ws.sumbottom;
    a.beta_d[ws.bside] = eta;
    a.beta_t[ws.bside] = (T)eta;
  }
}

// -------------------------------------------------------------- sweep ----
template <class T> struct SweepArgs {
  T* __restrict__ fout;
  const ElemRec<T>* __restrict__ rec;
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
  int E, V, Vp, EB, slots, nblocks, nvt, immat;
  T alpha, rgas;
};

// DTE = min(CSAFE/maxMU, DTEc)  (src/alotim2.f90:10-15, src/advnce.f90:258-262)
__device__ __forceinline__ double step_dt(const Ctrl* c) {
  const double mx = c->maxmu;
  const double dtb = (mx > 0.0) ? 0.9 * (1.0 / mx) : 1000000.0;
  return fmin(dtb, c->dtc);
}

// NFO of DG node i (src/gteqnf.f90:324-326)
template <class T>
__device__ __forceinline__ T feq_of(const ElemRec<T>& r, int i, T cx, T cy) {
  const T dx = r.ux[i] - cx, dy = r.uy[i] - cy;
  return r.A[i] * dexp<T>(-r.B[i] * (dx * dx + dy * dy));
}

// UMEAN of one element at one velocity (src/getelc.f90:54-83):
// 0.5*DTE*(div F - 1/3 sum MU (NFO - f)), div F = sum (N_i,x cx + N_i,y cy) f_i.
template <class T>
__device__ __forceinline__ T umean_of(const T* f, const T* q, const ElemRec<T>& r, T cx, T cy, T dth) {
  const T dive = (r.gx[0] * cx + r.gy[0] * cy) * f[0] + (r.gx[1] * cx + r.gy[1] * cy) * f[1] +
                 (r.gx[2] * cx + r.gy[2] * cy) * f[2];
  const T coll = r.mu[0] * (q[0] - f[0]) + r.mu[1] * (q[1] - f[1]) + r.mu[2] * (q[2] - f[2]);
  return (dive - coll * (T)(1.0 / 3.0)) * dth;
}

// Shared-memory carve-up of one sweep CTA (bytes): two stages, each =
// f rows [slots][3][32] + element records [EB] + halo record heads
// [slots-EB], 128-aligned; then the UMEAN tile [slots][32]; + 128 bytes of
// slack to align the base at run time.
template <class T> struct SweepSmem {
  unsigned f_bytes, rec_bytes, halo_bytes, stage_bytes, um_bytes, total;
  __host__ __device__ SweepSmem(int EB, int slots) {
    f_bytes = (unsigned)(slots * 3 * VTILE * sizeof(T));
    rec_bytes = (unsigned)(EB * sizeof(ElemRec<T>));
    halo_bytes = (unsigned)((slots - EB) * umean_part_bytes<T>());
    stage_bytes = (f_bytes + rec_bytes + halo_bytes + 127) / 128 * 128;
    um_bytes = (unsigned)(slots * VTILE * sizeof(T));
    total = 2 * stage_bytes + um_bytes + 128;
  }
};

template <class T, int M, int TY>
__global__ void __launch_bounds__(32 * TY) k_sweep(const __grid_constant__ CUtensorMap tm_blk,
                                                   const __grid_constant__ CUtensorMap tm_row3,
                                                   SweepArgs<T> a) {
  if (a.ctrl->done) return;
  constexpr int VT = VTILE;
  constexpr int EB = TY * M;
  constexpr unsigned HB = umean_part_bytes<T>();
  extern __shared__ __align__(128) unsigned char sm_raw[];
  __shared__ uint64_t bars[2];
  __shared__ double red_m[TY], red_s[TY];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const SweepSmem<T> L(EB, a.slots);
  // TMA destinations must be 128-byte aligned: align the base at run time
  unsigned char* base = sm_raw + ((128u - (smem_u32(sm_raw) & 127u)) & 127u);
  T* um_s = reinterpret_cast<T*>(base + 2 * L.stage_bytes);  // [slots][VT]
  const int ntiles = a.nblocks * a.nvt;
  const int G = gridDim.x;

  if (tx == 0 && ty == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // warp 0 issues the copies of tile t into stage s
  auto issue = [&](int t, int s) {
    const int b = t % a.nblocks, vt = t / a.nblocks;
    const int v0 = vt * VT, e0 = b * EB;
    const int nb = min(EB, a.E - e0);
    const int h0 = a.halo_off[b], nh = a.halo_off[b + 1] - h0;
    unsigned char* st = base + s * L.stage_bytes;
    T* dst = reinterpret_cast<T*>(st);
    unsigned char* recd = st + L.f_bytes;
    unsigned char* hald = recd + L.rec_bytes;
    if (tx == 0) {
      const unsigned bytes = (unsigned)((3 * EB + 3 * nh) * VT * sizeof(T)) +
                             (unsigned)(nb * sizeof(ElemRec<T>)) + (unsigned)nh * HB;
      mbar_expect_tx(&bars[s], bytes);
      tma_load_2d(dst, &tm_blk, v0, 3 * e0, &bars[s]);
      bulk_load(recd, a.rec + e0, (unsigned)(nb * sizeof(ElemRec<T>)), &bars[s]);
    }
    __syncwarp();
    for (int h = tx; h < nh; h += 32) {
      const int e = a.halo_list[h0 + h];
      tma_load_2d(dst + (size_t)(EB + h) * 3 * VT, &tm_row3, v0, 3 * e, &bars[s]);
      bulk_load(hald + (size_t)h * HB, a.rec + e, HB, &bars[s]);
    }
  };

  int t = blockIdx.x;
  if (ty == 0) {
    if (t < ntiles) issue(t, 0);
    if (t + G < ntiles) issue(t + G, 1);
  }
  const double dtd = step_dt(a.ctrl);
  const T dt = (T)dtd, dth = (T)(dtd * 0.5);
  double rmax = 0.0, rsq = 0.0;
  uint32_t par = 0;
  int s = 0;
  bool aborted = false;

  for (; t < ntiles; t += G) {
    // every thread waits for the stage itself; a timeout is voted on at the
    // end-of-tile barrier so that all threads leave together
    const bool ok = mbar_wait_bounded(&bars[s], (par >> s) & 1);
    par ^= 1u << s;
    const unsigned char* st = base + s * L.stage_bytes;
    const T* fs = reinterpret_cast<const T*>(st);
    const ElemRec<T>* recs = reinterpret_cast<const ElemRec<T>*>(st + L.f_bytes);
    const unsigned char* halr = st + L.f_bytes + L.rec_bytes;
    const int b = t % a.nblocks, vt = t / a.nblocks;
    const int v = vt * VT + tx;
    const bool vok = v < a.V;
    const T cx = vok ? a.cx[v] : (T)0, cy = vok ? a.cy[v] : (T)0;
    const int e0 = b * EB;
    const int nb = min(EB, a.E - e0);
    const int nh = a.halo_off[b + 1] - a.halo_off[b];

    // phase 1: NFO and N_i,x cx + N_i,y cy of the block (kept in
    // registers) and UMEAN of block + halo
    T q[M][3], sv[M][3], um[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int j = ty + TY * m;
      if (ok && j < nb) {
        const ElemRec<T>& r = recs[j];
        const T f[3] = {fs[(j * 3 + 0) * VT + tx], fs[(j * 3 + 1) * VT + tx], fs[(j * 3 + 2) * VT + tx]};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          q[m][i] = feq_of(r, i, cx, cy);
          sv[m][i] = r.gx[i] * cx + r.gy[i] * cy;
        }
        const T dive = sv[m][0] * f[0] + sv[m][1] * f[1] + sv[m][2] * f[2];
        const T coll = r.mu[0] * (q[m][0] - f[0]) + r.mu[1] * (q[m][1] - f[1]) + r.mu[2] * (q[m][2] - f[2]);
        um[m] = (dive - coll * (T)(1.0 / 3.0)) * dth;
        um_s[j * VT + tx] = um[m];
      }
    }
    for (int h = ty; ok && h < nh; h += TY) {
      const ElemRec<T>& r = *reinterpret_cast<const ElemRec<T>*>(halr + (size_t)h * HB);
      const int j = EB + h;
      const T f[3] = {fs[(j * 3 + 0) * VT + tx], fs[(j * 3 + 1) * VT + tx], fs[(j * 3 + 2) * VT + tx]};
      T qq[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) qq[i] = feq_of(r, i, cx, cy);
      um_s[j * VT + tx] = umean_of(f, qq, r, cx, cy, dth);
    }
    __syncthreads();

    // phase 2: volume + edge terms, increment, positivity, inflow reset
    T rmt = (T)0, sqt = (T)0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int j = ty + TY * m;
      if (ok && j < nb && vok) {
        const int e = e0 + j;
        const ElemRec<T>& r = recs[j];
        const T u = um[m];
        const T f[3] = {fs[(j * 3 + 0) * VT + tx], fs[(j * 3 + 1) * VT + tx], fs[(j * 3 + 2) * VT + tx]};
        // GETELC second half: RHS_i = AREA*(N_i,x FXME + N_i,y FYME)
        const T fm = ((f[0] - u) + (f[1] - u) + (f[2] - u)) * (T)(1.0 / 3.0);
        const T afm = r.area * fm;
        T rhs[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) rhs[i] = sv[m][i] * afm;
        // EDGFLXOPT / GETBOU, gathered per element
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int p = k, qn = (k + 1) % 3;
          const ElemEdge<T> ed = r.edge[k];
          const int kind = ed.info & 3;
          if (kind == 1) continue;  // inflow sides carry no flux
          const T sc = ed.nx * cx + ed.ny * cy;
          T up, uq;
          if (kind == 0) {
            // upwind values without divergence: read the own or the
            // neighbour's rows of the tile, whichever is upwind
            const bool left = (ed.info & 4) != 0;
            const bool mine = left ? (sc > (T)0) : (sc >= (T)0);
            const int sl = mine ? j : (ed.info >> 8);
            const int rp = mine ? p : ((ed.info >> 3) & 3), rq = mine ? qn : ((ed.info >> 5) & 3);
            const T un = mine ? u : um_s[sl * VT + tx];
            up = fs[(sl * 3 + rp) * VT + tx] - un;
            uq = fs[(sl * 3 + rq) * VT + tx] - un;
          } else if (kind == 2 || sc >= (T)0) {
            up = f[p] - u;
            uq = f[qn] - u;
          } else {
            // wall, molecules leaving the wall (src/getbou.f90:189-255): the
            // fully diffuse part ALPHA*ETA*Mw (ALPHA < 1 is not built)
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
          rhs[qn] -= ed.alen * (fnp + (T)2 * fnq);
        }
        // GETINC / CMMINC, ADTHEM, INFLOW
        T sq = (T)0, rm = (T)0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const T x = rhs[i] * dt;
          const T cdt = r.mu[i] * (q[m][i] - f[i]) * dt;
          const T d = r.mm[i] * x + cdt;
          T rr;
          if (a.immat == 1) {
            rr = fabs(d);
          } else {
            const T c = (x >= (T)0) ? a.cmax[3 * e + i] : a.cmin[3 * e + i];
            rr = c * x + cdt;
            rr = rr > (T)0 ? rr : (T)0;
          }
          rm = rr > rm ? rr : rm;
          sq += d * d;
          T fn = f[i] + d;
          if (fn < (T)0) fn = (T)0;
          if (r.inflow & (1 << i)) fn = a.nfinf[v];
          __stcs(a.fout + ((size_t)e * 3 + i) * a.Vp + v, fn);
        }
        rmt = rm > rmt ? rm : rmt;
        sqt += sq;
      }
    }
    rmax = fmax(rmax, (double)rmt);
    rsq += (double)sqt;
    // stage s and um_s are free; all threads learn whether any wait expired
    if (__syncthreads_or(ok ? 0 : 1)) {
      aborted = true;
      break;
    }
    if (ty == 0 && t + 2 * G < ntiles) {
      if (tx == 0) fence_proxy_async_smem();
      __syncwarp();
      issue(t + 2 * G, s);
    }
    s ^= 1;
  }
  if (aborted) {
    // drain this CTA's copies in flight (bounded) before leaving
    if (tx == 0 && ty == 0) {
      a.ctrl->timeout = 1;
      mbar_wait_bounded(&bars[0], par & 1);
      mbar_wait_bounded(&bars[1], (par >> 1) & 1);
    }
    return;
  }
  // per-CTA residual partials (deterministic final reduction in k_resid)
  rmax = warp_max(rmax);
  rsq = warp_sum(rsq);
  if (tx == 0) {
    red_m[ty] = rmax;
    red_s[ty] = rsq;
  }
  __syncthreads();
  if (tx == 0 && ty == 0) {
    double mm = 0, ss = 0;
    for (int w = 0; w < TY; ++w) {
      mm = fmax(mm, red_m[w]);
      ss += red_s[w];
    }
    a.part_max[blockIdx.x] = mm;
    a.part_sq[blockIdx.x] = ss;
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
    if (c->timeout) c->done = 1;
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
// reference DISNF(3,V,E) (old element order) <-> f rows (plan order, pitch Vp)
template <class S, class T>
__global__ void k_to_internal(const S* __restrict__ src, T* __restrict__ dst, const int* __restrict__ inv, int V,
                              int Vp) {
  const int eo = blockIdx.x;
  const size_t en = (size_t)inv[eo];
  const S* s = src + (size_t)eo * 3 * V;
  for (int i = 0; i < 3; ++i)
    for (int v = threadIdx.x; v < V; v += blockDim.x) dst[(en * 3 + i) * Vp + v] = (T)s[(size_t)v * 3 + i];
}

template <class T, class S>
__global__ void k_from_internal(const T* __restrict__ src, S* __restrict__ dst, const int* __restrict__ inv, int V,
                                int Vp) {
  const int eo = blockIdx.x;
  const size_t en = (size_t)inv[eo];
  S* d = dst + (size_t)eo * 3 * V;
  for (int i = 0; i < 3; ++i)
    for (int v = threadIdx.x; v < V; v += blockDim.x) d[(size_t)v * 3 + i] = (S)src[(en * 3 + i) * Vp + v];
}

// INICON2 (src/inicon2.f90:231-262) times an optional per-DG-node scale.
template <class T>
__global__ void k_init_uniform(T* __restrict__ f, const double* __restrict__ g, const double* __restrict__ scale,
                               double n1, int V, int Vp, size_t ndg) {
  const size_t dg = blockIdx.x;
  if (dg >= ndg) return;
  const double sc = scale ? scale[dg] : 1.0;
  for (int v = threadIdx.x; v < V; v += blockDim.x) {
    double val = n1 * g[v];
    if (scale) val = val * sc;
    f[dg * Vp + v] = (T)val;
  }
}

// Maxwellian from per-DG-node (n, u, v, T) (the warm start): the INICON2
// formula with RHO = n*M/NA, P = RHO*R*T, BETA^2 = RHO/(2P).
template <class T>
__global__ void k_init_maxwellian(T* __restrict__ f, const double* __restrict__ prm /* [dg][4] */,
                                  const double* __restrict__ cx, const double* __restrict__ cy, double MM,
                                  double R, int V, int Vp, size_t ndg) {
  const size_t dg = blockIdx.x;
  if (dg >= ndg) return;
  const double n = prm[4 * dg], u = prm[4 * dg + 1], w = prm[4 * dg + 2], t = prm[4 * dg + 3];
  const bool live = n >= TINY_D && t > 0.0;
  const double rho = n * MM, p = rho * R * t;
  const double b2 = live ? rho / (2 * p) : 0.0;
  for (int v = threadIdx.x; v < V; v += blockDim.x) {
    double val = 0.0;
    if (live) {
      const double dx = cx[v] - u, dy = cy[v] - w;
      val = n * ((b2 / PI_D) * exp(-(b2 * (dx * dx + dy * dy))));
    }
    f[dg * Vp + v] = (T)val;
  }
}

}  // namespace dgbgk

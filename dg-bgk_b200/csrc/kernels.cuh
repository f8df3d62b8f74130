// sm_100a kernels of the DG-BGK pseudo-time step.
//
// One step (src/advnce.f90:220-400) is four launches on one stream (five
// with ALPHA < 1: k_wspec after the sweep):
//   k_moments : MACROS passes 1+2 (src/macros.f90:80-154) fused with COMPMU
//               (src/compmu.f90:36-97) and the GTEQNF parameters
//               (src/gteqnf.f90:26-40).  Persistent warps take R whole
//               velocity rows of f at a time (32/R lanes per row) from a
//               per-warp ring of stages filled by 1-D bulk copies, so f is
//               read from HBM once for both passes; every access is a
//               16-byte vector.
//   k_wall    : FLUCON2 (src/flucon2.f90:134-233), one CTA per wall side.
//   k_sweep   : the whole velocity-loop body (GTEQNF, GETFLA, GETELC,
//               EDGFLXOPT/GETBOU, GETINC/CMMINC, ADTHEM, INFLOW;
//               src/advnce.f90:286-377) on tiles of (element block x one
//               64-byte velocity segment).  Persistent CTAs draw work units
//               (a block at several tiles); the block's records are staged
//               once per unit, the tiles' f rows arrive double-buffered (the
//               block's as 2-D TMA boxes, the halo's by cp.async), and each
//               thread works on whole elements at 8 (FP32) or 4 (FP64)
//               velocities.
//   k_resid   : GETRES + the residual bookkeeping (src/advnce.f90:385,
//               422-429), the convergence test and the step counter.
// Every device-side wait on an mbarrier is bounded: on expiry the kernel
// sets Ctrl::timeout, drains its own copies with a second bounded wait and
// returns; the host reports DGBGK_ECUDA.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "exp_tang.h"
#include "types.h"

namespace dgbgk {

constexpr double PI_D = 3.1416;  // the reference's PI
constexpr double TINY_D = 1e-20;
constexpr double LOG2E_D = 1.4426950408889634;  // log2(e)
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
// 1-D bulk copy global -> shared (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// -------------------------------------------------------------- cases ----
// One case (a mesh, its velocity grid and its state) as the kernels see it.
// Every launch works on a table of cases: a single handle is a table of one,
// a batch a table of many.  The work of the launch set is flattened: sweep
// units, moment row groups and wall sides of case c are [off[c], off[c+1]).
template <class T> struct alignas(64) CaseDev {
  CUtensorMap tm[2];  // f[b] as [3E rows][Vp] (sweep tile boxes, 64-byte swizzle)
  T* f[2];            // state, ping-pong; Ctrl::cur is the current one
  ElemRec<T>* rec;
  const int* halo_off;
  const int* halo_list;
  const T* swtab;  // [NTAB][Vp] sweep tables cx, cy, NFINF (, |c|^2), zero past V
  const T* cx;     // rows 0, 1, 2 of swtab
  const T* cy;
  const T* nfinf;
  const T* tabs;   // [MOM_TABS][Vp] moment tables: cx, cy, w = WEIGHT*JAC*FRAC, w*cx, w*cy; zero past V
  const T* bTw;    // per boundary side: wall temperature, wall velocity (x, y), ETA
  const T* bUw;
  T* bEta;
  double* bEtaD;
  const double* cxD;  // [V] FP64 velocity tables for FLUCON2
  const double* cyD;
  const double* wjf;
  const WallSide* walls;
  const T* cmax;   // IMMAT = 0 residual tables
  const T* cmin;
  double* nraw;    // per DG node: INT (number density before the 1e-20 test)
  double* disux;
  double* disuy;
  double* disps;
  double* mu;
  double* hist_linf;  // per step of an advance call
  double* hist_l2;
  double* hist_dt;
  Ctrl* ctrl;
  double MM, sigt;  // M/NA, PI*d*d
  T alpha, rgas;
  int E, V, Vp, nblocks, nvt;
  int tpu, nreg, ngrp, halve;  // velocity-tile groups of the sweep's units (sweep_group)
  int nwall;          // FLUCON2 wall sides
  unsigned rowbytes;  // V*sizeof(T) rounded up to 16
  // ALPHA < 1: the specular part of the wall flux (the host plan's tables)
  int spec;                 // 0: ALPHA = 1 or no wall side
  int immat;                // 1: lumped mass (GETINC), 0: CMMINC
  int n_spec_par, n_spec_slots;
  const int* rside;         // [B] reflection-table row, -1 off the walls
  const int* rf_i;          // [rows][V][2] mirrored grid velocities I1, I2; -1 where TEST >= 0
  const T* rf_z;            // [rows][V][2] ZD1, ZD2
  const int* welem;         // [slots] wall elements (plan order)
  T* wd;                    // deferred values: IMMAT = 1 [slots][3][Vp] DELUN without the specular part;
                            // IMMAT = 0 [2][slots][3][Vp] RHS*DTE without it, COLL*DTE
  const int* spec_par;      // items slot*V + v
  const int* spec_seq_off;  // [slots + 1]
  const int* spec_seq;
};

// Size of the next group of the sweep's tail when r tiles remain: half of
// them, rounded up (two or one at the end).
__host__ __device__ inline int sweep_tail_tiles(int r) { return r <= 2 ? r : (r + 1) / 2; }

// Tiles [vt0, vt0 + ntl) of velocity-tile group g: groups below nreg hold
// tpu tiles, the rest is one group or (halve) shrinking groups
// (sweep_tail_tiles).
template <class T> __device__ __forceinline__ void sweep_group(const CaseDev<T>& C, int g, int& vt0, int& ntl) {
  if (g < C.nreg) {
    vt0 = g * C.tpu;
    ntl = C.tpu;
    return;
  }
  int s = C.nreg * C.tpu, r = C.nvt - s;
  if (!C.halve) {
    vt0 = s;
    ntl = r;
    return;
  }
  for (int m = C.nreg; m < g; ++m) {
    const int n = sweep_tail_tiles(r);
    s += n;
    r -= n;
  }
  vt0 = s;
  ntl = sweep_tail_tiles(r);
}

// Moment tables: the row modes read the first three; the element mode of a
// single case (tables in shared memory) rows 2 to 4 in its first pass and 0
// to 2 in its second, of a batch (tables through L1) the first three.
constexpr int MOM_TABS = 5;
__host__ __device__ constexpr int mom_tables(int R) { return R == 3 ? 5 : 3; }

template <class T> struct BatchArgs {
  const CaseDev<T>* cases;  // [ncases]
  const int* unit_off;      // [ncases + 1] sweep work units
  const int* grp_off;       // [ncases + 1] moment row groups
  const int* wall_off;      // [ncases + 1] wall sides
  BatchCtl* ctl;
  int ncases;
  int max_halo;             // over the cases (sweep tile layout)
  int mom_stages;           // moment ring stages per warp
  unsigned mom_rowbytes;    // moment ring row size (max over the cases)
};

// The case c with off[c] <= x < off[c + 1] (cases with empty ranges are
// skipped: the largest c with off[c] <= x).
__device__ __forceinline__ int find_case(const int* __restrict__ off, int n, int x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------ moments ----

// sqrt by a reciprocal-square-root seed and one Newton step for 1/sqrt(x),
// y <- y (3 - x y^2)/2, in FP64 (relative error ~1e-14 from a ~1e-7 seed).
__device__ __forceinline__ float rsqrt_sfu(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double sqrt_newton(double x) {
  const float xf = (float)x;
  if (!(xf > 0.f)) return 0.0;
  const double y0 = (double)rsqrt_sfu(xf);
  const double y1 = y0 * (1.5 - 0.5 * x * y0 * y0);
  return x * y1;
}
// FP32 sqrt from the SFU (sqrt.approx: relative error ~2^-23; sqrt(0) = 0)
__device__ __forceinline__ float sqrt_fast(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Pass sums over one velocity row in shared memory by the L lanes of a
// group (lane sub takes 16-byte vectors sub, sub+L, ...).  FP64 storage:
// FP64 arithmetic.  FP32 storage: FP32 arithmetic; each lane's partial sums
// (V/(4L) vectors) are converted to FP64 before the group sum.
template <class T> struct RowMath;

template <> struct RowMath<double> {
  static __device__ __forceinline__ void pass1(const double* row, const double* tb, int Vp, int nq, int sub, int L,
                                               double& s0, double& s1, double& s2) {
    const double2* r = reinterpret_cast<const double2*>(row);
    const double2* cx = reinterpret_cast<const double2*>(tb);
    const double2* cy = reinterpret_cast<const double2*>(tb + Vp);
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
    for (int q = sub; q < nq; q += L) {
      const double2 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const double a0 = w.x * x.x, a1 = w.y * x.y;
      s0 += a0 + a1;
      s1 = fma(c.x, a0, fma(c.y, a1, s1));
      s2 = fma(d.x, a0, fma(d.y, a1, s2));
    }
  }
  static __device__ __forceinline__ void pass2(const double* row, const double* tb, int Vp, int nq, int sub, int L,
                                               double ux, double uy, double& sp, double& sc) {
    const double2* r = reinterpret_cast<const double2*>(row);
    const double2* cx = reinterpret_cast<const double2*>(tb);
    const double2* cy = reinterpret_cast<const double2*>(tb + Vp);
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
    for (int q = sub; q < nq; q += L) {
      const double2 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const double dx0 = c.x - ux, dy0 = d.x - uy, dx1 = c.y - ux, dy1 = d.y - uy;
      const double q0 = dx0 * dx0 + dy0 * dy0, q1 = dx1 * dx1 + dy1 * dy1;
      const double a0 = w.x * x.x, a1 = w.y * x.y;
      sp = fma(0.5 * q0, a0, fma(0.5 * q1, a1, sp));                // src/macros.f90:144-148
      sc = fma(sqrt_newton(q0), a0, fma(sqrt_newton(q1), a1, sc));  // src/compmu.f90:71-74
    }
  }
};

__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

template <> struct RowMath<float> {
  // on packed pairs (fma/add/mul.rn.f32x2): each sum as two partial sums,
  // the halves of one pair (the even and the odd values of a vector)
  static __device__ __forceinline__ void pass1(const float* row, const float* tb, int Vp, int nq, int sub, int L,
                                               double& s0, double& s1, double& s2) {
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* cx = reinterpret_cast<const float4*>(tb);
    const float4* cy = reinterpret_cast<const float4*>(tb + Vp);
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    float2 t0 = make_float2(0.f, 0.f), t1 = t0, t2 = t0;
    for (int q = sub; q < nq; q += L) {
      const float4 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const float2 al = __fmul2_rn(lo2(w), lo2(x)), ah = __fmul2_rn(hi2(w), hi2(x));
      t0 = __fadd2_rn(t0, __fadd2_rn(al, ah));
      t1 = __ffma2_rn(lo2(c), al, __ffma2_rn(hi2(c), ah, t1));
      t2 = __ffma2_rn(lo2(d), al, __ffma2_rn(hi2(d), ah, t2));
    }
    s0 += (double)t0.x + (double)t0.y;
    s1 += (double)t1.x + (double)t1.y;
    s2 += (double)t2.x + (double)t2.y;
  }
  static __device__ __forceinline__ void pass2(const float* row, const float* tb, int Vp, int nq, int sub, int L,
                                               double ux, double uy, double& sp, double& sc) {
    const float2 nx = make_float2(-(float)ux, -(float)ux), ny = make_float2(-(float)uy, -(float)uy);
    const float4* r = reinterpret_cast<const float4*>(row);
    const float4* cx = reinterpret_cast<const float4*>(tb);
    const float4* cy = reinterpret_cast<const float4*>(tb + Vp);
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    float2 tp = make_float2(0.f, 0.f), tc = tp;
    for (int q = sub; q < nq; q += L) {
      const float4 x = r[q], c = cx[q], d = cy[q], w = wj[q];
      const float2 el = __fadd2_rn(lo2(c), nx), eh = __fadd2_rn(hi2(c), nx);
      const float2 gl = __fadd2_rn(lo2(d), ny), gh = __fadd2_rn(hi2(d), ny);
      const float2 ql = __ffma2_rn(el, el, __fmul2_rn(gl, gl)), qh = __ffma2_rn(eh, eh, __fmul2_rn(gh, gh));
      const float2 al = __fmul2_rn(lo2(w), lo2(x)), ah = __fmul2_rn(hi2(w), hi2(x));
      tp = __ffma2_rn(ql, al, __ffma2_rn(qh, ah, tp));
      const float2 sl = make_float2(sqrt_fast(ql.x), sqrt_fast(ql.y));
      const float2 sh = make_float2(sqrt_fast(qh.x), sqrt_fast(qh.y));
      tc = __ffma2_rn(sl, al, __ffma2_rn(sh, ah, tc));
    }
    sp += 0.5 * ((double)tp.x + (double)tp.y);
    sc += (double)tc.x + (double)tc.y;
  }
};

// Pass sums over the three velocity rows of one element by all 32 lanes of
// a warp (lane l takes 16-byte vectors l, l+32, ...): the velocity tables
// are loaded once per vector for the three rows.  FP32 storage: FP32 lane
// partials, summed in FP64 across the warp; FP64 storage: FP64 throughout.
template <class T> struct ElemMath;

template <> struct ElemMath<float> {
  // Each sum runs as two partial sums, the even and the odd values of a
  // vector (shorter dependent chains: 0.1535 -> 0.1508 ms on the 200x100
  // channel; four partials were slower).  Where the two partial sums take
  // the same operations, they are the halves of one packed pair
  // (fma/add/mul.rn.f32x2: one instruction for two values; the same bits
  // as two scalar chains; 0.1527 -> 0.1456 ms).
  // pass 1.  TAB: from the tables w, w*cx, w*cy (three FMAs per value;
  // tables in shared memory); otherwise from w, cx, cy (w*f, then three
  // sums; the tables the second pass reads too, through L1)
  template <bool TAB>
  static __device__ __forceinline__ void pass1(const float* rows, unsigned pitch, const float* tb, int Vp, int nq,
                                               int lane, double (&s)[3][3]) {
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    const float4* wx = reinterpret_cast<const float4*>(tb + (TAB ? 3 : 0) * Vp);
    const float4* wy = reinterpret_cast<const float4*>(tb + (TAB ? 4 : 1) * Vp);
    if constexpr (TAB) {
      float2 t[3][3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) t[r][k] = make_float2(0.f, 0.f);
      for (int q = lane; q < nq; q += 32) {
        const float4 w = wj[q], c = wx[q], d = wy[q];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const float4 x =
              reinterpret_cast<const float4*>(reinterpret_cast<const unsigned char*>(rows) + r * pitch)[q];
          t[r][0] = __ffma2_rn(lo2(w), lo2(x), __ffma2_rn(hi2(w), hi2(x), t[r][0]));
          t[r][1] = __ffma2_rn(lo2(c), lo2(x), __ffma2_rn(hi2(c), hi2(x), t[r][1]));
          t[r][2] = __ffma2_rn(lo2(d), lo2(x), __ffma2_rn(hi2(d), hi2(x), t[r][2]));
        }
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) s[r][k] = (double)t[r][k].x + (double)t[r][k].y;
    } else {
      float t[3][3] = {};
      for (int q = lane; q < nq; q += 32) {
        const float4 w = wj[q], c = wx[q], d = wy[q];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const float4 x =
              reinterpret_cast<const float4*>(reinterpret_cast<const unsigned char*>(rows) + r * pitch)[q];
          const float a0 = w.x * x.x, a1 = w.y * x.y, a2 = w.z * x.z, a3 = w.w * x.w;
          t[r][0] += (a0 + a1) + (a2 + a3);
          t[r][1] = fmaf(c.x, a0, fmaf(c.y, a1, fmaf(c.z, a2, fmaf(c.w, a3, t[r][1]))));
          t[r][2] = fmaf(d.x, a0, fmaf(d.y, a1, fmaf(d.z, a2, fmaf(d.w, a3, t[r][2]))));
        }
      }
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) s[r][k] = (double)t[r][k];
    }
  }
  // pass 2 on packed pairs (c - u as c + (-u))
  static __device__ __forceinline__ void pass2(const float* rows, unsigned pitch, const float* tb, int Vp, int nq,
                                               int lane, const double (&u)[3][2], double (&s)[3][2]) {
    const float4* cx = reinterpret_cast<const float4*>(tb);
    const float4* cy = reinterpret_cast<const float4*>(tb + Vp);
    const float4* wj = reinterpret_cast<const float4*>(tb + 2 * Vp);
    float2 nu[3][2], t[3][2];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const float ux = (float)u[r][0], uy = (float)u[r][1];
      nu[r][0] = make_float2(-ux, -ux);
      nu[r][1] = make_float2(-uy, -uy);
      t[r][0] = t[r][1] = make_float2(0.f, 0.f);
    }
    for (int q = lane; q < nq; q += 32) {
      const float4 c = cx[q], d = cy[q], w = wj[q];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const float4 x = reinterpret_cast<const float4*>(reinterpret_cast<const unsigned char*>(rows) + r * pitch)[q];
        const float2 el = __fadd2_rn(lo2(c), nu[r][0]), eh = __fadd2_rn(hi2(c), nu[r][0]);
        const float2 gl = __fadd2_rn(lo2(d), nu[r][1]), gh = __fadd2_rn(hi2(d), nu[r][1]);
        const float2 ql = __ffma2_rn(el, el, __fmul2_rn(gl, gl)), qh = __ffma2_rn(eh, eh, __fmul2_rn(gh, gh));
        const float2 al = __fmul2_rn(lo2(w), lo2(x)), ah = __fmul2_rn(hi2(w), hi2(x));
        t[r][0] = __ffma2_rn(ql, al, __ffma2_rn(qh, ah, t[r][0]));  // src/macros.f90:144-148
        const float2 sl = make_float2(sqrt_fast(ql.x), sqrt_fast(ql.y));
        const float2 sh = make_float2(sqrt_fast(qh.x), sqrt_fast(qh.y));
        t[r][1] = __ffma2_rn(sl, al, __ffma2_rn(sh, ah, t[r][1]));  // src/compmu.f90:71-74
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      s[r][0] = 0.5 * ((double)t[r][0].x + (double)t[r][0].y);
      s[r][1] = (double)t[r][1].x + (double)t[r][1].y;
    }
  }
};

template <> struct ElemMath<double> {
  // pass 1, TAB as for FP32
  template <bool TAB>
  static __device__ __forceinline__ void pass1(const double* rows, unsigned pitch, const double* tb, int Vp, int nq,
                                               int lane, double (&s)[3][3]) {
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
    const double2* wx = reinterpret_cast<const double2*>(tb + (TAB ? 3 : 0) * Vp);
    const double2* wy = reinterpret_cast<const double2*>(tb + (TAB ? 4 : 1) * Vp);
#pragma unroll
    for (int r = 0; r < 3; ++r) s[r][0] = s[r][1] = s[r][2] = 0.0;
    for (int q = lane; q < nq; q += 32) {
      const double2 w = wj[q], c = wx[q], d = wy[q];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double2 x = reinterpret_cast<const double2*>(reinterpret_cast<const unsigned char*>(rows) + r * pitch)[q];
        if constexpr (TAB) {
          s[r][0] = fma(w.x, x.x, fma(w.y, x.y, s[r][0]));
          s[r][1] = fma(c.x, x.x, fma(c.y, x.y, s[r][1]));
          s[r][2] = fma(d.x, x.x, fma(d.y, x.y, s[r][2]));
        } else {
          const double a0 = w.x * x.x, a1 = w.y * x.y;
          s[r][0] += a0 + a1;
          s[r][1] = fma(c.x, a0, fma(c.y, a1, s[r][1]));
          s[r][2] = fma(d.x, a0, fma(d.y, a1, s[r][2]));
        }
      }
    }
  }
  static __device__ __forceinline__ void pass2(const double* rows, unsigned pitch, const double* tb, int Vp, int nq,
                                               int lane, const double (&u)[3][2], double (&s)[3][2]) {
    const double2* cx = reinterpret_cast<const double2*>(tb);
    const double2* cy = reinterpret_cast<const double2*>(tb + Vp);
    const double2* wj = reinterpret_cast<const double2*>(tb + 2 * Vp);
#pragma unroll
    for (int r = 0; r < 3; ++r) s[r][0] = s[r][1] = 0.0;
    for (int q = lane; q < nq; q += 32) {
      const double2 c = cx[q], d = cy[q], w = wj[q];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double2 x = reinterpret_cast<const double2*>(reinterpret_cast<const unsigned char*>(rows) + r * pitch)[q];
        const double dx0 = c.x - u[r][0], dy0 = d.x - u[r][1], dx1 = c.y - u[r][0], dy1 = d.y - u[r][1];
        const double q0 = dx0 * dx0 + dy0 * dy0, q1 = dx1 * dx1 + dy1 * dy1;
        const double a0 = w.x * x.x, a1 = w.y * x.y;
        s[r][0] = fma(0.5 * q0, a0, fma(0.5 * q1, a1, s[r][0]));                // src/macros.f90:144-148
        s[r][1] = fma(sqrt_newton(q0), a0, fma(sqrt_newton(q1), a1, s[r][1]));  // src/compmu.f90:71-74
      }
    }
  }
};

// MACROS / COMPMU / GTEQNF per DG node from its velocity sums
// (src/macros.f90:126-154, src/compmu.f90:86-97, src/gteqnf.f90:28-37):
// s0 = n (before the 1e-20 test), (ux, uy), nd = n or 0, sp = the pressure
// sum over M/NA, sc = the mean-relative-speed sum; writes the node's
// moments, MU and the sweep's NFO parameters, returns MU.
template <class T>
__device__ __forceinline__ double node_epilogue(const CaseDev<T>& C, int node, double s0, double ux, double uy,
                                                double nd, double sp, double sc) {
  const double ps = sp * C.MM;
  const double ct = (nd >= TINY_D) ? sc / nd : 0.0;
  const double mu = sqrt(2.0) * ct * C.sigt * nd;
  const int e = node / 3, i = node - 3 * (node / 3);
  ElemRec<T>& en = C.rec[e];
  // GTEQNF's parameters; FP64 in the expanded exponent form of the sweep
  // (ElemRec)
  if (ps >= TINY_D) {
    const double rho = C.MM * nd;
    const double b2 = rho / (2 * ps);
    const double a = nd * (b2 / PI_D);
    if (sizeof(T) == 4) {
      en.A[i] = (T)a;
      en.ex[i] = (T)(-b2 * LOG2E_D);
      en.ux[i] = (T)ux;
      en.uy[i] = (T)uy;
    } else {
      en.A[i] = (T)(log(a) - b2 * (ux * ux + uy * uy));
      en.ex[i] = (T)(-b2);
      en.ux[i] = (T)(2.0 * b2 * ux);
      en.uy[i] = (T)(2.0 * b2 * uy);
    }
  } else {
    en.A[i] = (T)(sizeof(T) == 4 ? 0.0 : -INFINITY);
    en.ex[i] = (T)0;
    en.ux[i] = (T)(sizeof(T) == 4 ? ux : 0.0);
    en.uy[i] = (T)(sizeof(T) == 4 ? uy : 0.0);
  }
  en.mu[i] = (T)mu;
  C.nraw[node] = s0;
  C.disux[node] = ux;
  C.disuy[node] = uy;
  C.disps[node] = ps;
  C.mu[node] = mu;
  return mu;
}

// Sum over the L lanes of an aligned lane group (every lane gets the same
// bits: each butterfly level adds the same two operands in either order).
template <int L> __device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Moment kernel: persistent warps over the flattened row groups of all the
// cases; each warp takes R DG nodes (velocity rows) at a time, L = 32/R
// lanes per row, from a per-warp ring of stages filled by 1-D bulk copies,
// so f is read from HBM once for both passes.  ONE: a single case, passed
// as a kernel parameter, with its velocity tables staged in shared memory;
// otherwise the case table, with the tables read through L1 (they differ
// from case to case).  MU's maximum goes to the case's control block once
// per warp and case.  Up to 20 warps per CTA for a single case (at
// most 96 registers), 16 for the case table.
template <class T, int R, bool ONE>
__global__ void __launch_bounds__(ONE ? 640 : 512, 1)
    k_moments(BatchArgs<T> a, int total_groups, const __grid_constant__ CaseDev<T> one) {
  // R = 1, 2, 4: R rows of any elements per warp step, 32/R lanes per row;
  // R = 3: the three rows of one element per warp step, all 32 lanes on
  // each (the velocity tables loaded once for the three rows)
  constexpr bool ELEM = R == 3;
  constexpr int L = ELEM ? 32 : 32 / R;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int grp = ELEM ? 0 : lane / L, sub = lane % L;
  const int nstage = a.mom_stages;
  // layout: [barriers][tables [3][Vp] (ONE)][rings: warp, stage, R rows]
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm_raw) + warp * nstage;
  T* tb1 = reinterpret_cast<T*>(sm_raw + 128 * (((size_t)nwarp * nstage * 8 + 127) / 128));
  constexpr int NTB = mom_tables(R);  // tables staged for a single case
  const size_t tbytes = ONE ? (NTB * (size_t)one.Vp * sizeof(T) + 127) / 128 * 128 : 0;
  const size_t stage_bytes = (size_t)R * a.mom_rowbytes;
  unsigned char* ring = reinterpret_cast<unsigned char*>(tb1) + tbytes + (size_t)warp * nstage * stage_bytes;
  if (ONE)
    for (int i = threadIdx.x; i < NTB * one.Vp; i += blockDim.x) tb1[i] = one.tabs[i];
  const int gw = blockIdx.x * nwarp + warp, stride = gridDim.x * nwarp;
  if (lane == 0) {
    for (int s = 0; s < nstage; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // lane 0: the rows of group g into stage s (none when the case is done)
  auto fill = [&](int s, int g) {
    const int c = ONE ? 0 : find_case(a.grp_off, a.ncases, g);
    const CaseDev<T>& C = ONE ? one : a.cases[c];
    const Ctrl* ctl = C.ctrl;
    const int r0 = (g - (ONE ? 0 : a.grp_off[c])) * R;
    const int nr = ctl->done ? 0 : min(R, 3 * C.E - r0);
    const T* f = C.f[ctl->cur];
    mbar_expect_tx(&bars[s], (unsigned)nr * C.rowbytes);
    for (int k = 0; k < nr; ++k)
      bulk_load(ring + (size_t)s * stage_bytes + (size_t)k * C.rowbytes, f + (size_t)(r0 + k) * C.Vp, C.rowbytes,
                &bars[s]);
  };
  if (lane == 0)
    for (int s = 0; s < nstage; ++s)
      if (gw + s * stride < total_groups) fill(s, gw + s * stride);
  uint32_t parity = 0;  // bit s: parity of stage s
  int s = 0;
  bool aborted = false;
  int mu_case = -1;
  double mumax = 0.0;
  // MU >= 0: the max of the bit patterns is the max of the values
  auto flush_mu = [&]() {
    const double m = warp_max(mumax);
    if (lane == 0 && mu_case >= 0 && m > 0.0)
      atomicMax(reinterpret_cast<unsigned long long*>(&(ONE ? one : a.cases[mu_case]).ctrl->maxmu),
                (unsigned long long)__double_as_longlong(m));
    mumax = 0.0;
  };
  int c = 0;
  for (int g = gw; g < total_groups; g += stride) {
    c = ONE ? 0 : find_case(a.grp_off, a.ncases, g);  // warp-uniform
    int ok = 1;
    if (lane == 0) ok = mbar_wait_bounded(&bars[s], (parity >> s) & 1) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) {
      aborted = true;
      break;
    }
    mbar_wait_bounded(&bars[s], (parity >> s) & 1);  // completed: returns at once
    parity ^= 1u << s;
    const CaseDev<T>& C = ONE ? one : a.cases[c];
    if (c != mu_case) {
      flush_mu();
      mu_case = c;
    }
    const int node0 = (g - (ONE ? 0 : a.grp_off[c])) * R;
    const T* tb = ONE ? tb1 : C.tabs;
    const bool live0 = !C.ctrl->done;
    const int nql = live0 ? (int)(C.rowbytes / 16) : 0;
    // this lane's node and its sums: s0 = n, ux, uy (MACROS pass 1), sp, sc
    // (pass 2: pressure and COMPMU's mean relative speed)
    int node;
    double s0, ux, uy, nd, sp, sc;
    if constexpr (ELEM) {
      const T* rows = reinterpret_cast<const T*>(ring + (size_t)s * stage_bytes);
      double m1[3][3], u[3][2], m2[3][2];
      ElemMath<T>::template pass1<ONE>(rows, C.rowbytes, tb, C.Vp, nql, lane, m1);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int k = 0; k < 3; ++k) m1[r][k] = group_sum<32>(m1[r][k]);
        u[r][0] = u[r][1] = 0.0;
        if (m1[r][0] >= TINY_D) {  // src/macros.f90:126-134
          const double inv = 1.0 / m1[r][0];
          u[r][0] = m1[r][1] * inv;
          u[r][1] = m1[r][2] * inv;
        }
      }
      ElemMath<T>::pass2(rows, C.rowbytes, tb, C.Vp, nql, lane, u, m2);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        m2[r][0] = group_sum<32>(m2[r][0]);
        m2[r][1] = group_sum<32>(m2[r][1]);
      }
      // lanes 0, 1, 2 write rows 0, 1, 2
      const int r = lane < 3 ? lane : 0;
      node = node0 + r;
      s0 = r == 0 ? m1[0][0] : r == 1 ? m1[1][0] : m1[2][0];
      ux = r == 0 ? u[0][0] : r == 1 ? u[1][0] : u[2][0];
      uy = r == 0 ? u[0][1] : r == 1 ? u[1][1] : u[2][1];
      sp = r == 0 ? m2[0][0] : r == 1 ? m2[1][0] : m2[2][0];
      sc = r == 0 ? m2[0][1] : r == 1 ? m2[1][1] : m2[2][1];
      nd = s0 >= TINY_D ? s0 : 0.0;
    } else {
      node = node0 + grp;
      const T* row = reinterpret_cast<const T*>(ring + (size_t)s * stage_bytes + (size_t)grp * C.rowbytes);
      const int nqr = node < 3 * C.E ? nql : 0;
      double s1 = 0, s2 = 0;
      s0 = 0;
      RowMath<T>::pass1(row, tb, C.Vp, nqr, sub, L, s0, s1, s2);
      s0 = group_sum<L>(s0);
      s1 = group_sum<L>(s1);
      s2 = group_sum<L>(s2);
      nd = ux = uy = 0;
      if (s0 >= TINY_D) {  // src/macros.f90:126-134
        nd = s0;
        const double inv = 1.0 / s0;
        ux = s1 * inv;
        uy = s2 * inv;
      }
      sp = sc = 0;
      RowMath<T>::pass2(row, tb, C.Vp, nqr, sub, L, ux, uy, sp, sc);
      sp = group_sum<L>(sp);
      sc = group_sum<L>(sc);
    }
    const bool live = live0 && node < 3 * C.E;
    __syncwarp();
    // the rows are consumed: refill this stage with the group nstage ahead
    if (lane == 0) {
      const int nxt = g + nstage * stride;
      if (nxt < total_groups) {
        fence_proxy_async_smem();
        fill(s, nxt);
      }
    }
    if ((ELEM ? lane < 3 : sub == 0) && live) mumax = fmax(mumax, node_epilogue(C, node, s0, ux, uy, nd, sp, sc));
    s = (s + 1 == nstage) ? 0 : s + 1;
  }
  if (aborted) {
    if (lane == 0) {
      (ONE ? one : a.cases[c]).ctrl->timeout = 1;
      for (int k = 0; k < nstage; ++k) mbar_wait_bounded(&bars[k], (parity >> k) & 1);
    }
    return;
  }
  flush_mu();
}

// --------------------------------------------------------- wall flux ----
// FLUCON2 (src/flucon2.f90:134-233): one CTA (WALL_THREADS threads) per
// wall side of any case, its threads strided over the velocities, then a
// block sum (a warp per side left the loads of a side in a serial chain:
// ~37 us on the 200x100 channel's 40 wall sides).
constexpr int WALL_THREADS = 256;
template <class T> __global__ void __launch_bounds__(WALL_THREADS) k_wall(BatchArgs<T> a, int total_walls) {
  __shared__ double part[WALL_THREADS / 32];
  const int w = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (w >= total_walls) return;
  const int c = find_case(a.wall_off, a.ncases, w);
  const CaseDev<T>& C = a.cases[c];
  if (C.ctrl->done) return;  // the same for the whole CTA
  const WallSide ws = C.walls[w - a.wall_off[c]];
  const T* f = C.f[C.ctrl->cur];
  const T* f1 = f + ((size_t)ws.elem * 3 + ws.in1) * C.Vp;
  const T* f2 = f + ((size_t)ws.elem * 3 + ws.in2) * C.Vp;
  double s = 0;
  for (int v = threadIdx.x; v < C.V; v += WALL_THREADS) {
    const double test = C.cxD[v] * ws.anx + C.cyD[v] * ws.any;
    if (test > 0.0) s += fabs(test) * (0.5 * ((double)f1[v] + (double)f2[v])) * C.wjf[v];
  }
  s = warp_sum(s);
  if (lane == 0) part[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
#pragma unroll
    for (int k = 0; k < WALL_THREADS / 32; ++k) t += part[k];
    const double eta = t / ws.sumbottom;
    C.bEtaD[ws.bside] = eta;
    C.bEta[ws.bside] = (T)eta;
  }
}

// -------------------------------------------------------------- sweep ----
// DTE = min(CSAFE/maxMU, DTEc)  (src/alotim2.f90:10-15, src/advnce.f90:258-262)
__device__ __forceinline__ double step_dt(const Ctrl* c) {
  const double mx = c->maxmu;
  const double dtb = (mx > 0.0) ? 0.9 * (1.0 / mx) : 1000000.0;
  return fmin(dtb, c->dtc);
}

// Sweep tile geometry.  A tile is one 64-byte segment of velocities (16 FP32
// or 8 FP64 values) of the three rows of every element of a block and of its
// halo: row r = 3*slot + i (block element j: slot j; halo element h: slot
// EB + h), 64 bytes per row, with the 16-byte chunks of a row permuted by the
// 64-byte swizzle (chunk c of row r at 16*(c ^ ((r >> 1) & 3))).  The block's
// rows arrive as 2-D TMA boxes that apply this swizzle, the halo rows by
// cp.async copies that apply it by hand; with it, eight threads that each
// read their own element's row with 16-byte vectors fall on eight distinct
// bank groups.  A work unit is one block at `tpu` consecutive velocity
// tiles: the block's element records and the halo's record heads are staged
// in shared memory once per unit, the f rows once per tile (double-buffered).
template <class T> struct SweepGeo {
  static constexpr int W = 16 / (int)sizeof(T);  // values per 16-byte vector
  static constexpr int VT = 64 / (int)sizeof(T);  // velocities per tile
  static constexpr int NCH = 4;                   // 16-byte chunks per row segment
  // threads per block element in the sweep, each taking NCH / TPE chunks.
  // Two for both precisions: on the Mach 2 channel (200x100, 24x48) four
  // threads per element made the FP32 sweep 0.42 -> 0.55 ms, and the FP64
  // sweep (16 warps per SM but 128 registers, spilling) slower than two
  // threads at 8 warps and 226 registers without spills
#ifndef DGBGK_SWEEP_TPE32
#define DGBGK_SWEEP_TPE32 2
#endif
#ifndef DGBGK_SWEEP_TPE64
#define DGBGK_SWEEP_TPE64 2
#endif
  static constexpr int TPE = sizeof(T) == 4 ? DGBGK_SWEEP_TPE32 : DGBGK_SWEEP_TPE64;
  static constexpr int CPT = NCH / TPE;           // chunks per thread
  static_assert(TPE == 2 || TPE == 4, "two or four threads per element");
  static constexpr int BOX_ROWS = 192;            // rows of one TMA box
  static constexpr int RW = (int)(sizeof(ElemRec<T>) / 16);                    // record words
  static constexpr int HW = (REC_HEAD_VALUES * (int)sizeof(T) + 15) / 16;        // head words
  static constexpr int HR = 16 * (HW | 1);  // halo head pitch (odd number of words)
  static constexpr int TPU_MAX = 16;
  // velocity tables staged per unit: cx, cy, NFINF (and |c|^2 for the FP64
  // exponent)
  static constexpr int NTAB = sizeof(T) == 8 ? 4 : 3;
  // one tile buffer, 1024-byte aligned
  static constexpr size_t tile_bytes(int EB, int max_halo) {
    return ((size_t)3 * (EB + max_halo) * 64 + 1023) / 1024 * 1024;
  }
  // alignment slack, two tiles, records [EB], halo heads [max_halo][HR],
  // velocity tables [NTAB][TPU_MAX * VT], halo row list [3 * max_halo]
  static constexpr size_t smem(int EB, int max_halo) {
    return 1024 + 2 * tile_bytes(EB, max_halo) + (size_t)EB * sizeof(ElemRec<T>) + (size_t)max_halo * HR +
           NTAB * (size_t)TPU_MAX * VT * sizeof(T) + ((size_t)3 * max_halo * 4 + 15) / 16 * 16;
  }
};


// A tensor map read from global memory (the batch's case table, written by
// a host copy) must be acquired by the tensormap proxy before a thread uses
// it; one fence per map and thread.  Maps passed as __grid_constant__
// parameters need none.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* p) {
  asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(p) : "memory");
}

// 2-D tiled TMA load (no multicast) of one box into shared memory.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// 2-D tiled TMA store of one box from shared memory (elements outside the
// tensor are not written), tracked by the issuing thread's bulk groups.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map), "r"(x),
               "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... all but the most recent one
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
// ... and their writes are complete
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared through L2 only (cp.async.cg).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// exp of the NFO exponent: FP64 by Tang's table-driven method (exp_tang.h,
// about one ulp, `tab` the CTA's 2^(j/64) table); FP32 2^x from the SFU
// (ex2.approx, relative error ~2^-22; the FP32 coefficient carries the
// log2(e) factor, applied in FP64 by the moment kernel; no table).
template <class T> __device__ __forceinline__ T nfo_exp(T x, const double* tab);
template <> __device__ __forceinline__ double nfo_exp<double>(double x, const double* tab) {
  return exp_tang(x, tab);
}
template <> __device__ __forceinline__ float nfo_exp<float>(float x, const double*) {
  float p;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p) : "f"(x));
  return p;
}

template <class T> struct Vec;
template <> struct Vec<float> {
  using type = float4;
  static __device__ __forceinline__ float get(const float4& v, int k) {
    return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
  }
  static __device__ __forceinline__ void set(float4& v, int k, float x) {
    if (k == 0)
      v.x = x;
    else if (k == 1)
      v.y = x;
    else if (k == 2)
      v.z = x;
    else
      v.w = x;
  }
};
template <> struct Vec<double> {
  using type = double2;
  static __device__ __forceinline__ double get(const double2& v, int k) { return k == 0 ? v.x : v.y; }
  static __device__ __forceinline__ void set(double2& v, int k, double x) {
    if (k == 0)
      v.x = x;
    else
      v.y = x;
  }
};
template <class T> __device__ __forceinline__ typename Vec<T>::type vld(const void* p) {
  return *reinterpret_cast<const typename Vec<T>::type*>(p);
}
template <class T> __device__ __forceinline__ void vst(void* p, const typename Vec<T>::type& v) {
  *reinterpret_cast<typename Vec<T>::type*>(p) = v;
}

// Phase 1 of the sweep on one 16-byte chunk of an element's three rows
// (tile byte offsets ro[0..2]): NFO (GTEQNF, src/gteqnf.f90:35-37) and
// UMEAN = 0.5*DTE*(div F - 1/3 sum_i MU_i (NFO_i - f_i)) with div F = sum_i
// (N_i,x cx + N_i,y cy) f_i (GETELC, src/getelc.f90:54-83).  The rows are
// overwritten in place with g = f - UMEAN, the value every edge flux and the
// volume term of this element use (src/getelc.f90:87-117,
// src/edgflxopt.f90:95-125); NFO and UMEAN are returned.  FP32: NFO =
// A*2^(ex*|c-u|^2) with the SFU's 2^x; FP64: NFO = exp(a0 + a1*cx + a2*cy +
// ex*|c|^2) (the exponent expanded, three FMAs; c2 = |c|^2 per velocity).
template <class T>
__device__ __forceinline__ void sweep_p1(const ElemRec<T>& r, const double* etab, unsigned char* tl,
                                         const unsigned (&ro)[3], const typename Vec<T>::type& cxv,
                                         const typename Vec<T>::type& cyv, const typename Vec<T>::type& c2v, T dth,
                                         T dth3, typename Vec<T>::type (&q)[3], typename Vec<T>::type& u) {
  using VO = Vec<T>;
  constexpr int W = SweepGeo<T>::W;
  typename VO::type f[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) f[i] = vld<T>(tl + ro[i]);
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const T cx = VO::get(cxv, w), cy = VO::get(cyv, w);
    const T f0 = VO::get(f[0], w), f1 = VO::get(f[1], w), f2 = VO::get(f[2], w);
    const T sx = r.gx[0] * f0 + r.gx[1] * f1 + r.gx[2] * f2;
    const T sy = r.gy[0] * f0 + r.gy[1] * f1 + r.gy[2] * f2;
    T coll = (T)0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      T qi;
      if constexpr (sizeof(T) == 8) {
        qi = exp_tang(fma(r.ux[i], cx, fma(r.uy[i], cy, fma(r.ex[i], VO::get(c2v, w), r.A[i]))), etab);
      } else {
        const T dx = r.ux[i] - cx, dy = r.uy[i] - cy;
        qi = r.A[i] * nfo_exp<T>(r.ex[i] * (dx * dx + dy * dy), etab);
      }
      VO::set(q[i], w, qi);
      coll += r.mu[i] * (qi - VO::get(f[i], w));
    }
    const T um = dth * (sx * cx + sy * cy) - dth3 * coll;
    VO::set(u, w, um);
#pragma unroll
    for (int i = 0; i < 3; ++i) VO::set(f[i], w, VO::get(f[i], w) - um);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) vst<T>(tl + ro[i], f[i]);
}

// max that keeps a NaN operand (max.NaN): the residual's "change the
// unknown receives" must carry a non-finite update into the L2 sum
__device__ __forceinline__ float fmax_nan(float a, float b) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ double fmax_nan(double a, double b) {
  return (a != a || b != b) ? a + b : fmax(a, b);
}

// Adds the per-warp residual partials (max |d|, sum of squares) to a case's
// accumulators.
template <int NW>
__device__ __forceinline__ void resid_add(Ctrl* ctrl, const double* red_m, const double* red_s) {
  double mm = 0, ss = 0;
  for (int w = 0; w < NW; ++w) {
    mm = fmax(mm, red_m[w]);
    ss += red_s[w];
  }
  atomicAdd(&ctrl->acc_sq, ss);
  atomicMax(reinterpret_cast<unsigned long long*>(&ctrl->acc_max), (unsigned long long)__double_as_longlong(mm));
}

// Persistent sweep kernel: EB block elements, TPE*EB threads.  Work units are
// (block b, group of `tpu` velocity tiles) with b fastest, handed out in
// order (the first by blockIdx, the rest from a device counter), so the CTAs
// running at one moment cover neighbouring blocks at the same velocities and
// the halo rows they read are L2 hits.  Per unit the block's element records
// and the halo's record heads are staged in shared memory; per tile the
// block's rows arrive as TMA boxes (completing on an mbarrier, bounded wait)
// and the halo's rows by cp.async copies, double-buffered so the next tile's
// rows load while this one is computed.  Per tile:
//  * phase 1: UMEAN and g = f - UMEAN of every block and halo element; a
//    block element's NFO and UMEAN stay in the registers of the thread that
//    updates it;
//  * phase 2, threads j, j+EB, .. (TPE of them) take NCH/TPE of block
//    element j's 16-byte velocity chunks each: the volume term (src/getelc.f90:87-117), the edge fluxes gathered
//    per element (EDGFLXOPT src/edgflxopt.f90:95-125; outflow and, with zero
//    length, inflow and wall sides read the element itself), the wall sides'
//    fluxes (GETBOU src/getbou.f90:142-281), GETINC/CMMINC, ADTHEM and INFLOW;
//    the new rows stay in registers.
// Two barriers per tile: at the top (tile k has landed; every thread is
// done with tile k - 1, whose new rows it then writes back into that tile's
// buffer) and after phase 1; after the second, thread 0 stores tile k - 1
// and the next tile's copies go into its buffer once the store has read it.
// The unit's last tile is written back and stored at the unit's end.
// ONE: a single case passed as a kernel parameter (its fields come from the
// constant bank, no registers); otherwise the case table.
// Upwinding: the own value is taken where SC = n.c > 0.  The reference takes
// it where SC > 0 for the ISIDE(3) element and SC >= 0 for the other; the
// two differ only at SC = 0, where the flux SC*value is zero either way.
// Residency: FP32, two CTAs per SM (128 registers); FP64 with 64-element
// blocks, three CTAs of 4 warps (168 registers, a few spilled: 1.02 ms per
// sweep on the 200x100 channel at 24x48 velocities, against 1.24 ms for one
// 8-warp CTA of 128 elements at 208 registers).
template <class T, int EB, int IMMAT, bool ONE>
__global__ void __launch_bounds__(SweepGeo<T>::TPE * EB, sizeof(T) == 4 ? 2 : (EB == 64 ? 3 : 1))
    k_sweep(BatchArgs<T> a, int total_units, const __grid_constant__ CaseDev<T> one) {
  using G = SweepGeo<T>;
  using VO = Vec<T>;
  using VecT = typename VO::type;
  constexpr int W = G::W, VT = G::VT, NCH = G::NCH, RW = G::RW, HW = G::HW, HR = G::HR;
  constexpr int TPE = G::TPE, CPT = G::CPT;
  constexpr int NT = TPE * EB, NW = NT / 32;
  constexpr int NBOX = (3 * EB + G::BOX_ROWS - 1) / G::BOX_ROWS;
  constexpr unsigned BOX_BYTES = G::BOX_ROWS * 64;
  static_assert(EB % 16 == 0, "whole warps");
  extern __shared__ __align__(128) unsigned char sm_raw[];
  // the next unit, handed from thread 0 to the CTA: two slots used in turn,
  // so thread 0 never overwrites the slot another warp may still be reading
  // (a unit of a finished case has no barrier of its own: with one slot,
  // thread 0 could loop round and replace the value before a slow warp read
  // it, and the warps would then disagree on the unit and on the barriers)
  __shared__ int s_unit[2];
  __shared__ double red_m[NW], red_s[NW];
  __shared__ uint64_t bars[2];  // TMA completion of tile buffer 0 / 1
  // FP64: the 2^(j/64) table of the NFO exp (one entry for FP32, unused)
  __shared__ double etab[sizeof(T) == 8 ? EXP_TAB : 1];
  const int tid = threadIdx.x;
  if (sizeof(T) == 8)
    for (int i = tid; i < EXP_TAB; i += NT) etab[i] = exp2((double)i / EXP_TAB);
  // tile buffers 1024-byte aligned (the swizzle pattern repeats every 512 B)
  unsigned char* const base = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
  const size_t tile_bytes = G::tile_bytes(EB, a.max_halo);
  ElemRec<T>* const recs = reinterpret_cast<ElemRec<T>*>(base + 2 * tile_bytes);
  unsigned char* const hrec = reinterpret_cast<unsigned char*>(recs + EB);
  T* const vtab = reinterpret_cast<T*>(hrec + (size_t)a.max_halo * HR);  // cx, cy, NFINF (, |c|^2)
  constexpr int UV = G::TPU_MAX * VT;
  int* const hrow = reinterpret_cast<int*>(vtab + G::NTAB * UV);  // f rows of the unit's halo, 3 per element
  const int j = tid % EB, hh = tid / EB;  // block element, and which of its TPE parts
  const T third = (T)(1.0 / 3.0);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t par = 0;  // bit b: parity of the next phase of bars[b]
  bool aborted = false;
  int abort_buf = 0;
  // the new block rows of tile vt (written into buffer bi by every thread,
  // each followed by a proxy fence, before a barrier) as NBOX box stores
  // issued by thread 0; rows past 3E are not written
  auto store = [&](const CUtensorMap* map, int vt, int bi, int y0) {
    const unsigned char* srcb = base + (size_t)bi * tile_bytes;
#pragma unroll
    for (int x = 0; x < NBOX; ++x) tma_store_2d(map, vt * VT, y0 + x * G::BOX_ROWS, srcb + x * BOX_BYTES);
    bulk_commit();
  };

  int unit = blockIdx.x, c = 0, iter = 0;
  // tiles this CTA has started: the two tile buffers are used in turn across
  // units, so a unit's first tile goes to the buffer its predecessor's last
  // tile did not use, whose box store was issued a tile earlier
  int gk = 0;
  // residual partials of the thread's values: a single case adds them to its
  // control block once per CTA (after the last unit), a batch once per unit
  double rmax = 0.0, rsq = 0.0;
  // the unit after this one, drawn ahead so the atomic's latency is hidden
  int next = (tid == 0 && unit < total_units) ? (int)gridDim.x + atomicAdd(&a.ctl->sweep_next, 1) : 0;
  while (unit < total_units) {
    c = ONE ? 0 : find_case(a.unit_off, a.ncases, unit);
    const CaseDev<T>& C = ONE ? one : a.cases[c];
    const bool active = !C.ctrl->done;  // the same for every thread
    if (!ONE && active && tid == 0) {
      tensormap_acquire(&C.tm[0]);
      tensormap_acquire(&C.tm[1]);
    }
    const CUtensorMap* last_map = nullptr;
    int last_vt = 0, last_bi = 0, last_y0 = 0;
    if (active) {
      const int lu = unit - (ONE ? 0 : a.unit_off[c]);
      const int b = lu % C.nblocks, vg = lu / C.nblocks;
      const int e0 = b * EB, nb = min(EB, C.E - e0);
      const int h0 = C.halo_off[b], nh = C.halo_off[b + 1] - h0;
      int vt0, ntl;
      sweep_group(C, vg, vt0, ntl);
      const int cur = C.ctrl->cur;
      const double dtd = step_dt(C.ctrl);
      const T dt = (T)dtd, dth = (T)(0.5 * dtd), dth3 = (T)(0.5 * dtd / 3.0);
      const int* __restrict__ hlist = C.halo_list + h0;

      // unit prologue, all of it asynchronous (the first tile's barrier
      // publishes it): tile 0's block rows as TMA boxes (thread 0, once the
      // buffer's last box store has read it) and its halo rows by cp.async,
      // row numbers from the halo list; the block's element records, the
      // halo's record heads and the unit's slices of the velocity tables
      // (cp.async, in one group with the halo rows); the halo row list of
      // the later tiles
      {
        const int bi0 = gk & 1;
        unsigned char* dst = base + (size_t)bi0 * tile_bytes;
        if (tid == 0) {
          bulk_wait_read1();  // the newest store reads the other buffer
          fence_proxy_async_smem();
          mbar_expect_tx(&bars[bi0], NBOX * BOX_BYTES);
#pragma unroll
          for (int x = 0; x < NBOX; ++x)
            tma_load_2d(dst + x * BOX_BYTES, &C.tm[cur], vt0 * VT, 3 * e0 + x * G::BOX_ROWS, &bars[bi0]);
        }
        const T* srcf = C.f[cur] + (size_t)vt0 * VT;
        for (int w = tid; w < nh * 12; w += NT) {
          const int row = w >> 2, cq = w & 3, h = row / 3;
          cp_async16(dst + (tile_row_off(3 * EB + row) ^ (16u * cq)),
                     srcf + (size_t)(hlist[h] * 3 + (row - 3 * h)) * C.Vp + cq * W);
        }
        const uint4* src = reinterpret_cast<const uint4*>(C.rec + e0);
        for (int w = tid; w < nb * RW; w += NT) cp_async16(reinterpret_cast<uint4*>(recs) + w, src + w);
        for (int w = tid; w < nh * HW; w += NT) {
          const int s = w / HW, k = w - s * HW;
          cp_async16(hrec + (size_t)s * HR + 16 * k, reinterpret_cast<const uint4*>(C.rec + hlist[s]) + k);
        }
        // table t's values [vt0*VT, (vt0 + ntl)*VT) to vtab + t*UV, 16 bytes a copy
        constexpr int TW = VT * (int)sizeof(T) / 16;  // 16-byte words of one tile's values
        const int nw = ntl * TW;
        for (int w = tid; w < G::NTAB * nw; w += NT) {
          const int t = w / nw, x = w - t * nw;
          cp_async16(reinterpret_cast<uint4*>(vtab + t * UV) + x,
                     reinterpret_cast<const uint4*>(C.swtab + (size_t)t * C.Vp + (size_t)vt0 * VT) + x);
        }
        cp_async_commit();
        for (int s = tid; s < 3 * nh; s += NT) {
          const int h = s / 3;
          hrow[s] = hlist[h] * 3 + (s - 3 * h);
        }
      }
      // copies of tile vt (k >= 1) into buffer bi: the block's rows (3*e0 ..)
      // as NBOX TMA boxes issued by thread 0 once the buffer's last box store
      // has read it (rows past 3E read as zeros), the halo rows (tile rows
      // 3*EB ..) by cp.async, four threads per 64-byte row
      auto issue = [&](int vt, int bi) {
        unsigned char* dst = base + (size_t)bi * tile_bytes;
        const T* src = C.f[cur] + (size_t)vt * VT;
        for (int w = tid; w < nh * 12; w += NT) {
          const int row = w >> 2, cq = w & 3;
          cp_async16(dst + (tile_row_off(3 * EB + row) ^ (16u * cq)), src + (size_t)hrow[row] * C.Vp + cq * W);
        }
        if (tid == 0) {
          bulk_wait_read0();
          fence_proxy_async_smem();  // the buffer's previous generic accesses
          mbar_expect_tx(&bars[bi], NBOX * BOX_BYTES);
#pragma unroll
          for (int x = 0; x < NBOX; ++x)
            tma_load_2d(dst + x * BOX_BYTES, &C.tm[cur], vt * VT, 3 * e0 + x * G::BOX_ROWS, &bars[bi]);
        }
      };
      const unsigned hx = 16u * CPT * hh;  // the thread's first chunk, as an offset XOR
      // block element j's own rows at the thread's first chunk
      unsigned own[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) own[i] = tile_row_off(3 * j + i) ^ hx;
      // the new rows of the previous tile, written back after the next
      // tile's first barrier
      VecT outv[CPT][3];
      auto put_rows = [&](unsigned char* t) {
        if (j < nb) {
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc)
#pragma unroll
            for (int i = 0; i < 3; ++i) vst<T>(t + (own[i] ^ (16u * cc)), outv[cc][i]);
        }
        fence_proxy_async_smem();
      };

      for (int k = 0; k < ntl; ++k, ++gk) {
        const int bi = gk & 1;
        unsigned char* const tl = base + (size_t)bi * tile_bytes;
        // thread 0 waits for the boxes (the others wait in the barrier, not
        // spinning); every thread waits for its own halo copies
        const uint32_t ph = (par >> bi) & 1u;
        const bool ok = tid != 0 || mbar_wait_bounded(&bars[bi], ph);
        par ^= 1u << bi;
        cp_async_wait<0>();
        // tile k has landed (or the wait expired), and every thread has
        // written and fenced its new rows of tile k - 1
        if (__syncthreads_or(ok ? 0 : 1)) {
          aborted = true;
          abort_buf = bi;
          break;
        }
        if (tid != 0) mbar_try_wait(&bars[bi], ph);  // completed: acquires the box data
        // every thread is past its phase-2 reads of tile k - 1: its new rows
        // replace the block rows in its buffer, for the box store
        if (k > 0) put_rows(base + (size_t)(bi ^ 1) * tile_bytes);
        const int vb0 = (vt0 + k) * VT;
        const T* vx = vtab + k * VT;
        const T* vy = vtab + UV + k * VT;
        const T* vn = vtab + 2 * UV + k * VT;
        const T* vc2 = vtab + (G::NTAB - 1) * UV + k * VT;  // |c|^2 (FP64; unused in FP32)

        // ---- phase 1: block element j (chunks CPT*hh ..), then the halo
        // chunk by chunk
        VecT qr[CPT][3], ur[CPT];
        if (j < nb) {
          const ElemRec<T>& r = recs[j];
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc) {
            const int cq = CPT * hh + cc;
            const unsigned ro[3] = {own[0] ^ (16u * cc), own[1] ^ (16u * cc), own[2] ^ (16u * cc)};
            sweep_p1<T>(r, etab, tl, ro, vld<T>(vx + cq * W), vld<T>(vy + cq * W), vld<T>(vc2 + cq * W), dth, dth3,
                        qr[cc], ur[cc]);
          }
        }
        for (int w = tid; w < nh * NCH; w += NT) {
          const int hs = w >> 2, cq = w & 3;
          const ElemRec<T>& r = *reinterpret_cast<const ElemRec<T>*>(hrec + (size_t)hs * HR);
          const int r0 = 3 * (EB + hs);
          const unsigned ro[3] = {tile_row_off(r0) ^ (16u * cq), tile_row_off(r0 + 1) ^ (16u * cq),
                                  tile_row_off(r0 + 2) ^ (16u * cq)};
          VecT qd[3], ud;
          sweep_p1<T>(r, etab, tl, ro, vld<T>(vx + cq * W), vld<T>(vy + cq * W), vld<T>(vc2 + cq * W), dth, dth3, qd,
                      ud);
        }
        __syncthreads();
        // tile k - 1's new rows are in place: store them, then load tile k + 1
        // into that buffer once the store has read it
        if (tid == 0 && k > 0) store(&C.tm[cur ^ 1], vt0 + k - 1, bi ^ 1, 3 * e0);
        if (k + 1 < ntl) {
          issue(vt0 + k + 1, bi ^ 1);
          cp_async_commit();
        }

        // ---- phase 2: the update of block element j, chunks CPT*hh ..
        // CPT*hh + CPT - 1 (row offsets own[], srcp[], srcq[] are at chunk
        // CPT*hh; chunk CPT*hh + cc of the same row is at offset ^ 16*cc)
        T rmt = (T)0, sqt = (T)0;
        if (j < nb) {
          const ElemRec<T>& r = recs[j];
          // per edge: the flux source's rows, AL*n where the edge carries
          // the element-centric flux (zero on inflow and wall sides, whose
          // flux the wall path adds); MU*DTE, MM*DTE
          const int flags = r.flags;
          unsigned srcp[3], srcq[3];
          T anx[3], any[3], mudt[3], mmdt[3], cmx[3], cmn[3];
#pragma unroll
          for (int k2 = 0; k2 < 3; ++k2) {
            srcp[k2] = r.edge[k2].offp ^ hx;
            srcq[k2] = r.edge[k2].offq ^ hx;
            const bool fl = (flags & (FLAG_FLUX0 << k2)) != 0;
            anx[k2] = fl ? r.edge[k2].anx : (T)0;
            any[k2] = fl ? r.edge[k2].any : (T)0;
          }
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            mudt[i] = r.mu[i] * dt;
            mmdt[i] = r.mm[i] * dt;
            if (IMMAT == 0) {
              cmx[i] = C.cmax[3 * (e0 + j) + i];
              cmn[i] = C.cmin[3 * (e0 + j) + i];
            }
          }
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc) {
            const int cq = CPT * hh + cc;
            const unsigned cx16 = 16u * cc;
            const int vb = vb0 + cq * W;
            VecT(&out)[3] = outv[cc];
            if (vb >= C.V) {  // all past V: the padding stays zero
#pragma unroll
              for (int i = 0; i < 3; ++i) out[i] = VecT{};
              continue;
            }
            const VecT cxv = vld<T>(vx + cq * W), cyv = vld<T>(vy + cq * W);
            VecT g[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) g[i] = vld<T>(tl + (own[i] ^ cx16));
            // GETELC second half, the volume term RHS_i = AREA/3 (N_i,x cx +
            // N_i,y cy) sum(g) (src/getelc.f90:87-117).  For P1,
            // AREA/3 grad N_i = -(EL/6) n of the edge opposite node i, so an
            // element whose three sides are interior (AL*n of every edge at
            // hand) takes RHS_i = -AL*c.n(edge (i+1) mod 3) * sum(g), added
            // in the edge loop below (sgm = sum(g)); the others use the
            // gradients, with RHS_3 = -(RHS_1 + RHS_2) from the gradients
            // summing to zero (sgm = 0)
            T rhs[3][W], sgm[W];
            if (flags & FLAG_INTERIOR) {
#pragma unroll
              for (int w = 0; w < W; ++w) {
                sgm[w] = VO::get(g[0], w) + VO::get(g[1], w) + VO::get(g[2], w);
                rhs[0][w] = rhs[1][w] = rhs[2][w] = (T)0;
              }
            } else {
              const T area3 = r.area * third;
#pragma unroll
              for (int w = 0; w < W; ++w) {
                const T cx = VO::get(cxv, w), cy = VO::get(cyv, w);
                const T s3 = (VO::get(g[0], w) + VO::get(g[1], w) + VO::get(g[2], w)) * area3;
                rhs[0][w] = (r.gx[0] * cx + r.gy[0] * cy) * s3;
                rhs[1][w] = (r.gx[1] * cx + r.gy[1] * cy) * s3;
                rhs[2][w] = -(rhs[0][w] + rhs[1][w]);
                sgm[w] = (T)0;
              }
            }
            // edge fluxes (EDGFLXOPT, src/edgflxopt.f90:95-125): RHS_p -=
            // AL*SC*(2 u_p + u_q), RHS_q -= AL*SC*(u_p + 2 u_q), (u_p, u_q)
            // the element's own values where AL*SC > 0, the source's
            // otherwise; AL*SC is zero on sides without the element-centric
            // flux.  The node opposite the edge takes the volume term.
#pragma unroll
            for (int k2 = 0; k2 < 3; ++k2) {
              const int p = k2, qn = (k2 + 1) % 3, op = (k2 + 2) % 3;
              const VecT gp = vld<T>(tl + (srcp[k2] ^ cx16)), gq = vld<T>(tl + (srcq[k2] ^ cx16));
#pragma unroll
              for (int w = 0; w < W; ++w) {
                const T as = anx[k2] * VO::get(cxv, w) + any[k2] * VO::get(cyv, w);
                const bool mine = as > (T)0;
                const T up = mine ? VO::get(g[p], w) : VO::get(gp, w);
                const T uq = mine ? VO::get(g[qn], w) : VO::get(gq, w);
                rhs[p][w] -= as * ((T)2 * up + uq);
                rhs[qn][w] -= as * (up + (T)2 * uq);
                rhs[op][w] -= as * sgm[w];
              }
            }
            // ALPHA < 1: bit 3*w + i marks node i at velocity vb + w as
            // deferred (its update gets the specular part in k_wspec)
            unsigned dmask = 0u;
            if (flags & 0x38) {
              // wall sides; molecules leaving the wall (src/getbou.f90:189-255)
              // carry the diffuse part ALPHA*ETA*Mw here, the specular part
              // (1-ALPHA)*Rf in k_wspec
              const bool spec = C.spec != 0;
#pragma unroll
              for (int k2 = 0; k2 < 3; ++k2) {
                if (!(flags & (8 << k2))) continue;
                const int p = k2, qn = (k2 + 1) % 3;
                const int bs = r.bside[k2];
                const T twr = (T)2 * C.rgas * C.bTw[bs];
                const T uwx = C.bUw[2 * bs], uwy = C.bUw[2 * bs + 1], eta = C.bEta[bs];
                const T wnx = r.edge[k2].anx, wny = r.edge[k2].any;  // AL*n of the wall side
                // with the specular part, the wall branch is taken where the
                // host's FP64 TEST < 0 (the items of k_wspec are built from it)
                const int* rfi = spec ? C.rf_i + (size_t)C.rside[bs] * C.V * 2 : nullptr;
#pragma unroll
                for (int w = 0; w < W; ++w) {
                  const T cx = VO::get(cxv, w), cy = VO::get(cyv, w);
                  const T asw = wnx * cx + wny * cy;  // AL * (n.c), the sign of TEST
                  const bool own = spec ? !(vb + w < C.V && rfi[2 * (vb + w)] >= 0) : asw >= (T)0;
                  T up, uq;
                  if (own) {
                    up = VO::get(g[p], w);
                    uq = VO::get(g[qn], w);
                  } else {
                    T mw;
                    if (uwx == (T)0 && uwy == (T)0) {
                      const T spd = sqrt(cx * cx + cy * cy);
                      mw = dexp<T>(-(spd * spd) / twr);
                    } else {
                      const T dx = cx - uwx, dy = cy - uwy;
                      mw = dexp<T>(-(dx * dx + dy * dy) / twr);
                    }
                    up = uq = C.alpha * (mw * eta);
                    if (spec) dmask |= ((1u << p) | (1u << qn)) << (3 * w);
                  }
                  rhs[p][w] -= asw * ((T)2 * up + uq);
                  rhs[qn][w] -= asw * (up + (T)2 * uq);
                }
              }
            }
            // GETINC / CMMINC, ADTHEM (f >= 0), INFLOW; the padding past V
            // stays zero
            // defer: some node of this chunk waits for the specular part
            // (only wall elements with ALPHA < 1; the other variant has no
            // per-value test)
            auto finish = [&](auto full, auto defer) {
#pragma unroll
              for (int w = 0; w < W; ++w) {
                const bool live = decltype(full)::value || vb + w < C.V;
                const T u = VO::get(ur[cc], w);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                  const T f = VO::get(g[i], w) + u;
                  const T qmf = VO::get(qr[cc][i], w) - f;
                  T d, rr, x = (T)0, cdt = (T)0;
                  if (IMMAT == 1) {
                    d = mmdt[i] * rhs[i][w] + mudt[i] * qmf;
                    rr = fabs(d);
                  } else {
                    x = rhs[i][w] * dt;
                    cdt = mudt[i] * qmf;
                    d = r.mm[i] * x + cdt;
                    rr = ((x >= (T)0) ? cmx[i] : cmn[i]) * x + cdt;
                    rr = rr > (T)0 ? rr : (T)0;
                  }
                  // L2 residual: the change the unknown receives (-f where
                  // the clip applies, i.e. where d < -f; none at
                  // inflow-reset nodes); a non-finite d or f reaches the sum
                  T ch;
                  if constexpr (sizeof(T) == 4)
                    ch = fmax_nan(d, -f);
                  else
                    ch = (f + d < (T)0) ? -f : d;
                  T fn = fmax(f + d, (T)0);
                  if (live) {
                    if (decltype(defer)::value && ((dmask >> (3 * w + i)) & 1u)) {
                      // deferred: k_wspec adds the specular part, clips and
                      // counts the residual
                      const size_t o = ((size_t)r.wslot * 3 + i) * C.Vp + vb + w;
                      if (IMMAT == 1) {
                        C.wd[o] = d;
                      } else {
                        C.wd[o] = x;
                        C.wd[(size_t)C.n_spec_slots * 3 * C.Vp + o] = cdt;
                      }
                    } else {
                      rmt = fmax(rmt, rr);
                      if (!(flags & (1 << i))) sqt += ch * ch;
                    }
                  } else {
                    fn = (T)0;
                  }
                  VO::set(out[i], w, fn);
                }
              }
            };
            if (dmask != 0u) {
              if (vb + W <= C.V)
                finish(std::true_type(), std::true_type());
              else
                finish(std::false_type(), std::true_type());
            } else {
              if (vb + W <= C.V)
                finish(std::true_type(), std::false_type());
              else
                finish(std::false_type(), std::false_type());
            }
            if (flags & 7) {
              const VecT nf = vld<T>(vn + cq * W);  // zero past V
#pragma unroll
              for (int i = 0; i < 3; ++i)
                if (flags & (1 << i)) out[i] = nf;
            }
          }
        }
        rmax = fmax(rmax, (double)rmt);
        rsq += (double)sqt;
      }
      if (aborted) {
        // a bounded wait expired (the vote made every thread leave the tile
        // loop together): drain this CTA's copies in flight, bounded, and
        // report through the case's control block
        if (tid == 0) {
          C.ctrl->timeout = 1;
          mbar_wait_bounded(&bars[abort_buf], ((par >> abort_buf) & 1u) ^ 1u);
          bulk_wait0();
        }
        return;
      }
      // a batch: the unit's residual, per warp
      if (!ONE) {
        rmax = warp_max(rmax);
        rsq = warp_sum(rsq);
        if ((tid & 31) == 0) {
          red_m[tid >> 5] = rmax;
          red_s[tid >> 5] = rsq;
        }
        rmax = rsq = 0.0;
      }
      last_map = &C.tm[cur ^ 1];
      last_vt = vt0 + ntl - 1;
      last_bi = (gk - 1) & 1;
      last_y0 = 3 * e0;
      // the last tile's new rows, once every thread is past its reads
      __syncthreads();
      put_rows(base + (size_t)last_bi * tile_bytes);
    }
    // every thread is past phase 2 of the unit's last tile and has written
    // its rows: store the last tile and (a batch) add the unit's residual to
    // its case (the sum of squares can differ in its last bits between runs:
    // the order of the atomics varies); the records, tables and halo list
    // may be replaced
    if (tid == 0) s_unit[iter & 1] = next;
    __syncthreads();
    if (tid == 0 && last_map) {
      store(last_map, last_vt, last_bi, last_y0);
      if (!ONE) resid_add<NW>(C.ctrl, red_m, red_s);
    }
    unit = s_unit[iter & 1];
    ++iter;
    if (tid == 0 && unit < total_units) next = (int)gridDim.x + atomicAdd(&a.ctl->sweep_next, 1);
  }
  // a single case: the CTA's residual (only a CTA that updated values; the
  // case's flag is the same for all of them)
  if (ONE && gk > 0) {
    rmax = warp_max(rmax);
    rsq = warp_sum(rsq);
    if ((tid & 31) == 0) {
      red_m[tid >> 5] = rmax;
      red_s[tid >> 5] = rsq;
    }
    __syncthreads();
    if (tid == 0) resid_add<NW>(one.ctrl, red_m, red_s);
  }
  if (tid == 0) bulk_wait0();  // the last box stores are complete before the CTA exits
}

// ------------------------------------------------ specular wall part ----
// GETBOU's specular part for ALPHA < 1 (src/getbou.f90:189-255): a molecule
// leaving wall side k of element e at velocity v carries UNSID =
// (1-ALPHA)*Rf + ALPHA*ETA*Mw with Rf = (ZD2*f(I1) + ZD1*f(I2)) / (ZD1 +
// ZD2) of the element's own nodes at the mirrored grid velocities.  The
// reference reads f(I) from DISNF while its velocity loop updates it in
// place: the new value for I < v, the old one for I > v.  The sweep has
// applied the diffuse part and stored the deferred nodes' partial update
// (wd); the specular part is linear in RHS: with IMMAT = 1, DELUN +=
// MMAT*DTE*dRHS with dRHS the edge term of (1-ALPHA)*Rf; with IMMAT = 0
// CMMINC (src/cmminc.f90:22-41) on RHS*DTE + dRHS*DTE, its residual from the
// CMMAT row's largest or smallest entry; then ADTHEM's clip, INFLOW's reset
// and the residual.  seq = 0: the items whose mirrored velocities include no earlier
// deferred one, a thread each; seq = 1: the others, one thread per wall
// element in velocity order (after the parallel ones).
template <class T> __global__ void __launch_bounds__(256) k_wspec(const __grid_constant__ CaseDev<T> C, int seq) {
  if (C.ctrl->done) return;
  const T dt = (T)step_dt(C.ctrl);
  const int cur = C.ctrl->cur;
  const T* __restrict__ fo = C.f[cur];
  T* fnw = C.f[cur ^ 1];
  const T om = (T)1 - C.alpha;
  double mx = 0.0, sq = 0.0;
  auto item = [&](int it) {
    const int s = it / C.V, v = it - s * C.V;
    const int e = C.welem[s];
    const ElemRec<T>& r = C.rec[e];
    const T cx = C.cx[v], cy = C.cy[v];
    T drhs[3] = {(T)0, (T)0, (T)0};
    unsigned mask = 0u;
    auto F = [&](int node, int I) {
      const size_t o = ((size_t)e * 3 + node) * C.Vp + I;
      return I < v ? fnw[o] : fo[o];
    };
    for (int k = 0; k < 3; ++k) {
      if (!(r.flags & (8 << k))) continue;
      const size_t o = ((size_t)C.rside[r.bside[k]] * C.V + v) * 2;
      const int i1 = C.rf_i[o], i2 = C.rf_i[o + 1];
      if (i1 < 0) continue;
      const T zd1 = C.rf_z[o], zd2 = C.rf_z[o + 1];
      const int p = k, q = (k + 1) % 3;
      const T dp = om * ((zd2 * F(p, i1) + zd1 * F(p, i2)) / (zd1 + zd2));
      const T dq = om * ((zd2 * F(q, i1) + zd1 * F(q, i2)) / (zd1 + zd2));
      const T as = r.edge[k].anx * cx + r.edge[k].any * cy;  // AL * (n.c)
      drhs[p] -= as * ((T)2 * dp + dq);
      drhs[q] -= as * (dp + (T)2 * dq);
      mask |= (1u << p) | (1u << q);
    }
    for (int i = 0; i < 3; ++i) {
      if (!((mask >> i) & 1u)) continue;
      const size_t o = ((size_t)e * 3 + i) * C.Vp + v;
      const size_t od = ((size_t)s * 3 + i) * C.Vp + v;
      T d, rr;
      if (C.immat == 1) {
        d = C.wd[od] + (r.mm[i] * dt) * drhs[i];
        rr = fabs(d);
      } else {
        // CMMINC (src/cmminc.f90:22-41) on the whole RHS*DTE
        const T x = C.wd[od] + dt * drhs[i], cdt = C.wd[(size_t)C.n_spec_slots * 3 * C.Vp + od];
        d = r.mm[i] * x + cdt;
        rr = ((x >= (T)0) ? C.cmax[3 * (size_t)e + i] : C.cmin[3 * (size_t)e + i]) * x + cdt;
        rr = rr > (T)0 ? rr : (T)0;
      }
      const T f = fo[o];
      T f1 = f + d;
      const T ch = (f1 < (T)0) ? -f : d;
      f1 = f1 > (T)0 ? f1 : (T)0;
      mx = fmax(mx, (double)rr);
      if (r.flags & (1 << i))
        f1 = C.nfinf[v];
      else
        sq += (double)ch * (double)ch;
      fnw[o] = f1;
    }
  };
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  if (!seq) {
    for (int it = tid; it < C.n_spec_par; it += nt) item(C.spec_par[it]);
  } else {
    for (int s = tid; s < C.n_spec_slots; s += nt)
      for (int j = C.spec_seq_off[s]; j < C.spec_seq_off[s + 1]; ++j) item(C.spec_seq[j]);
  }
  mx = warp_max(mx);
  sq = warp_sum(sq);
  if ((threadIdx.x & 31) == 0 && (mx > 0.0 || sq > 0.0)) {
    atomicAdd(&C.ctrl->acc_sq, sq);
    atomicMax(reinterpret_cast<unsigned long long*>(&C.ctrl->acc_max), (unsigned long long)__double_as_longlong(mx));
  }
}

// ----------------------------------------------------------- residual ----
// GETRES + the residual bookkeeping (src/advnce.f90:385, 422-429) per case,
// one thread per case: the step's max and L2 residual into the history, the
// non-finite and convergence tests, the step counter and the buffer swap;
// the step's accumulators are cleared for the next step.
template <class T> __device__ __forceinline__ void resid_book(const CaseDev<T>& C, double mm, double sq) {
  Ctrl* c = C.ctrl;
  const int st = c->step;
  const double l2 = sqrt(sq);
  C.hist_linf[st] = mm;
  C.hist_l2[st] = l2;
  C.hist_dt[st] = step_dt(c);
  if (!isfinite(l2) || !isfinite(mm)) {
    c->nonfinite = 1;
    c->done = 1;
  }
  if (c->timeout) c->done = 1;
  if (c->ref == 0.0 && l2 > 0.0) c->ref = l2;
  c->acc_sq = 0.0;
  c->acc_max = 0.0;
  c->maxmu = 0.0;
  c->cur ^= 1;
  c->step = st + 1;
  if (c->step >= c->max_steps) c->done = 1;
  if (c->tol > 0.0 && l2 <= c->tol * c->ref) c->done = 1;
}
template <class T> __global__ void k_resid(BatchArgs<T> a) {
  if (threadIdx.x != 0) return;
  if (blockIdx.x == 0) a.ctl->sweep_next = 0;
  const CaseDev<T>& C = a.cases[blockIdx.x];
  if (C.ctrl->done) return;
  resid_book(C, C.ctrl->acc_max, C.ctrl->acc_sq);
}

// ------------------------------------------------- velocity-space shards ----
// A handle that holds only some speed rings of the velocity grid (the
// reference's V-communicator partition, src/spectralbgk.f90:163-199)
// forms partial velocity sums; the caller adds them up over the shards
// between the phases of a step, as the reference's MPI_ALLREDUCEs over
// MPI_COMM_V do (src/macros.f90:114-119, 153-154; src/compmu.f90:80-81;
// src/flucon2.f90:215-216).  Exchange buffers (device, the caller's):
//   sums1 [3][3E]: n, n*ux, n*uy per DG node (MACROS pass 1);
//   sums2 [2][3E] + [nwall]: the pressure sum over M/NA, COMPMU's mean
//          relative-speed sum, FLUCON2's wall sums;
//   res [2]: the step's max residual and sum of squared changes.
// One warp per DG node (a row of f in global memory, 16-byte vectors).
template <class T>
__global__ void __launch_bounds__(256) k_shard_sums1(const __grid_constant__ CaseDev<T> C, double* __restrict__ sums1) {
  if (C.ctrl->done) return;
  const int lane = threadIdx.x & 31, node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (node >= 3 * C.E) return;
  const T* row = C.f[C.ctrl->cur] + (size_t)node * C.Vp;
  double s0 = 0, s1 = 0, s2 = 0;
  RowMath<T>::pass1(row, C.tabs, C.Vp, (int)(C.rowbytes / 16), lane, 32, s0, s1, s2);
  s0 = group_sum<32>(s0);
  s1 = group_sum<32>(s1);
  s2 = group_sum<32>(s2);
  if (lane == 0) {
    const size_t n3 = 3 * (size_t)C.E;
    sums1[node] = s0;
    sums1[n3 + node] = s1;
    sums1[2 * n3 + node] = s2;
  }
}
// the bulk velocity of a node from the summed pass-1 sums (src/macros.f90:126-134)
__device__ __forceinline__ void shard_u(const double* __restrict__ sums1, size_t n3, int node, double& s0,
                                        double& ux, double& uy) {
  s0 = sums1[node];
  ux = uy = 0.0;
  if (s0 >= TINY_D) {
    ux = sums1[n3 + node] / s0;
    uy = sums1[2 * n3 + node] / s0;
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_shard_sums2(const __grid_constant__ CaseDev<T> C,
                                                     const double* __restrict__ sums1, double* __restrict__ sums2) {
  if (C.ctrl->done) return;
  const int lane = threadIdx.x & 31, node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (node >= 3 * C.E) return;
  const size_t n3 = 3 * (size_t)C.E;
  double s0, ux, uy;
  shard_u(sums1, n3, node, s0, ux, uy);
  const T* row = C.f[C.ctrl->cur] + (size_t)node * C.Vp;
  double sp = 0, sc = 0;
  RowMath<T>::pass2(row, C.tabs, C.Vp, (int)(C.rowbytes / 16), lane, 32, ux, uy, sp, sc);
  sp = group_sum<32>(sp);
  sc = group_sum<32>(sc);
  if (lane == 0) {
    sums2[node] = sp;
    sums2[n3 + node] = sc;
  }
}
// FLUCON2's sum over this shard's outgoing velocities, one CTA per wall side
template <class T>
__global__ void __launch_bounds__(WALL_THREADS) k_shard_wall(const __grid_constant__ CaseDev<T> C,
                                                             double* __restrict__ wsum) {
  __shared__ double part[WALL_THREADS / 32];
  if (C.ctrl->done) return;
  const WallSide ws = C.walls[blockIdx.x];
  const T* f = C.f[C.ctrl->cur];
  const T* f1 = f + ((size_t)ws.elem * 3 + ws.in1) * C.Vp;
  const T* f2 = f + ((size_t)ws.elem * 3 + ws.in2) * C.Vp;
  double t = 0;
  for (int v = threadIdx.x; v < C.V; v += WALL_THREADS) {
    const double test = C.cxD[v] * ws.anx + C.cyD[v] * ws.any;
    if (test > 0.0) t += fabs(test) * (0.5 * ((double)f1[v] + (double)f2[v])) * C.wjf[v];
  }
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0;
#pragma unroll
    for (int k = 0; k < WALL_THREADS / 32; ++k) u += part[k];
    wsum[blockIdx.x] = u;
  }
}
// the nodes' moments, MU and NFO parameters and the walls' ETA from the
// summed partials
template <class T>
__global__ void __launch_bounds__(256) k_shard_fin(const __grid_constant__ CaseDev<T> C,
                                                   const double* __restrict__ sums1, const double* __restrict__ sums2) {
  if (C.ctrl->done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n3 = 3 * (size_t)C.E;
  double mu = 0.0;
  if (t < (int)n3) {
    double s0, ux, uy;
    shard_u(sums1, n3, t, s0, ux, uy);
    mu = node_epilogue(C, t, s0, ux, uy, s0 >= TINY_D ? s0 : 0.0, sums2[t], sums2[n3 + t]);
  }
  if (t < C.nwall) {
    const WallSide ws = C.walls[t];
    const double eta = sums2[2 * n3 + t] / ws.sumbottom;
    C.bEtaD[ws.bside] = eta;
    C.bEta[ws.bside] = (T)eta;
  }
  const double m = warp_max(mu);
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(&C.ctrl->maxmu), (unsigned long long)__double_as_longlong(m));
}
// the step's residual partials out; after the sum / max over the shards,
// the bookkeeping of k_resid with the global values
template <class T> __global__ void k_shard_respart(const __grid_constant__ CaseDev<T> C, double* __restrict__ res) {
  if (threadIdx.x != 0 || C.ctrl->done) return;
  res[0] = C.ctrl->acc_max;
  res[1] = C.ctrl->acc_sq;
}
template <class T>
__global__ void k_shard_resid(const __grid_constant__ CaseDev<T> C, const double* __restrict__ res, BatchCtl* ctl) {
  if (threadIdx.x != 0) return;
  ctl->sweep_next = 0;
  if (C.ctrl->done) return;
  resid_book(C, res[0], res[1]);
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

// mesh node q's ND, RHO, UVEL, VVEL, PS, TEMP into out[k*stride + q]
__device__ __forceinline__ void nodal_one(const NodalArgs& a, int q, double* out, int stride) {
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
  out[q] = nd;
  out[stride + q] = rho;
  out[2 * stride + q] = u;
  out[3 * stride + q] = v;
  out[4 * stride + q] = ps;
  out[5 * stride + q] = t;
}

__global__ void k_nodal(NodalArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.NP) return;
  nodal_one(a, q, a.nd, (int)(a.rho - a.nd));
}

// ------------------------------------------------ observables on device ----
// GETMAC's nodal fields and GETFOR's lift and drag (src/getmac.f90:98-123,
// src/getfor.f90:29-49) recorded without a host round trip.  A record is
// [ITIME, LIFT, DRAG, 0][ND | RHO | UVEL | VVEL | PS | TEMP] (6*NPOIN).
// Ring mode (inside the step graph, right after the moment kernel, whose
// moments are those of the state after the previous step): the record of
// ITIME = itime0 + step is taken when that is a multiple of `every`, into
// slot count % cap of the ring, and count is bumped.  Direct mode
// (force_itime >= 0): one record into `direct`, unconditionally.
struct OutArgs {
  NodalArgs nod;  // its nd .. temp pointers unused
  const Ctrl* ctrl;
  const ForceSide* fs;
  int nfs;
  int every, cap;
  double* ring;   // [cap][4 + 6*NP]
  int* count;
  double* direct;
  int force_itime;
};
__device__ __forceinline__ int out_itime(const OutArgs& o) {
  if (o.force_itime >= 0) return o.force_itime;
  const Ctrl* c = o.ctrl;
  if (c->done || c->step == 0) return -1;
  const int it = c->itime0 + c->step;
  return (it % o.every == 0) ? it : -1;
}
__device__ __forceinline__ double* out_record(const OutArgs& o) {
  if (o.direct) return o.direct;
  return o.ring + (size_t)(*o.count % o.cap) * (4 + 6 * (size_t)o.nod.NP);
}
__global__ void k_out_nodal(OutArgs o) {
  if (out_itime(o) < 0) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= o.nod.NP) return;
  nodal_one(o.nod, q, out_record(o) + 4, o.nod.NP);
}
constexpr int FORCE_THREADS = 256;
__global__ void __launch_bounds__(FORCE_THREADS) k_out_forces(OutArgs o) {
  const int it = out_itime(o);
  if (it < 0) return;
  double* rec = out_record(o);
  const double* ps = rec + 4 + 4 * (size_t)o.nod.NP;
  double lift = 0.0, drag = 0.0;
  for (int k = threadIdx.x; k < o.nfs; k += FORCE_THREADS) {
    const ForceSide s = o.fs[k];
    const double pav = 0.5 * (ps[s.ip1] + ps[s.ip2]);
    lift -= pav * s.ly;
    drag -= pav * s.lx;
  }
  __shared__ double red[2][FORCE_THREADS / 32];
  lift = warp_sum(lift);
  drag = warp_sum(drag);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = lift;
    red[1][threadIdx.x >> 5] = drag;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double l = 0.0, d = 0.0;
    for (int w = 0; w < FORCE_THREADS / 32; ++w) {
      l += red[0][w];
      d += red[1][w];
    }
    rec[0] = (double)it;
    rec[1] = l;
    rec[2] = d;
    rec[3] = 0.0;
    if (!o.direct) {
      __threadfence();
      *o.count += 1;
    }
  }
}

// ---------------------------------------------- vector extrapolation ----
// Reduced-rank extrapolation of the pseudo-time iterates (no counterpart in
// the reference; it changes the path to the fixed point, not the fixed
// point): snapshots x_0 .. x_{n-1} of the state, differences
// u_j = x_{j+1} - x_j.  k_gram accumulates G_ab = u_a . u_b (a <= b < n-1)
// in FP64 (per-thread partials, a warp and block reduction, one atomic per
// block and entry); k_combine writes max(sum_j gamma_j x_j, 0).
constexpr int RRE_MAX = 11;  // snapshots (10 differences, 55 products)
template <class T>
__global__ void __launch_bounds__(256) k_gram(const T* __restrict__ snaps, size_t stride, int n, size_t N,
                                              double* __restrict__ G) {
  constexpr int MD = RRE_MAX - 1, NPAIR = MD * (MD + 1) / 2;
  const int m = n - 1;
  double acc[NPAIR];
#pragma unroll
  for (int q = 0; q < NPAIR; ++q) acc[q] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    double u[MD];
    double prev = (double)snaps[i];
#pragma unroll
    for (int j = 0; j < MD; ++j) {
      if (j < m) {
        const double x = (double)snaps[(size_t)(j + 1) * stride + i];
        u[j] = x - prev;
        prev = x;
      } else {
        u[j] = 0.0;
      }
    }
#pragma unroll
    for (int a = 0; a < MD; ++a)
#pragma unroll
      for (int b = a; b < MD; ++b) {
        const int q = a * MD - a * (a - 1) / 2 + (b - a);
        acc[q] = fma(u[a], u[b], acc[q]);
      }
  }
  __shared__ double red[8];
#pragma unroll
  for (int a = 0; a < MD; ++a)
#pragma unroll
    for (int b = a; b < MD; ++b) {
      if (b >= m) continue;  // uniform over the block
      const int q = a * MD - a * (a - 1) / 2 + (b - a);
      const double v = warp_sum(acc[q]);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(&G[a * m + b], t);
      }
      __syncthreads();
    }
}

template <class T>
__global__ void __launch_bounds__(256) k_combine(const T* __restrict__ snaps, size_t stride, int m,
                                                 const double* __restrict__ gamma, size_t N, T* __restrict__ out) {
  __shared__ double g[RRE_MAX];
  if (threadIdx.x < RRE_MAX) g[threadIdx.x] = (int)threadIdx.x < m ? gamma[threadIdx.x] : 0.0;
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    double x = 0.0;
    for (int j = 0; j < m; ++j) x = fma(g[j], (double)snaps[(size_t)j * stride + i], x);
    out[i] = (T)(x > 0.0 ? x : 0.0);
  }
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

// INICON2 (src/inicon2.f90:143-174) times an optional per-DG-node scale.
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

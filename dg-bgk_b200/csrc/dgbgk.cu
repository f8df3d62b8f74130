// C ABI of the DG-BGK sweep on B200 (sm_100a): handle management, device
// memory, the captured two-step CUDA graph and the state transfers.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dgbgk.h"
#include "kernels.cuh"
#include "plan.h"

namespace dgbgk {
static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
}  // namespace dgbgk

using namespace dgbgk;

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) {                                                               \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" #x ")");       \
      return DGBGK_ECUDA;                                                                  \
    }                                                                                      \
  } while (0)

#define TRY(x)                \
  do {                        \
    int rc_ = (x);            \
    if (rc_ != 0) return rc_; \
  } while (0)

namespace {

template <class X> int dalloc(X** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc((void**)p, n * sizeof(X)));
  return 0;
}
template <class X> int upload(X** p, const std::vector<X>& v, cudaStream_t s) {
  TRY(dalloc(p, v.size()));
  if (!v.empty()) CK(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, s));
  return 0;
}
template <class X> void dfree(X*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

struct ImplBase {
  virtual ~ImplBase() {}
  virtual int set_state(const void* src, bool f32) = 0;
  virtual int get_state(void* dst, bool f32) = 0;
  virtual int init_uniform(double t1, double p1, double u0, double v0, const double* scale) = 0;
  virtual int init_maxwellian(const double* n, const double* u, const double* v, const double* t) = 0;
  virtual int advance(int max_steps, double tol, int* steps, double* linf, double* l2, double* dt) = 0;
  virtual int macros(double* nd, double* rho, double* u, double* v, double* ps, double* temp) = 0;
  virtual int node_fields(double* nd, double* ux, double* uy, double* ps, double* mu) = 0;
  virtual int wall_eta(double* eta) = 0;
  virtual void info(int* out) = 0;
  virtual int profile(int nsteps, double* ms) = 0;
  virtual int macros_noalloc(double* scratch, double* nd, double* rho, double* u, double* v, double* ps,
                             double* temp) = 0;
  // the state in the reference layout DISNF(3,VNPNT,NELEM), FP64, from / to
  // a device buffer (the stream is synchronised on return)
  virtual int export_device(double* buf) = 0;
  // reduced-rank extrapolation: snapshot slots of the state (slot < 0 frees
  // them), and the extrapolated state from slots 0 .. n-1
  virtual int snapshot(int slot) = 0;
  virtual int extrapolate(int n, double* gamma) = 0;
  virtual int import_device(const double* buf) = 0;
  // device observables (GETFOR, and GETMAC every `every` steps into a ring)
  virtual int forces(double* lift, double* drag) = 0;
  virtual int set_output(int every, int cap) = 0;
  virtual int output_count(int* n) = 0;
  virtual int get_output(int k, int* itime, double* const* fields, double* lift, double* drag) = 0;
  Plan pl;
  int device = 0;
  int prec = 64;
  int nsm = 148;
  double ref_host = 0.0;
  float last_ms = 0.f;
  int mom_rows_req = 0;  // moment rows per warp step asked for at create (0: the heuristic)
  long long itime_total = 0;  // steps run since the state was last set (the reference's ITIME)
  bool shard = false;         // a velocity shard: its steps run through the shard phases
  // velocity-shard step phases (the caller sums the partials between them)
  virtual int shard_begin(int max_steps, double tol) = 0;
  virtual int shard_phase(int k, double* sums1, double* sums2, double* res) = 0;
  virtual int shard_end(int* steps, double* linf, double* l2, double* dt, int* done) = 0;
  virtual void* stream_ptr() = 0;
  virtual int shard_poll(int* done) = 0;

  // bumped when the case's device table entry changes (buffers moved,
  // re-blocked): a batch holding the case rebuilds its table
  unsigned gen = 0;
  // bumped when the state is written from outside the time loop: a batch
  // lets a case it stopped after a divergence run again
  unsigned epoch = 0;
};

// A set of cases launched together (one handle, or a batch): the case table
// and the flattened work offsets on the device, and the launch shapes.
template <class T> struct LaunchSet {
  CaseDev<T>* d_cases = nullptr;
  int* d_off = nullptr;  // [3][n + 1]: sweep units, moment row groups, wall sides
  BatchCtl* d_ctl = nullptr;
  BatchArgs<T> args{};
  int n = 0, cap = 0, total_units = 0, total_groups = 0, total_walls = 0;
  int eb = 128, immat = 1;
  bool one = false;       // a single case: the kernels take it as a parameter
  CaseDev<T> one_case{};  // that case (zeros for a batch)
  std::vector<CaseDev<T>> spec_cases;  // cases with ALPHA < 1 wall sides (k_wspec runs per case)
  int mom_rows = 1, mom_warps = 1, mom_grid = 1, sweep_grid = 1;
  size_t mom_smem = 0, sweep_smem = 0;
  // the wall kernel's branch: it runs beside the moment kernel (both read
  // the state only; the sweep reads the wall's ETA and waits for both)
  cudaStream_t st_wall = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  LaunchSet() = default;
  LaunchSet(const LaunchSet&) = delete;
  LaunchSet& operator=(const LaunchSet&) = delete;
  ~LaunchSet() {
    release();
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st_wall) cudaStreamDestroy(st_wall);
  }
  int ensure_wall_branch() {
    if (!st_wall) CK(cudaStreamCreateWithFlags(&st_wall, cudaStreamNonBlocking));
    if (!ev_fork) CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    if (!ev_join) CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    return 0;
  }
  void release() {
    dfree(d_cases);
    dfree(d_off);
    dfree(d_ctl);
    cap = 0;
  }
};

template <class T> using MomFn = void (*)(BatchArgs<T>, int, const CaseDev<T>);
template <class T, bool ONE> MomFn<T> mom_fn1(int R) {
  return R == 4 ? k_moments<T, 4, ONE> : R == 3 ? k_moments<T, 3, ONE> : R == 2 ? k_moments<T, 2, ONE> : k_moments<T, 1, ONE>;
}
template <class T> MomFn<T> mom_fn(int R, bool one) { return one ? mom_fn1<T, true>(R) : mom_fn1<T, false>(R); }
template <class T> using SweepFn = void (*)(BatchArgs<T>, int, const CaseDev<T>);
template <class T, bool ONE> SweepFn<T> sweep_fn1(int eb, int immat) {
  if (eb == 64) return immat == 1 ? k_sweep<T, 64, 1, ONE> : k_sweep<T, 64, 0, ONE>;
  return immat == 1 ? k_sweep<T, 128, 1, ONE> : k_sweep<T, 128, 0, ONE>;
}
template <class T> SweepFn<T> sweep_fn(int eb, int immat, bool one) {
  return one ? sweep_fn1<T, true>(eb, immat) : sweep_fn1<T, false>(eb, immat);
}

// Lets a kernel take as much dynamic shared memory as the device allows.
// The attribute is process-wide state of the function, shared by every
// handle, so it is raised to the limit (each launch still asks for exactly
// what it needs) rather than set to one handle's size.
inline int allow_max_smem(const void* fn) {
  int dev = 0, optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, fn));
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  return 0;
}

// Resident sweep CTAs per SM for a tile shape (0: does not fit).
template <class T> int sweep_per_sm(int eb, int immat, int max_halo, bool one) {
  const size_t smem = SweepGeo<T>::smem(eb, max_halo);
  if (smem > 227 * 1024) return 0;
  SweepFn<T> fn = sweep_fn<T>(eb, immat, one);
  if (allow_max_smem((const void*)fn) != 0) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, SweepGeo<T>::TPE * eb, smem) !=
      cudaSuccess)
    return 0;
  return per_sm;
}

// Velocity tiles per sweep work unit for a set of cases: about `upc` units
// per resident CTA over the whole set, equal groups of tiles per case.
inline int tiles_per_unit(long total_tiles, int grid0, int upc, int nvt) {
  int t = (int)std::min<long>(16, std::max<long>(1, total_tiles / ((long)upc * grid0)));
  const int ng = (nvt + t - 1) / t;
  return (nvt + ng - 1) / ng;
}

// The sweep's velocity-tile groups of a case (a work unit is one element
// block at one group): groups of t tiles and the rest.  A single case
// (halve) ends with t to 2t - 1 tiles in groups of decreasing size
// (sweep_tail_tiles), so that the units handed out last, which set the
// launch's tail, are short; in a batch only the last case's units end the
// launch, and the extra units would cost more than they save (measured on
// eight 100x100 channels: FP64 batch step +6%).
template <class T> void set_groups(CaseDev<T>& k, int nvt, int t, bool halve) {
  t = std::max(1, std::min(t, nvt));
  k.tpu = t;
  k.halve = halve ? 1 : 0;
  if (!halve) {
    k.nreg = (nvt - 1) / t;
    k.ngrp = k.nreg + 1;
    return;
  }
  k.nreg = std::max(0, nvt / t - 1);
  int r = nvt - k.nreg * t, m = 0;
  while (r > 0) {
    r -= sweep_tail_tiles(r);
    ++m;
  }
  k.ngrp = k.nreg + m;
}

// Uploads the case table and picks the launch shapes.  Moments: per-warp
// rings of R-row stages; picks (R, warps per CTA, ring stages) with the most
// resident warps per SM (shared memory and registers), then the most rows in
// flight, then the fewest rows per warp step (FP32 takes the element mode
// first, below).  Measured on B200 at 24x48 velocities, one row per warp
// step against two or four: warps count for more than stages (FP64: 20 warps
// with one-stage rings 0.344 ms, 16 with one 0.372, 10 with two 0.486; FP32:
// 20 with one 0.204, 16 with two 0.207).
template <class T>
int build_launch_set(LaunchSet<T>& L, const std::vector<CaseDev<T>>& cs, int eb, int immat, int max_halo, int nsm,
                     cudaStream_t st, int force_rows = 0) {
  const int n = (int)cs.size();
  const bool one = n == 1;
  L.spec_cases.clear();
  for (const auto& c : cs)
    if (c.spec) L.spec_cases.push_back(c);
  unsigned maxrow = 16;
  for (const auto& c : cs) maxrow = std::max(maxrow, c.rowbytes);
  // one case: its moment tables sit in shared memory
  const size_t cap = 227 * 1024;
  long best = -1;
  for (int R : {4, 3, 2, 1})
    for (int w : {20, 16, 15, 14, 13, 12, 10, 8, 6, 5, 4, 3, 2, 1})
      for (int sg : {3, 2, 1}) {
        if (force_rows > 0 && R != force_rows) continue;
        const size_t tbytes = one ? (mom_tables(R) * (size_t)cs[0].Vp * sizeof(T) + 127) / 128 * 128 : 0;
        if (w > 16 && !one) continue;  // 640 threads: the single-case kernel only
        const size_t bytes = 128 * (((size_t)w * sg * 8 + 127) / 128) + tbytes + (size_t)w * sg * R * maxrow;
        if (bytes > cap) continue;
        // resident CTAs per SM (shared memory and registers)
        const void* mfn = (const void*)mom_fn<T>(R, one);
        int blocks = 0;
        TRY(allow_max_smem(mfn));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, mfn, w * 32, bytes));
        blocks = std::min(blocks, 4);
        if (blocks < 1) continue;
        long score = ((long)blocks * w * 1024 + (long)blocks * w * (sg - 1) * R) * 8 + (8 - R);
        // FP32: the element mode (R = 3: three rows per warp step sharing
        // the velocity tables) first, while it keeps 8 or more warps per SM
        // (measured on the 200x100 channel at 24x48 velocities: 0.158 ms,
        // against 0.191 with one row per warp step; FP64 loses occupancy
        // with it: 0.387 against 0.325)
        if (R == 3 && force_rows == 0) score = (sizeof(T) == 4 && blocks * w >= 8) ? score + (1L << 40) : -1;
        if (score > best) {
          best = score;
          L.mom_rows = R;
          L.mom_warps = w;
          L.args.mom_stages = sg;
          L.mom_smem = bytes;
        }
      }
  if (best < 0) {
    set_error("velocity rows too long for the moment kernel's shared-memory ring");
    return DGBGK_EUNSUP;
  }
  std::vector<int> off(3 * (size_t)(n + 1), 0);
  for (int c = 0; c < n; ++c) {
    const auto& k = cs[c];
    const int units = k.nblocks * k.ngrp;
    const int groups = (3 * k.E + L.mom_rows - 1) / L.mom_rows;
    off[c + 1] = off[c] + units;
    off[(n + 1) + c + 1] = off[(n + 1) + c] + groups;
    off[2 * (n + 1) + c + 1] = off[2 * (n + 1) + c] + k.nwall;
  }
  if (n > L.cap) {
    L.release();
    TRY(dalloc(&L.d_cases, n));
    TRY(dalloc(&L.d_off, 3 * (size_t)(n + 1)));
    TRY(dalloc(&L.d_ctl, 1));
    L.cap = n;
  }
  CK(cudaMemcpyAsync(L.d_cases, cs.data(), n * sizeof(CaseDev<T>), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(L.d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(L.d_ctl, 0, sizeof(BatchCtl), st));
  L.n = n;
  L.one = one;
  L.one_case = one ? cs[0] : CaseDev<T>{};
  L.eb = eb;
  L.immat = immat;
  L.total_units = off[n];
  L.total_groups = off[(n + 1) + n];
  L.total_walls = off[2 * (n + 1) + n];
  if (L.total_walls > 0) TRY(L.ensure_wall_branch());
  L.args.cases = L.d_cases;
  L.args.unit_off = L.d_off;
  L.args.grp_off = L.d_off + (n + 1);
  L.args.wall_off = L.d_off + 2 * (n + 1);
  L.args.ctl = L.d_ctl;
  L.args.ncases = n;
  L.args.max_halo = max_halo;
  L.args.mom_rowbytes = maxrow;
  // moments: persistent grid
  MomFn<T> mf = mom_fn<T>(L.mom_rows, one);
  TRY(allow_max_smem((const void*)mf));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)mf, L.mom_warps * 32, L.mom_smem));
  per_sm = std::max(per_sm, 1);
  L.mom_grid = std::max(1, std::min((L.total_groups + L.mom_warps - 1) / L.mom_warps, per_sm * nsm));
  // sweep: persistent grid
  const int sps = sweep_per_sm<T>(eb, immat, max_halo, one);
  if (sps < 1) {
    set_error("sweep kernel does not fit on an SM with this tile");
    return DGBGK_EUNSUP;
  }
  L.sweep_smem = SweepGeo<T>::smem(eb, max_halo);
  L.sweep_grid = std::max(1, std::min(L.total_units, sps * nsm));
  return 0;
}

// Reports a failed launch with its kernel and configuration.
inline int launch_check(const char* what, int grid, int block, size_t smem) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return 0;
  set_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " (launch of " + what + ": grid " +
            std::to_string(grid) + ", block " + std::to_string(block) + ", dynamic smem " + std::to_string(smem) +
            ")");
  return DGBGK_ECUDA;
}

// One pseudo-time step of every case of the set: moments, wall flux, sweep,
// residual bookkeeping.
template <class T>
int enqueue_step(const LaunchSet<T>& L, cudaStream_t st, float* ms = nullptr, const OutArgs* out = nullptr) {
  cudaEvent_t ev[5];
  if (ms)
    for (auto& e : ev) CK(cudaEventCreate(&e));
  if (ms) cudaEventRecord(ev[0], st);
  // the wall flux on its own branch beside the moments (not when timing the
  // kernels one by one)
  const bool branch = !ms && L.total_walls > 0 && L.st_wall;
  if (branch) {
    CK(cudaEventRecord(L.ev_fork, st));
    CK(cudaStreamWaitEvent(L.st_wall, L.ev_fork, 0));
    k_wall<T><<<L.total_walls, WALL_THREADS, 0, L.st_wall>>>(L.args, L.total_walls);
    TRY(launch_check("k_wall", L.total_walls, WALL_THREADS, 0));
    CK(cudaEventRecord(L.ev_join, L.st_wall));
  }
  mom_fn<T>(L.mom_rows, L.one)<<<L.mom_grid, L.mom_warps * 32, L.mom_smem, st>>>(L.args, L.total_groups,
                                                                                 L.one_case);
  TRY(launch_check("k_moments", L.mom_grid, L.mom_warps * 32, L.mom_smem));
  if (out) {  // the previous step's GETMAC / GETFOR record, when due
    const int g = (out->nod.NP + 255) / 256;
    k_out_nodal<<<g, 256, 0, st>>>(*out);
    TRY(launch_check("k_out_nodal", g, 256, 0));
    k_out_forces<<<1, FORCE_THREADS, 0, st>>>(*out);
    TRY(launch_check("k_out_forces", 1, FORCE_THREADS, 0));
  }
  if (ms) cudaEventRecord(ev[1], st);
  if (branch) {
    CK(cudaStreamWaitEvent(st, L.ev_join, 0));
  } else if (L.total_walls > 0) {
    k_wall<T><<<L.total_walls, WALL_THREADS, 0, st>>>(L.args, L.total_walls);
    TRY(launch_check("k_wall", L.total_walls, WALL_THREADS, 0));
  }
  if (ms) cudaEventRecord(ev[2], st);
  constexpr int TPE = SweepGeo<T>::TPE;
  sweep_fn<T>(L.eb, L.immat, L.one)<<<L.sweep_grid, TPE * L.eb, L.sweep_smem, st>>>(L.args, L.total_units,
                                                                                     L.one_case);
  TRY(launch_check("k_sweep", L.sweep_grid, TPE * L.eb, L.sweep_smem));
  // the specular part of ALPHA < 1 wall sides: the parallel items, then the
  // ones that wait on earlier deferred velocities
  for (const auto& c : L.spec_cases) {
    if (c.n_spec_par > 0) {
      const int g = std::min(4 * 148, (c.n_spec_par + 255) / 256);
      k_wspec<T><<<g, 256, 0, st>>>(c, 0);
      TRY(launch_check("k_wspec", g, 256, 0));
    }
    if (c.spec_seq) {
      const int g = (c.n_spec_slots + 255) / 256;
      k_wspec<T><<<g, 256, 0, st>>>(c, 1);
      TRY(launch_check("k_wspec", g, 256, 0));
    }
  }
  if (ms) cudaEventRecord(ev[3], st);
  k_resid<T><<<L.n, 32, 0, st>>>(L.args);
  TRY(launch_check("k_resid", L.n, 32, 0));
  if (ms) {
    cudaEventRecord(ev[4], st);
    cudaEventSynchronize(ev[4]);
    for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return 0;
}

// Reduced-rank extrapolation coefficients from the m x m Gram matrix G of
// the snapshot differences (upper triangle accumulated by k_gram): solve
// G gamma = 1 and scale to sum(gamma) = 1.  G is overwritten.
int rre_coeffs(std::vector<double>& G, int m, std::vector<double>& g) {
  // G gamma = 1 (upper triangle accumulated), a tiny ridge, Gaussian
  // elimination with partial pivoting, then sum(gamma) = 1
  double tr = 0;
  for (int a = 0; a < m; ++a) {
    for (int b = 0; b < a; ++b) G[a * m + b] = G[b * m + a];
    tr += G[a * m + a];
  }
  if (!(tr > 0) || !std::isfinite(tr)) {
    set_error("dgbgk_extrapolate: the snapshots do not differ");
    return DGBGK_EINVAL;
  }
  for (int a = 0; a < m; ++a) G[a * m + a] += 1e-14 * tr;
  g.assign(m, 1.0);
  for (int c = 0; c < m; ++c) {
    int pv = c;
    for (int r = c + 1; r < m; ++r)
      if (std::fabs(G[r * m + c]) > std::fabs(G[pv * m + c])) pv = r;
    if (pv != c) {
      for (int k = 0; k < m; ++k) std::swap(G[c * m + k], G[pv * m + k]);
      std::swap(g[c], g[pv]);
    }
    for (int r = c + 1; r < m; ++r) {
      const double fct = G[r * m + c] / G[c * m + c];
      for (int k = c; k < m; ++k) G[r * m + k] -= fct * G[c * m + k];
      g[r] -= fct * g[c];
    }
  }
  for (int c = m - 1; c >= 0; --c) {
    for (int k = c + 1; k < m; ++k) g[c] -= G[c * m + k] * g[k];
    g[c] /= G[c * m + c];
  }
  double sum = 0;
  for (double x : g) sum += x;
  for (auto& x : g) x /= sum;
  for (double x : g)
    if (!std::isfinite(x)) {
      set_error("dgbgk_extrapolate: singular difference system");
      return DGBGK_ENONFINITE;
    }
  return 0;
}

template <class T> struct Impl : ImplBase {
  static constexpr int GRAPH_STEPS = 2;  // pseudo-time steps per graph launch
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evpoll[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec = nullptr;
  int cur = 0;  // host copy of Ctrl::cur
  int tpu = 1;  // velocity tiles per sweep work unit
  int Vp = 0;
  // device arrays
  T* f[2] = {nullptr, nullptr};
  ElemRec<T>* rec = nullptr;
  int *halo_off = nullptr, *halo_list = nullptr;
  T *cmax = nullptr, *cmin = nullptr;
  T* tabs = nullptr;  // moment tables [MOM_TABS][Vp]
  double *nraw = nullptr, *disux = nullptr, *disuy = nullptr, *disps = nullptr, *mu = nullptr;
  T* swtab = nullptr;  // [NTAB][Vp] the sweep's velocity tables (cx, cy, NFINF, FP64: |c|^2)
  double *cxD = nullptr, *cyD = nullptr, *wjf = nullptr;
  T *bTw = nullptr, *bUw = nullptr, *bEta = nullptr;
  double* bEtaD = nullptr;
  WallSide* walls = nullptr;
  int *node_off = nullptr, *node_dg = nullptr;
  double* node_ae = nullptr;
  double *hist_linf = nullptr, *hist_l2 = nullptr, *hist_dt = nullptr;
  int hist_cap = 0;
  Ctrl* ctrl = nullptr;
  Ctrl* hctrl = nullptr;  // pinned: [0] upload, [1..2] polls
  void* staging = nullptr;
  size_t staging_bytes = 0;
  int* d_inv = nullptr;
  // ALPHA < 1 wall sides
  int *rside = nullptr, *rf_i = nullptr, *welem = nullptr, *spec_par = nullptr, *spec_seq_off = nullptr,
      *spec_seq = nullptr;
  T *rf_z = nullptr, *wd = nullptr;
  // extrapolation snapshots [snap_cap][3E*Vp] (slots 0 .. snap_n - 1 taken)
  // and the Gram / coefficient buffers
  T* snaps = nullptr;
  int snap_cap = 0, snap_n = 0;
  double *d_gram = nullptr, *d_gamma = nullptr;
  CaseDev<T> hc;          // this case's table entry
  LaunchSet<T> single;    // this case alone
  // device observables: GETFOR's sides, the output ring and one direct record
  ForceSide* d_fs = nullptr;
  int out_every = 0, out_cap = 0;
  double* out_ring = nullptr;
  int* out_count = nullptr;
  double* out_direct = nullptr;

  ~Impl() override {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
    single.release();
    dfree(d_inv);
    dfree(f[0]);
    dfree(f[1]);
    dfree(rec);
    dfree(tabs);
    dfree(halo_off);
    dfree(halo_list);
    dfree(cmax);
    dfree(cmin);
    dfree(nraw);
    dfree(disux);
    dfree(disuy);
    dfree(disps);
    dfree(mu);
    dfree(swtab);
    dfree(cxD);
    dfree(cyD);
    dfree(wjf);
    dfree(bTw);
    dfree(bUw);
    dfree(bEta);
    dfree(bEtaD);
    dfree(walls);
    dfree(node_off);
    dfree(node_dg);
    dfree(node_ae);
    dfree(hist_linf);
    dfree(hist_l2);
    dfree(hist_dt);
    dfree(ctrl);
    dfree(rside);
    dfree(rf_i);
    dfree(rf_z);
    dfree(welem);
    dfree(wd);
    dfree(spec_par);
    dfree(spec_seq_off);
    dfree(spec_seq);
    dfree(snaps);
    dfree(d_gram);
    dfree(d_gamma);
    dfree(d_fs);
    dfree(out_ring);
    dfree(out_count);
    dfree(out_direct);
    if (staging) cudaFree(staging);
    if (hctrl) cudaFreeHost(hctrl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto& e : evpoll)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int nvt() const { return (pl.V + SweepGeo<T>::VT - 1) / SweepGeo<T>::VT; }
  // measured on B200 (channel 200x100, 24x48 velocities): FP32 sweep 0.414 ms
  // at 128 elements per tile, 0.50 at 64; FP64 1.24 ms at 128 (one CTA of
  // 8 warps per SM), 1.02 at 64 (three CTAs of 4 warps)
  static int default_eb() { return sizeof(T) == 8 ? 64 : 128; }

  int init(int tile_elems) {
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    for (auto& e : evpoll) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    Vp = ((pl.V + 31) / 32) * 32;
    const size_t n = (size_t)3 * pl.E * Vp;
    TRY(dalloc(&f[0], n));
    TRY(dalloc(&f[1], n));
    CK(cudaMemsetAsync(f[0], 0, n * sizeof(T), st));
    CK(cudaMemsetAsync(f[1], 0, n * sizeof(T), st));
    std::vector<T> cm(pl.cmax.begin(), pl.cmax.end()), cn(pl.cmin.begin(), pl.cmin.end());
    TRY(upload(&cmax, cm, st));
    TRY(upload(&cmin, cn, st));
    const size_t ndg = 3 * (size_t)pl.E;
    TRY(dalloc(&nraw, ndg));
    TRY(dalloc(&disux, ndg));
    TRY(dalloc(&disuy, ndg));
    TRY(dalloc(&disps, ndg));
    TRY(dalloc(&mu, ndg));
    // sweep velocity tables, zero past V: cx, cy, NFINF and (FP64) |c|^2
    // rounded once from the FP64 cx*cx + cy*cy
    std::vector<T> sw(SweepGeo<T>::NTAB * (size_t)Vp, (T)0);
    for (int v = 0; v < pl.V; ++v) {
      sw[v] = (T)pl.cx[v];
      sw[Vp + v] = (T)pl.cy[v];
      sw[2 * (size_t)Vp + v] = (T)pl.nfinf[v];
      if (SweepGeo<T>::NTAB == 4) sw[3 * (size_t)Vp + v] = (T)(pl.cx[v] * pl.cx[v] + pl.cy[v] * pl.cy[v]);
    }
    TRY(upload(&swtab, sw, st));
    TRY(upload(&cxD, pl.cx, st));
    TRY(upload(&cyD, pl.cy, st));
    TRY(upload(&wjf, pl.wjf, st));
    std::vector<T> tb(MOM_TABS * (size_t)Vp, (T)0);  // zero past V; products rounded once from FP64
    for (int v = 0; v < pl.V; ++v) {
      tb[v] = (T)pl.cx[v];
      tb[Vp + v] = (T)pl.cy[v];
      tb[2 * (size_t)Vp + v] = (T)pl.wjf[v];
      tb[3 * (size_t)Vp + v] = (T)(pl.wjf[v] * pl.cx[v]);
      tb[4 * (size_t)Vp + v] = (T)(pl.wjf[v] * pl.cy[v]);
    }
    TRY(upload(&tabs, tb, st));
    std::vector<T> tw(pl.bTw.begin(), pl.bTw.end()), uw(pl.bUw.begin(), pl.bUw.end()),
        z(std::max(pl.B, 1), (T)0);
    TRY(upload(&bTw, tw, st));
    TRY(upload(&bUw, uw, st));
    TRY(upload(&bEta, z, st));
    std::vector<double> zd(std::max(pl.B, 1), 0.0);
    TRY(upload(&bEtaD, zd, st));
    TRY(upload(&walls, pl.walls, st));
    TRY(upload(&node_off, pl.node_off, st));
    TRY(upload(&node_dg, pl.node_dg, st));
    TRY(upload(&node_ae, pl.node_ae, st));
    TRY(upload(&d_fs, pl.fsides, st));
    if (pl.spec) {
      std::vector<T> rz(pl.rf_z.begin(), pl.rf_z.end());
      TRY(upload(&rside, pl.rside, st));
      TRY(upload(&rf_i, pl.rf_i, st));
      TRY(upload(&rf_z, rz, st));
      TRY(upload(&welem, pl.welem, st));
      // deferred wall values: IMMAT = 1 DELUN without the specular part;
      // IMMAT = 0 RHS*DTE and COLL*DTE (two halves), whose CMMINC residual
      // needs them apart
      TRY(dalloc(&wd, std::max<size_t>(1, (pl.immat == 0 ? 2 : 1) * pl.welem.size() * 3 * (size_t)Vp)));
      std::vector<int> one1(1, 0);
      TRY(upload(&spec_par, pl.spec_par.empty() ? one1 : pl.spec_par, st));
      TRY(upload(&spec_seq_off, pl.spec_seq_off, st));
      if (!pl.spec_seq.empty()) TRY(upload(&spec_seq, pl.spec_seq, st));
    }
    TRY(dalloc(&ctrl, 1));
    CK(cudaMallocHost((void**)&hctrl, 3 * sizeof(Ctrl)));
    std::memset(hctrl, 0, 3 * sizeof(Ctrl));
    CK(cudaMemcpyAsync(ctrl, hctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    TRY(ensure_hist(1024));
    TRY(set_tile(tile_elems, 8));
    CK(cudaStreamSynchronize(st));
    return 0;
  }

  // f[b] as a [3E rows][Vp] tensor; box = one 64-byte velocity segment of
  // BOX_ROWS rows, 64-byte swizzle (the sweep's tile layout)
  int make_tensor_maps() {
    auto enc = tensor_map_encoder();
    if (!enc) {
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return DGBGK_ECUDA;
    }
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    cuuint64_t dims[2] = {(cuuint64_t)Vp, (cuuint64_t)3 * pl.E};
    cuuint64_t strides[1] = {(cuuint64_t)Vp * sizeof(T)};
    cuuint32_t box[2] = {(cuuint32_t)SweepGeo<T>::VT, (cuuint32_t)SweepGeo<T>::BOX_ROWS};
    cuuint32_t estr[2] = {1, 1};
    for (int b = 0; b < 2; ++b) {
      CUresult r = enc(&hc.tm[b], dt, 2, f[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed for the state buffer");
        return DGBGK_ECUDA;
      }
    }
    return 0;
  }

  // this case's table entry (the tensor maps are set by make_tensor_maps)
  void fill_case() {
    hc.f[0] = f[0];
    hc.f[1] = f[1];
    hc.rec = rec;
    hc.halo_off = halo_off;
    hc.halo_list = halo_list;
    hc.swtab = swtab;
    hc.cx = swtab;
    hc.cy = swtab + Vp;
    hc.nfinf = swtab + 2 * (size_t)Vp;
    hc.tabs = tabs;
    hc.bTw = bTw;
    hc.bUw = bUw;
    hc.bEta = bEta;
    hc.bEtaD = bEtaD;
    hc.cxD = cxD;
    hc.cyD = cyD;
    hc.wjf = wjf;
    hc.walls = walls;
    hc.cmax = cmax;
    hc.cmin = cmin;
    hc.nraw = nraw;
    hc.disux = disux;
    hc.disuy = disuy;
    hc.disps = disps;
    hc.mu = mu;
    hc.hist_linf = hist_linf;
    hc.hist_l2 = hist_l2;
    hc.hist_dt = hist_dt;
    hc.ctrl = ctrl;
    hc.MM = pl.M / 6.022e26;
    hc.sigt = 3.1416 * pl.d * pl.d;
    hc.alpha = (T)pl.alpha;
    hc.rgas = (T)pl.rgas;
    hc.E = pl.E;
    hc.V = pl.V;
    hc.Vp = Vp;
    hc.nblocks = pl.nblocks;
    hc.nvt = nvt();
    set_groups(hc, nvt(), tpu, true);
    hc.nwall = (int)pl.walls.size();
    hc.rowbytes = (unsigned)(((size_t)pl.V * sizeof(T) + 15) / 16 * 16);
    hc.spec = pl.spec ? 1 : 0;
    hc.immat = pl.immat;
    hc.n_spec_par = (int)pl.spec_par.size();
    hc.n_spec_slots = (int)pl.welem.size();
    hc.rside = rside;
    hc.rf_i = rf_i;
    hc.rf_z = rf_z;
    hc.welem = welem;
    hc.wd = wd;
    hc.spec_par = spec_par;
    hc.spec_seq_off = spec_seq_off;
    hc.spec_seq = spec_seq;
  }

  // the one-case launch set
  int refresh() {
    ++gen;
    fill_case();
    TRY(build_launch_set(single, std::vector<CaseDev<T>>{hc}, pl.EB, pl.immat, pl.max_halo, nsm, st, mom_rows_req));
    drop_graphs();
    return 0;
  }

  // Sweep tile: EB elements per CTA (TPE*EB threads) x one 64-byte velocity
  // segment; `upc` work units per resident CTA picks the tiles per unit.
  int set_tile(int tile_elems, int upc) {
    const int eb = tile_elems > 0 ? tile_elems : default_eb();
    if (eb != 64 && eb != 128) {
      set_error("tile_elems must be 64 or 128");
      return DGBGK_EINVAL;
    }
    if (pl.EB != eb || halo_off == nullptr) {
      build_blocks(pl, eb);
      dfree(halo_off);
      dfree(halo_list);
      dfree(rec);
      TRY(upload(&halo_off, pl.halo_off, st));
      TRY(upload(&halo_list, pl.halo_list, st));
      // element records: geometry, mass matrix and edges (the node
      // parameters are filled by the moment kernel before every sweep)
      std::vector<ElemRec<T>> r(pl.E);
      std::memset((void*)r.data(), 0, r.size() * sizeof(ElemRec<T>));
      for (int e = 0; e < pl.E; ++e) {
        const auto& g = pl.geo[e];
        int flags = g.inflow & 7, interior = 0;
        for (int k = 0; k < 3; ++k) {
          r[e].gx[k] = (T)g.gx[k];
          r[e].gy[k] = (T)g.gy[k];
          r[e].mm[k] = (T)g.mm[k];
          const size_t i = 3 * (size_t)e + k;
          const PlanEdge& pe = pl.edge[i];
          r[e].edge[k].anx = (T)(pe.alen * pe.nx);
          r[e].edge[k].any = (T)(pe.alen * pe.ny);
          // the flux source's rows: the neighbour's (its slot and local
          // nodes) across an interior side, the element's own otherwise
          const int inf = edge_info(pl, i, e % eb);
          const int slot = inf >> 8, kind = inf & 3;
          r[e].edge[k].offp = tile_row_off(3 * slot + ((inf >> 3) & 3));
          r[e].edge[k].offq = tile_row_off(3 * slot + ((inf >> 5) & 3));
          if (kind == 0 || kind == 2) flags |= FLAG_FLUX0 << k;
          if (kind == 0) ++interior;
          const bool wall = kind == 3;
          r[e].bside[k] = wall ? pe.bside : -1;
          if (wall) flags |= 8 << k;
        }
        if (interior == 3) flags |= FLAG_INTERIOR;
        const int j = e % eb;
        r[e].own01 = tile_row_off(3 * j) | (tile_row_off(3 * j + 1) << 16);
        r[e].own2 = tile_row_off(3 * j + 2);
        r[e].area = (T)g.area;
        r[e].flags = flags;
        r[e].wslot = pl.spec ? pl.wslot[e] : -1;
      }
      TRY(upload(&rec, r, st));
    }
    if (SweepGeo<T>::smem(pl.EB, pl.max_halo) > 227 * 1024) {
      set_error("sweep tile needs more than 227 KB of shared memory");
      return DGBGK_EUNSUP;
    }
    TRY(make_tensor_maps());
    const int sps = sweep_per_sm<T>(pl.EB, pl.immat, pl.max_halo, true);
    if (sps < 1) {
      set_error("sweep kernel does not fit on an SM with this tile");
      return DGBGK_EUNSUP;
    }
    tpu = tiles_per_unit((long)pl.nblocks * nvt(), sps * nsm, upc, nvt());
    return refresh();
  }

  int ensure_hist(int n) {
    if (n <= hist_cap) return 0;
    dfree(hist_linf);
    dfree(hist_l2);
    dfree(hist_dt);
    TRY(dalloc(&hist_linf, n));
    TRY(dalloc(&hist_l2, n));
    TRY(dalloc(&hist_dt, n));
    hist_cap = n;
    if (halo_off) TRY(refresh());
    return 0;
  }

  void drop_graphs() {
    if (gexec) {
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
  }
  // GRAPH_STEPS pseudo-time steps as one graph (the buffer swap is on the
  // device, so one graph serves every step)
  int build_graph() {
    if (gexec) return 0;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    const OutArgs oa = out_args(-1, nullptr);
    for (int k = 0; k < GRAPH_STEPS && rc == 0; ++k) rc = enqueue_step(single, st, nullptr, out_every > 0 ? &oa : nullptr);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != 0) return rc;
    CK(e);
    CK(cudaGraphInstantiate(&gexec, g, 0));
    cudaGraphDestroy(g);
    return 0;
  }

  void fill_ctrl(Ctrl& h, int max_steps, double tol) const {
    std::memset(&h, 0, sizeof(Ctrl));
    h.max_steps = max_steps;
    h.tol = tol;
    h.ref = ref_host;
    h.dtc = pl.dtc;
    h.cur = cur;
    h.itime0 = (int)itime_total;
  }
  int upload_ctrl(int max_steps, double tol) {
    fill_ctrl(hctrl[0], max_steps, tol);
    CK(cudaMemcpyAsync(ctrl, &hctrl[0], sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    return 0;
  }

  int finish_status(const Ctrl& c) {
    if (c.timeout) {
      set_error("a bounded device wait expired (asynchronous copy did not complete)");
      return DGBGK_ECUDA;
    }
    if (c.nonfinite) {
      set_error("non-finite residual: the state diverged");
      return DGBGK_ENONFINITE;
    }
    return 0;
  }

  // after an advance: step count, history, reference and current buffer
  int collect(const Ctrl& c, int* steps, double* linf, double* l2, double* dt) {
    const int ns = c.step;
    if (steps) *steps = ns;
    ref_host = c.ref;
    cur = c.cur;
    itime_total += ns;
    if (ns > 0) {
      if (linf) CK(cudaMemcpy(linf, hist_linf, ns * sizeof(double), cudaMemcpyDeviceToHost));
      if (l2) CK(cudaMemcpy(l2, hist_l2, ns * sizeof(double), cudaMemcpyDeviceToHost));
      if (dt) CK(cudaMemcpy(dt, hist_dt, ns * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return finish_status(c);
  }

  // Velocity shard: one step in four phases on the handle's stream,
  //   1: pass-1 partial sums -> sums1;
  //   2: pass-2 partial sums with the summed sums1 -> sums2 (+ the walls);
  //   3: moments, MU, parameters, ETA from the summed sums; the sweep of the
  //      shard's velocities; residual partials -> res;
  //   4: the step's bookkeeping with the reduced res;
  // the caller sums sums1 and sums2 and takes the max (res[0]) and sum
  // (res[1]) over the shards between them, on this stream.
  int shard_begin(int max_steps, double tol) override {
    CK(cudaSetDevice(device));
    TRY(ensure_hist(std::max(max_steps, 1)));
    TRY(upload_ctrl(max_steps, tol));
    CK(cudaEventRecord(ev0, st));
    return 0;
  }
  int shard_phase(int k, double* sums1, double* sums2, double* res) override {
    const int n3 = 3 * pl.E;
    const int gw = (n3 * 32 + 255) / 256;  // a warp per DG node
    const CaseDev<T>& C = single.one_case;
    if (k == 1) {
      k_shard_sums1<T><<<gw, 256, 0, st>>>(C, sums1);
    } else if (k == 2) {
      k_shard_sums2<T><<<gw, 256, 0, st>>>(C, sums1, sums2);
      if (single.total_walls > 0) k_shard_wall<T><<<single.total_walls, WALL_THREADS, 0, st>>>(C, sums2 + 2 * (size_t)n3);
    } else if (k == 3) {
      const int nt = std::max(n3, (int)pl.walls.size());
      k_shard_fin<T><<<(nt + 255) / 256, 256, 0, st>>>(C, sums1, sums2);
      constexpr int TPE = SweepGeo<T>::TPE;
      sweep_fn<T>(single.eb, single.immat, true)<<<single.sweep_grid, TPE * single.eb, single.sweep_smem, st>>>(
          single.args, single.total_units, single.one_case);
      k_shard_respart<T><<<1, 32, 0, st>>>(C, res);
    } else if (k == 4) {
      k_shard_resid<T><<<1, 32, 0, st>>>(C, res, single.args.ctl);
    } else if (k == 0) {  // before phases 1, 2 and 5 outside a step: the kernels run
      TRY(aux_ctrl());
    } else if (k == 5) {  // the moments of the current state from the summed sums (no sweep)
      const int nt = std::max(n3, (int)pl.walls.size());
      k_shard_fin<T><<<(nt + 255) / 256, 256, 0, st>>>(C, sums1, sums2);
    } else {
      set_error("dgbgk_shard_phase: phase 0 to 5");
      return DGBGK_EINVAL;
    }
    CK(cudaGetLastError());
    return 0;
  }
  int shard_end(int* steps, double* linf, double* l2, double* dt, int* done) override {
    CK(cudaEventRecord(ev1, st));
    CK(cudaMemcpyAsync(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&last_ms, ev0, ev1));
    if (done) *done = hctrl[1].done;
    return collect(hctrl[1], steps, linf, l2, dt);
  }
  void* stream_ptr() override { return (void*)st; }
  int shard_poll(int* done) override {
    CK(cudaMemcpyAsync(&hctrl[2], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *done = hctrl[2].done;
    return 0;
  }

  int advance(int max_steps, double tol, int* steps, double* linf, double* l2, double* dt) override {
    if (shard) {
      set_error("dgbgk_advance: a velocity shard steps through dgbgk_shard_*");
      return DGBGK_EINVAL;
    }
    if (max_steps < 0) {
      set_error("max_steps < 0");
      return DGBGK_EINVAL;
    }
    if (steps) *steps = 0;
    if (max_steps == 0) return 0;
    CK(cudaSetDevice(device));
    TRY(ensure_hist(max_steps));
    TRY(build_graph());
    TRY(upload_ctrl(max_steps, tol));
    CK(cudaEventRecord(ev0, st));
    const int launches = (max_steps + GRAPH_STEPS - 1) / GRAPH_STEPS;
    const int chunk = 32;
    int issued = 0, chunks = 0;
    bool stop = false;
    while (issued < launches && !stop) {
      const int n = std::min(chunk, launches - issued);
      for (int i = 0; i < n; ++i) CK(cudaGraphLaunch(gexec, st));
      issued += n;
      const int slot = 1 + (chunks & 1);
      CK(cudaMemcpyAsync(&hctrl[slot], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(evpoll[chunks & 1], st));
      ++chunks;
      if (chunks >= 2) {  // look at the chunk before the one just issued
        const int pslot = 1 + (chunks & 1);
        CK(cudaEventSynchronize(evpoll[chunks & 1]));
        if (hctrl[pslot].done) stop = true;
      }
    }
    CK(cudaEventRecord(ev1, st));
    CK(cudaMemcpyAsync(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&last_ms, ev0, ev1));
    const int rc = collect(hctrl[1], steps, linf, l2, dt);
    // the call's last step, when its record is due (the graph takes a
    // step's record at the start of the next one)
    if (rc == 0 && out_every > 0 && hctrl[1].step > 0 && itime_total % out_every == 0) {
      TRY(moments_now());
      TRY(record(out_args((int)itime_total, nullptr)));
      CK(cudaStreamSynchronize(st));
    }
    return rc;
  }

  OutArgs out_args(int force_itime, double* direct) const {
    OutArgs o{};
    o.nod = NodalArgs{node_off, node_dg, node_ae, nraw, disux, disuy, disps, nullptr, nullptr, nullptr,
                      nullptr, nullptr, nullptr, pl.NP, pl.M / 6.022e26, pl.rgas};
    o.ctrl = ctrl;
    o.fs = d_fs;
    o.nfs = (int)pl.fsides.size();
    o.every = out_every > 0 ? out_every : 1;
    o.cap = out_cap > 0 ? out_cap : 1;
    o.ring = out_ring;
    o.count = out_count;
    o.direct = direct;
    o.force_itime = force_itime;
    return o;
  }
  int record(const OutArgs& o) {
    k_out_nodal<<<(pl.NP + 255) / 256, 256, 0, st>>>(o);
    CK(cudaGetLastError());
    k_out_forces<<<1, FORCE_THREADS, 0, st>>>(o);
    CK(cudaGetLastError());
    return 0;
  }
  size_t rec_len() const { return 4 + 6 * (size_t)pl.NP; }

  int forces(double* lift, double* drag) override {
    CK(cudaSetDevice(device));
    if (!out_direct) TRY(dalloc(&out_direct, rec_len()));
    TRY(moments_now());
    TRY(record(out_args((int)itime_total, out_direct)));
    double hdr[4];
    CK(cudaMemcpyAsync(hdr, out_direct, sizeof hdr, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    TRY(finish_status(hctrl[1]));
    if (lift) *lift = hdr[1];
    if (drag) *drag = hdr[2];
    return 0;
  }
  int set_output(int every, int cap) override {
    CK(cudaSetDevice(device));
    if (every < 0 || (every > 0 && cap < 1)) {
      set_error("dgbgk_set_output: every >= 0 and, with every > 0, capacity >= 1");
      return DGBGK_EINVAL;
    }
    CK(cudaStreamSynchronize(st));
    dfree(out_ring);
    dfree(out_count);
    out_every = every;
    out_cap = every > 0 ? cap : 0;
    if (every > 0) {
      TRY(dalloc(&out_ring, (size_t)cap * rec_len()));
      TRY(dalloc(&out_count, 1));
      CK(cudaMemsetAsync(out_count, 0, sizeof(int), st));
      CK(cudaStreamSynchronize(st));
    }
    drop_graphs();  // the step graph takes the record kernels or leaves them out
    return 0;
  }
  int output_count(int* n) override {
    CK(cudaSetDevice(device));
    int c = 0;
    if (out_count) {
      CK(cudaMemcpyAsync(&c, out_count, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    *n = c;
    return 0;
  }
  int get_output(int k, int* itime, double* const* fields, double* lift, double* drag) override {
    int count = 0;
    TRY(output_count(&count));
    const int n = std::min(count, out_cap);
    if (k < 0 || k >= n) {
      set_error("dgbgk_get_output: record " + std::to_string(k) + " not in the ring (" + std::to_string(n) +
                " held)");
      return DGBGK_EINVAL;
    }
    const int slot = (count - n + k) % out_cap;
    std::vector<double> h(rec_len());
    CK(cudaMemcpyAsync(h.data(), out_ring + (size_t)slot * rec_len(), h.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (itime) *itime = (int)h[0];
    if (lift) *lift = h[1];
    if (drag) *drag = h[2];
    for (int f = 0; f < 6; ++f)
      if (fields[f]) std::memcpy(fields[f], h.data() + 4 + (size_t)f * pl.NP, pl.NP * sizeof(double));
    return 0;
  }

  int profile(int nsteps, double* ms) override {
    CK(cudaSetDevice(device));
    TRY(ensure_hist(std::max(nsteps, 1)));
    TRY(upload_ctrl(nsteps, 0.0));
    double acc[4] = {0, 0, 0, 0};
    for (int s = 0; s < nsteps; ++s) {
      float k[4] = {0, 0, 0, 0};
      TRY(enqueue_step(single, st, k));
      for (int i = 0; i < 4; ++i) acc[i] += k[i];
    }
    CK(cudaMemcpy(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 4; ++k) ms[k] = nsteps > 0 ? acc[k] / nsteps : 0.0;
    return collect(hctrl[1], nullptr, nullptr, nullptr, nullptr);
  }

  // auxiliary kernels run with done = 0
  int aux_ctrl() { return upload_ctrl(1, 0.0); }

  int set_state(const void* src, bool f32) override {
    CK(cudaSetDevice(device));
    const size_t n = (size_t)3 * pl.E * pl.V;
    const size_t bytes = n * (f32 ? sizeof(float) : sizeof(double));
    TRY(ensure_staging(bytes));
    CK(cudaMemcpyAsync(staging, src, bytes, cudaMemcpyHostToDevice, st));
    TRY(upload_perm());
    if (f32)
      k_to_internal<float, T><<<pl.E, 256, 0, st>>>((const float*)staging, f[0], d_inv, pl.V, Vp);
    else
      k_to_internal<double, T><<<pl.E, 256, 0, st>>>((const double*)staging, f[0], d_inv, pl.V, Vp);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    cur = 0;
    ++epoch;
    itime_total = 0;  // a new state: ITIME starts again
    return 0;
  }
  int get_state(void* dst, bool f32) override {
    CK(cudaSetDevice(device));
    const size_t n = (size_t)3 * pl.E * pl.V;
    const size_t bytes = n * (f32 ? sizeof(float) : sizeof(double));
    TRY(ensure_staging(bytes));
    TRY(upload_perm());
    if (f32)
      k_from_internal<T, float><<<pl.E, 256, 0, st>>>(f[cur], (float*)staging, d_inv, pl.V, Vp);
    else
      k_from_internal<T, double><<<pl.E, 256, 0, st>>>(f[cur], (double*)staging, d_inv, pl.V, Vp);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, staging, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  int export_device(double* buf) override {
    CK(cudaSetDevice(device));
    TRY(upload_perm());
    k_from_internal<T, double><<<pl.E, 256, 0, st>>>(f[cur], buf, d_inv, pl.V, Vp);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  int import_device(const double* buf) override {
    CK(cudaSetDevice(device));
    TRY(upload_perm());
    k_to_internal<double, T><<<pl.E, 256, 0, st>>>(buf, f[0], d_inv, pl.V, Vp);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    cur = 0;
    ++epoch;
    itime_total = 0;  // a new state: ITIME starts again
    return 0;
  }
  // the capacity to grow to for slot `slot`: doubling (a march takes its
  // slots in order; growing one slot at a time copied the slots taken
  // O(m^2) times and freed and allocated device memory m times)
  int snap_grow(int slot) const { return std::min(RRE_MAX, std::max(slot + 1, 2 * snap_cap)); }
  // room for `cap` snapshot slots, keeping the slots taken so far (the
  // caller has let every queued copy into them finish)
  int grow_snaps(int cap) {
    const size_t N = (size_t)3 * pl.E * Vp;
    T* nb = nullptr;
    CK(cudaMalloc((void**)&nb, (size_t)cap * N * sizeof(T)));
    if (snaps) {
      if (snap_n > 0)
        CK(cudaMemcpyAsync(nb, snaps, (size_t)snap_n * N * sizeof(T), cudaMemcpyDeviceToDevice, st));
      CK(cudaStreamSynchronize(st));
      cudaFree(snaps);
    }
    snaps = nb;
    snap_cap = cap;
    return 0;
  }
  int snapshot(int slot) override {
    CK(cudaSetDevice(device));
    const size_t N = (size_t)3 * pl.E * Vp;
    if (slot < 0) {  // free the snapshots
      CK(cudaStreamSynchronize(st));
      dfree(snaps);
      snap_cap = snap_n = 0;
      return 0;
    }
    if (slot >= RRE_MAX) {
      set_error("dgbgk_snapshot: slot beyond the extrapolation limit of " + std::to_string(RRE_MAX) + " snapshots");
      return DGBGK_EINVAL;
    }
    if (slot >= snap_cap) TRY(grow_snaps(snap_grow(slot)));
    snap_n = std::max(snap_n, slot + 1);
    // waited for: measured on the bench's eight channels, leaving the copy
    // queued on the case's stream made the extrapolated march slower (the
    // snapshot calls 0.20 -> 0.43 ms each)
    CK(cudaMemcpyAsync(snaps + (size_t)slot * N, f[cur], N * sizeof(T), cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  int extrapolate(int n, double* gamma) override {
    CK(cudaSetDevice(device));
    if (n < 2 || n > snap_n) {
      set_error("dgbgk_extrapolate: needs 2 <= n <= the snapshots taken");
      return DGBGK_EINVAL;
    }
    const int m = n - 1;
    const size_t N = (size_t)3 * pl.E * Vp;
    if (!d_gram) TRY(dalloc(&d_gram, (size_t)RRE_MAX * RRE_MAX));
    if (!d_gamma) TRY(dalloc(&d_gamma, (size_t)RRE_MAX));
    CK(cudaMemsetAsync(d_gram, 0, (size_t)m * m * sizeof(double), st));
    const int grid = (int)std::min<size_t>((size_t)4 * nsm, (N + 255) / 256);
    k_gram<T><<<grid, 256, 0, st>>>(snaps, N, n, N, d_gram);
    CK(cudaGetLastError());
    std::vector<double> G((size_t)m * m), g;
    CK(cudaMemcpyAsync(G.data(), d_gram, G.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    TRY(rre_coeffs(G, m, g));
    if (gamma) std::copy(g.begin(), g.end(), gamma);
    CK(cudaMemcpyAsync(d_gamma, g.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
    // gamma is staged by the copy before it returns (pageable source); the
    // new state is written on the case's stream, which every later use of
    // it follows or waits for
    k_combine<T><<<grid, 256, 0, st>>>(snaps, N, m, d_gamma, N, f[cur]);
    CK(cudaGetLastError());
    ++epoch;
    return 0;
  }
  int upload_perm() {
    if (d_inv) return 0;
    TRY(upload(&d_inv, pl.inv, st));
    return 0;
  }
  int ensure_staging(size_t bytes) {
    if (bytes <= staging_bytes) return 0;
    if (staging) cudaFree(staging);
    staging = nullptr;
    staging_bytes = 0;
    CK(cudaMalloc(&staging, bytes));
    staging_bytes = bytes;
    return 0;
  }

  int init_uniform(double t1, double p1, double u0, double v0, const double* scale) override {
    CK(cudaSetDevice(device));
    // INICON2 (src/inicon2.f90:120-174) evaluated per velocity in double
    const double PI = 3.1416, NA = 6.022e26;
    const double rho1 = (p1 * 100000.0) / (pl.rgas * t1);
    const double n1 = rho1 * NA / pl.M;
    const double tmp1 = rho1 / (2 * p1 * 100000.0);
    const double beta1 = std::sqrt(tmp1);
    std::vector<double> g(pl.V, 0.0);
    const bool vacuum = !(n1 >= 1e-20);
    if (!vacuum) {
      const double co = (beta1 * beta1) / PI;
      for (int v = 0; v < pl.V; ++v) {
        double ux = pl.cx[v], uy = pl.cy[v];
        double tmp = (ux - u0) * (ux - u0) + (uy - v0) * (uy - v0);
        double speed = std::sqrt(tmp);
        tmp = -((beta1 * beta1) * (speed * speed));
        g[v] = co * std::exp(tmp);
      }
    }
    std::vector<double> sc;
    if (scale) {
      sc.resize(3 * (size_t)pl.E);
      for (int en = 0; en < pl.E; ++en)
        for (int i = 0; i < 3; ++i) sc[3 * (size_t)en + i] = scale[3 * (size_t)pl.perm[en] + i];
    }
    double *dg = nullptr, *dsc = nullptr;
    TRY(upload(&dg, g, st));
    if (scale) TRY(upload(&dsc, sc, st));
    const size_t ndg = (size_t)3 * pl.E;
    k_init_uniform<T><<<(unsigned)ndg, 128, 0, st>>>(f[0], dg, dsc, vacuum ? 0.0 : n1, pl.V, Vp, ndg);
    cudaError_t e = cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaFree(dg);
    if (dsc) cudaFree(dsc);
    CK(e);
    cur = 0;
    ++epoch;
    itime_total = 0;  // a new state: ITIME starts again
    return 0;
  }

  int init_maxwellian(const double* n, const double* u, const double* v, const double* t) override {
    CK(cudaSetDevice(device));
    std::vector<double> prm(4 * 3 * (size_t)pl.E);
    for (int en = 0; en < pl.E; ++en)
      for (int i = 0; i < 3; ++i) {
        size_t o = 3 * (size_t)pl.perm[en] + i, d = 3 * (size_t)en + i;
        prm[4 * d] = n[o];
        prm[4 * d + 1] = u[o];
        prm[4 * d + 2] = v[o];
        prm[4 * d + 3] = t[o];
      }
    double* dp = nullptr;
    TRY(upload(&dp, prm, st));
    const size_t ndg = (size_t)3 * pl.E;
    k_init_maxwellian<T><<<(unsigned)ndg, 128, 0, st>>>(f[0], dp, cxD, cyD, pl.M / 6.022e26, pl.rgas, pl.V, Vp,
                                                         ndg);
    cudaError_t e = cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaFree(dp);
    CK(e);
    cur = 0;
    ++epoch;
    itime_total = 0;  // a new state: ITIME starts again
    return 0;
  }

  // the moments of the current state (a velocity shard has them from its
  // last phase 3 or 5: the sums are over every shard)
  int moments_now() {
    if (shard) return 0;
    TRY(aux_ctrl());
    mom_fn<T>(single.mom_rows, true)<<<single.mom_grid, single.mom_warps * 32, single.mom_smem, st>>>(
        single.args, single.total_groups, single.one_case);
    CK(cudaGetLastError());
    return 0;
  }

  int macros(double* nd, double* rho, double* u, double* v, double* ps, double* temp) override {
    CK(cudaSetDevice(device));
    TRY(moments_now());
    double* out = nullptr;
    TRY(dalloc(&out, 6 * (size_t)pl.NP));
    NodalArgs a{node_off, node_dg, node_ae, nraw, disux, disuy, disps, out, out + pl.NP, out + 2 * pl.NP,
                out + 3 * pl.NP, out + 4 * pl.NP, out + 5 * pl.NP, pl.NP, pl.M / 6.022e26, pl.rgas};
    k_nodal<<<(pl.NP + 255) / 256, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h(6 * (size_t)pl.NP);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    cudaFree(out);
    CK(e);
    CK(cudaMemcpy(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    TRY(finish_status(hctrl[1]));
    double* dsts[6] = {nd, rho, u, v, ps, temp};
    for (int k = 0; k < 6; ++k)
      if (dsts[k]) std::memcpy(dsts[k], h.data() + (size_t)k * pl.NP, pl.NP * sizeof(double));
    return 0;
  }

  // dgbgk_get_macros without any allocation: the nodal fields are staged in
  // the caller-supplied device scratch (the library's static array) and
  // copied straight into the caller's host arrays.
  int macros_noalloc(double* scratch, double* nd, double* rho, double* u, double* v, double* ps,
                     double* temp) override {
    CK(cudaSetDevice(device));
    TRY(moments_now());
    const int NP = pl.NP;
    NodalArgs a{node_off, node_dg, node_ae, nraw,          disux,  disuy,          disps,
                scratch,  scratch + NP, scratch + 2 * NP, scratch + 3 * NP, scratch + 4 * NP,
                scratch + 5 * NP, NP, pl.M / 6.022e26, pl.rgas};
    k_nodal<<<(NP + 255) / 256, 256, 0, st>>>(a);
    CK(cudaGetLastError());
    double* dsts[6] = {nd, rho, u, v, ps, temp};
    for (int k = 0; k < 6; ++k)
      if (dsts[k])
        CK(cudaMemcpyAsync(dsts[k], scratch + (size_t)k * NP, NP * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return finish_status(hctrl[1]);
  }

  int node_fields(double* nd, double* ux, double* uy, double* ps, double* muo) override {
    CK(cudaSetDevice(device));
    TRY(moments_now());
    const size_t ndg = 3 * (size_t)pl.E;
    std::vector<double> h(5 * ndg);
    CK(cudaMemcpyAsync(h.data(), nraw, ndg * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h.data() + ndg, disux, ndg * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h.data() + 2 * ndg, disuy, ndg * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h.data() + 3 * ndg, disps, ndg * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h.data() + 4 * ndg, mu, ndg * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    TRY(finish_status(hctrl[1]));
    double* dsts[5] = {nd, ux, uy, ps, muo};
    for (int k = 0; k < 5; ++k) {
      if (!dsts[k]) continue;
      for (int eo = 0; eo < pl.E; ++eo)
        for (int i = 0; i < 3; ++i) {
          double x = h[(size_t)k * ndg + 3 * (size_t)pl.inv[eo] + i];
          if (k == 0 && !(x >= 1e-20)) x = 0.0;  // DISND stays 0 below 1e-20
          dsts[k][3 * (size_t)eo + i] = x;
        }
    }
    return 0;
  }

  int wall_eta(double* eta) override {
    CK(cudaSetDevice(device));
    TRY(aux_ctrl());
    CK(cudaMemsetAsync(bEtaD, 0, std::max(pl.B, 1) * sizeof(double), st));
    if (single.total_walls > 0) {
      k_wall<T><<<single.total_walls, WALL_THREADS, 0, st>>>(single.args, single.total_walls);
      CK(cudaGetLastError());
    }
    if (pl.B) CK(cudaMemcpyAsync(eta, bEtaD, pl.B * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
  }

  void info(int* o) override {
    o[0] = pl.E;
    o[1] = pl.NP;
    o[2] = pl.B;
    o[3] = pl.S;
    o[4] = pl.V;
    o[5] = prec;
    o[6] = pl.EB;
    o[7] = SweepGeo<T>::VT;
    o[8] = pl.nblocks;
    o[9] = pl.max_halo;
  }
};

}  // namespace

struct dgbgk_handle {
  std::unique_ptr<ImplBase> impl;
};

extern "C" {

const char* dgbgk_last_error(void) { return g_err.c_str(); }

int dgbgk_create(const dgbgk_mesh* mesh, const dgbgk_vspace* vs, const dgbgk_params* prm,
                 dgbgk_handle** out) {
  if (!mesh || !vs || !prm || !out) {
    set_error("dgbgk_create: NULL argument");
    return DGBGK_EINVAL;
  }
  *out = nullptr;
  if (prm->precision != 64 && prm->precision != 32) {
    set_error("dgbgk_create: precision must be 32 or 64");
    return DGBGK_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    set_error("dgbgk_create: no CUDA device available (this library has no CPU fallback)");
    return DGBGK_ECUDA;
  }
  if (prm->device < 0 || prm->device >= ndev) {
    set_error("dgbgk_create: bad device ordinal");
    return DGBGK_EINVAL;
  }
  CK(cudaSetDevice(prm->device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, prm->device));
  if (prop.major != 10) {
    set_error("dgbgk_create: this build targets sm_100a (B200); found sm_" + std::to_string(prop.major) +
              std::to_string(prop.minor));
    return DGBGK_ECUDA;
  }
  std::unique_ptr<ImplBase> impl;
  if (prm->precision == 64)
    impl.reset(new Impl<double>());
  else
    impl.reset(new Impl<float>());
  impl->device = prm->device;
  impl->prec = prm->precision;
  if (prm->moment_rows < 0 || prm->moment_rows > 4) {
    set_error("dgbgk_create: moment_rows must be 0 (the library's choice) or 1 to 4");
    return DGBGK_EINVAL;
  }
  impl->mom_rows_req = prm->moment_rows;
  impl->shard = prm->shard != 0;
  if (impl->shard && prm->alpha < 1.0) {
    set_error("dgbgk_create: a velocity shard needs ALPHA = 1 (the specular part reads mirrored velocities)");
    return DGBGK_EUNSUP;
  }
  std::string err;
  const int eb0 = prm->tile_elems > 0      ? prm->tile_elems
                  : prm->precision == 64 ? Impl<double>::default_eb()
                                         : Impl<float>::default_eb();
  int rc = build_plan(*mesh, *vs, *prm, eb0, impl->pl, &err);
  if (rc != 0) {
    set_error(err);
    return rc;
  }
  if (prm->precision == 64)
    rc = static_cast<Impl<double>*>(impl.get())->init(eb0);
  else
    rc = static_cast<Impl<float>*>(impl.get())->init(eb0);
  if (rc != 0) return rc;
  *out = new dgbgk_handle{std::move(impl)};
  return DGBGK_OK;
}

#define HCHECK(h)               \
  do {                          \
    if (!(h) || !(h)->impl) {   \
      set_error("NULL handle"); \
      return DGBGK_EINVAL;      \
    }                           \
  } while (0)

int dgbgk_set_state(dgbgk_handle* h, const double* disnf) {
  HCHECK(h);
  if (!disnf) return set_error("NULL state"), DGBGK_EINVAL;
  return h->impl->set_state(disnf, false);
}
int dgbgk_set_state_f32(dgbgk_handle* h, const float* disnf) {
  HCHECK(h);
  if (!disnf) return set_error("NULL state"), DGBGK_EINVAL;
  return h->impl->set_state(disnf, true);
}
int dgbgk_get_state(dgbgk_handle* h, double* disnf) {
  HCHECK(h);
  if (!disnf) return set_error("NULL state"), DGBGK_EINVAL;
  return h->impl->get_state(disnf, false);
}
int dgbgk_get_state_f32(dgbgk_handle* h, float* disnf) {
  HCHECK(h);
  if (!disnf) return set_error("NULL state"), DGBGK_EINVAL;
  return h->impl->get_state(disnf, true);
}
int dgbgk_init_uniform(dgbgk_handle* h, double t1, double p1, double u0, double v0, const double* scale) {
  HCHECK(h);
  return h->impl->init_uniform(t1, p1, u0, v0, scale);
}
int dgbgk_init_maxwellian(dgbgk_handle* h, const double* n, const double* u, const double* v, const double* t) {
  HCHECK(h);
  if (!n || !u || !v || !t) return set_error("NULL field"), DGBGK_EINVAL;
  return h->impl->init_maxwellian(n, u, v, t);
}
int dgbgk_advance(dgbgk_handle* h, int max_steps, double tol_rel, int* steps_done, double* res_linf,
                  double* res_l2, double* dte) {
  HCHECK(h);
  return h->impl->advance(max_steps, tol_rel, steps_done, res_linf, res_l2, dte);
}
int dgbgk_set_residual_reference(dgbgk_handle* h, double r) {
  HCHECK(h);
  if (!(r >= 0)) return set_error("bad residual reference"), DGBGK_EINVAL;
  h->impl->ref_host = r;
  return 0;
}
int dgbgk_get_residual_reference(dgbgk_handle* h, double* r) {
  HCHECK(h);
  if (!r) return set_error("NULL pointer"), DGBGK_EINVAL;
  *r = h->impl->ref_host;
  return 0;
}
int dgbgk_snapshot(dgbgk_handle* h, int slot) {
  HCHECK(h);
  return h->impl->snapshot(slot);
}
int dgbgk_extrapolate(dgbgk_handle* h, int n, double* gamma) {
  HCHECK(h);
  return h->impl->extrapolate(n, gamma);
}
int dgbgk_copy_state(dgbgk_handle* dst, const dgbgk_handle* src) {
  HCHECK(dst);
  HCHECK(src);
  ImplBase* d = dst->impl.get();
  ImplBase* s_ = src->impl.get();
  if (d->device != s_->device || d->pl.E != s_->pl.E || d->pl.V != s_->pl.V || d->pl.NP != s_->pl.NP ||
      d->pl.B != s_->pl.B)
    return set_error("dgbgk_copy_state: the handles differ in device, mesh or velocity grid"), DGBGK_EINVAL;
  if (d == s_) return 0;
  CK(cudaSetDevice(d->device));
  double* buf = nullptr;
  CK(cudaMalloc(&buf, (size_t)3 * d->pl.E * d->pl.V * sizeof(double)));
  int rc = s_->export_device(buf);
  if (rc == 0) rc = d->import_device(buf);
  cudaFree(buf);
  if (rc == 0) d->ref_host = s_->ref_host;
  if (rc == 0) d->itime_total = s_->itime_total;
  return rc;
}
int dgbgk_get_macros(dgbgk_handle* h, double* nd, double* rho, double* u, double* v, double* ps, double* temp) {
  HCHECK(h);
  return h->impl->macros(nd, rho, u, v, ps, temp);
}
int dgbgk_get_forces(dgbgk_handle* h, double* lift, double* drag) {
  HCHECK(h);
  return h->impl->forces(lift, drag);
}
int dgbgk_set_output(dgbgk_handle* h, int every, int capacity) {
  HCHECK(h);
  if (h->impl->shard) return set_error("dgbgk_set_output: not for a velocity shard"), DGBGK_EINVAL;
  return h->impl->set_output(every, capacity);
}
int dgbgk_output_count(dgbgk_handle* h, int* count) {
  HCHECK(h);
  if (!count) return set_error("NULL pointer"), DGBGK_EINVAL;
  return h->impl->output_count(count);
}
int dgbgk_get_output(dgbgk_handle* h, int k, int* itime, double* nd, double* rho, double* u, double* v, double* ps,
                     double* temp, double* lift, double* drag) {
  HCHECK(h);
  double* const fields[6] = {nd, rho, u, v, ps, temp};
  return h->impl->get_output(k, itime, fields, lift, drag);
}
int dgbgk_get_node_fields(dgbgk_handle* h, double* disnd, double* disux, double* disuy, double* disps,
                          double* mu) {
  HCHECK(h);
  return h->impl->node_fields(disnd, disux, disuy, disps, mu);
}
int dgbgk_get_wall_eta(dgbgk_handle* h, double* eta) {
  HCHECK(h);
  if (!eta) return set_error("NULL pointer"), DGBGK_EINVAL;
  return h->impl->wall_eta(eta);
}
int dgbgk_info(dgbgk_handle* h, int* out10) {
  HCHECK(h);
  if (!out10) return set_error("NULL pointer"), DGBGK_EINVAL;
  h->impl->info(out10);
  return 0;
}
int dgbgk_last_timing(dgbgk_handle* h, double* total_ms) {
  HCHECK(h);
  if (!total_ms) return set_error("NULL pointer"), DGBGK_EINVAL;
  *total_ms = h->impl->last_ms;
  return 0;
}
int dgbgk_profile_steps(dgbgk_handle* h, int nsteps, double* kernel_ms) {
  HCHECK(h);
  if (!kernel_ms || nsteps < 1) return set_error("bad arguments"), DGBGK_EINVAL;
  return h->impl->profile(nsteps, kernel_ms);
}
#define SCHECK(h)                                                                   \
  do {                                                                              \
    HCHECK(h);                                                                      \
    if (!(h)->impl->shard) return set_error("not a velocity shard"), DGBGK_EINVAL; \
  } while (0)
int dgbgk_shard_stream(dgbgk_handle* h, void** stream) {
  SCHECK(h);
  if (!stream) return set_error("NULL pointer"), DGBGK_EINVAL;
  *stream = h->impl->stream_ptr();
  return 0;
}
int dgbgk_shard_sizes(dgbgk_handle* h, long long* n_sums1, long long* n_sums2) {
  SCHECK(h);
  const long long n3 = 3LL * h->impl->pl.E;
  if (n_sums1) *n_sums1 = 3 * n3;
  if (n_sums2) *n_sums2 = 2 * n3 + (long long)h->impl->pl.walls.size();
  return 0;
}
int dgbgk_shard_begin(dgbgk_handle* h, int max_steps, double tol) {
  SCHECK(h);
  if (max_steps < 1) return set_error("dgbgk_shard_begin: max_steps >= 1"), DGBGK_EINVAL;
  return h->impl->shard_begin(max_steps, tol);
}
int dgbgk_shard_phase(dgbgk_handle* h, int phase, double* sums1, double* sums2, double* res) {
  SCHECK(h);
  if ((phase >= 1 && phase != 4 && !sums1) || ((phase == 2 || phase == 3 || phase == 5) && !sums2) ||
      ((phase == 3 || phase == 4) && !res))
    return set_error("dgbgk_shard_phase: NULL exchange buffer"), DGBGK_EINVAL;
  return h->impl->shard_phase(phase, sums1, sums2, res);
}
int dgbgk_shard_poll(dgbgk_handle* h, int* done) {
  SCHECK(h);
  if (!done) return set_error("NULL pointer"), DGBGK_EINVAL;
  return h->impl->shard_poll(done);
}
int dgbgk_shard_end(dgbgk_handle* h, int* steps_done, double* res_linf, double* res_l2, double* dte, int* done) {
  SCHECK(h);
  return h->impl->shard_end(steps_done, res_linf, res_l2, dte, done);
}
void dgbgk_destroy(dgbgk_handle* h) { delete h; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches: many handles advanced by one launch set (one persistent launch
// per kernel and step, captured in a CUDA graph).
namespace {

// 1 when every case of the set is done
template <class T> __global__ void k_all_done(BatchArgs<T> a, int* out) {
  int active = 0;
  for (int c = threadIdx.x; c < a.ncases; c += blockDim.x) active |= !a.cases[c].ctrl->done;
  active = __syncthreads_or(active);
  if (threadIdx.x == 0) *out = !active;
}

struct BatchBase {
  virtual ~BatchBase() {}
  virtual int advance(int max_steps, double tol, int* steps, double* l2) = 0;
  virtual void info(int* out) const = 0;
  virtual int tuning(int n, double* ms) const = 0;
  virtual int snapshot(int slot, const int* which) = 0;
  virtual int extrapolate(int n, const int* which, int* status, double* gamma) = 0;
  float last_ms = 0.f;
  std::vector<int> last_rc;  // per case: the status of the last advance
  std::vector<int> active;   // per case: 0 = left out of the advances (dgbgk_batch_set_active)
};

template <class T> struct BatchImpl : BatchBase {
  static constexpr int GRAPH_STEPS = 2;
  std::vector<Impl<T>*> cs;
  LaunchSet<T> L;
  int device = 0, nsm = 148, eb = 128, upc = 8, immat = 1, max_halo = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec = nullptr;
  int* d_done = nullptr;
  int* h_done = nullptr;  // pinned [2]
  double* h_l2 = nullptr;  // pinned [ncases]: the cases' last L2 residuals
  // extrapolation of the whole batch: pinned Gram matrices and coefficients
  // [ncases][RRE_MAX^2], [ncases][RRE_MAX]; the event the cases' streams
  // wait on after work queued on the batch's stream
  double *h_gram = nullptr, *h_gamma = nullptr;
  cudaEvent_t ev_q = nullptr;
  int rows = 0;           // moment rows per warp step (0: the heuristic)
  // ms per step: (eb 64, 128) x (upc 2, 4, 8, 16), then moment rows 1, 2, 3, 4;
  // 0 = not tried
  std::vector<double> tune_ms;
  // per case: the handle's table generation the launch set was built from
  std::vector<unsigned> gens;
  // per case: a non-zero status that stops the case (divergence, expired
  // wait) and the state epoch it belongs to; a new state clears it
  std::vector<int> stop_rc;
  std::vector<unsigned> stop_epoch;

  ~BatchImpl() override {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    if (gexec) cudaGraphExecDestroy(gexec);
    L.release();
    dfree(d_done);
    if (h_done) cudaFreeHost(h_done);
    if (h_l2) cudaFreeHost(h_l2);
    if (h_gram) cudaFreeHost(h_gram);
    if (h_gamma) cudaFreeHost(h_gamma);
    if (ev_q) cudaEventDestroy(ev_q);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto& e : evp)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int init(std::vector<Impl<T>*> cases) {
    cs = std::move(cases);
    device = cs[0]->device;
    nsm = cs[0]->nsm;
    immat = cs[0]->pl.immat;
    for (auto* c : cs) {
      if (c->device != device || c->pl.immat != immat) {
        set_error("dgbgk_batch_create: cases must share the device, the precision and IMMAT");
        return DGBGK_EINVAL;
      }
    }
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    for (auto& e : evp) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TRY(dalloc(&d_done, 1));
    CK(cudaMallocHost((void**)&h_done, 2 * sizeof(int)));
    CK(cudaMallocHost((void**)&h_l2, cs.size() * sizeof(double)));
    tune_ms.assign(12, 0.0);
    active.assign(cs.size(), 1);
    stop_rc.assign(cs.size(), 0);
    stop_epoch.assign(cs.size(), 0);
    last_rc.assign(cs.size(), 0);
    return 0;
  }

  // the case runs in the next advance: active and not stopped (a stop
  // lapses once the case's state was written anew)
  bool runs(size_t i) {
    if (stop_rc[i] != 0 && stop_epoch[i] != cs[i]->epoch) stop_rc[i] = 0;
    return active[i] && stop_rc[i] == 0;
  }

  // Re-blocks every case to EB = e and gives each case its tiles per unit
  // from the whole batch's work (about u units per resident CTA).
  int configure(int e, int u) {
    for (auto* c : cs) {
      TRY(c->set_tile(e, u));
      CK(cudaStreamSynchronize(c->st));
    }
    max_halo = 0;
    long tiles = 0;
    for (auto* c : cs) {
      max_halo = std::max(max_halo, c->pl.max_halo);
      tiles += (long)c->pl.nblocks * c->nvt();
    }
    const int sps = sweep_per_sm<T>(e, immat, max_halo, cs.size() == 1);
    if (sps < 1) {
      set_error("dgbgk_batch: the sweep tile does not fit on an SM");
      return DGBGK_EUNSUP;
    }
    std::vector<CaseDev<T>> table;
    for (auto* c : cs) {
      set_groups(c->hc, c->nvt(), tiles_per_unit(tiles, sps * nsm, u, c->nvt()), cs.size() == 1);
      table.push_back(c->hc);
    }
    TRY(build_launch_set(L, table, e, immat, max_halo, nsm, st, rows));
    gens.clear();
    for (auto* c : cs) gens.push_back(c->gen);
    eb = e;
    upc = u;
    if (gexec) {
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
    return 0;
  }

  // every case's control block for an advance; a case that does not run
  // is uploaded finished (the kernels skip it; its step count stays 0)
  int upload_ctrls(int max_steps, double tol) {
    for (size_t i = 0; i < cs.size(); ++i) {
      Impl<T>* c = cs[i];
      c->fill_ctrl(c->hctrl[0], max_steps, tol);
      if (!runs(i)) c->hctrl[0].done = 1;
      CK(cudaMemcpyAsync(c->ctrl, &c->hctrl[0], sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    }
    return 0;
  }

  // Autotuner: times `steps` steps (after one untimed) of every candidate
  // tile shape on the cases' current states, restoring the states after
  // each, and keeps the fastest.
  int autotune(int fixed_eb, int fixed_upc, int fixed_rows, int steps) {
    std::vector<T*> backup(cs.size(), nullptr);
    int rc = 0;
    for (size_t i = 0; i < cs.size() && rc == 0; ++i) {
      const size_t n = (size_t)3 * cs[i]->pl.E * cs[i]->Vp;
      rc = dalloc(&backup[i], n);
      if (rc == 0 && cudaMemcpyAsync(backup[i], cs[i]->f[cs[i]->cur], n * sizeof(T), cudaMemcpyDeviceToDevice, st) !=
                         cudaSuccess)
        rc = DGBGK_ECUDA;
    }
    auto restore = [&]() -> int {
      for (size_t i = 0; i < cs.size(); ++i) {
        const size_t n = (size_t)3 * cs[i]->pl.E * cs[i]->Vp;
        CK(cudaMemcpyAsync(cs[i]->f[cs[i]->cur], backup[i], n * sizeof(T), cudaMemcpyDeviceToDevice, st));
      }
      CK(cudaStreamSynchronize(st));
      return 0;
    };
    // ms per step of the current configuration (one untimed step first)
    auto trial = [&](double* per) -> int {
      TRY(upload_ctrls(steps + 1, 0.0));
      TRY(enqueue_step(L, st));
      CK(cudaEventRecord(ev0, st));
      for (int k = 0; k < steps; ++k) TRY(enqueue_step(L, st));
      CK(cudaEventRecord(ev1, st));
      float ms = 0.f;
      CK(cudaEventSynchronize(ev1));
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      *per = ms / std::max(steps, 1);
      return restore();
    };
    const int ebs[2] = {64, 128}, upcs[4] = {2, 4, 8, 16}, rws[4] = {1, 2, 3, 4};
    double best = 1e300;
    int beb = fixed_eb > 0 ? fixed_eb : 128, bupc = fixed_upc > 0 ? fixed_upc : 8;
    for (int ie = 0; ie < 2 && rc == 0; ++ie) {
      if (fixed_eb > 0 && ebs[ie] != fixed_eb) continue;
      for (int iu = 0; iu < 4 && rc == 0; ++iu) {
        if (fixed_upc > 0 && upcs[iu] != fixed_upc) continue;
        rc = configure(ebs[ie], upcs[iu]);
        if (rc == DGBGK_EUNSUP) {  // shape does not fit: skip it
          rc = 0;
          continue;
        }
        double per = 0;
        if (rc == 0) rc = trial(&per);
        if (rc == 0) {
          tune_ms[ie * 4 + iu] = per;
          if (per < best) {
            best = per;
            beb = ebs[ie];
            bupc = upcs[iu];
          }
        }
      }
    }
    // then the moment kernel's rows per warp step for the chosen sweep shape
    int brows = 0;
    best = 1e300;
    for (int ir = 0; ir < 4 && rc == 0; ++ir) {
      if (fixed_rows > 0 && rws[ir] != fixed_rows) continue;
      rows = rws[ir];
      rc = configure(beb, bupc);
      if (rc == DGBGK_EUNSUP) {
        rc = 0;
        continue;
      }
      double per = 0;
      if (rc == 0) rc = trial(&per);
      if (rc == 0) {
        tune_ms[8 + ir] = per;
        if (per < best) {
          best = per;
          brows = rws[ir];
        }
      }
    }
    rows = brows;
    for (T* p : backup) dfree(p);
    TRY(rc);
    return configure(beb, bupc);
  }

  int build_graph() {
    if (gexec) return 0;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    for (int k = 0; k < GRAPH_STEPS && rc == 0; ++k) rc = enqueue_step(L, st);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != 0) return rc;
    CK(e);
    CK(cudaGraphInstantiate(&gexec, g, 0));
    cudaGraphDestroy(g);
    return 0;
  }

  int advance(int max_steps, double tol, int* steps, double* l2) override {
    if (max_steps < 0) {
      set_error("max_steps < 0");
      return DGBGK_EINVAL;
    }
    CK(cudaSetDevice(device));
    for (auto* c : cs)
      if (c->hist_cap < max_steps) TRY(c->ensure_hist(max_steps));
    // a case's table entry changed since the launch set was built (its
    // history grew above, or it was re-blocked or grown on its own or by
    // another batch): rebuild the table before any launch reads it
    bool stale = gens.size() != cs.size();
    for (size_t i = 0; i < cs.size() && !stale; ++i) stale = gens[i] != cs[i]->gen;
    if (stale) TRY(configure(eb, upc));
    for (auto* c : cs) CK(cudaStreamSynchronize(c->st));
    TRY(build_graph());
    TRY(upload_ctrls(max_steps, tol));
    CK(cudaEventRecord(ev0, st));
    const int launches = max_steps > 0 ? (max_steps + GRAPH_STEPS - 1) / GRAPH_STEPS : 0;
    const int chunk = 32;
    int issued = 0, chunks = 0;
    bool stop = false;
    while (issued < launches && !stop) {
      const int n = std::min(chunk, launches - issued);
      for (int i = 0; i < n; ++i) CK(cudaGraphLaunch(gexec, st));
      issued += n;
      k_all_done<T><<<1, 256, 0, st>>>(L.args, d_done);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(&h_done[chunks & 1], d_done, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(evp[chunks & 1], st));
      ++chunks;
      if (chunks >= 2) {  // look at the chunk before the one just issued
        CK(cudaEventSynchronize(evp[chunks & 1]));
        if (h_done[chunks & 1]) stop = true;
      }
    }
    CK(cudaEventRecord(ev1, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&last_ms, ev0, ev1));
    int rc = 0;
    last_rc.assign(cs.size(), 0);
    // the running cases' control blocks, then their last L2 residuals: one
    // wait for each set of copies
    auto running = [&](size_t i) { return active[i] && stop_rc[i] == 0; };
    for (size_t i = 0; i < cs.size(); ++i)
      if (running(i)) CK(cudaMemcpyAsync(&cs[i]->hctrl[1], cs[i]->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int> ns(cs.size(), 0);
    for (size_t i = 0; i < cs.size(); ++i) {
      Impl<T>* c = cs[i];
      if (steps) steps[i] = 0;
      if (l2) l2[i] = 0.0;
      if (!active[i]) continue;
      if (stop_rc[i] != 0) {  // stopped before this advance: keeps its status
        last_rc[i] = stop_rc[i];
        if (rc == 0) rc = stop_rc[i];
        continue;
      }
      const int r = c->collect(c->hctrl[1], &ns[i], nullptr, nullptr, nullptr);
      last_rc[i] = r;
      if (r != 0) {
        stop_rc[i] = r;
        stop_epoch[i] = c->epoch;
        if (rc == 0) rc = r;
      }
      if (steps) steps[i] = ns[i];
      if (l2 && ns[i] > 0)
        CK(cudaMemcpyAsync(&h_l2[i], c->hist_l2 + ns[i] - 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (l2) {
      CK(cudaStreamSynchronize(st));
      for (size_t i = 0; i < cs.size(); ++i)
        if (ns[i] > 0) l2[i] = h_l2[i];
    }
    return rc;
  }

  // every later use of a case on its own stream follows the work just
  // queued on the batch's stream
  int release_to_cases(const std::vector<int>& sel) {
    if (!ev_q) CK(cudaEventCreateWithFlags(&ev_q, cudaEventDisableTiming));
    CK(cudaEventRecord(ev_q, st));
    for (int i : sel) CK(cudaStreamWaitEvent(cs[i]->st, ev_q, 0));
    return 0;
  }

  // dgbgk_snapshot(slot) of the selected cases, the copies queued on the
  // batch's stream (no wait; the next advance follows them)
  int snapshot(int slot, const int* which) override {
    CK(cudaSetDevice(device));
    if (slot < 0 || slot >= RRE_MAX) {
      set_error("dgbgk_batch_snapshot: slot outside 0 .. " + std::to_string(RRE_MAX - 1));
      return DGBGK_EINVAL;
    }
    std::vector<int> sel;
    bool grow = false;
    for (size_t i = 0; i < cs.size(); ++i)
      if (!which || which[i]) {
        sel.push_back((int)i);
        grow |= slot >= cs[i]->snap_cap;
      }
    if (grow) CK(cudaStreamSynchronize(st));  // copies into the old slots land first
    for (int i : sel) {
      Impl<T>* c = cs[i];
      CK(cudaStreamSynchronize(c->st));  // the case's own queued work on its state
      if (slot >= c->snap_cap) TRY(c->grow_snaps(c->snap_grow(slot)));
      c->snap_n = std::max(c->snap_n, slot + 1);
      const size_t N = (size_t)3 * c->pl.E * c->Vp;
      CK(cudaMemcpyAsync(c->snaps + (size_t)slot * N, c->f[c->cur], N * sizeof(T), cudaMemcpyDeviceToDevice, st));
    }
    return release_to_cases(sel);
  }

  // dgbgk_extrapolate(n) of the selected cases: all Gram matrices formed
  // before one wait, then each case's coefficients and combination
  int extrapolate(int n, const int* which, int* status, double* gamma) override {
    CK(cudaSetDevice(device));
    const int m = n - 1;
    const size_t GS = (size_t)RRE_MAX * RRE_MAX;
    if (!h_gram) CK(cudaMallocHost((void**)&h_gram, cs.size() * GS * sizeof(double)));
    if (!h_gamma) CK(cudaMallocHost((void**)&h_gamma, cs.size() * RRE_MAX * sizeof(double)));
    std::vector<int> sel;
    int rc = 0;
    for (size_t i = 0; i < cs.size(); ++i) {
      status[i] = 0;
      if (which && !which[i]) continue;
      if (n < 2 || n > cs[i]->snap_n) {
        status[i] = DGBGK_EINVAL;
        set_error("dgbgk_batch_extrapolate: needs 2 <= n <= the snapshots taken");
        if (rc == 0) rc = DGBGK_EINVAL;
        continue;
      }
      sel.push_back((int)i);
    }
    CK(cudaStreamSynchronize(st));  // the gamma buffer's earlier copies
    for (int i : sel) {
      Impl<T>* c = cs[i];
      CK(cudaStreamSynchronize(c->st));
      if (!c->d_gram) TRY(dalloc(&c->d_gram, GS));
      if (!c->d_gamma) TRY(dalloc(&c->d_gamma, (size_t)RRE_MAX));
      const size_t N = (size_t)3 * c->pl.E * c->Vp;
      CK(cudaMemsetAsync(c->d_gram, 0, (size_t)m * m * sizeof(double), st));
      const int grid = (int)std::min<size_t>((size_t)4 * nsm, (N + 255) / 256);
      k_gram<T><<<grid, 256, 0, st>>>(c->snaps, N, n, N, c->d_gram);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h_gram + i * GS, c->d_gram, (size_t)m * m * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    std::vector<int> done;
    for (int i : sel) {
      Impl<T>* c = cs[i];
      std::vector<double> G(h_gram + i * GS, h_gram + i * GS + (size_t)m * m), g;
      const int r = rre_coeffs(G, m, g);
      status[i] = r;
      if (r != 0) {
        if (rc == 0) rc = r;
        continue;
      }
      if (gamma) std::copy(g.begin(), g.end(), gamma + (size_t)i * m);
      std::copy(g.begin(), g.end(), h_gamma + (size_t)i * RRE_MAX);
      CK(cudaMemcpyAsync(c->d_gamma, h_gamma + (size_t)i * RRE_MAX, m * sizeof(double), cudaMemcpyHostToDevice, st));
      const size_t N = (size_t)3 * c->pl.E * c->Vp;
      const int grid = (int)std::min<size_t>((size_t)4 * nsm, (N + 255) / 256);
      k_combine<T><<<grid, 256, 0, st>>>(c->snaps, N, m, c->d_gamma, N, c->f[c->cur]);
      CK(cudaGetLastError());
      ++c->epoch;
      done.push_back(i);
    }
    TRY(release_to_cases(done));
    return rc;
  }

  void info(int* o) const override {
    o[0] = (int)cs.size();
    o[1] = eb;
    o[2] = upc;
    o[3] = L.total_units;
    o[4] = L.sweep_grid;
    o[5] = L.mom_grid;
    o[6] = L.mom_rows;
  }
  int tuning(int n, double* ms) const override {
    for (int i = 0; i < n && i < (int)tune_ms.size(); ++i) ms[i] = tune_ms[i];
    return 0;
  }
};

}  // namespace

struct dgbgk_batch {
  std::unique_ptr<BatchBase> impl;
};

extern "C" {

void dgbgk_batch_default_params(dgbgk_batch_params* p) {
  if (!p) return;
  p->tile_elems = 0;
  p->units_per_cta = 0;
  p->tune_steps = 4;
  p->moment_rows = 0;
}

int dgbgk_batch_create(dgbgk_handle* const* cases, int ncases, const dgbgk_batch_params* prm,
                       dgbgk_batch** out) {
  if (!cases || ncases < 1 || !out) {
    set_error("dgbgk_batch_create: no cases");
    return DGBGK_EINVAL;
  }
  *out = nullptr;
  dgbgk_batch_params p;
  dgbgk_batch_default_params(&p);
  if (prm) p = *prm;
  const int prec = cases[0] && cases[0]->impl ? cases[0]->impl->prec : 0;
  for (int i = 0; i < ncases; ++i) {
    if (!cases[i] || !cases[i]->impl || cases[i]->impl->prec != prec) {
      set_error("dgbgk_batch_create: NULL handle or mixed precision");
      return DGBGK_EINVAL;
    }
    if (cases[i]->impl->shard) {
      set_error("dgbgk_batch_create: a velocity shard steps through dgbgk_shard_*");
      return DGBGK_EINVAL;
    }
  }
  for (int i = 0; i < ncases; ++i)
    for (int k = 0; k < i; ++k)
      if (cases[i] == cases[k]) {
        set_error("dgbgk_batch_create: a handle appears twice");
        return DGBGK_EINVAL;
      }
  std::unique_ptr<BatchBase> b;
  int rc = 0;
  if (prec == 64) {
    auto* bi = new BatchImpl<double>();
    b.reset(bi);
    std::vector<Impl<double>*> v;
    for (int i = 0; i < ncases; ++i) v.push_back(static_cast<Impl<double>*>(cases[i]->impl.get()));
    rc = bi->init(v);
    if (rc == 0) rc = bi->autotune(p.tile_elems, p.units_per_cta, p.moment_rows, std::max(1, p.tune_steps));
  } else {
    auto* bi = new BatchImpl<float>();
    b.reset(bi);
    std::vector<Impl<float>*> v;
    for (int i = 0; i < ncases; ++i) v.push_back(static_cast<Impl<float>*>(cases[i]->impl.get()));
    rc = bi->init(v);
    if (rc == 0) rc = bi->autotune(p.tile_elems, p.units_per_cta, p.moment_rows, std::max(1, p.tune_steps));
  }
  if (rc != 0) return rc;
  *out = new dgbgk_batch{std::move(b)};
  return DGBGK_OK;
}

int dgbgk_batch_advance(dgbgk_batch* b, int max_steps, double tol, int* steps_done, double* res_l2_last) {
  if (!b || !b->impl) return set_error("NULL batch"), DGBGK_EINVAL;
  return b->impl->advance(max_steps, tol, steps_done, res_l2_last);
}

int dgbgk_batch_set_active(dgbgk_batch* b, const int* active) {
  if (!b || !b->impl || !active) return set_error("NULL batch"), DGBGK_EINVAL;
  for (size_t i = 0; i < b->impl->active.size(); ++i) b->impl->active[i] = active[i] != 0;
  return DGBGK_OK;
}

int dgbgk_batch_snapshot(dgbgk_batch* b, int slot, const int* which) {
  if (!b || !b->impl) return set_error("NULL batch"), DGBGK_EINVAL;
  return b->impl->snapshot(slot, which);
}

int dgbgk_batch_extrapolate(dgbgk_batch* b, int n, const int* which, int* status, double* gamma) {
  if (!b || !b->impl || !status) return set_error("NULL batch or status"), DGBGK_EINVAL;
  return b->impl->extrapolate(n, which, status, gamma);
}

int dgbgk_batch_status(const dgbgk_batch* b, int* status) {
  if (!b || !b->impl || !status) return set_error("NULL batch"), DGBGK_EINVAL;
  for (size_t i = 0; i < b->impl->last_rc.size(); ++i) status[i] = b->impl->last_rc[i];
  return DGBGK_OK;
}

int dgbgk_batch_info(const dgbgk_batch* b, int* out) {
  if (!b || !b->impl || !out) return set_error("NULL batch"), DGBGK_EINVAL;
  b->impl->info(out);
  return DGBGK_OK;
}

int dgbgk_batch_tuning(const dgbgk_batch* b, int n, double* ms_per_step) {
  if (!b || !b->impl || !ms_per_step) return set_error("NULL batch"), DGBGK_EINVAL;
  return b->impl->tuning(n, ms_per_step);
}

int dgbgk_batch_last_timing(const dgbgk_batch* b, double* total_ms) {
  if (!b || !b->impl || !total_ms) return set_error("NULL batch"), DGBGK_EINVAL;
  *total_ms = b->impl->last_ms;
  return DGBGK_OK;
}

void dgbgk_batch_destroy(dgbgk_batch* b) { delete b; }

}  // extern "C"

// ---------------------------------------------------------------------------
// dgbgk_get_macros_noalloc: scratch in a file-scope device array.
//
// The array lives in every GPU's memory that loads this library, for the
// life of the process (6 * DGBGK_NOALLOC_MAX_NPOIN doubles, ~6.3 MB).  Host
// code must not use its name as a pointer (that is a host-side stand-in);
// the device address is taken once per device with cudaGetSymbolAddress
// while that device is current, on the first call made on the device.
// The nodal gather writes every one of the 6*NPOIN entries it uses, so no
// part of the array needs clearing between calls.
static __device__ __align__(256) double g_macros_scratch[6 * DGBGK_NOALLOC_MAX_NPOIN];

namespace {
constexpr int kMaxDevices = 64;
double* g_macros_scratch_dev[kMaxDevices] = {};
std::mutex g_macros_scratch_mu;

int macros_scratch_on(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("dgbgk_get_macros_noalloc: device ordinal out of range");
    return DGBGK_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_macros_scratch_mu);
  if (!g_macros_scratch_dev[device]) {
    void* p = nullptr;
    CK(cudaSetDevice(device));
    CK(cudaGetSymbolAddress(&p, g_macros_scratch));
    g_macros_scratch_dev[device] = static_cast<double*>(p);
  }
  *out = g_macros_scratch_dev[device];
  return 0;
}
}  // namespace

extern "C" {

int dgbgk_get_macros_noalloc(dgbgk_handle* h, double* nd, double* rho, double* u, double* v, double* ps,
                             double* temp) {
  HCHECK(h);
  if (h->impl->pl.NP > DGBGK_NOALLOC_MAX_NPOIN) {
    set_error("dgbgk_get_macros_noalloc: NPOIN = " + std::to_string(h->impl->pl.NP) +
              " exceeds DGBGK_NOALLOC_MAX_NPOIN = " + std::to_string(DGBGK_NOALLOC_MAX_NPOIN));
    return DGBGK_EINVAL;
  }
  double* scratch = nullptr;
  TRY(macros_scratch_on(h->impl->device, &scratch));
  return h->impl->macros_noalloc(scratch, nd, rho, u, v, ps, temp);
}

}  // extern "C"

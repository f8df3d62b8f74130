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
  Plan pl;
  int device = 0;
  int prec = 64;
  int nsm = 148;
  double ref_host = 0.0;
  float last_ms = 0.f;
};

template <class T> struct Impl : ImplBase {
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evpoll[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int cur = 0;
  int tpu = 1;  // velocity tiles per sweep work unit
  int Vp = 0;
  // device arrays
  T* f[2] = {nullptr, nullptr};
  CUtensorMap tm[2];  // f[b] as a 2-D tensor of rows (sweep tile boxes)
  ElemRec<T>* rec = nullptr;
  int *halo_off = nullptr, *halo_list = nullptr;
  T *cmax = nullptr, *cmin = nullptr;
  T* tabs = nullptr;  // moment tables [3][Vp]
  double *nraw = nullptr, *disux = nullptr, *disuy = nullptr, *disps = nullptr, *mu = nullptr;
  T *cxT = nullptr, *cyT = nullptr, *nfT = nullptr;
  double *cxD = nullptr, *cyD = nullptr, *wjf = nullptr;
  T *bTw = nullptr, *bUw = nullptr, *bEta = nullptr;
  double* bEtaD = nullptr;
  WallSide* walls = nullptr;
  int *node_off = nullptr, *node_dg = nullptr;
  double* node_ae = nullptr;
  double *part_max = nullptr, *part_sq = nullptr;
  int nparts = 0, sweep_grid = 0, part_cap = 0;
  int mom_grid = 0, mom_warps = 0, mom_stages = 0, mom_rows = 4;
  size_t mom_smem = 0;
  double *hist_linf = nullptr, *hist_l2 = nullptr, *hist_dt = nullptr;
  int hist_cap = 0;
  Ctrl* ctrl = nullptr;
  Ctrl* hctrl = nullptr;  // pinned: [0] upload, [1..2] polls
  void* staging = nullptr;
  size_t staging_bytes = 0;
  int* d_inv = nullptr;

  ~Impl() override {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
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
    dfree(cxT);
    dfree(cyT);
    dfree(nfT);
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
    dfree(part_max);
    dfree(part_sq);
    dfree(hist_linf);
    dfree(hist_l2);
    dfree(hist_dt);
    dfree(ctrl);
    if (staging) cudaFree(staging);
    if (hctrl) cudaFreeHost(hctrl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto& e : evpoll)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int nvt() const { return (pl.V + SweepGeo<T>::VT - 1) / SweepGeo<T>::VT; }
  static int default_eb() { return 128; }
  size_t sweep_smem() const { return SweepGeo<T>::smem(pl.EB, pl.max_halo); }

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
    // sweep velocity tables, zero past V
    std::vector<T> a(Vp, (T)0), b(Vp, (T)0), c(Vp, (T)0);
    for (int v = 0; v < pl.V; ++v) {
      a[v] = (T)pl.cx[v];
      b[v] = (T)pl.cy[v];
      c[v] = (T)pl.nfinf[v];
    }
    TRY(upload(&cxT, a, st));
    TRY(upload(&cyT, b, st));
    TRY(upload(&nfT, c, st));
    TRY(upload(&cxD, pl.cx, st));
    TRY(upload(&cyD, pl.cy, st));
    TRY(upload(&wjf, pl.wjf, st));
    std::vector<T> tb(3 * (size_t)Vp, (T)0);  // zero past V
    for (int v = 0; v < pl.V; ++v) {
      tb[v] = (T)pl.cx[v];
      tb[Vp + v] = (T)pl.cy[v];
      tb[2 * (size_t)Vp + v] = (T)pl.wjf[v];
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
    TRY(dalloc(&ctrl, 1));
    CK(cudaMallocHost((void**)&hctrl, 3 * sizeof(Ctrl)));
    std::memset(hctrl, 0, 3 * sizeof(Ctrl));
    CK(cudaMemcpyAsync(ctrl, hctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    TRY(config_moments());
    TRY(set_tile(tile_elems));
    TRY(ensure_hist(1024));
    CK(cudaStreamSynchronize(st));
    return 0;
  }

  // Moment kernel: per-warp rings of velocity rows, persistent grid.  Picks
  // the (warps per CTA, ring stages) with the most resident warps per SM.
  // Moment kernel: per-warp rings of R-row stages, persistent grid.  Picks
  // (rows per warp step R, warps per CTA, ring stages) with the most resident
  // warps per SM, then the most rows in flight, then the fewest rows per warp
  // step (measured on B200 at 24x48 velocities: one row per warp step was
  // fastest in FP32 and FP64).
  int config_moments() {
    const size_t rowbytes = ((size_t)pl.V * sizeof(T) + 15) / 16 * 16;
    const size_t tbytes = 3 * (size_t)Vp * sizeof(T);
    const size_t cap = 227 * 1024, sm_total = 228 * 1024;
    long best = -1;
    for (int R : {4, 2, 1})
      for (int w : {16, 12, 10, 8, 6, 5, 4, 3, 2, 1})
        for (int sg : {3, 2}) {
          const size_t bytes =
              128 * (((size_t)w * sg * 8 + 127) / 128) + tbytes + (size_t)w * sg * R * rowbytes;
          if (bytes > cap) continue;
          const int blocks = (int)std::min<size_t>(4, sm_total / (bytes + 1024));
          if (blocks < 1) continue;
          const long score = ((long)blocks * w * 1024 + (long)blocks * w * (sg - 1) * R) * 8 + (8 - R);
          if (score > best) {
            best = score;
            mom_rows = R;
            mom_warps = w;
            mom_stages = sg;
            mom_smem = bytes;
          }
        }
    if (best < 0) {
      set_error("velocity rows too long for the moment kernel's shared-memory ring");
      return DGBGK_EUNSUP;
    }
    const int warps = mom_warps;
    MomFn fn = mom_fn();
    CK(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mom_smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, warps * 32, mom_smem));
    if (per_sm < 1) per_sm = 1;
    const int ngroups = (3 * pl.E + mom_rows - 1) / mom_rows;
    const int need = (ngroups + warps - 1) / warps;
    mom_grid = std::max(1, std::min(need, per_sm * nsm));
    return 0;
  }
  using MomFn = void (*)(MomArgs<T>);
  MomFn mom_fn() const { return mom_rows == 4 ? k_moments<T, 4> : mom_rows == 2 ? k_moments<T, 2> : k_moments<T, 1>; }

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
      CUresult r = enc(&tm[b], dt, 2, f[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed for the state buffer");
        return DGBGK_ECUDA;
      }
    }
    return 0;
  }

  using SweepFn = void (*)(const CUtensorMap, const CUtensorMap, SweepArgs<T>);
  SweepFn sweep_fn() const {
    if (pl.EB == 64) return pl.immat == 1 ? k_sweep<T, 64, 1> : k_sweep<T, 64, 0>;
    return pl.immat == 1 ? k_sweep<T, 128, 1> : k_sweep<T, 128, 0>;
  }

  // Sweep tile: EB elements per CTA (2*EB threads) x one 64-byte velocity
  // segment.
  int set_tile(int tile_elems) {
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
        int flags = g.inflow & 7;
        for (int k = 0; k < 3; ++k) {
          r[e].gx[k] = (T)g.gx[k];
          r[e].gy[k] = (T)g.gy[k];
          r[e].mm[k] = (T)g.mm[k];
          const size_t i = 3 * (size_t)e + k;
          r[e].edge[k].nx = (T)pl.edge[i].nx;
          r[e].edge[k].ny = (T)pl.edge[i].ny;
          r[e].edge[k].alen = (T)pl.edge[i].alen;
          r[e].edge[k].info = edge_info(pl, i, e % eb);
          const bool wall = (pl.edge[i].low & 3) == 3;
          r[e].bside[k] = wall ? pl.edge[i].bside : -1;
          if (wall) flags |= 8 << k;
        }
        r[e].area = (T)g.area;
        r[e].flags = flags;
      }
      TRY(upload(&rec, r, st));
    }
    if (sweep_smem() > 227 * 1024) {
      set_error("sweep tile needs more than 227 KB of shared memory");
      return DGBGK_EUNSUP;
    }
    TRY(make_tensor_maps());
    SweepFn fn = sweep_fn();
    CK(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem()));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, 2 * pl.EB, sweep_smem()));
    if (per_sm < 1) {
      set_error("sweep kernel does not fit on an SM with this tile");
      return DGBGK_EUNSUP;
    }
    // velocity tiles per work unit: about eight units per resident CTA, so
    // the dynamic hand-out balances, and equal groups of tiles
    const int grid0 = per_sm * nsm;
    const long total = (long)pl.nblocks * nvt();
    tpu = (int)std::min<long>(SweepGeo<T>::TPU_MAX, std::max<long>(1, total / (8L * grid0)));
    const int ngroups = (nvt() + tpu - 1) / tpu;
    tpu = (nvt() + ngroups - 1) / ngroups;
    const int nunits = pl.nblocks * ngroups;
    sweep_grid = std::max(1, std::min(nunits, grid0));
    if (sweep_grid > part_cap) {
      dfree(part_max);
      dfree(part_sq);
      TRY(dalloc(&part_max, sweep_grid));
      TRY(dalloc(&part_sq, sweep_grid));
      part_cap = sweep_grid;
    }
    nparts = sweep_grid;
    drop_graphs();
    return 0;
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
    drop_graphs();
    return 0;
  }

  // -------------------------------------------------------- launches ----
  int launch_moments(int src) {
    MomArgs<T> a;
    a.f = f[src];
    a.tabs = tabs;
    a.rec = rec;
    a.nraw = nraw;
    a.disux = disux;
    a.disuy = disuy;
    a.disps = disps;
    a.mu = mu;
    a.ctrl = ctrl;
    a.ndg = 3 * pl.E;
    a.V = pl.V;
    a.Vp = Vp;
    a.nstage = mom_stages;
    a.rowbytes = (unsigned)(((size_t)pl.V * sizeof(T) + 15) / 16 * 16);
    a.MM = pl.M / 6.022e26;
    a.sigt = 3.1416 * pl.d * pl.d;
    CK(cudaMemsetAsync(&ctrl->maxmu, 0, sizeof(double), st));
    mom_fn()<<<mom_grid, mom_warps * 32, mom_smem, st>>>(a);
    CK(cudaGetLastError());
    return 0;
  }
  int launch_wall(int src) {
    if (pl.walls.empty()) return 0;
    WallArgs<T> a{f[src], walls, cxD, cyD, wjf, bEta, bEtaD, ctrl, (int)pl.walls.size(), pl.V, Vp};
    k_wall<T><<<(a.nwall + 7) / 8, 256, 0, st>>>(a);
    CK(cudaGetLastError());
    return 0;
  }
  int launch_sweep(int src) {
    SweepArgs<T> a;
    a.fin = f[src];
    a.fout = f[1 - src];
    a.rec = rec;
    a.halo_off = halo_off;
    a.halo_list = halo_list;
    a.cx = cxT;
    a.cy = cyT;
    a.nfinf = nfT;
    a.bTw = bTw;
    a.bUw = bUw;
    a.bEta = bEta;
    a.cmax = cmax;
    a.cmin = cmin;
    a.part_max = part_max;
    a.part_sq = part_sq;
    a.ctrl = ctrl;
    a.E = pl.E;
    a.V = pl.V;
    a.Vp = Vp;
    a.nblocks = pl.nblocks;
    a.max_halo = pl.max_halo;
    a.nvt = nvt();
    a.tpu = tpu;
    a.alpha = (T)pl.alpha;
    a.rgas = (T)pl.rgas;
    sweep_fn()<<<sweep_grid, 2 * pl.EB, sweep_smem(), st>>>(tm[src], tm[1 - src], a);
    CK(cudaGetLastError());
    return 0;
  }
  int launch_resid() {
    ResidArgs a{part_max, part_sq, hist_linf, hist_l2, hist_dt, ctrl};
    k_resid<<<1, 1024, 0, st>>>(a);
    CK(cudaGetLastError());
    return 0;
  }
  int enqueue_step(int src) {
    TRY(launch_moments(src));
    TRY(launch_wall(src));
    TRY(launch_sweep(src));
    TRY(launch_resid());
    return 0;
  }

  void drop_graphs() {
    for (auto& g : gexec)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  // Two pseudo-time steps (f[s] -> f[1-s] -> f[s]) as one graph.
  int build_graph(int s) {
    if (gexec[s]) return 0;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(s);
    if (rc == 0) rc = enqueue_step(1 - s);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != 0) return rc;
    CK(e);
    CK(cudaGraphInstantiate(&gexec[s], g, 0));
    cudaGraphDestroy(g);
    return 0;
  }

  int upload_ctrl(int max_steps, double tol) {
    Ctrl& h = hctrl[0];
    std::memset(&h, 0, sizeof(Ctrl));
    h.max_steps = max_steps;
    h.tol = tol;
    h.ref = ref_host;
    h.dtc = pl.dtc;
    h.nparts = nparts;
    CK(cudaMemcpyAsync(ctrl, &h, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
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

  int advance(int max_steps, double tol, int* steps, double* linf, double* l2, double* dt) override {
    if (max_steps < 0) {
      set_error("max_steps < 0");
      return DGBGK_EINVAL;
    }
    if (steps) *steps = 0;
    if (max_steps == 0) return 0;
    CK(cudaSetDevice(device));
    TRY(ensure_hist(max_steps));
    const int s0 = cur;
    TRY(build_graph(s0));
    TRY(upload_ctrl(max_steps, tol));
    CK(cudaEventRecord(ev0, st));
    const int launches = (max_steps + 1) / 2;
    const int chunk = 32;
    int issued = 0, chunks = 0;
    bool stop = false;
    while (issued < launches && !stop) {
      const int n = std::min(chunk, launches - issued);
      for (int i = 0; i < n; ++i) CK(cudaGraphLaunch(gexec[s0], st));
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
    const Ctrl c = hctrl[1];
    const int ns = c.step;
    if (steps) *steps = ns;
    ref_host = c.ref;
    if (ns > 0) {
      if (linf) CK(cudaMemcpy(linf, hist_linf, ns * sizeof(double), cudaMemcpyDeviceToHost));
      if (l2) CK(cudaMemcpy(l2, hist_l2, ns * sizeof(double), cudaMemcpyDeviceToHost));
      if (dt) CK(cudaMemcpy(dt, hist_dt, ns * sizeof(double), cudaMemcpyDeviceToHost));
    }
    cur = s0 ^ (ns & 1);
    return finish_status(c);
  }

  int profile(int nsteps, double* ms) override {
    CK(cudaSetDevice(device));
    TRY(ensure_hist(std::max(nsteps, 1)));
    TRY(upload_ctrl(nsteps, 0.0));
    cudaEvent_t ev[5];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    int rc = 0;
    for (int s = 0; s < nsteps && rc == 0; ++s) {
      cudaEventRecord(ev[0], st);
      rc = launch_moments(cur);
      cudaEventRecord(ev[1], st);
      if (rc == 0) rc = launch_wall(cur);
      cudaEventRecord(ev[2], st);
      if (rc == 0) rc = launch_sweep(cur);
      cudaEventRecord(ev[3], st);
      if (rc == 0) rc = launch_resid();
      cudaEventRecord(ev[4], st);
      cudaEventSynchronize(ev[4]);
      for (int k = 0; k < 4; ++k) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        acc[k] += t;
      }
      cur ^= 1;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    CK(cudaMemcpy(&hctrl[1], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    ref_host = hctrl[1].ref;
    for (int k = 0; k < 4; ++k) ms[k] = nsteps > 0 ? acc[k] / nsteps : 0.0;
    return finish_status(hctrl[1]);
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
    // INICON2 (src/inicon2.f90:216-251) evaluated per velocity in double
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
    return 0;
  }

  int moments_now() {
    TRY(aux_ctrl());
    TRY(launch_moments(cur));
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
    TRY(launch_wall(cur));
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
  std::string err;
  const int eb0 = prm->tile_elems > 0 ? prm->tile_elems : 128;
  int rc = build_plan(*mesh, *vs, *prm, eb0, impl->pl, &err);
  if (rc != 0) {
    set_error(err);
    return rc;
  }
  if (impl->pl.alpha != 1.0 && impl->pl.has_wall_incoming) {
    set_error("dgbgk_create: wall accommodation ALPHA < 1 (specular part) is not supported by this build");
    return DGBGK_EUNSUP;
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
int dgbgk_get_macros(dgbgk_handle* h, double* nd, double* rho, double* u, double* v, double* ps, double* temp) {
  HCHECK(h);
  return h->impl->macros(nd, rho, u, v, ps, temp);
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
void dgbgk_destroy(dgbgk_handle* h) { delete h; }

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

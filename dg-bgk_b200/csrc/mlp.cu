// The warm-start network: an MLP with tanh hidden layers trained and run
// with the BF16 tensor-core GEMM of umma.cuh (FP32 accumulation, FP32
// master weights, Adam).  Layers: n_in (padded to 64) -> width x depth ->
// n_out.  All GEMMs are C = A B^T with both operands K-major, so the network
// keeps W and W^T in BF16 and every activation and gradient in both
// layouts:
//   forward   H_{l+1} = tanh(H_l W_l^T + b_l)       A = H_l,   B = W_l
//   output    P = H_L W_L^T + b_L                    (FP32)
//   loss      dP = 2 (P - T) / (B n_out)             (BF16, both layouts)
//   dW_l      = dZ_{l+1}^T H_l                        A = dZ^T,  B = H_l^T
//   dZ_l      = (dZ_{l+1} W_l) (1 - H_l^2)            A = dZ,    B = W_l^T
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/dgbgk.h"
#include "umma.cuh"

namespace dgbgk {
void set_error(const std::string& m);
}

using namespace dgbgk;
using namespace dgbgk::umma;

#define MCK(x)                                                                       \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess) {                                                         \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" #x ")"); \
      return DGBGK_ECUDA;                                                            \
    }                                                                                \
  } while (0)
#define MTRY(x)               \
  do {                        \
    int rc_ = (x);            \
    if (rc_ != 0) return rc_; \
  } while (0)

namespace {

constexpr int KPAD = 64;  // the input layer's K (n_in padded)

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
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

// [rows][cols] BF16 row-major as a TMA tensor; box = 64 columns x box_rows
// rows, 128-byte swizzle (the layout the GEMM's descriptors describe).
int bf16_map(CUtensorMap* m, const void* p, int rows, int cols, int box_rows) {
  auto enc = encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return DGBGK_ECUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(p), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for an MLP operand");
    return DGBGK_ECUDA;
  }
  return 0;
}

// One planned GEMM: its operand maps and epilogue.
struct Gemm {
  CUtensorMap ta, tb;
  GemmArgs g;
  int bn;
};

int plan_gemm(Gemm& G, const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, GemmArgs g) {
  if (M % BM || K % BK || N % 64) {
    set_error("MLP GEMM shape not a multiple of the tile");
    return DGBGK_EINVAL;
  }
  G.bn = (N % 128 == 0) ? 128 : 64;
  MTRY(bf16_map(&G.ta, A, M, K, BM));
  MTRY(bf16_map(&G.tb, B, N, K, G.bn));
  G.g = g;
  G.g.M = M;
  G.g.N = N;
  G.g.K = K;
  return 0;
}

int allow_smem(const void* fn, size_t bytes) {
  MCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return 0;
}

int run_gemm(const Gemm& G, cudaStream_t st) {
  dim3 grid(G.g.N / G.bn, G.g.M / BM);
  if (G.bn == 128) {
    MTRY(allow_smem((const void*)k_gemm<128>, Smem<128>::TOTAL));
    k_gemm<128><<<grid, 128, Smem<128>::TOTAL, st>>>(G.ta, G.tb, G.g);
  } else {
    MTRY(allow_smem((const void*)k_gemm<64>, Smem<64>::TOTAL));
    k_gemm<64><<<grid, 128, Smem<64>::TOTAL, st>>>(G.ta, G.tb, G.g);
  }
  MCK(cudaGetLastError());
  return 0;
}

// ----------------------------------------------------------- small kernels
// minibatch: rows idx[r] of the set -> X0 (BF16, padded to KPAD, both
// layouts) and T (FP32)
__global__ void k_gather(const float* __restrict__ xs, const float* __restrict__ ts, const int* __restrict__ idx,
                         int n_in, int n_out, int B, __nv_bfloat16* x0, __nv_bfloat16* x0T, float* t) {
  const int r = blockIdx.x;
  const int s = idx[r];
  for (int c = threadIdx.x; c < KPAD; c += blockDim.x) {
    const float v = c < n_in ? xs[(size_t)s * n_in + c] : 0.f;
    x0[(size_t)r * KPAD + c] = __float2bfloat16_rn(v);
    x0T[(size_t)c * B + r] = __float2bfloat16_rn(v);
  }
  for (int c = threadIdx.x; c < n_out; c += blockDim.x) t[(size_t)r * n_out + c] = ts[(size_t)s * n_out + c];
}

// MSE loss and its gradient: dP = 2 (P - T) / (B n_out) in both layouts;
// the loss sum goes to loss[0] (FP64 atomics of per-block sums)
__global__ void k_loss(const float* __restrict__ p, const float* __restrict__ t, int B, int n_out,
                       __nv_bfloat16* dp, __nv_bfloat16* dpT, double* loss) {
  const size_t n = (size_t)B * n_out;
  const float scale = 2.f / (float)n;
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = p[i] - t[i];
    acc += (double)d * d;
    const int r = (int)(i / n_out), c = (int)(i - (size_t)r * n_out);
    const __nv_bfloat16 g = __float2bfloat16_rn(scale * d);
    dp[i] = g;
    dpT[(size_t)c * B + r] = g;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    atomicAdd(loss, s / (double)n);
  }
}

// bias gradient: db[j] = sum over the batch of G[.., j], from G^T [N][B]
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ gT, int N, int B, float* db) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= N) return;
  float s = 0.f;
  for (int r = lane; r < B; r += 32) s += __bfloat162float(gT[(size_t)j * B + r]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) db[j] = s;
}

// Adam on FP32 masters; refreshes the BF16 copies W [out][in] and W^T
// [in][out].  Padded input columns (c >= in_live) stay zero.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       int rows, int cols, int in_live, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* wb, __nv_bfloat16* wbT) {
  const size_t n = (size_t)rows * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (size_t)r * cols);
    float x = w[i];
    if (c < in_live) {
      const float gi = g[i];
      const float mi = b1 * m[i] + (1.f - b1) * gi;
      const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
      m[i] = mi;
      v[i] = vi;
      x -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
      w[i] = x;
    }
    if (wb) {
      const __nv_bfloat16 xb = __float2bfloat16_rn(x);
      wb[i] = xb;
      wbT[(size_t)c * rows + r] = xb;
    }
  }
}

// FP32 -> BF16 copies of a weight matrix (both layouts)
__global__ void k_to_bf16(const float* __restrict__ w, int rows, int cols, __nv_bfloat16* wb, __nv_bfloat16* wbT) {
  const size_t n = (size_t)rows * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (size_t)r * cols);
    const __nv_bfloat16 xb = __float2bfloat16_rn(w[i]);
    wb[i] = xb;
    wbT[(size_t)c * rows + r] = xb;
  }
}

// zeroed device allocation; the memset is complete on return, so work on
// any stream may use the buffer
template <class X> int mall(X** p, size_t n) {
  *p = nullptr;
  MCK(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(X)));
  MCK(cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(X)));
  MCK(cudaDeviceSynchronize());
  return 0;
}
template <class X> void mfree(X*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

struct Layer {
  int in = 0, in_live = 0, out = 0;
  float *w = nullptr, *b = nullptr, *gw = nullptr, *gb = nullptr;
  float *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;
  __nv_bfloat16 *wb = nullptr, *wbT = nullptr;
};

}  // namespace

struct dgbgk_mlp {
  int device = 0, n_in = 0, width = 0, depth = 0, n_out = 0, B = 0;
  cudaStream_t st = nullptr;
  std::vector<Layer> L;                  // depth + 1 layers
  std::vector<__nv_bfloat16*> H, HT;     // activations 0..depth (0 = input), [B][in] and [in][B]
  std::vector<__nv_bfloat16*> G, GT;     // dZ of layers 1..depth, and dP (index depth+1)
  float *P = nullptr, *T = nullptr;
  double* loss = nullptr;                // one slot per training step (slot 0 otherwise)
  int loss_cap = 1;
  int* err = nullptr;
  float *xs = nullptr, *ts = nullptr;    // training set
  int nset = 0;
  int* idx = nullptr;
  int idx_cap = 0;
  float *xin = nullptr, *tin = nullptr;  // staging of one host batch
  int* iin = nullptr;
  long long adam_t = 0;
  std::vector<Gemm> fwd, bwd_dw, bwd_dx;

  ~dgbgk_mlp() {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    for (auto& l : L) {
      mfree(l.w), mfree(l.b), mfree(l.gw), mfree(l.gb), mfree(l.mw), mfree(l.vw), mfree(l.mb), mfree(l.vb);
      mfree(l.wb), mfree(l.wbT);
    }
    for (auto* p : H) mfree(p);
    for (auto* p : HT) mfree(p);
    for (auto* p : G) mfree(p);
    for (auto* p : GT) mfree(p);
    mfree(P), mfree(T), mfree(loss), mfree(err), mfree(xs), mfree(ts), mfree(idx);
    mfree(xin), mfree(tin), mfree(iin);
    if (st) cudaStreamDestroy(st);
  }

  int init(unsigned long long seed) {
    MCK(cudaSetDevice(device));
    MCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int nl = depth + 1;
    L.resize(nl);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < nl; ++l) {
      Layer& y = L[l];
      y.in = l == 0 ? KPAD : width;
      y.in_live = l == 0 ? n_in : width;
      y.out = l == depth ? n_out : width;
      const size_t nw = (size_t)y.out * y.in;
      MTRY(mall(&y.w, nw));
      MTRY(mall(&y.gw, nw));
      MTRY(mall(&y.mw, nw));
      MTRY(mall(&y.vw, nw));
      MTRY(mall(&y.b, y.out));
      MTRY(mall(&y.gb, y.out));
      MTRY(mall(&y.mb, y.out));
      MTRY(mall(&y.vb, y.out));
      MTRY(mall(&y.wb, nw));
      MTRY(mall(&y.wbT, nw));
      // Xavier-uniform weights, zero biases
      std::vector<float> hw(nw, 0.f);
      const float a = std::sqrt(6.f / (float)(y.in_live + y.out));
      std::uniform_real_distribution<float> U(-a, a);
      for (int r = 0; r < y.out; ++r)
        for (int c = 0; c < y.in_live; ++c) hw[(size_t)r * y.in + c] = U(rng);
      MCK(cudaMemcpyAsync(y.w, hw.data(), nw * 4, cudaMemcpyHostToDevice, st));
      MCK(cudaStreamSynchronize(st));
    }
    H.assign(nl, nullptr);
    HT.assign(nl, nullptr);
    for (int l = 0; l < nl; ++l) {
      const int c = L[l].in;
      MTRY(mall(&H[l], (size_t)B * c));
      MTRY(mall(&HT[l], (size_t)B * c));
    }
    G.assign(nl + 1, nullptr);
    GT.assign(nl + 1, nullptr);
    for (int l = 1; l <= nl; ++l) {
      const int c = l == nl ? n_out : width;
      MTRY(mall(&G[l], (size_t)B * c));
      MTRY(mall(&GT[l], (size_t)B * c));
    }
    MTRY(mall(&P, (size_t)B * n_out));
    MTRY(mall(&T, (size_t)B * n_out));
    MTRY(mall(&loss, 1));
    MTRY(mall(&err, 1));
    MTRY(mall(&xin, (size_t)B * n_in));
    MTRY(mall(&tin, (size_t)B * n_out));
    MTRY(mall(&iin, B));
    {
      std::vector<int> id(B);
      for (int r = 0; r < B; ++r) id[r] = r;
      MCK(cudaMemcpyAsync(iin, id.data(), B * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    MTRY(refresh_bf16());
    return plan();
  }

  int refresh_bf16() {
    for (auto& y : L) {
      k_to_bf16<<<256, 256, 0, st>>>(y.w, y.out, y.in, y.wb, y.wbT);
      MCK(cudaGetLastError());
    }
    return 0;
  }

  int plan() {
    const int nl = depth + 1;
    fwd.assign(nl, Gemm{});
    bwd_dw.assign(nl, Gemm{});
    bwd_dx.assign(nl, Gemm{});
    for (int l = 0; l < nl; ++l) {
      Layer& y = L[l];
      GemmArgs g{};
      g.err = err;
      g.bias = y.b;
      if (l < depth) {
        g.epi = EPI_TANH;
        g.out_bf = H[l + 1];
        g.out_bfT = HT[l + 1];
      } else {
        g.epi = EPI_LINEAR;
        g.out_f = P;
      }
      MTRY(plan_gemm(fwd[l], H[l], y.wb, B, y.out, y.in, g));
      // dW_l = G_{l+1}^T H_l: [out][in], K = B
      GemmArgs gw{};
      gw.err = err;
      gw.epi = EPI_F32;
      gw.out_f = y.gw;
      MTRY(plan_gemm(bwd_dw[l], GT[l + 1], HT[l], y.out, y.in, B, gw));
      // G_l = (G_{l+1} W_l) (1 - H_l^2): [B][in], K = out (not for the input layer)
      if (l > 0) {
        GemmArgs gx{};
        gx.err = err;
        gx.epi = EPI_DTANH;
        gx.aux = H[l];
        gx.out_bf = G[l];
        gx.out_bfT = GT[l];
        MTRY(plan_gemm(bwd_dx[l], G[l + 1], y.wbT, B, y.in, y.out, gx));
      }
    }
    return 0;
  }

  int forward() {
    for (int l = 0; l <= depth; ++l) MTRY(run_gemm(fwd[l], st));
    return 0;
  }

  // loss (into *lslot) and all gradients of the current minibatch (in H[0], T)
  int backward(double* lslot) {
    MCK(cudaMemsetAsync(lslot, 0, sizeof(double), st));
    k_loss<<<592, 256, 0, st>>>(P, T, B, n_out, G[depth + 1], GT[depth + 1], lslot);
    MCK(cudaGetLastError());
    for (int l = depth; l >= 0; --l) {
      MTRY(run_gemm(bwd_dw[l], st));
      k_bias_grad<<<(L[l].out + 7) / 8, 256, 0, st>>>(GT[l + 1], L[l].out, B, L[l].gb);
      MCK(cudaGetLastError());
      if (l > 0) MTRY(run_gemm(bwd_dx[l], st));
    }
    return 0;
  }

  int adam(float lr) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)adam_t), c2 = 1.f - std::pow(b2, (float)adam_t);
    for (auto& y : L) {
      k_adam<<<592, 256, 0, st>>>(y.w, y.mw, y.vw, y.gw, y.out, y.in, y.in_live, lr, b1, b2, eps, c1, c2, y.wb, y.wbT);
      k_adam<<<8, 256, 0, st>>>(y.b, y.mb, y.vb, y.gb, 1, y.out, y.out, lr, b1, b2, eps, c1, c2, nullptr, nullptr);
      MCK(cudaGetLastError());
    }
    return 0;
  }

  int check_err() {
    int e = 0;
    MCK(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    if (e) {
      set_error("MLP GEMM: a bounded device wait expired");
      return DGBGK_ECUDA;
    }
    return 0;
  }

  // n <= B host rows x[n][n_in] (and t[n][n_out]) -> the minibatch
  // buffers; rows past n repeat nothing meaningful (their inputs are zero
  // and their outputs are not read back)
  int load_batch_host(const float* x, const float* t, int n) {
    if (n < B) {
      MCK(cudaMemsetAsync(xin, 0, (size_t)B * n_in * 4, st));
      MCK(cudaMemsetAsync(tin, 0, (size_t)B * n_out * 4, st));
    }
    MCK(cudaMemcpyAsync(xin, x, (size_t)n * n_in * 4, cudaMemcpyHostToDevice, st));
    if (t) MCK(cudaMemcpyAsync(tin, t, (size_t)n * n_out * 4, cudaMemcpyHostToDevice, st));
    k_gather<<<B, 128, 0, st>>>(xin, tin, iin, n_in, n_out, B, H[0], HT[0], T);
    MCK(cudaGetLastError());
    return 0;
  }
};

extern "C" {

int dgbgk_mlp_create(int n_in, int width, int depth, int n_out, int batch, unsigned long long seed, int device,
                     dgbgk_mlp** out) {
  if (!out || n_in < 1 || n_in > KPAD || width < 128 || width % 128 || depth < 1 || n_out < 128 || n_out % 128 ||
      batch < 128 || batch % 128) {
    set_error("dgbgk_mlp_create: n_in <= 64, width/n_out/batch multiples of 128, depth >= 1");
    return DGBGK_EINVAL;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_error("dgbgk_mlp_create: no such CUDA device");
    return DGBGK_ECUDA;
  }
  cudaDeviceProp prop;
  MCK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("dgbgk_mlp_create: this build targets sm_100a (B200)");
    return DGBGK_ECUDA;
  }
  std::unique_ptr<dgbgk_mlp> m(new dgbgk_mlp());
  m->device = device;
  m->n_in = n_in;
  m->width = width;
  m->depth = depth;
  m->n_out = n_out;
  m->B = batch;
  MTRY(m->init(seed));
  *out = m.release();
  return DGBGK_OK;
}

long long dgbgk_mlp_param_count(const dgbgk_mlp* m) {
  if (!m) return -1;
  long long n = 0;
  for (const auto& y : m->L) n += (long long)y.out * y.in + y.out;
  return n;
}

// flat layout per layer: W [out][in] (input layer in = 64, columns past
// n_in zero), then b [out]
int dgbgk_mlp_get_params(dgbgk_mlp* m, float* p) {
  if (!m || !p) return set_error("NULL argument"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  size_t o = 0;
  for (const auto& y : m->L) {
    const size_t nw = (size_t)y.out * y.in;
    MCK(cudaMemcpyAsync(p + o, y.w, nw * 4, cudaMemcpyDeviceToHost, m->st));
    o += nw;
    MCK(cudaMemcpyAsync(p + o, y.b, y.out * 4, cudaMemcpyDeviceToHost, m->st));
    o += y.out;
  }
  MCK(cudaStreamSynchronize(m->st));
  return 0;
}

int dgbgk_mlp_set_params(dgbgk_mlp* m, const float* p) {
  if (!m || !p) return set_error("NULL argument"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  size_t o = 0;
  for (auto& y : m->L) {
    const size_t nw = (size_t)y.out * y.in;
    MCK(cudaMemcpyAsync(y.w, p + o, nw * 4, cudaMemcpyHostToDevice, m->st));
    o += nw;
    MCK(cudaMemcpyAsync(y.b, p + o, y.out * 4, cudaMemcpyHostToDevice, m->st));
    o += y.out;
  }
  MTRY(m->refresh_bf16());
  MCK(cudaStreamSynchronize(m->st));
  return 0;
}

// y[n][n_out] = network(x[n][n_in]); n rows in chunks of the batch size
int dgbgk_mlp_forward(dgbgk_mlp* m, const float* x, int n, float* y) {
  if (!m || !x || !y || n < 1) return set_error("NULL argument"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  for (int r0 = 0; r0 < n; r0 += m->B) {
    const int k = std::min(m->B, n - r0);
    MTRY(m->load_batch_host(x + (size_t)r0 * m->n_in, nullptr, k));
    MTRY(m->forward());
    MCK(cudaMemcpyAsync(y + (size_t)r0 * m->n_out, m->P, (size_t)k * m->n_out * 4, cudaMemcpyDeviceToHost, m->st));
    MCK(cudaStreamSynchronize(m->st));
    MTRY(m->check_err());
  }
  return 0;
}

// loss (mean squared error) and the gradient (flat, as the parameters) of
// one batch of exactly `batch` rows
int dgbgk_mlp_gradient(dgbgk_mlp* m, const float* x, const float* t, int n, double* loss, float* grad) {
  if (!m || !x || !t || n != m->B) return set_error("dgbgk_mlp_gradient: n must equal the batch size"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  MTRY(m->load_batch_host(x, t, n));
  MTRY(m->forward());
  MTRY(m->backward(m->loss));
  MTRY(m->check_err());
  if (loss) MCK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st));
  if (grad) {
    size_t o = 0;
    for (const auto& y : m->L) {
      const size_t nw = (size_t)y.out * y.in;
      MCK(cudaMemcpyAsync(grad + o, y.gw, nw * 4, cudaMemcpyDeviceToHost, m->st));
      o += nw;
      MCK(cudaMemcpyAsync(grad + o, y.gb, y.out * 4, cudaMemcpyDeviceToHost, m->st));
      o += y.out;
    }
  }
  MCK(cudaStreamSynchronize(m->st));
  return 0;
}

// the training set: x[n][n_in], t[n][n_out] (host), kept on the device
int dgbgk_mlp_set_data(dgbgk_mlp* m, const float* x, const float* t, int n) {
  if (!m || !x || !t || n < 1) return set_error("NULL argument"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  MCK(cudaStreamSynchronize(m->st));
  mfree(m->xs);
  mfree(m->ts);
  m->nset = 0;
  MTRY(mall(&m->xs, (size_t)n * m->n_in));
  MTRY(mall(&m->ts, (size_t)n * m->n_out));
  MCK(cudaMemcpyAsync(m->xs, x, (size_t)n * m->n_in * 4, cudaMemcpyHostToDevice, m->st));
  MCK(cudaMemcpyAsync(m->ts, t, (size_t)n * m->n_out * 4, cudaMemcpyHostToDevice, m->st));
  MCK(cudaStreamSynchronize(m->st));
  m->nset = n;
  return 0;
}

// `iters` Adam steps on minibatches drawn without replacement per epoch
// (std::mt19937_64 seeded with `seed`); loss_hist[iters] (may be NULL)
// receives each step's minibatch loss.
int dgbgk_mlp_train(dgbgk_mlp* m, int iters, float lr, unsigned long long seed, double* loss_hist) {
  if (!m || iters < 0 || m->nset < 1) return set_error("dgbgk_mlp_train: no training set"), DGBGK_EINVAL;
  MCK(cudaSetDevice(m->device));
  const int B = m->B;
  if (iters == 0) return 0;
  MCK(cudaStreamSynchronize(m->st));
  if (m->idx_cap < iters * B) {
    mfree(m->idx);
    MTRY(mall(&m->idx, (size_t)iters * B));
    m->idx_cap = iters * B;
  }
  if (m->loss_cap < iters) {
    mfree(m->loss);
    MTRY(mall(&m->loss, iters));
    m->loss_cap = iters;
  }
  std::vector<int> id((size_t)iters * B);
  std::mt19937_64 rng(seed);
  std::vector<int> perm(m->nset);
  for (int i = 0; i < m->nset; ++i) perm[i] = i;
  size_t pos = perm.size();
  for (size_t k = 0; k < id.size(); ++k) {
    if (pos == perm.size()) {
      std::shuffle(perm.begin(), perm.end(), rng);
      pos = 0;
    }
    id[k] = perm[pos++];
  }
  MCK(cudaMemcpyAsync(m->idx, id.data(), id.size() * sizeof(int), cudaMemcpyHostToDevice, m->st));
  for (int it = 0; it < iters; ++it) {
    k_gather<<<B, 128, 0, m->st>>>(m->xs, m->ts, m->idx + (size_t)it * B, m->n_in, m->n_out, B, m->H[0], m->HT[0],
                                    m->T);
    MCK(cudaGetLastError());
    MTRY(m->forward());
    MTRY(m->backward(m->loss + it));
    MTRY(m->adam(lr));
  }
  MTRY(m->check_err());
  if (loss_hist) {
    MCK(cudaMemcpyAsync(loss_hist, m->loss, iters * sizeof(double), cudaMemcpyDeviceToHost, m->st));
    MCK(cudaStreamSynchronize(m->st));
  }
  return 0;
}

void dgbgk_mlp_destroy(dgbgk_mlp* m) { delete m; }

}  // extern "C"

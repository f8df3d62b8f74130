// Blackwell (sm_100a) 5th-generation tensor-core GEMM for the warm-start
// MLP: C[M x N] = A[M x K] * B[N x K]^T with A and B in BF16, both K-major
// (row-major with the reduction index contiguous), accumulated in FP32 in
// tensor memory.
//
// One CTA computes one 128 x BN tile of C with 128 threads:
//   * warp 0, lane 0 loads 128 x 64 (A) and BN x 64 (B) BF16 boxes per
//     K-block with TMA (128-byte swizzle) into a ring of stages;
//   * warp 1, lane 0 issues tcgen05.mma (kind::f16, M = 128, N = BN, K = 16
//     per instruction, four per K-block) and frees each stage with
//     tcgen05.commit on the stage's "empty" mbarrier;
//   * all four warps read the accumulator with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31, i.e. rows 32w..32w+31 of the tile) and run the
//     epilogue.
// Every mbarrier wait is bounded; on expiry the CTA records an error flag,
// waits (bounded) for its own copies and MMAs, frees its tensor memory and
// returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace dgbgk {
namespace umma {

constexpr int BM = 128;        // tile rows (MMA M)
constexpr int BK = 64;         // K-block: 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 4;
constexpr unsigned WAIT_TRIES = 1u << 22;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
  for (unsigned i = 0; i < WAIT_TRIES; ++i) {
    if (bar_try(b, parity)) return true;
    if (i > 32) __nanosleep(128);
  }
  return false;
}
__device__ __forceinline__ void tma2d(void* dst, const CUtensorMap* m, int x, int y, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(saddr(dst)),
      "l"(m), "r"(x), "r"(y), "r"(saddr(b))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major BF16 tile whose 128-byte rows
// were written by TMA with the 128-byte swizzle: 8-row atoms of 1024 bytes
// stacked along M/N (stride byte offset 1024), descriptor version 1,
// layout type 2 (128-byte swizzle).  The start address advances by 32 bytes
// per K = 16 step inside the atom.
__device__ __forceinline__ uint64_t sdesc(const void* tile, int kbytes) {
  const uint64_t a = (uint64_t)((saddr(tile) + kbytes) >> 4) & 0x3FFFull;
  const uint64_t lbo = 1ull;               // unused by swizzled K-major layouts
  const uint64_t sbo = (1024ull >> 4);     // 8 rows x 128 bytes
  return a | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: D in FP32 (bits 4-5 = 1), A and B in
// BF16 (bits 7-9 = 1, bits 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(b))
               : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst_smem)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 32 columns of the warp's 32 TMEM lanes: thread t gets lane 32w+t
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Epilogue modes
enum Epi : int {
  EPI_TANH = 0,      // Y = tanh(C + bias): Y (BF16, [M][N]) and Y^T (BF16, [N][M])
  EPI_LINEAR = 1,    // Y = C + bias: FP32 [M][N]
  EPI_DTANH = 2,     // G = C * (1 - y^2), y = aux (BF16 [M][N]): G (BF16 [M][N]) and G^T (BF16 [N][M])
  EPI_F32 = 3,       // C: FP32 [M][N]
};

struct GemmArgs {
  const float* bias;        // [N] (EPI_TANH, EPI_LINEAR)
  const __nv_bfloat16* aux; // [M][N] (EPI_DTANH)
  __nv_bfloat16* out_bf;    // [M][N]
  __nv_bfloat16* out_bfT;   // [N][M]
  float* out_f;             // [M][N]
  int* err;                 // set when a bounded wait expired
  int M, N, K;
  int epi;
};

template <int BN>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;  // 16 KB
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int TOTAL = 1024 + STAGES * STAGE;  // + 1024 alignment slack
};

// C tile (blockIdx.y * 128, blockIdx.x * BN).  M, N, K: multiples of 128, BN, 64.
template <int BN>
__global__ void __launch_bounds__(128, 1) k_gemm(const __grid_constant__ CUtensorMap ta,
                                                 const __grid_constant__ CUtensorMap tb, GemmArgs g) {
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "MMA N");
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  __shared__ uint64_t full[STAGES], empty[STAGES], done;
  __shared__ uint32_t tmem_base;
  __shared__ int fail, issued, consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* base = sm_raw + ((1024u - (saddr(sm_raw) & 1023u)) & 1023u);
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int nk = g.K / BK;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], 1);
    }
    bar_init(&done, 1);
    fail = 0;
    issued = 0;
    consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_base, BN);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base;

  if (warp == 0 && lane == 0) {
    // producer: K-block kb into stage kb % STAGES once the MMAs of
    // kb - STAGES have released it
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !bar_wait(&empty[s], ((kb / STAGES) - 1) & 1)) {
        fail = 1;
        break;
      }
      unsigned char* st = base + s * Smem<BN>::STAGE;
      bar_expect(&full[s], Smem<BN>::STAGE);
      tma2d(st, &ta, kb * BK, m0, &full[s]);
      tma2d(st + Smem<BN>::A_BYTES, &tb, kb * BK, n0, &full[s]);
      issued = kb + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    constexpr uint32_t idesc = idesc_bf16(BM, BN);
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!bar_wait(&full[s], (kb / STAGES) & 1)) {
        fail = 1;
        break;
      }
      fence_after();
      const unsigned char* st = base + s * Smem<BN>::STAGE;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k)
        mma_bf16(tmem, sdesc(st, 32 * k), sdesc(st + Smem<BN>::A_BYTES, 32 * k), idesc, (kb | k) ? 1u : 0u);
      mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
      consumed = kb + 1;
    }
    mma_commit(&done);  // the accumulator is complete
  }
  __syncwarp();
  // every thread: wait for the accumulator
  const bool ok = bar_wait(&done, 0);
  fence_after();
  // the failing thread set `fail` before its own wait: the vote is uniform
  if (__syncthreads_or((!ok || fail) ? 1 : 0)) {
    if (tid == 0) {
      atomicExch(g.err, 1);
      // the box copies still in flight land before the CTA leaves (bounded)
      for (int kb = consumed; kb < issued; ++kb) bar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
    }
  } else {
    // epilogue: row m0 + 32*warp + lane, 32 columns at a time
    const int row = m0 + 32 * warp + lane;
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
      const int col = n0 + c0;
      if (g.epi == EPI_TANH || g.epi == EPI_LINEAR) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] += g.bias[col + i];
      }
      if (g.epi == EPI_TANH) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = tanhf(v[i]);
      } else if (g.epi == EPI_DTANH) {
        const __nv_bfloat16* y = g.aux + (size_t)row * g.N + col;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const float yy = __bfloat162float(y[i]);
          v[i] *= 1.f - yy * yy;
        }
      }
      if (g.epi == EPI_TANH || g.epi == EPI_DTANH) {
        __nv_bfloat16* o = g.out_bf + (size_t)row * g.N + col;
#pragma unroll
        for (int i = 0; i < 32; i += 2) *reinterpret_cast<__nv_bfloat162*>(o + i) = __floats2bfloat162_rn(v[i], v[i + 1]);
        // transposed copy: for a fixed column the 32 lanes write 32 consecutive rows
#pragma unroll
        for (int i = 0; i < 32; ++i) g.out_bfT[(size_t)(col + i) * g.M + row] = __float2bfloat16_rn(v[i]);
      } else {
        float* o = g.out_f + (size_t)row * g.N + col;
#pragma unroll
        for (int i = 0; i < 32; i += 4) *reinterpret_cast<float4*>(o + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, BN);
}

}  // namespace umma
}  // namespace dgbgk

// mlp.cu - the learned predictor's network: a BF16 tensor-core GEMM written
// for sm_100a (tcgen05.mma with the accumulator in tensor memory) and the
// forward pass, backward pass and Adam step of a small tanh MLP built on it.
//
// GEMM (one 128 x BN output tile per CTA, 128 threads):
//   * each K-block of 64 is staged into shared memory by all threads: FP32
//     operands are read from global memory (either orientation), rounded to
//     BF16 and stored in the canonical K-major, non-swizzled tcgen05 layout:
//     8-row x 16-byte core matrices, contiguous; the two 8-element K halves
//     of one MMA are LBO = 128 B apart, successive 8-row groups SBO = 1024 B;
//   * one elected thread issues four tcgen05.mma.kind::f16 (K = 16 each) per
//     K-block and commits them to an mbarrier; two shared-memory stages let
//     the next block load while the tensor core works on the current one;
//   * the FP32 accumulator (lane = row, column = n) is read back with
//     tcgen05.ld.32x32b: each warp reads its own 32 lanes, each thread one row.
// Every mbarrier wait is bounded (1 s); a wait that runs out sets the status
// flag, waits once more (bounded) for the work in flight, frees the tensor
// memory and returns.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <cuda_bf16.h>

#include "internal.h"
#include "learned.h"
#include "mlp_row.cuh"

namespace fastgpu {

namespace {

constexpr int kBM = 128;            // tile rows (= tensor-memory lanes)
constexpr int kBK = 64;             // K per shared-memory stage
constexpr uint64_t kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// true once the phase with this parity has completed, false after limit_ns
__device__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (!mbar_try(bar, parity))
    if (gtimer() - t0 > limit_ns) return false;
  return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// shared-memory matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor: D FP32, A and B BF16, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

template <int BN, bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128, 1)
    umma_gemm_bf16(int M, int N, int K, int kslice, const float *__restrict__ A, int lda, const float *__restrict__ B,
                   int ldb, float *__restrict__ C, int ldc, const float *__restrict__ bias,
                   const float *__restrict__ aux, int ldaux, int32_t *__restrict__ status) {
  constexpr int kNcols = BN < 32 ? 32 : BN;            // tensor-memory columns (power of 2, >= 32)
  constexpr int kAbytes = kBM * kBK * 2;
  constexpr int kBbytes = BN * kBK * 2;
  constexpr int kStage = kAbytes + kBbytes;
  constexpr uint32_t kSBO = (kBK / 8) * 128;           // next 8-row group
  constexpr uint32_t kLBO = 128;                       // next 8-element K half
  constexpr uint32_t kIdesc = idesc_bf16(kBM, BN);
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "M=128 needs N a multiple of 16 in [16, 256]");

  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int ok_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  // split K: this CTA reduces over [kbeg, kend); with several slices the
  // epilogue (store only) writes slice z's partial tile to C + z M ldc
  const int kbeg = blockIdx.z * kslice, kend = min(K, kbeg + kslice);
  const int nkb = (kend - kbeg + kBK - 1) / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kNcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    ok_sh = 1;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  int issued = 0;  // K-blocks committed (thread 0's count; used for the final wait)
  for (int kb = 0; kb < nkb; kb++) {
    const int s = kb & 1;
    uint8_t *sA = smem + s * kStage;
    uint8_t *sB = sA + kAbytes;
    if (kb >= 2) {
      // stage s was last read by the MMAs of block kb-2
      if (tid == 0 && !mbar_wait(&bars[s], ((kb - 2) >> 1) & 1, kWaitNs)) ok_sh = 0;
      __syncthreads();
      if (!ok_sh) break;
    }
    const int k0 = kbeg + kb * kBK;
    // A tile: 128 rows x 8 chunks of 8 K-values
    for (int u = tid; u < kBM * (kBK / 8); u += 128) {
      const int r = u % kBM, ch = u / kBM;
      const int gm = m0 + r, gk = k0 + ch * 8;
      float f[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int kk = gk + j;
        f[j] = (gm < M && kk < kend) ? (TA ? A[(int64_t)kk * lda + gm] : A[(int64_t)gm * lda + kk]) : 0.f;
      }
      uint4 p = make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
      *reinterpret_cast<uint4 *>(sA + ((r >> 3) * (kBK / 8) + ch) * 128 + (r & 7) * 16) = p;
    }
    // B tile: BN rows x 8 chunks
    for (int u = tid; u < BN * (kBK / 8); u += 128) {
      const int r = u % BN, ch = u / BN;
      const int gn = n0 + r, gk = k0 + ch * 8;
      float f[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int kk = gk + j;
        f[j] = (gn < N && kk < kend) ? (TB ? B[(int64_t)kk * ldb + gn] : B[(int64_t)gn * ldb + kk]) : 0.f;
      }
      uint4 p = make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
      *reinterpret_cast<uint4 *>(sB + ((r >> 3) * (kBK / 8) + ch) * 128 + (r & 7) * 16) = p;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; kk++) {
        const uint64_t da = smem_desc(a0 + kk * 256, kLBO, kSBO);
        const uint64_t db = smem_desc(b0 + kk * 256, kLBO, kSBO);
        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bars[s]))
                   : "memory");
    }
    issued = kb + 1;
  }

  // the last commit completes after every MMA before it
  if (tid == 0 && issued > 0) {
    const int kl = issued - 1;
    if (!mbar_wait(&bars[kl & 1], (kl >> 1) & 1, kWaitNs)) {
      ok_sh = 0;
      mbar_wait(&bars[kl & 1], (kl >> 1) & 1, kWaitNs);  // once more before the memory is freed
    }
  }
  __syncthreads();
  tc_fence_after();
  const bool ok = ok_sh != 0 && issued == nkb;
  if (!ok && tid == 0) atomicExch(status, 1);

  if (ok) {
    const int row = m0 + warp * 32 + lane;
    const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 8) {
      uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
                   : "r"(tbase + c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;"
                   : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7)::"memory");
      const float v[8] = {__uint_as_float(r0), __uint_as_float(r1), __uint_as_float(r2), __uint_as_float(r3),
                          __uint_as_float(r4), __uint_as_float(r5), __uint_as_float(r6), __uint_as_float(r7)};
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int col = n0 + c0 + j;
          if (col < N) {
            float x = v[j];
            if (EPI == kEpiBias || EPI == kEpiBiasTanh) x += bias[col];
            if (EPI == kEpiBiasTanh) x = tanhf(x);
            if (EPI == kEpiDTanh) {
              const float h = aux[(int64_t)row * ldaux + col];
              x *= 1.f - h * h;
            }
            C[((int64_t)blockIdx.z * M + row) * ldc + col] = x;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kNcols) : "memory");
}

template <int BN, bool TA, bool TB, int EPI>
cudaError_t launch_gemm(cudaStream_t s, int M, int N, int K, int splits, const float *A, int lda, const float *B,
                        int ldb, float *C, int ldc, const float *bias, const float *aux, int ldaux, int32_t *status) {
  constexpr int kStage = kBM * kBK * 2 + BN * kBK * 2;
  constexpr int kSmem = 2 * kStage;
  auto kern = umma_gemm_bf16<BN, TA, TB, EPI>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int kslice = (K + splits - 1) / splits;
  dim3 grid((M + kBM - 1) / kBM, (N + BN - 1) / BN, (K + kslice - 1) / kslice);
  kern<<<grid, 128, kSmem, s>>>(M, N, K, kslice, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
  return cudaGetLastError();
}

template <int BN, bool TA, bool TB>
cudaError_t launch_epi(cudaStream_t s, int epi, int M, int N, int K, int sp, const float *A, int lda, const float *B,
                       int ldb, float *C, int ldc, const float *bias, const float *aux, int ldaux, int32_t *status) {
  switch (epi) {
    case kEpiStore: return launch_gemm<BN, TA, TB, kEpiStore>(s, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
    case kEpiBias: return launch_gemm<BN, TA, TB, kEpiBias>(s, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
    case kEpiBiasTanh:
      return launch_gemm<BN, TA, TB, kEpiBiasTanh>(s, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
    case kEpiDTanh: return launch_gemm<BN, TA, TB, kEpiDTanh>(s, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
  }
  return cudaErrorInvalidValue;
}

template <int BN>
cudaError_t launch_bn(cudaStream_t s, int epi, bool ta, bool tb, int M, int N, int K, int sp, const float *A, int lda,
                      const float *B, int ldb, float *C, int ldc, const float *bias, const float *aux, int ldaux,
                      int32_t *status) {
  if (!ta && !tb) return launch_epi<BN, false, false>(s, epi, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
  if (!ta && tb) return launch_epi<BN, false, true>(s, epi, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
  if (ta && !tb) return launch_epi<BN, true, false>(s, epi, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
  return launch_epi<BN, true, true>(s, epi, M, N, K, sp, A, lda, B, ldb, C, ldc, bias, aux, ldaux, status);
}

// ---------------------------------------------------------------- MLP pieces

// G = 2 (Y - T) / (rows * cols); per-block partial sums of (Y - T)^2
__global__ void __launch_bounds__(256) mse_grad(int64_t n, float scale, const float *__restrict__ Y,
                                                const float *__restrict__ T, float *__restrict__ G,
                                                float *__restrict__ part) {
  __shared__ float sh[8];
  float acc = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = Y[i] - T[i];
    G[i] = 2.f * scale * d;
    acc += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; w++) t += sh[w];
    part[blockIdx.x] = t;
  }
}

__global__ void sum_parts(int nparts, float scale, const float *__restrict__ part, float *__restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float t = 0.f;
    for (int i = 0; i < nparts; i++) t += part[i];
    out[0] = t * scale;
  }
}

// db[n] = sum over rows of G[row][n]  (fixed order)
__global__ void col_sums(int rows, int cols, const float *__restrict__ G, float *__restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cols) return;
  float t = 0.f;
  for (int r = 0; r < rows; r++) t += G[(int64_t)r * cols + n];
  db[n] = t;
}

__global__ void adam_step(int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                          float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

constexpr int kLossBlocks = 64;

// C[m][n] = sum of the split-K partial tiles in slice order
__global__ void split_reduce(int M, int N, int splits, const float *__restrict__ ws, float *__restrict__ C, int ldc) {
  const int64_t mn = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < mn; i += (int64_t)gridDim.x * blockDim.x) {
    float t = 0.f;
    for (int z = 0; z < splits; z++) t += ws[z * mn + i];
    C[(i / N) * ldc + i % N] = t;
  }
}

// splitmix64: seeded, platform-independent initial weights
uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// one input row (FP32, global) through the network by one CTA
__global__ void __launch_bounds__(512) mlp_row_kernel(MlpRow m, const float *__restrict__ P,
                                                      const float *__restrict__ x, float *__restrict__ y) {
  __shared__ float in[kMlpRowMaxDim], tmp[kMlpRowMaxDim];
  for (int t = threadIdx.x; t < m.dims[0]; t += blockDim.x) in[t] = bf16_round(x[t]);
  __syncthreads();
  mlp_row_forward(m, P, in, tmp, y);
}

}  // namespace

int gemm_splits(int M, int N, int K, int epi) {
  if (epi != kEpiStore) return 1;
  const int tiles = ((M + kBM - 1) / kBM) * ((N + (N <= 64 ? 64 : 128) - 1) / (N <= 64 ? 64 : 128));
  if (tiles >= 32 || K < 1024) return 1;
  int sp = (K + 255) / 256;  // at least four K-blocks per slice
  const int cap = 128 / tiles;
  return sp < cap ? sp : (cap < 1 ? 1 : cap);
}

cudaError_t gemm_bf16(cudaStream_t s, int M, int N, int K, const float *A, int lda, bool ta, const float *B, int ldb,
                      bool tb, float *C, int ldc, int epi, const float *bias, const float *aux, int ldaux,
                      int32_t *status, float *ws) {
  if (M <= 0 || N <= 0 || K <= 0) return cudaErrorInvalidValue;
  const int sp = ws ? gemm_splits(M, N, K, epi) : 1;
  float *out = sp > 1 ? ws : C;
  const int ldo = sp > 1 ? N : ldc;
  cudaError_t e = N <= 64 ? launch_bn<64>(s, epi, ta, tb, M, N, K, sp, A, lda, B, ldb, out, ldo, bias, aux, ldaux, status)
                          : launch_bn<128>(s, epi, ta, tb, M, N, K, sp, A, lda, B, ldb, out, ldo, bias, aux, ldaux, status);
  if (e != cudaSuccess || sp == 1) return e;
  const int kslice = (K + sp - 1) / sp, z = (K + kslice - 1) / kslice;
  const int64_t mn = (int64_t)M * N;
  split_reduce<<<(unsigned)std::min<int64_t>(592, (mn + 255) / 256), 256, 0, s>>>(M, N, z, ws, C, ldc);
  return cudaGetLastError();
}

cudaError_t Mlp::init(const std::vector<int> &d, uint64_t seed) {
  release();
  dims = d;
  const int L = layers();
  w_off.assign(L, 0);
  b_off.assign(L, 0);
  int64_t off = 0;
  for (int l = 0; l < L; l++) {
    w_off[l] = off;
    off += (int64_t)dims[l + 1] * dims[l];
    b_off[l] = off;
    off += dims[l + 1];
  }
  nparams = off;
  std::vector<float> h(nparams, 0.f);
  uint64_t st = seed;
  for (int l = 0; l < L; l++) {
    // Glorot-uniform weights, zero biases
    const double a = std::sqrt(6.0 / (dims[l] + dims[l + 1]));
    for (int64_t i = 0; i < (int64_t)dims[l + 1] * dims[l]; i++) {
      const double u = (splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
      h[w_off[l] + i] = (float)((2.0 * u - 1.0) * a);
    }
  }
  cudaError_t e = cudaSuccess;
  for (float **p : {&d_params, &d_grads, &d_m, &d_v})
    if (e == cudaSuccess) e = cudaMalloc((void **)p, sizeof(float) * nparams);
  if (e == cudaSuccess) e = cudaMemcpy(d_params, h.data(), sizeof(float) * nparams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_m, 0, sizeof(float) * nparams);
  if (e == cudaSuccess) e = cudaMemset(d_v, 0, sizeof(float) * nparams);
  if (e == cudaSuccess) e = cudaMemset(d_grads, 0, sizeof(float) * nparams);
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_part, sizeof(float) * kLossBlocks);
  {
    // split-K partials of the weight gradients: at most 128 tiles of 128 x 128
    int64_t mx = 0;
    for (int l = 0; l < L; l++) mx = std::max<int64_t>(mx, (int64_t)dims[l + 1] * dims[l]);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_splitws, sizeof(float) * std::max<int64_t>(mx * 128, 128 * 128 * 128));
  }
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_status, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemset(d_status, 0, sizeof(int32_t));
  adam_t = 0;
  return e;
}

cudaError_t Mlp::reserve(int batch) {
  if (batch <= cap) return cudaSuccess;
  for (float *p : d_h) cudaFree(p);
  for (float *p : d_g) cudaFree(p);
  if (d_target) cudaFree(d_target);
  d_h.assign(dims.size(), nullptr);
  d_g.assign(dims.size(), nullptr);
  d_target = nullptr;
  cap = 0;
  cudaError_t e = cudaSuccess;
  for (size_t l = 0; l < dims.size() && e == cudaSuccess; l++) {
    e = cudaMalloc((void **)&d_h[l], sizeof(float) * (size_t)batch * dims[l]);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_g[l], sizeof(float) * (size_t)batch * dims[l]);
  }
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_target, sizeof(float) * (size_t)batch * dims.back());
  if (e == cudaSuccess) cap = batch;
  return e;
}

void Mlp::release() {
  for (float *p : d_h) if (p) cudaFree(p);
  for (float *p : d_g) if (p) cudaFree(p);
  d_h.clear();
  d_g.clear();
  for (float **p : {&d_params, &d_grads, &d_m, &d_v, &d_target, &d_part, &d_loss, &d_splitws})
    if (*p) { cudaFree(*p); *p = nullptr; }
  if (d_status) { cudaFree(d_status); d_status = nullptr; }
  cap = 0;
}

cudaError_t Mlp::forward(cudaStream_t s, int batch) {
  const int L = layers();
  for (int l = 0; l < L; l++) {
    const int in = dims[l], out = dims[l + 1];
    // h[l+1] = act(h[l] W_l^T + b_l)
    cudaError_t e = gemm_bf16(s, batch, out, in, d_h[l], in, false, d_params + w_off[l], in, false, d_h[l + 1], out,
                              l + 1 < L ? kEpiBiasTanh : kEpiBias, d_params + b_off[l], nullptr, 0, d_status);
    launches++;
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

bool Mlp::row_layout(MlpRow &r) const {
  const int L = layers();
  if (L < 1 || L > kMlpRowMaxLayers) return false;
  r.L = L;
  for (int l = 0; l <= L; l++) {
    if (dims[l] > kMlpRowMaxDim) return false;
    r.dims[l] = dims[l];
  }
  for (int l = 0; l < L; l++) {
    r.w_off[l] = w_off[l];
    r.b_off[l] = b_off[l];
  }
  return true;
}

cudaError_t Mlp::forward_row(cudaStream_t s) {
  MlpRow r;
  if (!row_layout(r)) return cudaErrorInvalidValue;
  mlp_row_kernel<<<1, 512, 0, s>>>(r, d_params, d_h[0], d_h[layers()]);
  launches++;
  return cudaGetLastError();
}

cudaError_t Mlp::backward(cudaStream_t s, int batch) {
  const int L = layers();
  const int out = dims[L];
  const int64_t n = (int64_t)batch * out;
  mse_grad<<<kLossBlocks, 256, 0, s>>>(n, 1.f / (float)n, d_h[L], d_target, d_g[L], d_part);
  sum_parts<<<1, 32, 0, s>>>(kLossBlocks, 1.f / (float)n, d_part, d_loss);
  launches += 2;
  for (int l = L - 1; l >= 0; l--) {
    const int fi = dims[l], fo = dims[l + 1];
    // dW_l[o][i] = sum_b g[l+1][b][o] h[l][b][i]
    cudaError_t e = gemm_bf16(s, fo, fi, batch, d_g[l + 1], fo, true, d_h[l], fi, true, d_grads + w_off[l], fi,
                              kEpiStore, nullptr, nullptr, 0, d_status, d_splitws);
    if (e != cudaSuccess) return e;
    col_sums<<<(fo + 127) / 128, 128, 0, s>>>(batch, fo, d_g[l + 1], d_grads + b_off[l]);
    launches += gemm_splits(fo, fi, batch, kEpiStore) > 1 ? 3 : 2;
    if (l > 0) {
      // g[l][b][i] = (sum_o g[l+1][b][o] W_l[o][i]) * (1 - h[l][b][i]^2)
      e = gemm_bf16(s, batch, fi, fo, d_g[l + 1], fo, false, d_params + w_off[l], fi, true, d_g[l], fi, kEpiDTanh,
                    nullptr, d_h[l], fi, d_status);
      launches++;
      if (e != cudaSuccess) return e;
    }
  }
  return cudaGetLastError();
}

cudaError_t Mlp::adam(cudaStream_t s, float lr, float beta1, float beta2, float eps) {
  adam_t++;
  const float c1 = 1.f - (float)std::pow((double)beta1, (double)adam_t);
  const float c2 = 1.f - (float)std::pow((double)beta2, (double)adam_t);
  adam_step<<<148, 256, 0, s>>>(nparams, lr, beta1, beta2, eps, c1, c2, d_params, d_grads, d_m, d_v);
  launches++;
  return cudaGetLastError();
}

}  // namespace fastgpu

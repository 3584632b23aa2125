// solve_kernels.cu - K.u solve on the node-block matrix (sm_100a).
//
// Replaces cSymSprsMatrix::MultVect (mlib/sysmat.cpp:942-963) and PCGSolver
// (mlib/sysmat.cpp:1061-1125).  The FP64 path is the reference's Jacobi PCG:
//
//   r = f, z = D^-1 r, p = z, dot0 = z.r
//   loop: w = K p; alpha = dot0 / p.w; u += alpha p; r -= alpha w; z = D^-1 r
//         err = |r| / |f|  (|f| > 1e11 replaced by 1);  stop if err < tol
//         dot1 = z.r; beta = dot1/dot0; dot0 = dot1; p = z + beta p
//
// The mixed path runs the same iteration in FP32 (FP32 matrix, vectors and
// products) and keeps FP64 only for the solution and the true residual: after
// every chunk of iterations the FP32 correction is flushed into the FP64
// solution, r = f - K u is recomputed with the FP64 matrix and replaces the
// FP32 recurrence residual while the search direction is kept ("reliable
// updates").  Convergence is decided on that FP64 residual.
//
// Layouts.  The assembly target is the node-block CSR with each 3x3 block
// stored contiguously (AoS).  For the solve, each block-row is transposed
// once per assembly into a row-local structure-of-arrays padded to a
// multiple of 4 blocks: with s = srow[n] and nbp the padded row length,
// entry k (0..8) of block p of row n sits at 9*s + k*nbp + p.  Every such
// segment starts on a 16-byte boundary, so a lane loads 4 FP32 blocks
// (float4 per entry) or 2 FP64 blocks (double2 per entry) at once and the
// lanes of a row read consecutive 16-byte words.  Padding blocks hold zeros
// and point at the row's own node.  Vectors are padded to 4 entries per node
// (x, y, z, 0) so a node's part of x is one 16-byte (FP32) or two 16-byte
// (FP64) loads.
//
// Every scalar lives on the device (PcgState) and every reduction uses a
// fixed grid and a fixed combination order, so the host never waits inside
// an iteration and a solve is bit-reproducible.  Kernels check state->done
// first, so iterations launched past convergence cost only their launch.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <cooperative_groups.h>

#include "internal.h"

namespace fastgpu {

constexpr int kSpmvThreads = 256;
constexpr int kVecThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-level fixed-order sum; returns the total in thread 0
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sbuf) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (lane < NT / 32) ? sbuf[lane] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

// padded node vectors
template <typename T> struct V4;
template <> struct V4<float> {
  static __device__ __forceinline__ void load(const float *p, float &a, float &b, float &c) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    a = v.x; b = v.y; c = v.z;
  }
  static __device__ __forceinline__ void store(float *p, float a, float b, float c) {
    *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, 0.f);
  }
};
template <> struct V4<double> {
  static __device__ __forceinline__ void load(const double *p, double &a, double &b, double &c) {
    const double2 v0 = *reinterpret_cast<const double2 *>(p);
    a = v0.x; b = v0.y; c = p[2];
  }
  static __device__ __forceinline__ void store(double *p, double a, double b, double c) {
    *reinterpret_cast<double2 *>(p) = make_double2(a, b);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(c, 0.0);
  }
};

// AoS blocks (FP64, or the FP32 tensor-core stiffness) -> padded row-local
// SoA, FP64 and FP32 copies
template <typename KT>
__global__ void __launch_bounds__(256)
aos_to_soa(int64_t nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ srow,
           const KT *__restrict__ K, double *__restrict__ Ks, float *__restrict__ Ks32) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < nrows; row += nwarps) {
    const int32_t b0 = rowptr[row], nb = rowptr[row + 1] - b0;
    const int32_t s0 = srow[row], nbp = srow[row + 1] - s0;
    const int64_t dst = 9 * (int64_t)s0;
    for (int p = lane; p < nb; p += 32) {
      const KT *src = K + 9 * ((int64_t)b0 + p);
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const double v = (double)src[k];
        if (Ks) Ks[dst + (int64_t)k * nbp + p] = v;
        if (Ks32) Ks32[dst + (int64_t)k * nbp + p] = (float)v;
      }
    }
  }
}

// Row epilogue shared by the SpMV kernels: y = K x (MODE 0, partial x.y) or
// y = b - K x (MODE 1, partial y.y).
template <typename XT, int MODE>
__device__ __forceinline__ void spmv_row_out(int64_t row, XT a0, XT a1, XT a2, const XT *__restrict__ x,
                                             const XT *__restrict__ b, XT *__restrict__ y, bool part,
                                             double &pacc) {
  if (MODE == 0) {
    V4<XT>::store(y + 4 * row, a0, a1, a2);
    if (part) {
      XT x0, x1, x2;
      V4<XT>::load(x + 4 * row, x0, x1, x2);
      pacc += (double)x0 * a0 + (double)x1 * a1 + (double)x2 * a2;
    }
  } else {
    XT b0, b1, b2;
    V4<XT>::load(b + 4 * row, b0, b1, b2);
    const XT y0 = b0 - a0, y1 = b1 - a1, y2 = b2 - a2;
    V4<XT>::store(y + 4 * row, y0, y1, y2);
    if (part) pacc += (double)y0 * y0 + (double)y1 * y1 + (double)y2 * y2;
  }
}

// matrix loads of the FP32 SpMV: plain, or cache-streaming (evict-first:
// the values and columns are read once per product, so the lines they take
// are the first to go and x, gathered many times, keeps its place in L1/L2)
template <bool CS, typename T>
__device__ __forceinline__ T ldm(const T *p) {
  if (CS) return __ldcs(p);
  return *p;
}

// FP32 SpMV: LPR lanes per block-row; a lane takes 4 blocks per trip (one
// int4 of columns, nine float4 of values, four float4 gathers of x): 14
// independent 16-byte loads in flight per lane.  CS: matrix loads streamed.
// Three CTAs per SM: at four the 52 registers of one trip's loads spill
// (measured 10 % slower in the PCG loop).
template <int MODE, int LPR, bool CS = false>
__global__ void __launch_bounds__(kSpmvThreads, 3)
spmv_f32(int64_t nrows, const int32_t *__restrict__ srow, const int32_t *__restrict__ scol,
         const float *__restrict__ val, const float *__restrict__ x, const float *__restrict__ b,
         float *__restrict__ y, double *__restrict__ part, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double sbuf[32];
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, q = lane % LPR;
  const int64_t warp = (blockIdx.x * (int64_t)kSpmvThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kSpmvThreads) >> 5;
  const float4 *__restrict__ x4 = reinterpret_cast<const float4 *>(x);
  double pacc = 0.0;
  for (int64_t row0 = warp * RPW; row0 < nrows; row0 += nwarps * RPW) {
    const int64_t row = row0 + lane / LPR;
    const bool live = row < nrows;
    int32_t s0 = 0, nbp = 0;
    if (live) {
      s0 = srow[row];
      nbp = srow[row + 1] - s0;
    }
    const float *__restrict__ vr = val + 9 * (int64_t)s0;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int j = 4 * q; j < nbp; j += 4 * LPR) {
      const int4 c = ldm<CS>(reinterpret_cast<const int4 *>(scol + s0 + j));
      float4 v[9];
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = ldm<CS>(reinterpret_cast<const float4 *>(vr + k * nbp + j));
      const float4 xa = x4[c.x], xb = x4[c.y], xc = x4[c.z], xd = x4[c.w];
      a0 += v[0].x * xa.x + v[1].x * xa.y + v[2].x * xa.z + v[0].y * xb.x + v[1].y * xb.y + v[2].y * xb.z +
            v[0].z * xc.x + v[1].z * xc.y + v[2].z * xc.z + v[0].w * xd.x + v[1].w * xd.y + v[2].w * xd.z;
      a1 += v[3].x * xa.x + v[4].x * xa.y + v[5].x * xa.z + v[3].y * xb.x + v[4].y * xb.y + v[5].y * xb.z +
            v[3].z * xc.x + v[4].z * xc.y + v[5].z * xc.z + v[3].w * xd.x + v[4].w * xd.y + v[5].w * xd.z;
      a2 += v[6].x * xa.x + v[7].x * xa.y + v[8].x * xa.z + v[6].y * xb.x + v[7].y * xb.y + v[8].y * xb.z +
            v[6].z * xc.x + v[7].z * xc.y + v[8].z * xc.z + v[6].w * xd.x + v[7].w * xd.y + v[8].w * xd.z;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (live && q == 0) spmv_row_out<float, MODE>(row, a0, a1, a2, x, b, y, part != nullptr, pacc);
  }
  if (part) {
    const double t = block_sum<kSpmvThreads>(pacc, sbuf);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

// FP32 SpMV with 16-bit column indices: each block-row stores its columns as
// offsets from the row's smallest column (every row of the mesh must span
// fewer than 65,536 nodes), 38 instead of 40 bytes per block for the matrix
// stream; otherwise spmv_f32<MODE, LPR> (the same sums in the same order).
template <int LPR>
__global__ void __launch_bounds__(kSpmvThreads, 3)
spmv_f32_c16(int64_t nrows, const int32_t *__restrict__ srow, const uint16_t *__restrict__ scol16,
             const int32_t *__restrict__ rowbase, const float *__restrict__ val, const float *__restrict__ x,
             float *__restrict__ y, double *__restrict__ part, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double sbuf[32];
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, q = lane % LPR;
  const int64_t warp = (blockIdx.x * (int64_t)kSpmvThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kSpmvThreads) >> 5;
  const float4 *__restrict__ x4 = reinterpret_cast<const float4 *>(x);
  double pacc = 0.0;
  for (int64_t row0 = warp * RPW; row0 < nrows; row0 += nwarps * RPW) {
    const int64_t row = row0 + lane / LPR;
    const bool live = row < nrows;
    int32_t s0 = 0, nbp = 0, base = 0;
    if (live) {
      s0 = srow[row];
      nbp = srow[row + 1] - s0;
      base = rowbase[row];
    }
    const float *__restrict__ vr = val + 9 * (int64_t)s0;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int j = 4 * q; j < nbp; j += 4 * LPR) {
      const ushort4 d = *reinterpret_cast<const ushort4 *>(scol16 + s0 + j);
      float4 v[9];
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = *reinterpret_cast<const float4 *>(vr + k * nbp + j);
      const float4 xa = x4[base + d.x], xb = x4[base + d.y], xc = x4[base + d.z], xd = x4[base + d.w];
      a0 += v[0].x * xa.x + v[1].x * xa.y + v[2].x * xa.z + v[0].y * xb.x + v[1].y * xb.y + v[2].y * xb.z +
            v[0].z * xc.x + v[1].z * xc.y + v[2].z * xc.z + v[0].w * xd.x + v[1].w * xd.y + v[2].w * xd.z;
      a1 += v[3].x * xa.x + v[4].x * xa.y + v[5].x * xa.z + v[3].y * xb.x + v[4].y * xb.y + v[5].y * xb.z +
            v[3].z * xc.x + v[4].z * xc.y + v[5].z * xc.z + v[3].w * xd.x + v[4].w * xd.y + v[5].w * xd.z;
      a2 += v[6].x * xa.x + v[7].x * xa.y + v[8].x * xa.z + v[6].y * xb.x + v[7].y * xb.y + v[8].y * xb.z +
            v[6].z * xc.x + v[7].z * xc.y + v[8].z * xc.z + v[6].w * xd.x + v[7].w * xd.y + v[8].w * xd.z;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (live && q == 0) spmv_row_out<float, 0>(row, a0, a1, a2, x, nullptr, y, part != nullptr, pacc);
  }
  if (part) {
    const double t = block_sum<kSpmvThreads>(pacc, sbuf);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

// FP32 SpMV with the matrix streamed through shared memory.  In the
// row-local SoA layout the values of consecutive block-rows are one
// contiguous range (and so are their column indices), so a tile of rows
// arrives with two cp.async.bulk copies (completion on an mbarrier, this
// GPU's memory only): the tile after the current one is requested before
// the current one is computed (two stages), and the bytes in flight are not
// bounded by registers.  Lanes then read values and columns from shared
// memory and gather x (L2-resident) from global memory; LPR lanes per row,
// 4 blocks per lane per trip, the same sums as spmv_f32.  Tiles and the grid
// are fixed per pattern, so the p.w partials (one per CTA) are too.  A wait
// that runs out (bounded) sets *status and the CTA stops.
constexpr int kBulkThreads = 256;
constexpr uint64_t kBulkWaitNs = 1000000000ull;

template <int LPR>
__global__ void __launch_bounds__(kBulkThreads, 2)
spmv_f32_bulk(int ntiles, const int32_t *__restrict__ tile_row, const int32_t *__restrict__ srow,
              const int32_t *__restrict__ scol, const float *__restrict__ val, const float *__restrict__ x,
              float *__restrict__ y, double *__restrict__ part, const int32_t *__restrict__ skip,
              int32_t *__restrict__ status, int vbytes, int cbytes) {
  if (skip && *skip) return;
  extern __shared__ __align__(128) uint8_t bsm[];
  __shared__ double sbuf[32];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int fail_sh;
  constexpr int RPW = 32 / LPR;
  constexpr int NWARP = kBulkThreads / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, q = lane % LPR;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((unsigned)__cvta_generic_to_shared(&bars[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((unsigned)__cvta_generic_to_shared(&bars[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail_sh = 0;
  }
  __syncthreads();
  auto issue = [&](int t, int st) {
    const int32_t b0 = srow[tile_row[t]], b1 = srow[tile_row[t + 1]];
    const uint32_t nv = 36u * (uint32_t)(b1 - b0), nc = 4u * (uint32_t)(b1 - b0);
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&bars[st]);
    uint8_t *dv = bsm + st * (vbytes + cbytes), *dc = dv + vbytes;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(nv + nc) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dv)),
                 "l"(val + 9 * (int64_t)b0), "r"(nv), "r"(bar)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dc)),
                 "l"(scol + b0), "r"(nc), "r"(bar)
                 : "memory");
  };
  auto wait = [&](int st, uint32_t parity) -> bool {
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&bars[st]);
    uint32_t ok = 0;
    uint64_t t0 = 0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (true) {
      asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                   "selp.b32 %0, 1, 0, p;\n\t}"
                   : "=r"(ok)
                   : "r"(bar), "r"(parity)
                   : "memory");
      if (ok) return true;
      uint64_t t1;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
      if (t1 - t0 > kBulkWaitNs) return false;
    }
  };
  const float4 *__restrict__ x4 = reinterpret_cast<const float4 *>(x);
  double pacc = 0.0;
  bool next_issued = false;
  if (tid == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
    const int st = k & 1;
    const int tn = t + gridDim.x;
    next_issued = tn < ntiles;
    if (tid == 0 && next_issued) issue(tn, st ^ 1);
    if (!wait(st, (uint32_t)((k >> 1) & 1))) atomicExch(&fail_sh, 1);
    __syncthreads();
    if (fail_sh) break;
    const float *sv = reinterpret_cast<const float *>(bsm + st * (vbytes + cbytes));
    const int32_t *sc = reinterpret_cast<const int32_t *>(bsm + st * (vbytes + cbytes) + vbytes);
    const int32_t r0 = tile_row[t], r1 = tile_row[t + 1];
    const int32_t base = srow[r0];
    for (int32_t rr = r0 + warp * RPW; rr < r1; rr += NWARP * RPW) {
      const int32_t row = rr + lane / LPR;
      const bool live = row < r1;
      int32_t s0 = 0, nbp = 0;
      if (live) {
        s0 = srow[row] - base;
        nbp = srow[row + 1] - srow[row];
      }
      const float *vr = sv + 9 * s0;
      float a0 = 0.f, a1 = 0.f, a2 = 0.f;
      for (int j = 4 * q; j < nbp; j += 4 * LPR) {
        const int4 c = *reinterpret_cast<const int4 *>(sc + s0 + j);
        const float4 xa = x4[c.x], xb = x4[c.y], xc = x4[c.z], xd = x4[c.w];
        float4 v[9];
#pragma unroll
        for (int kk = 0; kk < 9; kk++) v[kk] = *reinterpret_cast<const float4 *>(vr + kk * nbp + j);
        a0 += v[0].x * xa.x + v[1].x * xa.y + v[2].x * xa.z + v[0].y * xb.x + v[1].y * xb.y + v[2].y * xb.z +
              v[0].z * xc.x + v[1].z * xc.y + v[2].z * xc.z + v[0].w * xd.x + v[1].w * xd.y + v[2].w * xd.z;
        a1 += v[3].x * xa.x + v[4].x * xa.y + v[5].x * xa.z + v[3].y * xb.x + v[4].y * xb.y + v[5].y * xb.z +
              v[3].z * xc.x + v[4].z * xc.y + v[5].z * xc.z + v[3].w * xd.x + v[4].w * xd.y + v[5].w * xd.z;
        a2 += v[6].x * xa.x + v[7].x * xa.y + v[8].x * xa.z + v[6].y * xb.x + v[7].y * xb.y + v[8].y * xb.z +
              v[6].z * xc.x + v[7].z * xc.y + v[8].z * xc.z + v[6].w * xd.x + v[7].w * xd.y + v[8].w * xd.z;
      }
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      }
      if (live && q == 0) spmv_row_out<float, 0>(row, a0, a1, a2, x, nullptr, y, part != nullptr, pacc);
    }
    __syncthreads();  // this stage may be refilled by the next prefetch
  }
  if (fail_sh) {
    if (tid == 0) {
      atomicExch(status, 1);
      // copies in flight land before the shared memory goes away (bounded)
      wait(k & 1, (uint32_t)((k >> 1) & 1));
      if (next_issued) wait((k + 1) & 1, (uint32_t)(((k + 1) >> 1) & 1));
    }
    __syncthreads();
    return;
  }
  if (part) {
    const double tsum = block_sum<kBulkThreads>(pacc, sbuf);
    if (threadIdx.x == 0) part[blockIdx.x] = tsum;
  }
}

// FP64 SpMV: LPR lanes per block-row; a lane takes 2 blocks per trip (one
// int2 of columns, nine double2 of values, two gathers of x).
template <int MODE, int LPR>
__global__ void __launch_bounds__(kSpmvThreads, 4)
spmv_f64(int64_t nrows, const int32_t *__restrict__ srow, const int32_t *__restrict__ scol,
         const double *__restrict__ val, const double *__restrict__ x, const double *__restrict__ b,
         double *__restrict__ y, double *__restrict__ part, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double sbuf[32];
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, q = lane % LPR;
  const int64_t warp = (blockIdx.x * (int64_t)kSpmvThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kSpmvThreads) >> 5;
  double pacc = 0.0;
  for (int64_t row0 = warp * RPW; row0 < nrows; row0 += nwarps * RPW) {
    const int64_t row = row0 + lane / LPR;
    const bool live = row < nrows;
    int32_t s0 = 0, nbp = 0;
    if (live) {
      s0 = srow[row];
      nbp = srow[row + 1] - s0;
    }
    const double *__restrict__ vr = val + 9 * (int64_t)s0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 2 * q; j < nbp; j += 2 * LPR) {
      const int2 c = *reinterpret_cast<const int2 *>(scol + s0 + j);
      double2 v[9];
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = *reinterpret_cast<const double2 *>(vr + k * nbp + j);
      double xa0, xa1, xa2, xb0, xb1, xb2;
      V4<double>::load(x + 4 * (int64_t)c.x, xa0, xa1, xa2);
      V4<double>::load(x + 4 * (int64_t)c.y, xb0, xb1, xb2);
      a0 += v[0].x * xa0 + v[1].x * xa1 + v[2].x * xa2 + v[0].y * xb0 + v[1].y * xb1 + v[2].y * xb2;
      a1 += v[3].x * xa0 + v[4].x * xa1 + v[5].x * xa2 + v[3].y * xb0 + v[4].y * xb1 + v[5].y * xb2;
      a2 += v[6].x * xa0 + v[7].x * xa1 + v[8].x * xa2 + v[6].y * xb0 + v[7].y * xb1 + v[8].y * xb2;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (live && q == 0) spmv_row_out<double, MODE>(row, a0, a1, a2, x, b, y, part != nullptr, pacc);
  }
  if (part) {
    const double t = block_sum<kSpmvThreads>(pacc, sbuf);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

// single-block fixed-order sum of n partials
__device__ __forceinline__ double sum_partials(const double *p, int n, double *sbuf) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  return block_sum<256>(v, sbuf);
}

// z = Dinv r with Dinv stored as 3 padded rows per node
template <typename T>
__device__ __forceinline__ void apply_dinv(const T *D, T r0, T r1, T r2, T &z0, T &z1, T &z2) {
  z0 = D[0] * r0 + D[1] * r1 + D[2] * r2;
  z1 = D[4] * r0 + D[5] * r1 + D[6] * r2;
  z2 = D[8] * r0 + D[9] * r1 + D[10] * r2;
}

// ---- fused iteration kernels (kernel-per-step path)
// The scalars of one iteration come from fixed-order sums of per-block
// partials.  Instead of a single-block kernel between the vector kernels,
// every block of the next vector kernel forms the same sum itself (same block
// size, same order, hence the same bits) and takes the same decision; the
// last block to finish (a counter in the state) commits the scalars, so no
// block ever reads a value another block of the same launch has overwritten.

// true in exactly one thread of the last block to reach this point
__device__ __forceinline__ bool last_block(uint32_t *counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
    if (is_last) *counter = 0;
  }
  __syncthreads();
  return is_last && threadIdx.x == 0;
}

// alpha = dot0 / p.w (every block), then u += alpha p; r -= alpha w;
// z = Dinv r; partials r.r, z.r.  The last block stores p.w and alpha, or
// the breakdown state, which every block detects alike.
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_update_fused(int64_t nnode, T *__restrict__ u, T *__restrict__ r, T *__restrict__ z, const T *__restrict__ p,
                 const T *__restrict__ w, const T *__restrict__ dinv, PcgState *__restrict__ st,
                 const double *__restrict__ part_pw, int npw, double *__restrict__ part_rr,
                 double *__restrict__ part_zr) {
  if (st->done) return;
  __shared__ double sbuf[32];
  __shared__ double alpha_sh;
  __shared__ int bad_sh;
  const double pw = sum_partials(part_pw, npw, sbuf);
  if (threadIdx.x == 0) {
    const double al = st->dot0 / pw;
    // breakdown unless alpha > 0: p.Kp and z.r of one sign (an SPD system, or
    // a negative definite one such as the stiffness of a left-handed B-spline
    // parametrisation, which the reference's signed det J produces)
    bad_sh = (!(al > 0.0) || !isfinite(pw) || !isfinite(al)) ? 1 : 0;
    alpha_sh = al;
  }
  __syncthreads();
  const int bad = bad_sh;
  const double al = alpha_sh;
  double rr = 0.0, zr = 0.0;
  if (!bad) {
    const T alpha = (T)al;
    for (int64_t n = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; n < nnode;
         n += (int64_t)gridDim.x * kVecThreads) {
      T u0, u1, u2, p0, p1, p2, r0, r1, r2, w0, w1, w2, z0, z1, z2;
      V4<T>::load(u + 4 * n, u0, u1, u2);
      V4<T>::load(p + 4 * n, p0, p1, p2);
      V4<T>::load(r + 4 * n, r0, r1, r2);
      V4<T>::load(w + 4 * n, w0, w1, w2);
      u0 = u0 + alpha * p0; u1 = u1 + alpha * p1; u2 = u2 + alpha * p2;
      r0 = r0 + (-alpha) * w0; r1 = r1 + (-alpha) * w1; r2 = r2 + (-alpha) * w2;
      apply_dinv(dinv + 12 * n, r0, r1, r2, z0, z1, z2);
      V4<T>::store(u + 4 * n, u0, u1, u2);
      V4<T>::store(r + 4 * n, r0, r1, r2);
      V4<T>::store(z + 4 * n, z0, z1, z2);
      rr += (double)r0 * r0 + (double)r1 * r1 + (double)r2 * r2;
      zr += (double)z0 * r0 + (double)z1 * r1 + (double)z2 * r2;
    }
    const double t1 = block_sum<kVecThreads>(rr, sbuf);
    if (threadIdx.x == 0) part_rr[blockIdx.x] = t1;
    const double t2 = block_sum<kVecThreads>(zr, sbuf);
    if (threadIdx.x == 0) part_zr[blockIdx.x] = t2;
  }
  if (last_block(&st->arrive_update)) {
    st->pw = pw;
    if (bad) st->done = 3;
    else st->alpha = al;
  }
}

// err, convergence and beta from the r.r / z.r partials (every block), then
// p = z + beta p; the last block commits iter, rr, err, done, beta, dot0.
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_direction_fused(int64_t nnode, T *__restrict__ p, const T *__restrict__ z, PcgState *__restrict__ st,
                    const double *__restrict__ part_rr, const double *__restrict__ part_zr, int n) {
  if (st->done) return;
  __shared__ double sbuf[32];
  __shared__ double beta_sh, err_sh;
  __shared__ int done_sh;
  const double rr = sum_partials(part_rr, n, sbuf);
  const double zr = sum_partials(part_zr, n, sbuf);
  if (threadIdx.x == 0) {
    const int iter = st->iter + 1;
    const double err = sqrt(rr) / st->lenf;
    int done = 0;
    if (err < st->tol) done = 1;
    else if (!isfinite(err)) done = 3;
    else if (iter >= st->maxit) done = 2;
    done_sh = done;
    err_sh = err;
    beta_sh = zr / st->dot0;
  }
  __syncthreads();
  const int done = done_sh;
  if (!done) {
    const T beta = (T)beta_sh;
    for (int64_t k = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; k < nnode;
         k += (int64_t)gridDim.x * kVecThreads) {
      T p0, p1, p2, z0, z1, z2;
      V4<T>::load(p + 4 * k, p0, p1, p2);
      V4<T>::load(z + 4 * k, z0, z1, z2);
      V4<T>::store(p + 4 * k, z0 + beta * p0, z1 + beta * p1, z2 + beta * p2);
    }
  }
  if (last_block(&st->arrive_dir)) {
    st->iter += 1;
    st->rr = rr;
    st->err = err_sh;
    if (done) {
      st->done = done;
    } else {
      st->beta = beta_sh;
      st->dot0 = zr;
    }
  }
}

// z = Dinv r, p = z (if init_p); partials z.r and f.f
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_precond(int64_t nnode, const T *__restrict__ r, T *__restrict__ z, T *__restrict__ p, const T *__restrict__ dinv,
            const T *__restrict__ f, double *part_zr, double *part_ff) {
  __shared__ double sbuf[32];
  double zr = 0.0, ff = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; n < nnode; n += (int64_t)gridDim.x * kVecThreads) {
    T r0, r1, r2, z0, z1, z2;
    V4<T>::load(r + 4 * n, r0, r1, r2);
    apply_dinv(dinv + 12 * n, r0, r1, r2, z0, z1, z2);
    V4<T>::store(z + 4 * n, z0, z1, z2);
    if (p) V4<T>::store(p + 4 * n, z0, z1, z2);
    zr += (double)z0 * r0 + (double)z1 * r1 + (double)z2 * r2;
    if (f) {
      T f0, f1, f2;
      V4<T>::load(f + 4 * n, f0, f1, f2);
      ff += (double)f0 * f0 + (double)f1 * f1 + (double)f2 * f2;
    }
  }
  const double t1 = block_sum<kVecThreads>(zr, sbuf);
  if (threadIdx.x == 0) part_zr[blockIdx.x] = t1;
  if (part_ff) {
    const double t2 = block_sum<kVecThreads>(ff, sbuf);
    if (threadIdx.x == 0) part_ff[blockIdx.x] = t2;
  }
}

// FP64 start: state from z.r, f.f and the initial r.r (warm start) or f.f
__global__ void __launch_bounds__(256) pcg_init_scalar(PcgState *st, const double *part_zr, int nz,
                                                       const double *part_ff, int nf, const double *part_rr0,
                                                       int nr, double tol, const double *tol_dev, int maxit, int iter0) {
  if (tol_dev) tol = *tol_dev;
  __shared__ double sbuf[32];
  const double zr = sum_partials(part_zr, nz, sbuf);
  const double ff = sum_partials(part_ff, nf, sbuf);
  double rr0 = ff;
  if (part_rr0) rr0 = sum_partials(part_rr0, nr, sbuf);
  if (threadIdx.x == 0) {
    PcgState s{};
    s.dot0 = zr;
    double lenf = sqrt(ff);
    s.tol = tol;
    s.maxit = maxit;
    s.iter = iter0;
    if (lenf < tol) s.done = 1;        // PCGSolver returns at once for a null load
    if (lenf > 10e+10) lenf = 1.0;     // PCGSolver's large-load normaliser
    s.lenf = lenf;
    s.rr = rr0;
    s.err = sqrt(rr0) / lenf;
    s.err_true = s.err;
    if (!s.done && s.err < tol) s.done = 1;
    *st = s;
  }
}

// mixed path: u64 += x32, x32 = 0  (flush the FP32 correction)
__global__ void flush_correction(int64_t n4, double *__restrict__ u, float *__restrict__ x,
                                 const PcgState *__restrict__ st) {
  if (st->final) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    u[i] += (double)x[i];
    x[i] = 0.f;
  }
}

// mixed path: r32 = (float) r64; z32 = Dinv32 r32; p32 = z32 on the first update; partials z.r
__global__ void __launch_bounds__(kVecThreads)
replace_residual(int64_t nnode, const double *__restrict__ r64, float *__restrict__ r, float *__restrict__ z,
                 float *__restrict__ p, const float *__restrict__ dinv, const PcgState *__restrict__ st,
                 double *part_zr) {
  if (st->final) return;
  __shared__ double sbuf[32];
  const bool first = st->iter == 0;
  double zr = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; n < nnode; n += (int64_t)gridDim.x * kVecThreads) {
    double d0, d1, d2;
    V4<double>::load(r64 + 4 * n, d0, d1, d2);
    const float r0 = (float)d0, r1 = (float)d1, r2 = (float)d2;
    float z0, z1, z2;
    apply_dinv(dinv + 12 * n, r0, r1, r2, z0, z1, z2);
    V4<float>::store(r + 4 * n, r0, r1, r2);
    V4<float>::store(z + 4 * n, z0, z1, z2);
    if (first) V4<float>::store(p + 4 * n, z0, z1, z2);
    zr += (double)z0 * r0 + (double)z1 * r1 + (double)z2 * r2;
  }
  const double t = block_sum<kVecThreads>(zr, sbuf);
  if (threadIdx.x == 0) part_zr[blockIdx.x] = t;
}

// mixed path: the FP64 residual decides convergence; the iteration resumes otherwise
__global__ void __launch_bounds__(256) reliable_scalar(PcgState *st, const double *part_rr, int nr,
                                                       const double *part_zr, int nz) {
  __shared__ double sbuf[32];
  const double rr = sum_partials(part_rr, nr, sbuf);
  const double zr = sum_partials(part_zr, nz, sbuf);
  if (threadIdx.x == 0) {
    if (st->final || st->null_rhs || st->done >= 2) return;
    st->err_true = sqrt(rr) / st->lenf;
    st->rr = rr;
    st->err = st->err_true;
    st->updates += 1;
    st->best = 0;
    st->fresh = 0;
    if (!isfinite(st->err_true)) { st->done = 3; return; }
    if (st->err_true < st->tol) { st->done = 1; st->final = 1; st->best = 1; return; }
    // The FP64 residual must halve within 10 replacements (10 chunks of FP32
    // iterations) and must not grow 100x above its best; otherwise FP32
    // iterates cannot resolve this system (cond(K) * eps_fp32 near 1).  Where
    // the FP32 operator is not the rounded FP64 one (the tensor-core
    // stiffness against the element-by-element FP64 residual) the search
    // directions stop fitting the replaced residuals first: the recurrence
    // then starts afresh from the FP64 residual (restarted iterative
    // refinement, a fixed number of times) before stagnation is declared.
    const bool grew = st->updates > 1 && st->err_true > 100.0 * st->best_err;
    if (st->updates == 1 || st->err_true < st->best_err) st->best = 1;
    if (!grew && (st->updates == 1 || st->err_true < 0.5 * st->best_err)) {
      st->best_err = st->err_true;
      st->stall = 0;
    } else if (grew || ++st->stall >= 10) {
      if (st->restarts_left <= 0) { st->done = 4; return; }
      st->restarts_left--;
      st->restarts++;
      st->fresh = 1;
      st->stall = 0;
    }
    if (st->best) st->best_err = fmin(st->best_err, st->err_true);
    st->done = 0;
    st->dot0 = zr;
  }
}

// mixed path: a fresh start of the recurrence from the replaced residual
__global__ void restart_direction(int64_t n4, const float *__restrict__ z, float *__restrict__ p,
                                  const PcgState *__restrict__ st) {
  if (!st->fresh) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i];
}

// mixed path: remember the FP64 iterate with the smallest true residual
__global__ void keep_best(int64_t n4, const double *__restrict__ u, double *__restrict__ ubest,
                          const PcgState *__restrict__ st) {
  if (!st->best) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x)
    ubest[i] = u[i];
}

// mixed path start: lenf = |f| (with the reference's normaliser)
__global__ void __launch_bounds__(256) mixed_init_scalar(PcgState *st, const double *part_ff, int nf, double tol,
                                                         const double *tol_dev, int maxit, int restarts) {
  if (tol_dev) tol = *tol_dev;
  __shared__ double sbuf[32];
  const double ff = sum_partials(part_ff, nf, sbuf);
  if (threadIdx.x == 0) {
    PcgState s{};
    double lenf = sqrt(ff);
    s.tol = tol;
    s.maxit = maxit;
    s.restarts_left = restarts;
    if (lenf < tol) { s.done = 1; s.null_rhs = 1; }   // PCGSolver returns at once for a null load
    if (lenf > 10e+10) lenf = 1.0;
    s.lenf = lenf > 0.0 ? lenf : 1.0;
    *st = s;
  }
}

// Jacobi / block-Jacobi inverse per node from the diagonal block; 3 padded rows
template <typename T, typename KT>
__global__ void build_dinv(int64_t nnode, const int32_t *__restrict__ diag, const KT *__restrict__ K,
                           T *__restrict__ dinv, int block) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  T *D = dinv + 12 * n;
  const int32_t d = diag[n];
  double a[9];
  for (int k = 0; k < 9; k++) a[k] = (d >= 0) ? (double)K[(int64_t)d * 9 + k] : (k % 4 == 0 ? 1.0 : 0.0);
  double inv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!block) {
    inv[0] = 1.0 / a[0];
    inv[4] = 1.0 / a[4];
    inv[8] = 1.0 / a[8];
  } else {
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = -(a[3] * a[8] - a[5] * a[6]), c02 = a[3] * a[7] - a[4] * a[6];
    const double id = 1.0 / (a[0] * c00 + a[1] * c01 + a[2] * c02);
    inv[0] = c00 * id;
    inv[1] = -(a[1] * a[8] - a[2] * a[7]) * id;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    inv[3] = c01 * id;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    inv[5] = -(a[0] * a[5] - a[2] * a[3]) * id;
    inv[6] = c02 * id;
    inv[7] = -(a[0] * a[7] - a[1] * a[6]) * id;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  }
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) D[4 * i + j] = (T)inv[3 * i + j];
    D[4 * i + 3] = (T)0;
  }
}

__global__ void scatter_eq_to_node(int32_t neq, const int32_t *__restrict__ dof, const double *__restrict__ v,
                                   double *__restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < neq) out[dof[k]] = v[k];
}
__global__ void gather_node_to_eq(int32_t neq, const int32_t *__restrict__ dof, const double *__restrict__ v,
                                  double *__restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < neq) out[k] = v[dof[k]];
}

__global__ void __launch_bounds__(256) sumsq_kernel(int64_t n, const double *__restrict__ x, double *part) {
  __shared__ double sbuf[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += x[i] * x[i];
  const double t = block_sum<256>(s, sbuf);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
__global__ void __launch_bounds__(256) finish_sum(const double *part, int n, double *out) {
  __shared__ double sbuf[32];
  const double t = sum_partials(part, n, sbuf);
  if (threadIdx.x == 0) *out = t;
}

// ---------------------------------------------------------------------------
// host side

cudaEvent_t Ctx::take_event() {
  if (ev_pool.empty()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  cudaEvent_t e = ev_pool.back();
  ev_pool.pop_back();
  return e;
}
int64_t Ctx::begin_span(int kind) {
  if (!timing) return -1;
  Span sp{kind, span_ids++, false, take_event(), take_event()};
  cudaEventRecord(sp.a, stream);
  spans.push_back(sp);
  return sp.id;
}
void Ctx::end_span(int64_t id) {
  if (!timing) return;
  for (int i = (int)spans.size() - 1; i >= 0; i--) {
    Span &sp = spans[i];
    if (sp.closed || (id >= 0 && sp.id != id)) continue;
    cudaEventRecord(sp.b, stream);
    sp.closed = true;
    return;
  }
}
// call after the stream has been synchronised; open spans stay
void Ctx::harvest() {
  std::vector<Span> open;
  for (Span &sp : spans) {
    if (!sp.closed) {
      open.push_back(sp);
      continue;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) {
      kt_ms[sp.kind] += ms;
      kt_n[sp.kind] += 1;
    }
    ev_pool.push_back(sp.a);
    ev_pool.push_back(sp.b);
  }
  spans.swap(open);
}

static int spmv_grid(const Ctx &c) { return c.sm_count * 8; }

// partial buffers inside c.d_partials (16384 doubles)
static double *P_A(Ctx &c) { return c.d_partials; }           // [G]  p.w
static double *P_B(Ctx &c) { return c.d_partials + 2048; }    // [R]  r.r
static double *P_C(Ctx &c) { return c.d_partials + 4096; }    // [R]  z.r
static double *P_D(Ctx &c) { return c.d_partials + 6144; }    // [R]  f.f
static double *P_E(Ctx &c) { return c.d_partials + 8192; }    // [G]  true r.r

// lanes per block-row chosen at run time (fast_gpu_set_option / fast_gpu_autotune)
template <int MODE>
static void spmv64_go(const Ctx &c, int G, int64_t nn, const double *Ks, const double *x, const double *b, double *y,
                      double *part, const int32_t *skip) {
  switch (c.lpr64) {
    case 4: spmv_f64<MODE, 4><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, b, y, part, skip); break;
    case 8: spmv_f64<MODE, 8><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, b, y, part, skip); break;
    case 32: spmv_f64<MODE, 32><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, b, y, part, skip); break;
    default: spmv_f64<MODE, 16><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, b, y, part, skip);
  }
}
// tiles of the bulk-staged SpMV: up to kBulkRows consecutive block-rows, cut
// earlier when their values would pass kBulkTileBytes; built once per pattern
constexpr int kBulkRows = 16;
constexpr int64_t kBulkTileBytes = 48 * 1024;

cudaError_t ensure_bulk_tiles(Ctx &c) {
  if (c.d_tile_row) return cudaSuccess;
  std::vector<int32_t> tr(1, 0);
  int64_t vmax = 0;
  const int64_t n = c.nnode;
  for (int64_t r = 0; r < n;) {
    int64_t e = std::min<int64_t>(r + kBulkRows, n);
    while (e > r + 1 && 36 * (int64_t)(c.h_srow[e] - c.h_srow[r]) > kBulkTileBytes) e--;
    vmax = std::max<int64_t>(vmax, 36 * (int64_t)(c.h_srow[e] - c.h_srow[r]));
    tr.push_back((int32_t)e);
    r = e;
  }
  c.bulk_vbytes = (int)((vmax + 127) / 128 * 128);
  c.bulk_cbytes = (int)((vmax / 9 + 127) / 128 * 128);
  c.bulk_ntiles = (int)tr.size() - 1;
  cudaError_t e = cudaMalloc((void **)&c.d_tile_row, sizeof(int32_t) * tr.size());
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(c.d_tile_row, tr.data(), sizeof(int32_t) * tr.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  const int smem = 2 * (c.bulk_vbytes + c.bulk_cbytes);
  int per_sm = 0;
  for (auto kern : {spmv_f32_bulk<8>, spmv_f32_bulk<16>}) {
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    int a = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kern, kBulkThreads, smem)) != cudaSuccess) return e;
    per_sm = per_sm ? std::min(per_sm, a) : a;
  }
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  c.bulk_grid = (int)std::min<int64_t>((int64_t)per_sm * c.sm_count, c.bulk_ntiles);
  return cudaSuccess;
}

// 16-bit column offsets of the solve layout (once per pattern); not offered
// when a block-row spans 65,536 nodes or more
cudaError_t ensure_col16(Ctx &c) {
  if (c.d_scol16) return cudaSuccess;
  const int64_t n = c.nnode;
  std::vector<int32_t> base((size_t)n);
  std::vector<uint16_t> d16((size_t)c.nnzb_pad);
  for (int64_t i = 0; i < n; i++) {
    const int32_t s0 = c.h_srow[i], s1 = c.h_srow[i + 1];
    int32_t lo = c.h_scol[s0];
    for (int32_t k = s0; k < s1; k++) lo = std::min(lo, c.h_scol[k]);
    base[(size_t)i] = lo;
    for (int32_t k = s0; k < s1; k++) {
      const int64_t d = (int64_t)c.h_scol[k] - lo;
      if (d > 65535) return cudaErrorNotSupported;
      d16[(size_t)k] = (uint16_t)d;
    }
  }
  cudaError_t e = cudaMalloc((void **)&c.d_rowbase, sizeof(int32_t) * std::max<int64_t>(1, n));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c.d_scol16, sizeof(uint16_t) * std::max<int64_t>(4, c.nnzb_pad));
  if (e == cudaSuccess) e = cudaMemcpy(c.d_rowbase, base.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c.d_scol16, d16.data(), sizeof(uint16_t) * c.nnzb_pad, cudaMemcpyHostToDevice);
  return e;
}

// grid of the FP32 SpMV kernels: two full waves of their three resident CTAs
// per SM (the row groups are interleaved over the CTAs, so every CTA has the
// same work and a partial last wave would idle a third of the SMs' slots)
static int spmv32_grid(const Ctx &c) { return c.sm_count * 6; }

// CTAs (= p.w partials) of the FP32 SpMV in use
static int spmv32_parts(const Ctx &c) { return c.spmv32_bulk ? c.bulk_grid : spmv32_grid(c); }

static void spmv32_go(const Ctx &c, int G, int64_t nn, const float *Ks, const float *x, float *y, double *part,
                      const int32_t *skip) {
  if (c.spmv32_bulk) {
    const int smem = 2 * (c.bulk_vbytes + c.bulk_cbytes);
    if (c.lpr32 >= 16)
      spmv_f32_bulk<16><<<c.bulk_grid, kBulkThreads, smem, c.stream>>>(c.bulk_ntiles, c.d_tile_row, c.d_srow, c.d_scol, Ks,
                                                                        x, y, part, skip, c.d_status, c.bulk_vbytes,
                                                                        c.bulk_cbytes);
    else
      spmv_f32_bulk<8><<<c.bulk_grid, kBulkThreads, smem, c.stream>>>(c.bulk_ntiles, c.d_tile_row, c.d_srow, c.d_scol, Ks,
                                                                       x, y, part, skip, c.d_status, c.bulk_vbytes,
                                                                       c.bulk_cbytes);
    return;
  }
  if (c.spmv32_c16) {
    if (c.lpr32 >= 16)
      spmv_f32_c16<16><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol16, c.d_rowbase, Ks, x, y, part, skip);
    else
      spmv_f32_c16<8><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol16, c.d_rowbase, Ks, x, y, part, skip);
    return;
  }
  if (c.spmv32_stream) {
    if (c.lpr32 >= 16)
      spmv_f32<0, 16, true><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip);
    else
      spmv_f32<0, 8, true><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip);
    return;
  }
  switch (c.lpr32) {
    case 4: spmv_f32<0, 4><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip); break;
    case 16: spmv_f32<0, 16><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip); break;
    case 32: spmv_f32<0, 32><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip); break;
    default: spmv_f32<0, 8><<<G, kSpmvThreads, 0, c.stream>>>(nn, c.d_srow, c.d_scol, Ks, x, nullptr, y, part, skip);
  }
}

cudaError_t launch_to_soa(Ctx &c, const double *K, double *Ks, float *Ks32) {
  aos_to_soa<double><<<spmv_grid(c), 256, 0, c.stream>>>(c.nnode, c.d_rowptr, c.d_srow, K, Ks, Ks32);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_to_soa32(Ctx &c, const float *K32, float *Ks32) {
  aos_to_soa<float><<<spmv_grid(c), 256, 0, c.stream>>>(c.nnode, c.d_rowptr, c.d_srow, K32, nullptr, Ks32);
  c.launches++;
  return cudaGetLastError();
}

// r = f - g on the padded node vectors (g = K u from the element kernels),
// r.r per block; nothing while *skip is non-zero
__global__ void __launch_bounds__(kSpmvThreads)
sub_residual(int64_t n4, const double *__restrict__ f, const double *__restrict__ g, double *__restrict__ r,
             double *__restrict__ part, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double sbuf[32];
  double rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kSpmvThreads + threadIdx.x; i < n4; i += (int64_t)gridDim.x * kSpmvThreads) {
    const double v = f[i] - g[i];
    r[i] = v;
    rr += v * v;
  }
  const double t = block_sum<kSpmvThreads>(rr, sbuf);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void copy_unless(int64_t n, const double *__restrict__ a, double *__restrict__ b,
                            const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

cudaError_t launch_matfree_residual(Ctx &c, const double *f, const double *u, double *r, double *part,
                                    const int32_t *skip) {
  const int64_t n4 = 4 * c.nnode;
  cudaError_t e;
  const double *uu = u;
  if (c.has_ties()) {
    // the full displacement field, slaves from their masters, in the FP64
    // second search-direction buffer (unused by the mixed iteration)
    copy_unless<<<kRedBlocks, 256, 0, c.stream>>>(n4, u, c.d_p2, skip);
    c.launches++;
    if ((e = launch_tie_prolong(c, c.d_p2)) != cudaSuccess) return e;
    uu = c.d_p2;
  }
  if ((e = cudaMemsetAsync(c.d_gint, 0, sizeof(double) * n4, c.stream)) != cudaSuccess) return e;
  if ((e = launch_tl_at(c, nullptr, c.d_gint, false, true, uu, skip)) != cudaSuccess) return e;
  if (c.has_ties()) {
    if ((e = launch_tied_matvec(c, uu, c.d_gint, skip)) != cudaSuccess) return e;
    if ((e = launch_tie_restrict(c, c.d_gint)) != cudaSuccess) return e;
    if ((e = launch_zero_fixed(c, c.d_gint, skip)) != cudaSuccess) return e;
  }
  sub_residual<<<spmv_grid(c), kSpmvThreads, 0, c.stream>>>(n4, f, c.d_gint, r, part, skip);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_spmv(Ctx &c, const double *Ks, const double *x, double *y) {
  spmv64_go<0>(c, spmv_grid(c), c.nnode, Ks, x, nullptr, y, nullptr, nullptr);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_spmv32(Ctx &c, const float *Ks, const float *x, float *y) {
  spmv32_go(c, spmv32_grid(c), c.nnode, Ks, x, y, nullptr, nullptr);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_residual(Ctx &c, const double *Ks, const double *f, const double *u, double *r, double *rr_out) {
  double *part = P_E(c);
  if (Ks) {
    spmv64_go<1>(c, spmv_grid(c), c.nnode, Ks, u, f, r, part, nullptr);
    c.launches++;
  } else {
    cudaError_t e = launch_matfree_residual(c, f, u, r, part, nullptr);
    if (e != cudaSuccess) return e;
  }
  finish_sum<<<1, 256, 0, c.stream>>>(part, spmv_grid(c), rr_out);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_norm2(Ctx &c, const double *x, int64_t n, double *out_dev) {
  sumsq_kernel<<<kRedBlocks, 256, 0, c.stream>>>(n, x, c.d_partials);
  c.launches++;
  finish_sum<<<1, 256, 0, c.stream>>>(c.d_partials, kRedBlocks, out_dev);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_eq_to_node(Ctx &c, const double *eqv, double *nodev) {
  cudaError_t e = cudaMemsetAsync(nodev, 0, sizeof(double) * 4 * (size_t)c.nnode, c.stream);
  if (e != cudaSuccess) return e;
  if (c.neq > 0) {
    scatter_eq_to_node<<<(c.neq + 255) / 256, 256, 0, c.stream>>>(c.neq, c.d_dof_of_eq, eqv, nodev);
    c.launches++;
  }
  return cudaGetLastError();
}

cudaError_t launch_node_to_eq(Ctx &c, const double *nodev, double *eqv) {
  if (c.neq > 0) {
    gather_node_to_eq<<<(c.neq + 255) / 256, 256, 0, c.stream>>>(c.neq, c.d_dof_of_eq, nodev, eqv);
    c.launches++;
  }
  return cudaGetLastError();
}

cudaError_t launch_build_precond(Ctx &c, const double *K, int precond) {
  const int bs = 256;
  const unsigned g = (unsigned)((c.nnode + bs - 1) / bs);
  build_dinv<double, double><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K, c.d_dinv, precond);
  c.launches++;
  build_dinv<float, double><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K, c.s_dinv, precond);
  c.launches++;
  c.precond_built = precond;
  return cudaGetLastError();
}

cudaError_t launch_build_precond32(Ctx &c, const float *K32, int precond) {
  const int bs = 256;
  const unsigned g = (unsigned)((c.nnode + bs - 1) / bs);
  build_dinv<double, float><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K32, c.d_dinv, precond);
  c.launches++;
  build_dinv<float, float><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K32, c.s_dinv, precond);
  c.launches++;
  c.precond_built = precond;
  return cudaGetLastError();
}


// ---------------------------------------------------------------- persistent PCG
// For small systems the iteration is latency-bound (five kernels of a few
// microseconds each).  There one cooperative launch runs a whole chunk of
// iterations: each block owns a contiguous range of block-rows (nodes), and
// two grid barriers per iteration separate w = K p (with the p.w partials,
// the new search direction built on the fly) and the vector updates (with
// the r.r and z.r partials).  Every block sums the per-block partials itself, in the
// same fixed order, so the scalars agree in every block without a broadcast
// and a solve stays bit-reproducible.  Data written by other blocks during
// the launch (p and the partials) is read through L2 (ld.global.cg).  The
// scalars and the exit codes are exactly those of pcg_update_fused /
// pcg_direction_fused; block 0 writes them back to the PcgState at the end.
constexpr int kPersistThreads = 512;
constexpr uint64_t kBarrierWaitNs = 2000000000ull;  // one barrier wait; then the launch gives up

// Barrier over all blocks of a cooperative launch (grid_barrier below); the
// words are zeroed before a solve's first launch.
struct alignas(8) GridBarrier {
  unsigned int count;  // with gen: one 64-bit arrival counter (8-byte aligned)
  unsigned int gen;
  int32_t err;
  int32_t pad;
};
static_assert(sizeof(GridBarrier) <= Ctx::kBarrierBytes, "barrier words exceed their allocation");

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One 64-bit arrival counter (the count and gen words read as one), never
// reset within a solve: thread 0 of each block adds 1 with release semantics
// and polls with acquire loads until the counter reaches the next multiple of
// the grid.  (Measured against a sense-reversal barrier whose last arriver
// resets the count and advances a generation word behind full fences: 11.4
// against 13.6 us per FP32 PCG iteration on a 22,815-equation tangent; a flag
// barrier, each block posting its own word and block 0 releasing, was slower
// still.)  Every wait is bounded: when one runs out the error word is set and
// every block leaves at its next barrier.
__device__ bool grid_barrier(GridBarrier *b, int *ok_sh) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int32_t *verr = &b->err;
    int ok = *verr == 0;
    if (ok) {
      unsigned long long *ctr = reinterpret_cast<unsigned long long *>(&b->count);
      unsigned long long old, cur;
      asm volatile("atom.add.release.gpu.u64 %0, [%1], 1;" : "=l"(old) : "l"(ctr) : "memory");
      const unsigned long long target = (old / gridDim.x + 1) * gridDim.x;
      asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(cur) : "l"(ctr) : "memory");
      if (cur < target) {
        const uint64_t t0 = now_ns();
        do {
          if (*verr != 0) { ok = 0; break; }
          if (now_ns() - t0 > kBarrierWaitNs) { atomicExch(&b->err, 1); ok = 0; break; }
          asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(cur) : "l"(ctr) : "memory");
        } while (cur < target);
      }
    }
    *ok_sh = ok;
  }
  __syncthreads();
  return *ok_sh != 0;
}

template <typename T> struct V4cg;
template <> struct V4cg<float> {
  static __device__ __forceinline__ void load(const float *p, float &a, float &b, float &c) {
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(p));
    a = v.x; b = v.y; c = v.z;
  }
};
template <> struct V4cg<double> {
  static __device__ __forceinline__ void load(const double *p, double &a, double &b, double &c) {
    const double2 v0 = __ldcg(reinterpret_cast<const double2 *>(p));
    a = v0.x; b = v0.y; c = __ldcg(p + 2);
  }
};

// gather of the search direction: x_j = p_j (first iteration of a launch) or
// x_j = z_j + beta p_j (the direction of this iteration, built from the last
// one), read through L2
template <typename T>
struct DirGather {
  const T *p, *z;
  T beta;
  bool plain;
  __device__ __forceinline__ void load(int64_t j, T &a, T &b, T &c) const {
    V4cg<T>::load(p + 4 * j, a, b, c);
    if (!plain) {
      T z0, z1, z2;
      V4cg<T>::load(z + 4 * j, z0, z1, z2);
      a = z0 + beta * a;
      b = z1 + beta * b;
      c = z2 + beta * c;
    }
  }
};

__device__ __forceinline__ void persist_row_dir(const int32_t *__restrict__ scol, const float *__restrict__ vr,
                                                int32_t s0, int32_t nbp, int q, const DirGather<float> &x, float &a0,
                                                float &a1, float &a2) {
  for (int j = 4 * q; j < nbp; j += 64) {
    const int4 c = *reinterpret_cast<const int4 *>(scol + s0 + j);
    float4 v[9];
#pragma unroll
    for (int k = 0; k < 9; k++) v[k] = *reinterpret_cast<const float4 *>(vr + k * nbp + j);
    float xa0, xa1, xa2, xb0, xb1, xb2, xc0, xc1, xc2, xd0, xd1, xd2;
    x.load(c.x, xa0, xa1, xa2);
    x.load(c.y, xb0, xb1, xb2);
    x.load(c.z, xc0, xc1, xc2);
    x.load(c.w, xd0, xd1, xd2);
    a0 += v[0].x * xa0 + v[1].x * xa1 + v[2].x * xa2 + v[0].y * xb0 + v[1].y * xb1 + v[2].y * xb2 +
          v[0].z * xc0 + v[1].z * xc1 + v[2].z * xc2 + v[0].w * xd0 + v[1].w * xd1 + v[2].w * xd2;
    a1 += v[3].x * xa0 + v[4].x * xa1 + v[5].x * xa2 + v[3].y * xb0 + v[4].y * xb1 + v[5].y * xb2 +
          v[3].z * xc0 + v[4].z * xc1 + v[5].z * xc2 + v[3].w * xd0 + v[4].w * xd1 + v[5].w * xd2;
    a2 += v[6].x * xa0 + v[7].x * xa1 + v[8].x * xa2 + v[6].y * xb0 + v[7].y * xb1 + v[8].y * xb2 +
          v[6].z * xc0 + v[7].z * xc1 + v[8].z * xc2 + v[6].w * xd0 + v[7].w * xd1 + v[8].w * xd2;
  }
}
__device__ __forceinline__ void persist_row_dir(const int32_t *__restrict__ scol, const double *__restrict__ vr,
                                                int32_t s0, int32_t nbp, int q, const DirGather<double> &x,
                                                double &a0, double &a1, double &a2) {
  for (int j = 2 * q; j < nbp; j += 32) {
    const int2 c = *reinterpret_cast<const int2 *>(scol + s0 + j);
    double2 v[9];
#pragma unroll
    for (int k = 0; k < 9; k++) v[k] = *reinterpret_cast<const double2 *>(vr + k * nbp + j);
    double xa0, xa1, xa2, xb0, xb1, xb2;
    x.load(c.x, xa0, xa1, xa2);
    x.load(c.y, xb0, xb1, xb2);
    a0 += v[0].x * xa0 + v[1].x * xa1 + v[2].x * xa2 + v[0].y * xb0 + v[1].y * xb1 + v[2].y * xb2;
    a1 += v[3].x * xa0 + v[4].x * xa1 + v[5].x * xa2 + v[3].y * xb0 + v[4].y * xb1 + v[5].y * xb2;
    a2 += v[6].x * xa0 + v[7].x * xa1 + v[8].x * xa2 + v[6].y * xb0 + v[7].y * xb1 + v[8].y * xb2;
  }
}

// sum of the G per-block partials at part[0..G), the same in every block
__device__ __forceinline__ double persist_sum(const double *part, int G, double *sbuf, double *bc) {
  const double v = threadIdx.x < G ? __ldcg(part + threadIdx.x) : 0.0;
  const double t = block_sum<kPersistThreads>(v, sbuf);
  if (threadIdx.x == 0) *bc = t;
  __syncthreads();
  const double r = *bc;
  __syncthreads();
  return r;
}

template <typename T>
__global__ void __launch_bounds__(kPersistThreads, 1)
pcg_persistent(int64_t nnode, const int32_t *__restrict__ srow, const int32_t *__restrict__ scol,
               const T *__restrict__ val, T *u, T *r, T *z, T *p, T *p2, T *w, const T *__restrict__ dinv,
               PcgState *st, double *part_pw, double *part_rr, double *part_zr, GridBarrier *bar, int iters) {
  __shared__ double sbuf[32];
  __shared__ double bc;
  __shared__ int ok_sh;
  if (st->done) return;  // the same value in every block: no block waits alone
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, q = lane & 15;
  double dot0 = st->dot0, alpha = st->alpha, beta = st->beta, rr = st->rr, err = st->err, pw = st->pw;
  int iter = st->iter, done = 0;
  const double tol = st->tol, lenf = st->lenf;
  const int maxit = st->maxit;
  const int64_t rb = (nnode + G - 1) / G;
  const int64_t r0 = min(nnode, (int64_t)b * rb), r1 = min(nnode, r0 + rb);
  // The direction of iteration k+1 is p = z + beta p_k.  Instead of a third
  // barrier before the SpMV, each block builds it on the fly from z and the
  // last direction (both final after the second barrier) for every gathered
  // node, and stores it for its own nodes in the other buffer.
  T *pcur = p, *pnxt = p2;
  bool first = true;
  int it = 0;
  for (; it < iters; it++) {
    const DirGather<T> dir{pcur, z, (T)beta, first};
    T *pdir = first ? pcur : pnxt;
    // w = K p on the block's rows, partial p.w, own rows of p stored
    double pacc = 0.0;
    for (int64_t row0 = r0 + 2 * (tid >> 5); row0 < r1; row0 += 2 * (kPersistThreads / 32)) {
      const int64_t row = row0 + (lane >> 4);
      const bool live = row < r1;
      int32_t s0 = 0, nbp = 0;
      if (live) {
        s0 = srow[row];
        nbp = srow[row + 1] - s0;
      }
      T a0 = 0, a1 = 0, a2 = 0;
      persist_row_dir(scol, val + 9 * (int64_t)s0, s0, nbp, q, dir, a0, a1, a2);
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      }
      if (live && q == 0) {
        V4<T>::store(w + 4 * row, a0, a1, a2);
        T x0, x1, x2;
        dir.load(row, x0, x1, x2);
        if (!first) V4<T>::store(pdir + 4 * row, x0, x1, x2);
        pacc += (double)x0 * a0 + (double)x1 * a1 + (double)x2 * a2;
      }
    }
    pcur = pdir;
    pnxt = (pdir == p) ? p2 : p;
    first = false;
    double t = block_sum<kPersistThreads>(pacc, sbuf);
    if (tid == 0) part_pw[b] = t;
    if (!grid_barrier(bar, &ok_sh)) { done = kDoneBarrierTimeout; break; }
    pw = persist_sum(part_pw, G, sbuf, &bc);
    alpha = dot0 / pw;
    if (!(alpha > 0.0) || !isfinite(pw) || !isfinite(alpha)) { done = 3; break; }
    // u += alpha p; r -= alpha w; z = Dinv r; partials r.r, z.r
    const T al = (T)alpha;
    double rra = 0.0, zra = 0.0;
    for (int64_t n = r0 + tid; n < r1; n += kPersistThreads) {
      T u0, u1, u2, p0, p1, p2_, x0, x1, x2, w0, w1, w2, z0, z1, z2;
      V4<T>::load(u + 4 * n, u0, u1, u2);
      V4<T>::load(pcur + 4 * n, p0, p1, p2_);
      V4<T>::load(r + 4 * n, x0, x1, x2);
      V4<T>::load(w + 4 * n, w0, w1, w2);
      u0 = u0 + al * p0; u1 = u1 + al * p1; u2 = u2 + al * p2_;
      x0 = x0 + (-al) * w0; x1 = x1 + (-al) * w1; x2 = x2 + (-al) * w2;
      apply_dinv(dinv + 12 * n, x0, x1, x2, z0, z1, z2);
      V4<T>::store(u + 4 * n, u0, u1, u2);
      V4<T>::store(r + 4 * n, x0, x1, x2);
      V4<T>::store(z + 4 * n, z0, z1, z2);
      rra += (double)x0 * x0 + (double)x1 * x1 + (double)x2 * x2;
      zra += (double)z0 * x0 + (double)z1 * x1 + (double)z2 * x2;
    }
    t = block_sum<kPersistThreads>(rra, sbuf);
    if (tid == 0) part_rr[b] = t;
    t = block_sum<kPersistThreads>(zra, sbuf);
    if (tid == 0) part_zr[b] = t;
    if (!grid_barrier(bar, &ok_sh)) { done = kDoneBarrierTimeout; break; }
    rr = persist_sum(part_rr, G, sbuf, &bc);
    const double zr = persist_sum(part_zr, G, sbuf, &bc);
    iter += 1;
    err = sqrt(rr) / lenf;
    if (err < tol) { done = 1; break; }
    if (!isfinite(err)) { done = 3; break; }
    if (iter >= maxit) { done = 2; break; }
    beta = zr / dot0;
    dot0 = zr;
  }
  // leave the direction the per-kernel iteration expects in p: the next one
  // (z + beta p) when the chunk ran out, else the last one used
  if (done != kDoneBarrierTimeout) {
    const bool next = (done == 0);
    if (next || pcur != p) {
      const T be = (T)beta;
      for (int64_t n = r0 + tid; n < r1; n += kPersistThreads) {
        T p0, p1, p2_, z0, z1, z2;
        V4<T>::load(pcur + 4 * n, p0, p1, p2_);
        if (next) {
          V4<T>::load(z + 4 * n, z0, z1, z2);
          p0 = z0 + be * p0; p1 = z1 + be * p1; p2_ = z2 + be * p2_;
        }
        V4<T>::store(p + 4 * n, p0, p1, p2_);
      }
    }
  }
  if (b == 0 && tid == 0) {
    st->dot0 = dot0;
    st->alpha = alpha;
    st->beta = beta;
    st->rr = rr;
    st->err = err;
    st->pw = pw;
    st->iter = iter;
    st->done = done;
  }
}

// ---------------------------------------------------------------- batched PCG
// Many independent problems held in one block-diagonal matrix (problem k owns
// the node rows [noff[k], noff[k+1]) and no block couples two problems).  A
// thread-block cluster of kBatchCluster CTAs runs PCGSolver's iteration on one
// problem: each CTA owns a contiguous share of the problem's rows; the dot
// products are summed per CTA, exchanged through distributed shared memory and
// added in rank order (the same fixed order in every CTA, so the scalars agree
// and a solve is bit-reproducible); the hardware cluster barrier separates the
// phases.  No cluster ever waits on another.  order[] lists the problems
// largest first, so the block scheduler starts the long ones early.
constexpr int kBatchThreads = 256;
constexpr int kBatchCluster = 2;  // measured: 2 -> 1.83 s, 4 -> 1.91 s, 8 -> 2.11 s on the 1024-cantilever ensemble

template <int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(kBatchThreads, 2)
pcg_batch(const int32_t *__restrict__ order, const int64_t *__restrict__ noff, const int32_t *__restrict__ srow,
          const int32_t *__restrict__ scol, const double *__restrict__ val, double *u, double *r, double *z,
          double *p, double *w, const double *__restrict__ f, const double *__restrict__ dinv, double tol,
          int maxit, int warm, int32_t *__restrict__ iters, double *__restrict__ errs,
          int32_t *__restrict__ done_out) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double sbuf[32];
  __shared__ double slots[8];   // this CTA's partial sums, rotated so a slot is rewritten only 8 sums later
  const int rank = (int)cl.block_rank();
  const int k = order[blockIdx.x / CS];
  const int64_t P0 = noff[k], P1 = noff[k + 1];
  const int64_t chunk = (P1 - P0 + CS - 1) / CS;
  const int64_t n0 = min(P1, P0 + rank * chunk), n1 = min(P1, n0 + chunk);
  const int tid = threadIdx.x, lane = tid & 31, q = lane & 15;
  int slot = 0;
  // cluster-wide fixed-order sum of one value per thread
  auto csum = [&](double v) -> double {
    const double t = block_sum<kBatchThreads>(v, sbuf);
    if (tid == 0) slots[slot] = t;
    cl.sync();
    double out = 0.0;
    for (int rr = 0; rr < CS; rr++) out += cl.map_shared_rank(slots, rr)[slot];
    slot = (slot + 1) & 7;
    return out;
  };
  // y = K x on this CTA's rows, x gathered over the problem through L2;
  // returns the cluster sum of x.y (or, with b, y = b - K x and of y.y)
  auto spmv = [&](const double *x, const double *b, double *y) -> double {
    double acc = 0.0;
    for (int64_t row0 = n0 + 2 * (tid >> 5); row0 < n1; row0 += 2 * (kBatchThreads / 32)) {
      const int64_t row = row0 + (lane >> 4);
      const bool live = row < n1;
      int32_t s0 = 0, nbp = 0;
      if (live) {
        s0 = srow[row];
        nbp = srow[row + 1] - s0;
      }
      const double *vr = val + 9 * (int64_t)s0;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int j = 2 * q; j < nbp; j += 32) {
        const int2 c = *reinterpret_cast<const int2 *>(scol + s0 + j);
        double2 v[9];
#pragma unroll
        for (int kk = 0; kk < 9; kk++) v[kk] = *reinterpret_cast<const double2 *>(vr + kk * nbp + j);
        double xa0, xa1, xa2, xb0, xb1, xb2;
        V4cg<double>::load(x + 4 * (int64_t)c.x, xa0, xa1, xa2);
        V4cg<double>::load(x + 4 * (int64_t)c.y, xb0, xb1, xb2);
        a0 += v[0].x * xa0 + v[1].x * xa1 + v[2].x * xa2 + v[0].y * xb0 + v[1].y * xb1 + v[2].y * xb2;
        a1 += v[3].x * xa0 + v[4].x * xa1 + v[5].x * xa2 + v[3].y * xb0 + v[4].y * xb1 + v[5].y * xb2;
        a2 += v[6].x * xa0 + v[7].x * xa1 + v[8].x * xa2 + v[6].y * xb0 + v[7].y * xb1 + v[8].y * xb2;
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      }
      if (live && q == 0) {
        if (b) {
          double b0, b1, b2;
          V4<double>::load(b + 4 * row, b0, b1, b2);
          a0 = b0 - a0; a1 = b1 - a1; a2 = b2 - a2;
          acc += a0 * a0 + a1 * a1 + a2 * a2;
        } else {
          double x0, x1, x2;
          V4<double>::load(x + 4 * row, x0, x1, x2);
          acc += x0 * a0 + x1 * a1 + x2 * a2;
        }
        V4<double>::store(y + 4 * row, a0, a1, a2);
      }
    }
    return csum(acc);
  };
  // |f| with the reference's normaliser
  double ff = 0.0;
  for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) {
    double f0, f1, f2;
    V4<double>::load(f + 4 * n, f0, f1, f2);
    ff += f0 * f0 + f1 * f1 + f2 * f2;
  }
  double lenf = sqrt(csum(ff));
  int it = 0, done = 0;
  double err = 0.0;
  if (lenf < tol) {
    // PCGSolver returns u = 0 at once for a load below the tolerance
    for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) V4<double>::store(u + 4 * n, 0.0, 0.0, 0.0);
    done = 1;
  } else {
    if (lenf > 1e11) lenf = 1.0;
    if (warm) {
      cl.sync();
      spmv(u, f, r);  // r = f - K u (u gathered over the problem)
    } else {
      for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) {
        double f0, f1, f2;
        V4<double>::load(f + 4 * n, f0, f1, f2);
        V4<double>::store(u + 4 * n, 0.0, 0.0, 0.0);
        V4<double>::store(r + 4 * n, f0, f1, f2);
      }
    }
    double zr = 0.0;
    for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) {
      double r0, r1, r2, z0, z1, z2;
      V4<double>::load(r + 4 * n, r0, r1, r2);
      apply_dinv(dinv + 12 * n, r0, r1, r2, z0, z1, z2);
      V4<double>::store(z + 4 * n, z0, z1, z2);
      V4<double>::store(p + 4 * n, z0, z1, z2);
      zr += z0 * r0 + z1 * r1 + z2 * r2;
    }
    double dot0 = csum(zr);  // its cluster barrier also publishes p
    while (!done && it < maxit) {
      const double pw = spmv(p, nullptr, w);
      const double alpha = dot0 / pw;
      if (!(alpha > 0.0) || !isfinite(pw) || !isfinite(alpha)) { done = 3; break; }
      double rra = 0.0, zra = 0.0;
      for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) {
        double u0, u1, u2, p0, p1, p2, r0, r1, r2, w0, w1, w2, z0, z1, z2;
        V4<double>::load(u + 4 * n, u0, u1, u2);
        V4<double>::load(p + 4 * n, p0, p1, p2);
        V4<double>::load(r + 4 * n, r0, r1, r2);
        V4<double>::load(w + 4 * n, w0, w1, w2);
        u0 += alpha * p0; u1 += alpha * p1; u2 += alpha * p2;
        r0 += (-alpha) * w0; r1 += (-alpha) * w1; r2 += (-alpha) * w2;
        apply_dinv(dinv + 12 * n, r0, r1, r2, z0, z1, z2);
        V4<double>::store(u + 4 * n, u0, u1, u2);
        V4<double>::store(r + 4 * n, r0, r1, r2);
        V4<double>::store(z + 4 * n, z0, z1, z2);
        rra += r0 * r0 + r1 * r1 + r2 * r2;
        zra += z0 * r0 + z1 * r1 + z2 * r2;
      }
      const double rr = csum(rra);
      const double zr1 = csum(zra);
      it++;
      err = sqrt(rr) / lenf;
      if (err < tol) { done = 1; break; }
      if (!isfinite(err)) { done = 3; break; }
      const double beta = zr1 / dot0;
      dot0 = zr1;
      for (int64_t n = n0 + tid; n < n1; n += kBatchThreads) {
        double p0, p1, p2, z0, z1, z2;
        V4<double>::load(p + 4 * n, p0, p1, p2);
        V4<double>::load(z + 4 * n, z0, z1, z2);
        V4<double>::store(p + 4 * n, z0 + beta * p0, z1 + beta * p1, z2 + beta * p2);
      }
      __threadfence();
      cl.sync();  // the next SpMV gathers p of the whole problem
    }
    if (!done) done = 2;
  }
  if (rank == 0 && tid == 0) {
    iters[k] = it;
    errs[k] = err;
    done_out[k] = done;
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

cudaError_t launch_pcg_batch(Ctx &c, int nprob, const int32_t *d_order, const int64_t *d_noff, double tol, int maxit,
                             bool warm, int32_t *d_iters, double *d_errs, int32_t *d_done) {
  pcg_batch<kBatchCluster><<<nprob * kBatchCluster, kBatchThreads, 0, c.stream>>>(
      d_order, d_noff, c.d_srow, c.d_scol, c.d_Ks, c.d_u, c.d_r, c.d_z, c.d_p, c.d_w, c.d_f, c.d_dinv, tol, maxit,
      warm ? 1 : 0, d_iters, d_errs, d_done);
  c.launches++;
  return cudaGetLastError();
}

// k iterations of the persistent kernel; false when the system is too large
// for it (the caller then uses the per-kernel iteration)
// (reset_barrier false: inside a graph's loop body, where the barrier words
// were reset before the loop and every completed launch leaves them reset)
template <typename T>
static cudaError_t launch_persistent(Ctx &c, const T *val, T *u, T *r, T *z, T *p, T *p2, T *w, const T *dinv,
                                     int k, bool reset_barrier = true) {
  cudaError_t e = reset_barrier ? cudaMemsetAsync(c.d_bar, 0, sizeof(GridBarrier), c.stream) : cudaSuccess;
  if (e != cudaSuccess) return e;
  int64_t nn = c.nnode;
  const int32_t *srow = c.d_srow, *scol = c.d_scol;
  PcgState *st = c.d_state;
  double *pa = c.d_partials, *pb = c.d_partials + 2048, *pc = c.d_partials + 4096;
  GridBarrier *bar = static_cast<GridBarrier *>(c.d_bar);
  // a cooperative launch (all blocks resident), also as a node of a captured graph
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(c.persist_grid);
  cfg.blockDim = dim3(kPersistThreads);
  cfg.stream = c.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, pcg_persistent<T>, nn, srow, scol, val, u, r, z, p, p2, w, dinv, st, pa, pb, pc, bar, k);
  c.launches++;
  return e;
}

// small enough, and one block of the kernel fits on every SM (sized once)
static bool use_persistent(Ctx &c) {
  if (c.nnode <= 0 || c.nnode > c.persist_max_nodes) return false;
  if (c.persist_grid == 0) {
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, pcg_persistent<double>, kPersistThreads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, pcg_persistent<float>, kPersistThreads, 0) != cudaSuccess ||
        a < 1 || b < 1) {
      cudaGetLastError();
      c.persist_max_nodes = 0;
      return false;
    }
    c.persist_grid = 1;  // sized per system below (partials: at most 2048 blocks)
  }
  {
    // one block per SM (measured faster than fewer, fuller blocks), not more than one per 32 rows
    int64_t g = (c.nnode + 31) / 32;
    if (g > c.sm_count) g = c.sm_count;
    c.persist_grid = (int)(g < 1 ? 1 : g);
  }
  return true;
}

// Pipelined host loop: launch a chunk, then look at the state copied after the
// previous chunk; returns when done or when maxit iterations were launched.
// Full chunks run as a CUDA graph captured on first use (the scalars live on
// the device, so the same graph serves every chunk and every later solve of
// this context); live kernel timing launches the kernels directly instead.
template <typename LaunchChunk>
static cudaError_t drive(Ctx &c, int maxit, int chunk, cudaGraphExec_t *graph, int *graph_chunk,
                         int64_t *graph_kernels, LaunchChunk launch_chunk) {
  cudaError_t e;
  cudaEvent_t ev;
  if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
  const bool use_graph = graph != nullptr && !c.timing;
  int launched = 0;
  bool pending = false;
  while (true) {
    const int k = (maxit - launched < chunk) ? (maxit - launched) : chunk;
    if (use_graph && k == chunk) {
      if (!*graph || *graph_chunk != chunk) {
        if (*graph) cudaGraphExecDestroy(*graph);
        *graph = nullptr;
        cudaGraph_t g = nullptr;
        const int64_t before = c.launches;
        if ((e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) break;
        cudaError_t el = launch_chunk(k);
        e = cudaStreamEndCapture(c.stream, &g);
        if (el != cudaSuccess) e = el;
        if (e == cudaSuccess) e = cudaGraphInstantiate(graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) { *graph = nullptr; break; }
        *graph_chunk = chunk;
        *graph_kernels = c.launches - before;
        c.launches = before;
      }
      if ((e = cudaGraphLaunch(*graph, c.stream)) != cudaSuccess) break;
      c.launches += *graph_kernels;
    } else {
      if ((e = launch_chunk(k)) != cudaSuccess) break;
    }
    launched += k;
    if (pending) {
      if ((e = cudaEventSynchronize(ev)) != cudaSuccess) break;
      if (c.h_state->done) break;
    }
    if ((e = cudaMemcpyAsync(c.h_state, c.d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess)
      break;
    if ((e = cudaEventRecord(ev, c.stream)) != cudaSuccess) break;
    pending = true;
    if (launched >= maxit) {
      e = cudaEventSynchronize(ev);
      break;
    }
  }
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(c.h_state, c.d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess)
    return e;
  return cudaStreamSynchronize(c.stream);
}

// ---- the two PCG paths in pieces: initialisation and one chunk of
// iterations, stream-ordered on c.stream (kernel-per-step form)

static void fp64_init(Ctx &c, bool warm, double tol, const double *tol_dev, int maxit, int iter0) {
  const int64_t nn = c.nnode;
  const int G = spmv_grid(c), R = kRedBlocks;
  PcgState *st = c.d_state;
  if (warm) {
    spmv64_go<1>(c, G, nn, c.d_Ks, c.d_u, c.d_f, c.d_r, P_E(c), nullptr);
    c.launches++;
  } else {
    cudaMemsetAsync(c.d_u, 0, sizeof(double) * 4 * nn, c.stream);
    cudaMemcpyAsync(c.d_r, c.d_f, sizeof(double) * 4 * nn, cudaMemcpyDeviceToDevice, c.stream);
  }
  pcg_precond<double><<<R, kVecThreads, 0, c.stream>>>(nn, c.d_r, c.d_z, c.d_p, c.d_dinv, c.d_f, P_C(c), P_D(c));
  pcg_init_scalar<<<1, 256, 0, c.stream>>>(st, P_C(c), R, P_D(c), R, warm ? P_E(c) : nullptr, G, tol, tol_dev, maxit,
                                           iter0);
  c.launches += 2;
}

static void fp64_chunk(Ctx &c, int k) {
  const int64_t nn = c.nnode;
  const int G = spmv_grid(c), R = kRedBlocks;
  PcgState *st = c.d_state;
  for (int i = 0; i < k; i++) {
    c.begin_span(0);
    spmv64_go<0>(c, G, nn, c.d_Ks, c.d_p, nullptr, c.d_w, P_A(c), &st->done);
    c.end_span();
    pcg_update_fused<double><<<R, kVecThreads, 0, c.stream>>>(nn, c.d_u, c.d_r, c.d_z, c.d_p, c.d_w, c.d_dinv, st,
                                                               P_A(c), G, P_B(c), P_C(c));
    pcg_direction_fused<double><<<R, kVecThreads, 0, c.stream>>>(nn, c.d_p, c.d_z, st, P_B(c), P_C(c), R);
    c.launches += 3;
  }
}

static void mixed_init(Ctx &c, bool warm, double tol, const double *tol_dev, int maxit) {
  const int64_t nn = c.nnode;
  const int R = kRedBlocks;
  if (!warm) cudaMemsetAsync(c.d_u, 0, sizeof(double) * 4 * nn, c.stream);
  cudaMemsetAsync(c.s_x, 0, sizeof(float) * 4 * nn, c.stream);
  sumsq_kernel<<<R, 256, 0, c.stream>>>(4 * nn, c.d_f, P_D(c));
  // the tensor-core stiffness may restart its recurrence (see reliable_scalar)
  mixed_init_scalar<<<1, 256, 0, c.stream>>>(c.d_state, P_D(c), R, tol, tol_dev, maxit, c.K32_current ? 40 : 0);
  c.launches += 2;
}

// mixed path: flush the FP32 correction into the FP64 solution, recompute
// r = f - K u in FP64 (from the FP64 matrix, or element by element when the
// stiffness is the tensor-core FP32 one) and restart the FP32 recurrence from it
static void mixed_reliable(Ctx &c) {
  const int64_t nn = c.nnode;
  const int G = spmv_grid(c), R = kRedBlocks;
  PcgState *st = c.d_state;
  flush_correction<<<R, 256, 0, c.stream>>>(4 * nn, c.d_u, c.s_x, st);
  if (c.K32_current) {
    launch_matfree_residual(c, c.d_f, c.d_u, c.d_r, P_E(c), &st->final);  // counts its own launches
  } else {
    c.begin_span(0);
    spmv64_go<1>(c, G, nn, c.d_Ks, c.d_u, c.d_f, c.d_r, P_E(c), &st->final);
    c.end_span();
    c.launches++;
  }
  replace_residual<<<R, kVecThreads, 0, c.stream>>>(nn, c.d_r, c.s_r, c.s_z, c.s_p, c.s_dinv, st, P_C(c));
  reliable_scalar<<<1, 256, 0, c.stream>>>(st, P_E(c), G, P_C(c), R);
  keep_best<<<R, 256, 0, c.stream>>>(4 * nn, c.d_u, c.d_ubest, st);
  c.launches += 4;
  if (c.K32_current) {
    restart_direction<<<R, 256, 0, c.stream>>>(4 * nn, c.s_z, c.s_p, st);
    c.launches++;
  }
}

static void mixed_chunk(Ctx &c, int k) {
  const int64_t nn = c.nnode;
  const int G = spmv32_grid(c), R = kRedBlocks;
  PcgState *st = c.d_state;
  for (int i = 0; i < k; i++) {
    c.begin_span(1);
    spmv32_go(c, G, nn, c.d_Ks32, c.s_p, c.s_w, P_A(c), &st->done);
    c.end_span();
    pcg_update_fused<float><<<R, kVecThreads, 0, c.stream>>>(nn, c.s_x, c.s_r, c.s_z, c.s_p, c.s_w, c.s_dinv, st,
                                                              P_A(c), spmv32_parts(c), P_B(c), P_C(c));
    pcg_direction_fused<float><<<R, kVecThreads, 0, c.stream>>>(nn, c.s_p, c.s_z, st, P_B(c), P_C(c), R);
    c.launches += 3;
  }
  mixed_reliable(c);
}

cudaError_t pcg_fp64(Ctx &c, bool warm, double tol, int maxit, int chunk, int iter0) {
  cudaError_t e;
  fp64_init(c, warm, tol, nullptr, maxit, iter0);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (use_persistent(c)) {
    const int pchunk = chunk < 64 ? 64 : chunk;  // each chunk is one launch: read the state back less often
    return drive(c, maxit, pchunk, nullptr, nullptr, nullptr, [&](int k) -> cudaError_t {
      return launch_persistent<double>(c, c.d_Ks, c.d_u, c.d_r, c.d_z, c.d_p, c.d_p2, c.d_w, c.d_dinv, k);
    });
  }
  return drive(c, maxit, chunk, &c.graph_fp64, &c.graph_fp64_chunk, &c.graph_fp64_kernels, [&](int k) -> cudaError_t {
    fp64_chunk(c, k);
    return cudaGetLastError();
  });
}

// FP32 PCG with FP64 reliable updates every `chunk` iterations.
cudaError_t pcg_mixed(Ctx &c, bool warm, double tol, int maxit, int chunk) {
  cudaError_t e;
  mixed_init(c, warm, tol, nullptr, maxit);
  mixed_reliable(c);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (use_persistent(c)) {
    return drive(c, maxit, chunk, nullptr, nullptr, nullptr, [&](int k) -> cudaError_t {
      cudaError_t el = launch_persistent<float>(c, c.d_Ks32, c.s_x, c.s_r, c.s_z, c.s_p, c.s_p2, c.s_w, c.s_dinv, k);
      if (el != cudaSuccess) return el;
      mixed_reliable(c);
      return cudaGetLastError();
    });
  }
  return drive(c, maxit, chunk, &c.graph_mixed, &c.graph_mixed_chunk, &c.graph_mixed_kernels,
               [&](int k) -> cudaError_t {
    mixed_chunk(c, k);
    return cudaGetLastError();
  });
}

// ---- a whole solve inside a CUDA graph
// keeps the WHILE node looping while the iteration runs (done == 0)
__global__ void pcg_loop_cond(cudaGraphConditionalHandle h, const PcgState *__restrict__ st) {
  cudaGraphSetConditional(h, st->done == 0 ? 1u : 0u);
}

cudaError_t record_pcg(Ctx &c, bool mixed, bool warm, double tol, const double *tol_dev, int maxit, int chunk) {
  cudaError_t e;
  if (mixed) {
    mixed_init(c, warm, tol, tol_dev, maxit);
    mixed_reliable(c);
  } else {
    fp64_init(c, warm, tol, tol_dev, maxit, 0);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // small systems iterate in the persistent cooperative kernel (as the
  // launched solves do), a chunk per loop pass; its barrier words reset once
  const bool persist = use_persistent(c);
  if (persist && (e = cudaMemsetAsync(c.d_bar, 0, sizeof(GridBarrier), c.stream)) != cudaSuccess) return e;
  // the WHILE node, appended to the graph being captured on c.stream
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  if ((e = cudaStreamGetCaptureInfo(c.stream, &cs, nullptr, &g, &deps, &ndeps)) != cudaSuccess) return e;
  if (cs != cudaStreamCaptureStatusActive || !g) return cudaErrorStreamCaptureUnmatched;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, g, deps, ndeps, &np)) != cudaSuccess) return e;
  if ((e = cudaStreamUpdateCaptureDependencies(c.stream, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return e;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  // the loop body: one chunk and the condition, captured on the side stream
  if (!c.side_stream && (e = cudaStreamCreateWithFlags(&c.side_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return e;
  cudaStream_t main = c.stream;
  c.stream = c.side_stream;
  e = cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t el = cudaSuccess;
    if (persist && mixed) {
      el = launch_persistent<float>(c, c.d_Ks32, c.s_x, c.s_r, c.s_z, c.s_p, c.s_p2, c.s_w, c.s_dinv, chunk, false);
      mixed_reliable(c);
    } else if (persist) {
      el = launch_persistent<double>(c, c.d_Ks, c.d_u, c.d_r, c.d_z, c.d_p, c.d_p2, c.d_w, c.d_dinv,
                                     chunk < 64 ? 64 : chunk, false);
    } else if (mixed) {
      mixed_chunk(c, chunk);
    } else {
      fp64_chunk(c, chunk);
    }
    if (el != cudaSuccess) (void)cudaGetLastError();
    pcg_loop_cond<<<1, 1, 0, c.stream>>>(h, c.d_state);
    c.launches++;
    if (el == cudaSuccess) el = cudaGetLastError();
    e = cudaStreamEndCapture(c.stream, &body);
    if (e == cudaSuccess) e = el;
  }
  c.stream = main;
  return e;
}

}  // namespace fastgpu

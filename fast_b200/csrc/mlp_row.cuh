// mlp_row.cuh - one input row through the tanh MLP of learned.h on the CUDA
// cores, by one CTA.  The arithmetic is the tensor-core forward's (operands
// rounded to BF16, products exact in FP32, FP32 sums, bias then tanh on the
// hidden layers); only the order of the sums differs: each output is summed
// by one warp, lane-strided over the inputs, then across the lanes by a fixed
// butterfly, so the result is the same on every run.
//
// A single load-step prediction feeds one row through the network; the
// tensor-core GEMM pads that row to a 128-row tile per layer and launches
// once per layer, while this form runs all layers in the CTA that produced
// the input, with the activations in shared memory and the weights read once
// from L2.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>

namespace fastgpu {

constexpr int kMlpRowMaxLayers = 9;
constexpr int kMlpRowMaxDim = 1025;  // 1 + history 16 x 64 modes; hidden width <= 1024
constexpr int kMlpRowUnroll = 8;     // inputs per lane per trip

// layer sizes and parameter offsets (layer l: W_l [dims[l+1]][dims[l]]
// row-major at w_off[l], b_l at b_off[l])
struct MlpRow {
  int L;
  int dims[kMlpRowMaxLayers + 1];
  int64_t w_off[kMlpRowMaxLayers], b_off[kMlpRowMaxLayers];
};

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// in: the input row in shared memory, already rounded to BF16 values; tmp:
// shared scratch of the widest layer; y (global): the network output.
// Every thread of the block calls it; blockDim.x is a multiple of 32.
__device__ inline void mlp_row_forward(const MlpRow &m, const float *__restrict__ P, float *in, float *tmp,
                                       float *__restrict__ y) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float *a = in, *b = tmp;
  for (int l = 0; l < m.L; l++) {
    const int fi = m.dims[l], fo = m.dims[l + 1];
    const bool last = l + 1 == m.L;
    const float *W = P + m.w_off[l];
    const float *bias = P + m.b_off[l];
    for (int j0 = 4 * warp; j0 < fo; j0 += 4 * nw) {
      // four outputs per warp at a time, eight inputs per lane per trip: all
      // 32 weight loads of a trip are in flight together (L2 latency, not
      // bandwidth, bounds one CTA); the sums run over k in increasing order
      const float *w0 = W + (int64_t)j0 * fi;
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      const int nr = min(4, fo - j0);
      for (int k0 = 0; k0 < fi; k0 += 32 * kMlpRowUnroll) {
        float wv[4][kMlpRowUnroll], xv[kMlpRowUnroll];
#pragma unroll
        for (int u = 0; u < kMlpRowUnroll; u++) {
          const int k = k0 + 32 * u + lane;
          const bool in = k < fi;
          xv[u] = in ? a[k] : 0.f;
#pragma unroll
          for (int r = 0; r < 4; r++) wv[r][u] = (in && r < nr) ? __ldg(w0 + (int64_t)r * fi + k) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kMlpRowUnroll; u++)
#pragma unroll
          for (int r = 0; r < 4; r++) acc[r] = fmaf(bf16_round(wv[r][u]), xv[u], acc[r]);
      }
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], s);
      if (lane < nr) {
        float v = acc[0];
#pragma unroll
        for (int r = 1; r < 4; r++)
          if (lane == r) v = acc[r];
        v += bias[j0 + lane];
        if (last) {
          y[j0 + lane] = v;
        } else {
          b[j0 + lane] = bf16_round(tanhf(v));
        }
      }
    }
    __syncthreads();
    float *t = a;
    a = b;
    b = t;
  }
}

}  // namespace fastgpu

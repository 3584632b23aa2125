// pod.cu - FP64 dense kernels for the proper orthogonal decomposition (POD)
// of converged displacement snapshots, and a small symmetric eigen-solver.
//
// The POD basis is found by a randomized range finder with power iterations
// (Halko, Martinsson & Tropp, SIAM Review 53 (2011), Alg. 4.4) over the
// snapshot matrix S (n equations x m snapshots), so the only large products
// are S Omega and S^T Q with a thin right-hand side: dgemm below, split over
// K for the long reductions.  The small l x l symmetric eigenproblems are
// solved on the host by cyclic Jacobi rotations (Golub & Van Loan, Matrix
// Computations, 4th ed., Alg. 8.5.3).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "internal.h"
#include "learned.h"

namespace fastgpu {

namespace {

constexpr int kT = 64;     // output tile
constexpr int kKB = 16;    // K per shared-memory step
constexpr int kKSlice = 2048;  // K per split

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) dgemm_tile(int M, int N, int K, int kslice, const double *__restrict__ A,
                                                  int lda, const double *__restrict__ B, int ldb,
                                                  double *__restrict__ C, int ldc, double *__restrict__ ws) {
  __shared__ double As[kKB][kT + 1];
  __shared__ double Bs[kKB][kT + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * kT, n0 = blockIdx.y * kT;
  const int kbeg = blockIdx.z * kslice, kend = min(K, kbeg + kslice);
  double acc[4][4] = {};
  for (int k0 = kbeg; k0 < kend; k0 += kKB) {
    for (int u = tid; u < kT * kKB; u += 256) {
      // coalesced along whichever index is contiguous in memory
      int mm, kk;
      if (TA) { mm = u % kT; kk = u / kT; } else { kk = u % kKB; mm = u / kKB; }
      const int gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < kend) ? (TA ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk]) : 0.0;
      int nn, k2;
      if (TB) { k2 = u % kKB; nn = u / kKB; } else { nn = u % kT; k2 = u / kT; }
      const int gn = n0 + nn, gk2 = k0 + k2;
      Bs[k2][nn] = (gn < N && gk2 < kend) ? (TB ? B[(int64_t)gn * ldb + gk2] : B[(int64_t)gk2 * ldb + gn]) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kKB; k++) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[k][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  for (int i = 0; i < 4; i++) {
    const int gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
    for (int j = 0; j < 4; j++) {
      const int gn = n0 + tx * 4 + j;
      if (gn >= N) continue;
      if (gridDim.z == 1)
        C[(int64_t)gm * ldc + gn] = acc[i][j];
      else
        ws[((int64_t)blockIdx.z * M + gm) * N + gn] = acc[i][j];
    }
  }
}

// C[m][n] = sum over splits in order
__global__ void dgemm_reduce(int M, int N, int splits, const double *__restrict__ ws, double *__restrict__ C,
                             int ldc) {
  const int64_t mn = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < mn; i += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int z = 0; z < splits; z++) t += ws[z * mn + i];
    C[(i / N) * ldc + (i % N)] = t;
  }
}

}  // namespace

// Per-block partial sums of C[a][b] = sum_i A[i lda + a] B[i ldb + b]: with
// few outputs the block's threads split the rows into groups (combined in
// shared memory in a fixed order); with many, each thread owns outputs.
template <int NT>
__global__ void __launch_bounds__(NT) skinny_atb_part(int64_t n, int p, int q, const double *__restrict__ A, int lda,
                                                      const double *__restrict__ B, int ldb,
                                                      double *__restrict__ part) {
  __shared__ double red[NT];
  const int pq = p * q, tid = threadIdx.x;
  if (pq <= NT) {
    const int groups = NT / pq;
    const int o = tid % pq, g = tid / pq;
    double acc = 0.0;
    if (g < groups) {
      const int a = o / q, b = o % q;
      for (int64_t i = (int64_t)blockIdx.x * groups + g; i < n; i += (int64_t)gridDim.x * groups)
        acc = fma(A[i * lda + a], B[i * ldb + b], acc);
    }
    red[tid] = acc;
    __syncthreads();
    if (tid < pq) {
      double t = 0.0;
      for (int gg = 0; gg < groups; gg++) t += red[gg * pq + tid];
      part[(int64_t)blockIdx.x * pq + tid] = t;
    }
  } else {
    for (int o = tid; o < pq; o += NT) {
      const int a = o / q, b = o % q;
      double acc = 0.0;
      for (int64_t i = blockIdx.x; i < n; i += gridDim.x) acc = fma(A[i * lda + a], B[i * ldb + b], acc);
      part[(int64_t)blockIdx.x * pq + o] = acc;
    }
  }
}

// The same partial sums for many outputs (p q > NT, p, q <= 64): each block
// takes a contiguous range of rows in tiles of TR rows staged in shared
// memory (coalesced row loads), and each thread keeps up to kMaxOut / NT
// outputs in registers, summing its tile rows in order.
constexpr int kTiledMaxCols = 64;
template <int NT, int TR>
__global__ void __launch_bounds__(NT) skinny_atb_tiled(int64_t n, int p, int q, const double *__restrict__ A, int lda,
                                                       const double *__restrict__ B, int ldb,
                                                       double *__restrict__ part) {
  constexpr int MO = kSkinnyMaxOut / NT;
  __shared__ double As[TR][kTiledMaxCols], Bs[TR][kTiledMaxCols];
  const int pq = p * q, tid = threadIdx.x;
  double acc[MO];
#pragma unroll
  for (int m = 0; m < MO; m++) acc[m] = 0.0;
  const int64_t r0 = n * blockIdx.x / gridDim.x, r1 = n * (blockIdx.x + 1) / gridDim.x;
  for (int64_t t0 = r0; t0 < r1; t0 += TR) {
    const int nr = (int)(r1 - t0 < TR ? r1 - t0 : TR);
    for (int e = tid; e < nr * p; e += NT) {
      const int r = e / p, c = e - r * p;
      As[r][c] = A[(t0 + r) * lda + c];
    }
    for (int e = tid; e < nr * q; e += NT) {
      const int r = e / q, c = e - r * q;
      Bs[r][c] = B[(t0 + r) * ldb + c];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < MO; m++) {
      const int o = tid + m * NT;
      if (o < pq) {
        const int a = o / q, b = o - a * q;
        double t = acc[m];
        for (int r = 0; r < nr; r++) t = fma(As[r][a], Bs[r][b], t);
        acc[m] = t;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int m = 0; m < MO; m++) {
    const int o = tid + m * NT;
    if (o < pq) part[(int64_t)blockIdx.x * pq + o] = acc[m];
  }
}

// one warp per output entry: lane l sums the partials l, l+32, ... in order,
// then a fixed butterfly combines the lanes (deterministic)
__global__ void skinny_finish(int nblk, int p, int q, const double *__restrict__ part, double *__restrict__ C,
                              int ldc) {
  const int pq = p * q;
  const int lane = threadIdx.x & 31;
  const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (o >= pq) return;
  double t = 0.0;
  for (int b = lane; b < nblk; b += 32) t += part[(int64_t)b * pq + o];
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) t += __shfl_xor_sync(0xffffffffu, t, m);
  if (lane == 0) C[(int64_t)(o / q) * ldc + o % q] = t;
}

cudaError_t skinny_atb(cudaStream_t s, int64_t n, int p, int q, const double *A, int lda, const double *B, int ldb,
                       double *C, int ldc, double *ws) {
  if (n <= 0 || p <= 0 || q <= 0 || p * q > kSkinnyMaxOut || !ws) return cudaErrorInvalidValue;
  if (p * q > 256 && p <= kTiledMaxCols && q <= kTiledMaxCols)
    skinny_atb_tiled<256, 32><<<kSkinnyBlocks, 256, 0, s>>>(n, p, q, A, lda, B, ldb, ws);
  else
    skinny_atb_part<256><<<kSkinnyBlocks, 256, 0, s>>>(n, p, q, A, lda, B, ldb, ws);
  skinny_finish<<<(p * q + 7) / 8, 256, 0, s>>>(kSkinnyBlocks, p, q, ws, C, ldc);
  return cudaGetLastError();
}

int dgemm_splits(int M, int N, int K) {
  const int tiles = ((M + kT - 1) / kT) * ((N + kT - 1) / kT);
  if (tiles >= 148) return 1;
  return std::max(1, std::min((K + kKSlice - 1) / kKSlice, 296 / tiles));
}

cudaError_t dgemm(cudaStream_t s, int M, int N, int K, const double *A, int lda, bool ta, const double *B, int ldb,
                  bool tb, double *C, int ldc, double *ws) {
  if (M <= 0 || N <= 0 || K <= 0) return cudaErrorInvalidValue;
  const int splits = dgemm_splits(M, N, K);
  const int kslice = ((K + splits - 1) / splits + kKB - 1) / kKB * kKB;
  const int z = (K + kslice - 1) / kslice;
  dim3 grid((M + kT - 1) / kT, (N + kT - 1) / kT, z);
  if (z > 1 && !ws) return cudaErrorInvalidValue;
#define DG(TA_, TB_) dgemm_tile<TA_, TB_><<<grid, 256, 0, s>>>(M, N, K, kslice, A, lda, B, ldb, C, ldc, ws)
  if (!ta && !tb) DG(false, false);
  else if (!ta && tb) DG(false, true);
  else if (ta && !tb) DG(true, false);
  else DG(true, true);
#undef DG
  if (z > 1) dgemm_reduce<<<std::min<int64_t>(592, ((int64_t)M * N + 255) / 256), 256, 0, s>>>(M, N, z, ws, C, ldc);
  return cudaGetLastError();
}

void sym_eig(int n, std::vector<double> a, std::vector<double> &w, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  auto A = [&](int i, int j) -> double & { return a[(size_t)i * n + j]; };
  double total = 0.0;
  for (double x : a) total += x * x;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) off += A(i, j) * A(i, j);
    if (off <= 1e-30 * total || off == 0.0) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = A(p, q);
        if (apq == 0.0) continue;
        // rotation that zeroes A(p, q)
        const double tau = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; k++) {  // A <- A J (columns p, q)
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {  // A <- J^T A (rows p, q)
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - s * vkq;
          V[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A(x, x) > A(y, y); });
  std::vector<double> Vs((size_t)n * n);
  w.assign(n, 0.0);
  for (int j = 0; j < n; j++) {
    w[j] = A(order[j], order[j]);
    for (int k = 0; k < n; k++) Vs[(size_t)k * n + j] = V[(size_t)k * n + order[j]];
  }
  V.swap(Vs);
}

}  // namespace fastgpu

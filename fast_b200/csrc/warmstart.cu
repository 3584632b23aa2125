// warmstart.cu - the learned load-step predictor (fast_gpu_ws_* and
// fast_gpu_mlp_* in include/fast_gpu.h).  No counterpart in the reference:
// cCtrlNR::Solver (ctrl/ctrlnr.cpp:47-270) starts every load step from the
// last converged displacements.
//
// Training data are whole load-control trajectories (the converged u of every
// step).  Their POD basis Phi comes from a randomized range finder over the
// snapshot matrix in FP64 on the device; the POD coefficients a_s = Phi^T u_s
// of every snapshot then give one training sample per step s >= 2:
//   x = [lambda_s, a_{s-1}/sigma, da_{s-1}/delta, ..., da_{s-H+1}/delta]
//   t = (da_s - rho da_{s-1}) / tau          da_j = a_j - a_{j-1},  a_j = 0 for j <= 0,
//                                            rho = dlambda_s / dlambda_{s-1}
// i.e. the last H coefficient sets, given as the latest set and its H-1
// backward differences (each scaled by its own per-mode RMS, so that the BF16
// inputs keep the increments' digits), and as target what the secant
// increment misses inside the basis.  Prediction adds that correction to the
// secant start; the Newton driver accepts it only when its residual is below
// the secant start's.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "learned.h"
#include "mlp_row.cuh"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

// Phi_node[4 n + i][m] = Phi[eq][m] for the equation eq of DOF i of node n
__global__ void ws_phi_to_node(int32_t neq, int k, const int32_t *__restrict__ dof, const double *__restrict__ phi,
                               double *__restrict__ phin) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)neq * k) return;
  const int64_t e = t / k;
  const int m = (int)(t % k);
  phin[(int64_t)dof[e] * k + m] = phi[t];
}

// Y = K Phi_node with the assembled node-block matrix (AoS row-major 3x3
// blocks, full pattern): one thread per (node row, mode); rows node-padded
__global__ void ws_block_spmm(int64_t nnode, int k, const int32_t *__restrict__ rowptr,
                              const int32_t *__restrict__ col, const double *__restrict__ K,
                              const double *__restrict__ phin, double *__restrict__ Y) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nnode * k) return;
  const int64_t i = t / k;
  const int m = (int)(t % k);
  double y0 = 0.0, y1 = 0.0, y2 = 0.0;
  const int32_t b0 = rowptr[i], b1 = rowptr[i + 1];
#pragma unroll 4
  for (int32_t b = b0; b < b1; b++) {
    const double *v = K + 9 * (int64_t)b;
    const int64_t j = col[b];
    const double x0 = phin[(4 * j + 0) * k + m], x1 = phin[(4 * j + 1) * k + m], x2 = phin[(4 * j + 2) * k + m];
    y0 += v[0] * x0 + v[1] * x1 + v[2] * x2;
    y1 += v[3] * x0 + v[4] * x1 + v[5] * x2;
    y2 += v[6] * x0 + v[7] * x1 + v[8] * x2;
  }
  Y[(4 * i + 0) * k + m] = y0;
  Y[(4 * i + 1) * k + m] = y1;
  Y[(4 * i + 2) * k + m] = y2;
  Y[(4 * i + 3) * k + m] = 0.0;
}

// network input from the coefficient ring: slot[j] holds a_{s-j} (-1: zero)
struct FeatArgs {
  int k, kk, H;
  double lambda;
  int slot[18];
};

// input t of the network; the ring slot cur_slot is read from cur (shared
// memory: the coefficients this block has just formed)
__device__ float ws_feature(const FeatArgs &a, int t, const double *ring, int cur_slot, const double *cur,
                            const double *__restrict__ sigma, const double *__restrict__ delta) {
  if (t == 0) return (float)a.lambda;
  const int h = (t - 1) / a.kk, j = (t - 1) % a.kk;
  if (j >= a.k) return 0.f;
  auto coef = [&](int sl) -> double {
    if (sl < 0) return 0.0;
    return sl == cur_slot ? cur[j] : __ldcg(ring + sl * 64 + j);
  };
  // block 0: a_{s-1} / sigma;  block h >= 1: (a_{s-h} - a_{s-h-1}) / delta
  const double p = coef(a.slot[h == 0 ? 1 : h]);
  if (h == 0) return (float)(p / sigma[j]);
  return (float)((p - coef(a.slot[h + 1])) / delta[j]);
}

// what the last block of ws_project needs for the network step
struct NetArgs {
  FeatArgs f;
  MlpRow m;
  int cur_slot;
  const float *params;
  const double *ring, *sigma, *delta;
  float *x;  // network input (kept for fast_gpu_ws_last_input)
  float *y;  // network output
};

constexpr int kProjBlocks = 148, kProjThreads = 256;

// out[m] = sum_i (a[i] - b[i]) Phi[i][m] for m < k (b may be null), Phi
// [n][k] row-major.  A warp takes one row at a time (lane = mode), each block
// a fixed set of rows; the last block to finish adds the block partials in
// block order, so the sums do not depend on which block that is.  With
// with_net that block goes on to build the network input from out and the
// coefficient ring and runs the network (mlp_row.cuh).  The ticket is back
// at 0 when the kernel ends.
__global__ void __launch_bounds__(kProjThreads) ws_project(int32_t n, int k, const double *__restrict__ a,
                                                           const double *__restrict__ b, const double *__restrict__ phi,
                                                           double *part, unsigned int *ticket, double *out,
                                                           int with_net, NetArgs na) {
  constexpr int NW = kProjThreads / 32;
  __shared__ double red[NW][64];
  __shared__ double cur[64];
  __shared__ float xin[kMlpRowMaxDim], tmp[kMlpRowMaxDim];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
  for (int64_t r = (int64_t)blockIdx.x * NW + warp; r < n; r += (int64_t)gridDim.x * NW) {
    const double v = b ? a[r] - b[r] : a[r];
    const double *pr = phi + r * k;
    if (lane < k) s0 = fma(v, pr[lane], s0);
    if (lane + 32 < k) s1 = fma(v, pr[lane + 32], s1);
  }
  red[warp][lane] = s0;
  red[warp][lane + 32] = s1;
  __syncthreads();
  if (threadIdx.x < k) {
    double t = 0.0;
    for (int w = 0; w < NW; w++) t += red[w][threadIdx.x];
    part[blockIdx.x * 64 + threadIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < k) {
    double t = 0.0;
    for (unsigned g = 0; g < gridDim.x; g++) t += __ldcg(part + g * 64 + threadIdx.x);
    cur[threadIdx.x] = t;
    out[threadIdx.x] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  if (!with_net) return;
  __syncthreads();
  const int nin = 1 + na.f.H * na.f.kk;
  for (int t = threadIdx.x; t < nin; t += blockDim.x) {
    const float v = ws_feature(na.f, t, na.ring, na.cur_slot, cur, na.sigma, na.delta);
    na.x[t] = v;
    xin[t] = bf16_round(v);
  }
  __syncthreads();
  mlp_row_forward(na.m, na.params, xin, tmp, na.y);
}

// start = u_last + rho (u_last - u_prev) + Phi (tau * y)   (y: network output, or none)
__global__ void ws_start(int32_t n, int k, double rho, const double *__restrict__ ul, const double *__restrict__ up,
                         const double *__restrict__ phi, const double *__restrict__ tau, const float *__restrict__ y,
                         double *__restrict__ out) {
  __shared__ double cf[64];
  if (threadIdx.x < k) cf[threadIdx.x] = y ? tau[threadIdx.x] * (double)y[threadIdx.x] : 0.0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double t = ul[i] + rho * (ul[i] - up[i]);
    if (y)
      for (int m = 0; m < k; m++) t += phi[i * k + m] * cf[m];
    out[i] = t;
  }
}

// Cholesky factor L of the (symmetrised) reduced tangent, one block; ok = 0
// when a pivot is not positive
__global__ void ws_chol(int k, const double *__restrict__ E, double *__restrict__ L, int32_t *__restrict__ ok) {
  __shared__ double A[64][65];
  __shared__ int bad;
  __shared__ double dmax;
  for (int t = threadIdx.x; t < k * k; t += blockDim.x) {
    const int i = t / k, j = t % k;
    A[i][j] = 0.5 * (E[i * k + j] + E[j * k + i]);
  }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < k; i++) m = fmax(m, fabs(A[i][i]));
    dmax = m;
  }
  __syncthreads();
  for (int j = 0; j < k; j++) {
    if (threadIdx.x == 0) {
      double d = A[j][j];
      for (int p = 0; p < j; p++) d -= A[j][p] * A[j][p];
      if (!(d > 1e-14 * dmax)) { bad = 1; d = 1.0; }
      A[j][j] = sqrt(d);
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) {
      double v = A[i][j];
      for (int p = 0; p < j; p++) v -= A[i][p] * A[j][p];
      A[i][j] = v / A[j][j];
    }
    __syncthreads();
  }
  __syncthreads();
  // the factor L (lower triangle, row-major); the reduced solves run two
  // triangular solves on it
  for (int t = threadIdx.x; t < k * k; t += blockDim.x) {
    const int i = t / k, j = t % k;
    L[t] = j <= i ? A[i][j] : 0.0;
  }
  if (threadIdx.x == 0) *ok = bad ? 0 : 1;
}

// da = (L L^T)^-1 t (L from ws_chol), or 0 when the factor failed or |t| <=
// tol |tf|, then u += Phi da.  Every block forms da itself (its first warp:
// a forward and a backward substitution, each row's sum split over the lanes
// and combined by a fixed butterfly); block 0 also stores it.
__global__ void ws_reduced_add(int32_t n, int k, const double *__restrict__ L, const int32_t *__restrict__ ok,
                               const double *__restrict__ t, const double *__restrict__ tf, double tol,
                               const double *__restrict__ phi, double *__restrict__ u, double *__restrict__ da_out) {
  __shared__ double da[64], y[64], ts[64], Ls[64 * 64];
  // the factor and t into shared memory first (all threads, coalesced): the
  // two substitutions below are chains of k dependent steps each
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) Ls[e] = L[e];
  if (threadIdx.x < k) ts[threadIdx.x] = t[threadIdx.x];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double tn = 0.0, fn = 0.0;
    for (int j = lane; j < k; j += 32) { tn += t[j] * t[j]; fn += tf[j] * tf[j]; }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
      tn += __shfl_xor_sync(0xffffffffu, tn, m);
      fn += __shfl_xor_sync(0xffffffffu, fn, m);
    }
    const bool skip = !*ok || !(sqrt(tn) > tol * sqrt(fn));
    if (skip) {
      for (int i = lane; i < k; i += 32) da[i] = 0.0;
    } else {
      // L y = t
      for (int i = 0; i < k; i++) {
        double s = 0.0;
        for (int p = lane; p < i; p += 32) s += Ls[i * k + p] * y[p];
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        if (lane == 0) y[i] = (ts[i] - s) / Ls[i * k + i];
        __syncwarp();
      }
      // L^T da = y
      for (int i = k - 1; i >= 0; i--) {
        double s = 0.0;
        for (int p = i + 1 + lane; p < k; p += 32) s += Ls[p * k + i] * da[p];
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        if (lane == 0) da[i] = (y[i] - s) / Ls[i * k + i];
        __syncwarp();
      }
    }
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < k) da_out[threadIdx.x] = da[threadIdx.x];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int m = 0; m < k; m++) v += phi[i * k + m] * da[m];
    u[i] += v;
  }
}

uint64_t mix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double gauss(uint64_t &st) {  // Box-Muller
  const double u1 = ((mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

}  // namespace

struct fast_gpu_ws {
  Ctx *c = nullptr;
  fast_gpu_ws_opts o{};
  int32_t n = 0;
  // training trajectories (device snapshots, host load factors)
  std::vector<double *> traj;
  std::vector<std::vector<double>> lam;
  // POD
  int k = 0;
  double *d_phi = nullptr;       // [n][k]
  double energy = 0.0;
  std::vector<double> sigma, delta, tau;   // per-mode scales of a, da and the target
  // network
  Mlp net;
  bool trained = false;
  int in_dim = 0;
  std::vector<float> hx, ht;     // scaled samples
  int samples = 0, epochs = 0;
  float first_loss = 0.f, last_loss = 0.f;
  double basis_ms = 0.0, train_ms = 0.0;
  int64_t launches = 0;
  // dgemm split workspace and prediction scratch
  double *d_ws = nullptr;
  size_t ws_cap = 0;
  double *d_coef = nullptr;      // [2][64]: Phi^T r, Phi^T f
  double *d_delta = nullptr;     // [64] reduced correction
  int last_step = 0;             // step of the last prediction (a smaller one starts a new solve)
  // POD coefficients of recent converged steps (device ring), by step
  static constexpr int kRing = 18;
  double *d_ring = nullptr;      // [kRing][64]
  int ring_step[kRing];
  double *d_scales = nullptr;    // [3][64] sigma, delta, tau
  // Galerkin refinement of the start in the basis
  int use_network = 1, gal_iters = 0;
  double gal_tol = 1e-3;
  double *d_phin = nullptr;      // [nnode*4][k] basis in the node-padded layout
  double *d_Y = nullptr;         // [nnode*4][k] K Phi
  double *d_Er = nullptr;        // [64*64] Phi^T K Phi
  double *d_L = nullptr;         // [64*64] its Cholesky factor (lower, row-major)
  int32_t *d_ok = nullptr;
  double *d_g = nullptr;         // [n] internal force of the refined start
  unsigned int *d_ticket = nullptr;       // finishing-block counter of ws_project
  double *d_skinny = nullptr;    // [kSkinnyBlocks][kSkinnyMaxOut] partials of the skinny products
  int64_t n_pred = 0, n_gal = 0;
  double pred_ms = 0.0;

  bool fail(const std::string &m) { c->err = "ws: " + m; return false; }
  cudaError_t ensure_ws(int M, int N, int K) {
    const int s = dgemm_splits(M, N, K);
    const size_t need = s > 1 ? (size_t)s * M * N : 0;
    if (need <= ws_cap) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return e;
    if (d_ws) cudaFree(d_ws);
    d_ws = nullptr;
    ws_cap = 0;
    e = cudaMalloc((void **)&d_ws, sizeof(double) * need);
    if (e == cudaSuccess) ws_cap = need;
    return e;
  }
  cudaError_t gemm(int M, int N, int K, const double *A, int lda, bool ta, const double *B, int ldb, bool tb,
                   double *C, int ldc) {
    cudaError_t e = ensure_ws(M, N, K);
    if (e != cudaSuccess) return e;
    launches += dgemm_splits(M, N, K) > 1 ? 2 : 1;
    return dgemm(c->stream, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, d_ws);
  }
  // out = Phi^T (a - b) (b may be null), one launch; with na the network
  // step follows in the same launch
  cudaError_t project(const double *a, const double *b, double *out, const NetArgs *na) {
    launches++;
    ws_project<<<kProjBlocks, kProjThreads, 0, c->stream>>>(n, k, a, b, d_phi, d_skinny, d_ticket, out,
                                                            na ? 1 : 0, na ? *na : NetArgs{});
    return cudaGetLastError();
  }
  cudaError_t atb(int64_t rows, int p, int q, const double *A, int lda, const double *B, int ldb, double *C,
                  int ldc) {
    launches += 2;
    return skinny_atb(c->stream, rows, p, q, A, lda, B, ldb, C, ldc, d_skinny);
  }
  // Q = Y V_r Lambda_r^{-1/2} from the eigenpairs of Y^T Y (rank-revealing
  // orthonormalisation of the rows x l matrix Y); returns the rank r
  int orth(int rows, int l, double *Y, double *Q, cudaError_t &e);
};

int fast_gpu_ws::orth(int rows, int l, double *Y, double *Q, cudaError_t &e) {
  double *d_g = nullptr, *d_t = nullptr;
  std::vector<double> G((size_t)l * l), w, V;
  int r = 0;
  e = cudaMalloc((void **)&d_g, sizeof(double) * l * l);
  if (e == cudaSuccess) e = gemm(l, l, rows, Y, l, true, Y, l, false, d_g, l);
  if (e == cudaSuccess) e = cudaMemcpyAsync(G.data(), d_g, sizeof(double) * l * l, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) {
    sym_eig(l, G, w, V);
    const double wmax = w.empty() ? 0.0 : w[0];
    while (r < l && w[r] > 1e-24 * wmax && w[r] > 0.0) r++;
    std::vector<double> T((size_t)l * std::max(r, 1), 0.0);
    for (int i = 0; i < l; i++)
      for (int j = 0; j < r; j++) T[(size_t)i * r + j] = V[(size_t)i * l + j] / std::sqrt(w[j]);
    if (r > 0) {
      e = cudaMalloc((void **)&d_t, sizeof(double) * l * r);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_t, T.data(), sizeof(double) * l * r, cudaMemcpyHostToDevice, c->stream);
      if (e == cudaSuccess) e = gemm(rows, r, l, Y, l, false, d_t, r, false, Q, r);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
  }
  if (d_g) cudaFree(d_g);
  if (d_t) cudaFree(d_t);
  return r;
}

#define WCK(call)                                                          \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      w->c->err = std::string("ws: ") + #call + ": " + cudaGetErrorString(_e); \
      return FAST_GPU_ECUDA;                                               \
    }                                                                      \
  } while (0)

extern "C" int fast_gpu_ws_create(fast_gpu_ctx *ctx, const fast_gpu_ws_opts *opts, fast_gpu_ws **out) {
  if (!ctx || !opts || !out) return FAST_GPU_EINVAL;
  *out = nullptr;
  if (ctx->neq <= 0) { ctx->err = "ws_create: no mesh"; return FAST_GPU_ESTATE; }
  if (opts->modes <= 0 || opts->modes > 64 || opts->history <= 0 || opts->history > 16 || opts->width <= 0 ||
      opts->width > 1024 || opts->hidden <= 0 || opts->hidden > 8 || opts->oversample < 0 || opts->power_iters < 0) {
    ctx->err = "ws_create: options out of range (modes 1..64, history 1..16, width 1..1024, hidden 1..8)";
    return FAST_GPU_EINVAL;
  }
  fast_gpu_ws *w = new (std::nothrow) fast_gpu_ws;
  if (!w) return FAST_GPU_ENOMEM;
  w->c = ctx;
  w->o = *opts;
  w->n = ctx->neq;
  w->in_dim = 1 + opts->history * opts->modes;
  std::vector<int> dims{w->in_dim};
  for (int i = 0; i < opts->hidden; i++) dims.push_back(opts->width);
  dims.push_back(opts->modes);
  cudaError_t e = w->net.init(dims, opts->seed);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_coef, sizeof(double) * 2 * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_delta, sizeof(double) * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_ring, sizeof(double) * fast_gpu_ws::kRing * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_scales, sizeof(double) * 3 * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_Er, sizeof(double) * 64 * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_L, sizeof(double) * 64 * 64);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_ok, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_g, sizeof(double) * (size_t)w->n);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_skinny, sizeof(double) * kSkinnyBlocks * kSkinnyMaxOut);
  if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_ticket, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(w->d_ticket, 0, sizeof(unsigned int));
  for (int i = 0; i < fast_gpu_ws::kRing; i++) w->ring_step[i] = -1;
  if (e != cudaSuccess) {
    ctx->err = std::string("ws_create: ") + cudaGetErrorString(e);
    fast_gpu_ws_destroy(w);
    return FAST_GPU_ENOMEM;
  }
  *out = w;
  return FAST_GPU_OK;
}

extern "C" void fast_gpu_ws_destroy(fast_gpu_ws *w) {
  if (!w) return;
  if (w->c) cudaStreamSynchronize(w->c->stream);
  for (double *p : w->traj) cudaFree(p);
  for (double *p : {w->d_phi, w->d_ws, w->d_coef, w->d_delta, w->d_ring, w->d_scales, w->d_phin, w->d_Y, w->d_Er,
                    w->d_L, w->d_g, w->d_skinny})
    if (p) cudaFree(p);
  if (w->d_ok) cudaFree(w->d_ok);
  if (w->d_ticket) cudaFree(w->d_ticket);
  w->net.release();
  delete w;
}

extern "C" int fast_gpu_ws_add_trajectory(fast_gpu_ws *w, int32_t steps, const double *lambda,
                                          const double *u_steps) {
  if (!w || steps <= 0 || !lambda || !u_steps) return FAST_GPU_EINVAL;
  double *d = nullptr;
  const size_t bytes = sizeof(double) * (size_t)steps * w->n;
  WCK(cudaMalloc((void **)&d, bytes));
  cudaError_t e = cudaMemcpy(d, u_steps, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    w->c->err = std::string("ws_add_trajectory: ") + cudaGetErrorString(e);
    return FAST_GPU_ECUDA;
  }
  w->traj.push_back(d);
  w->lam.emplace_back(lambda, lambda + steps);
  w->trained = false;
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_build_basis(fast_gpu_ws *w, double *captured_energy) {
  if (!w) return FAST_GPU_EINVAL;
  Ctx &c = *w->c;
  int m = 0;
  for (auto &l : w->lam) m += (int)l.size();
  if (m < w->o.modes) { c.err = "ws_build_basis: fewer snapshots than modes"; return FAST_GPU_ESTATE; }
  const auto t0 = std::chrono::steady_clock::now();
  const int n = w->n;
  const int l = std::min(m, w->o.modes + w->o.oversample);
  // S: [m][n], the snapshots as rows
  double *S = nullptr, *Om = nullptr, *Y = nullptr, *Q = nullptr, *Z = nullptr, *Zq = nullptr, *d_u = nullptr,
         *d_fro = nullptr;
  int rc = FAST_GPU_OK;
  cudaError_t e = cudaMalloc((void **)&S, sizeof(double) * (size_t)m * n);
  if (e == cudaSuccess) e = cudaMalloc((void **)&Om, sizeof(double) * (size_t)m * l);
  if (e == cudaSuccess) e = cudaMalloc((void **)&Y, sizeof(double) * (size_t)n * l);
  if (e == cudaSuccess) e = cudaMalloc((void **)&Q, sizeof(double) * (size_t)n * l);
  if (e == cudaSuccess) e = cudaMalloc((void **)&Z, sizeof(double) * (size_t)m * l);
  if (e == cudaSuccess) e = cudaMalloc((void **)&Zq, sizeof(double) * (size_t)m * l);
  if (e == cudaSuccess) e = cudaMalloc((void **)&d_fro, sizeof(double));
  size_t row = 0;
  for (size_t t = 0; t < w->traj.size() && e == cudaSuccess; t++) {
    const size_t cnt = w->lam[t].size();
    e = cudaMemcpyAsync(S + row * n, w->traj[t], sizeof(double) * cnt * n, cudaMemcpyDeviceToDevice, c.stream);
    row += cnt;
  }
  std::vector<double> hom((size_t)m * l);
  uint64_t st = w->o.seed ^ 0x5DEECE66Dull;
  for (double &x : hom) x = gauss(st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Om, hom.data(), sizeof(double) * hom.size(), cudaMemcpyHostToDevice, c.stream);
  int r = l;
  // Y = S^T Omega ... in snapshot-as-row terms: Y[n][l] = S^T[n][m] Om[m][l]
  if (e == cudaSuccess) e = w->gemm(n, l, m, S, n, true, Om, l, false, Y, l);
  if (e == cudaSuccess) r = w->orth(n, l, Y, Q, e);
  for (int it = 0; it < w->o.power_iters && e == cudaSuccess && r > 0; it++) {
    e = w->gemm(m, r, n, S, n, false, Q, r, false, Z, r);            // Z = S Q       [m][r]
    int r2 = r;
    if (e == cudaSuccess) r2 = w->orth(m, r, Z, Zq, e);
    if (e == cudaSuccess && r2 > 0) e = w->gemm(n, r2, m, S, n, true, Zq, r2, false, Y, r2);  // Y = S^T Zq
    if (e == cudaSuccess && r2 > 0) r = w->orth(n, r2, Y, Q, e);
  }
  std::vector<double> B2, ev, U;
  if (e == cudaSuccess && r > 0) e = w->gemm(m, r, n, S, n, false, Q, r, false, Z, r);  // Z = S Q = B^T
  if (e == cudaSuccess && r > 0) {
    double *d_b = nullptr;
    e = cudaMalloc((void **)&d_b, sizeof(double) * r * r);
    if (e == cudaSuccess) e = w->gemm(r, r, m, Z, r, true, Z, r, false, d_b, r);  // B B^T = Z^T Z
    B2.resize((size_t)r * r);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B2.data(), d_b, sizeof(double) * r * r, cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (d_b) cudaFree(d_b);
  }
  const int k = std::min(w->o.modes, r);
  double kept = 0.0, fro = 0.0;
  if (e == cudaSuccess && k > 0) {
    sym_eig(r, B2, ev, U);
    for (int j = 0; j < k; j++) kept += std::max(0.0, ev[j]);
    std::vector<double> Uk((size_t)r * k);
    for (int i = 0; i < r; i++)
      for (int j = 0; j < k; j++) Uk[(size_t)i * k + j] = U[(size_t)i * r + j];
    e = cudaMalloc((void **)&d_u, sizeof(double) * r * k);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_u, Uk.data(), sizeof(double) * r * k, cudaMemcpyHostToDevice, c.stream);
    if (w->d_phi) { cudaFree(w->d_phi); w->d_phi = nullptr; }
    if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_phi, sizeof(double) * (size_t)n * k);
    if (e == cudaSuccess) e = w->gemm(n, k, r, Q, r, false, d_u, k, false, w->d_phi, k);  // Phi = Q U_k
    for (double **p : {&w->d_phin, &w->d_Y})
      if (*p) { cudaFree(*p); *p = nullptr; }
    const size_t nrow = 4 * (size_t)c.nnode;
    if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_phin, sizeof(double) * nrow * k);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w->d_Y, sizeof(double) * nrow * k);
    if (e == cudaSuccess) e = cudaMemsetAsync(w->d_phin, 0, sizeof(double) * nrow * k, c.stream);
    if (e == cudaSuccess) {
      const int64_t tot = (int64_t)n * k;
      ws_phi_to_node<<<(unsigned)((tot + 255) / 256), 256, 0, c.stream>>>(n, k, c.d_dof_of_eq, w->d_phi, w->d_phin);
      w->launches++;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_norm2(c, S, (int64_t)m * n, d_fro);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&fro, d_fro, sizeof(double), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  }
  if (e == cudaSuccess && k > 0) {
    w->k = k;
    w->energy = fro > 0 ? kept / fro : 0.0;
    if (captured_energy) *captured_energy = w->energy;
    w->trained = false;
  } else if (e != cudaSuccess) {
    c.err = std::string("ws_build_basis: ") + cudaGetErrorString(e);
    rc = FAST_GPU_ECUDA;
  } else {
    c.err = "ws_build_basis: snapshots have rank 0";
    rc = FAST_GPU_ESTATE;
  }
  for (double *p : {S, Om, Y, Q, Z, Zq, d_u, d_fro})
    if (p) cudaFree(p);
  w->basis_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

namespace {

// scaled samples from the POD coefficients of every snapshot
void build_samples(fast_gpu_ws *w, const std::vector<double> &A) {
  const int k = w->k, H = w->o.history, in = w->in_dim;
  const int kk = w->o.modes;  // network output width (modes beyond k stay zero)
  size_t off = 0;
  std::vector<size_t> toff;
  for (size_t t = 0; t < w->lam.size(); t++) { toff.push_back(off); off += w->lam[t].size(); }
  auto coef = [&](size_t t, long s, int j) -> double {  // a_s of trajectory t (s = 1..S), 0 for s <= 0
    return s <= 0 ? 0.0 : A[(toff[t] + (size_t)(s - 1)) * k + j];
  };
  auto lamv = [&](size_t t, long s) -> double { return s <= 0 ? 0.0 : w->lam[t][(size_t)(s - 1)]; };
  struct Sm { size_t t; long s; double rho; };
  std::vector<Sm> list;
  for (size_t t = 0; t < w->lam.size(); t++) {
    const long S = (long)w->lam[t].size();
    for (long s = 2; s <= S; s++) {
      const double d1 = lamv(t, s - 1) - lamv(t, s - 2);
      list.push_back({t, s, d1 != 0.0 ? (lamv(t, s) - lamv(t, s - 1)) / d1 : 1.0});
    }
  }
  const size_t ns = list.size();
  // per-mode RMS scales: a over all snapshots, da_{s-1} and the target over the samples
  auto floor_scale = [](std::vector<double> &v, double rel) {
    double mx = 0.0;
    for (double x : v) mx = std::max(mx, x);
    for (double &x : v) x = std::max(x, rel * mx + 1e-300);
  };
  w->sigma.assign(k, 0.0);
  w->delta.assign(k, 0.0);
  w->tau.assign(k, 0.0);
  const size_t rows = A.size() / k;
  for (size_t r = 0; r < rows; r++)
    for (int j = 0; j < k; j++) w->sigma[j] += A[r * k + j] * A[r * k + j];
  std::vector<double> raw(ns * k);
  for (size_t i = 0; i < ns; i++) {
    const Sm &m = list[i];
    for (int j = 0; j < k; j++) {
      const double d1 = coef(m.t, m.s - 1, j) - coef(m.t, m.s - 2, j);
      w->delta[j] += d1 * d1;
      raw[i * k + j] = coef(m.t, m.s, j) - coef(m.t, m.s - 1, j) - m.rho * d1;
      w->tau[j] += raw[i * k + j] * raw[i * k + j];
    }
  }
  for (int j = 0; j < k; j++) {
    w->sigma[j] = std::sqrt(w->sigma[j] / std::max<size_t>(1, rows));
    w->delta[j] = std::sqrt(w->delta[j] / std::max<size_t>(1, ns));
    w->tau[j] = std::sqrt(w->tau[j] / std::max<size_t>(1, ns));
  }
  floor_scale(w->sigma, 1e-12);
  floor_scale(w->delta, 1e-12);
  floor_scale(w->tau, 1e-6);
  w->hx.assign(ns * in, 0.f);
  w->ht.assign(ns * kk, 0.f);
  for (size_t i = 0; i < ns; i++) {
    const Sm &m = list[i];
    float *x = &w->hx[i * in];
    x[0] = (float)lamv(m.t, m.s);
    for (int j = 0; j < k; j++) x[1 + j] = (float)(coef(m.t, m.s - 1, j) / w->sigma[j]);
    for (int h = 1; h < H; h++)
      for (int j = 0; j < k; j++)
        x[1 + h * kk + j] = (float)((coef(m.t, m.s - h, j) - coef(m.t, m.s - h - 1, j)) / w->delta[j]);
    for (int j = 0; j < k; j++) w->ht[i * kk + j] = (float)(raw[i * k + j] / w->tau[j]);
  }
  w->samples = (int)ns;
}

}  // namespace

extern "C" int fast_gpu_ws_train(fast_gpu_ws *w, int32_t epochs, float lr, float *loss_history) {
  if (!w || epochs < 0 || !(lr > 0.f)) return FAST_GPU_EINVAL;
  Ctx &c = *w->c;
  if (!w->d_phi || w->k <= 0) { c.err = "ws_train: build the basis first"; return FAST_GPU_ESTATE; }
  const auto t0 = std::chrono::steady_clock::now();
  const int n = w->n, k = w->k;
  int m = 0;
  for (auto &l : w->lam) m += (int)l.size();
  // POD coefficients of every snapshot: A[m][k] = S Phi
  std::vector<double> A((size_t)m * k);
  {
    double *d_a = nullptr;
    WCK(cudaMalloc((void **)&d_a, sizeof(double) * (size_t)m * k));
    size_t row = 0;
    cudaError_t e = cudaSuccess;
    for (size_t t = 0; t < w->traj.size() && e == cudaSuccess; t++) {
      const int cnt = (int)w->lam[t].size();
      e = w->gemm(cnt, k, n, w->traj[t], n, false, w->d_phi, k, false, d_a + row * k, k);
      row += cnt;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(A.data(), d_a, sizeof(double) * A.size(), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFree(d_a);
    WCK(e);
  }
  build_samples(w, A);
  const int ns = w->samples;
  if (ns <= 0) { c.err = "ws_train: trajectories need at least 2 steps"; return FAST_GPU_ESTATE; }
  Mlp &net = w->net;
  WCK(net.reserve(ns));
  WCK(cudaMemcpyAsync(net.d_h[0], w->hx.data(), sizeof(float) * w->hx.size(), cudaMemcpyHostToDevice, c.stream));
  WCK(cudaMemcpyAsync(net.d_target, w->ht.data(), sizeof(float) * w->ht.size(), cudaMemcpyHostToDevice, c.stream));
  WCK(cudaMemsetAsync(net.d_status, 0, sizeof(int32_t), c.stream));
  float *d_hist = nullptr;
  WCK(cudaMalloc((void **)&d_hist, sizeof(float) * std::max(1, epochs)));
  cudaError_t e = cudaSuccess;
  const int64_t l0 = net.launches;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ep++) {
    const float lr_t = (float)(0.5 * lr * (1.0 + std::cos(3.141592653589793 * ep / std::max(1, epochs))));
    e = net.forward(c.stream, ns);
    if (e == cudaSuccess) e = net.backward(c.stream, ns);
    if (e == cudaSuccess) e = net.adam(c.stream, lr_t, 0.9f, 0.999f, 1e-8f);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_hist + ep, net.d_loss, sizeof(float), cudaMemcpyDeviceToDevice, c.stream);
  }
  std::vector<float> hh(std::max(1, epochs));
  int32_t status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(hh.data(), d_hist, sizeof(float) * hh.size(), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, net.d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFree(d_hist);
  w->launches += net.launches - l0;
  c.launches += net.launches - l0;
  WCK(e);
  if (status) { c.err = "ws_train: a tensor-core wait timed out"; return FAST_GPU_ECUDA; }
  if (loss_history && epochs > 0) std::memcpy(loss_history, hh.data(), sizeof(float) * epochs);
  w->epochs = epochs;
  if (epochs > 0) { w->first_loss = hh[0]; w->last_loss = hh[epochs - 1]; }
  {
    std::vector<double> sc(3 * 64, 1.0);
    for (int j = 0; j < w->k; j++) {
      sc[j] = w->sigma[j];
      sc[64 + j] = w->delta[j];
      sc[128 + j] = w->tau[j];
    }
    WCK(cudaMemcpy(w->d_scales, sc.data(), sizeof(double) * sc.size(), cudaMemcpyHostToDevice));
  }
  w->trained = true;
  w->last_step = 0;
  for (int i = 0; i < fast_gpu_ws::kRing; i++) w->ring_step[i] = -1;
  w->train_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_predict(void *user, int32_t step, double lambda, const double *d_u_last,
                                   const double *d_u_prev, const double *d_f, double *d_u_pred) {
  // Everything below is stream-ordered device work: no host synchronisation.
  fast_gpu_ws *w = static_cast<fast_gpu_ws *>(user);
  if (!w || !d_u_last || !d_u_prev || !d_u_pred || step < 2) return FAST_GPU_EINVAL;
  if (!w->trained) return FAST_GPU_ESTATE;
  if (w->gal_iters > 0 && !d_f) return FAST_GPU_EINVAL;
  const auto t0 = std::chrono::steady_clock::now();
  Ctx &c = *w->c;
  const int n = w->n, k = w->k, kk = w->o.modes, H = w->o.history;
  constexpr int R = fast_gpu_ws::kRing;
  const int64_t l_start = w->launches;
  if (step <= w->last_step)  // a new solve
    for (int i = 0; i < R; i++) w->ring_step[i] = -1;
  w->last_step = step;
  // load factors of the two previous steps: proportional loading with equal steps
  const double lam1 = lambda * (step - 1) / step, lam2 = lambda * (step - 2) / step;
  const double rho = (lam1 - lam2) != 0.0 ? (lambda - lam1) / (lam1 - lam2) : 1.0;
  const double *tau = w->d_scales + 128;
  const float *y = nullptr;
  const int64_t span_net = c.begin_span(FAST_KERNEL_PREDICT_NET);
  if (w->use_network) {
    Mlp &net = w->net;
    WCK(net.reserve(1));
    const int s1 = (step - 1) % R, s2 = (step - 2) % R;
    // a_{s-2} = Phi^T u_prev unless the ring has it from the last prediction
    // (then it was that step's u_last)
    if (step - 2 >= 1 && w->ring_step[s2] != step - 2) {
      WCK(w->project(d_u_prev, nullptr, w->d_ring + s2 * 64, nullptr));
      w->ring_step[s2] = step - 2;
    }
    NetArgs na{};
    na.f.k = k;
    na.f.kk = kk;
    na.f.H = H;
    na.f.lambda = lambda;
    for (int j = 0; j < 18; j++) na.f.slot[j] = -1;
    w->ring_step[s1] = step - 1;
    for (int j = 1; j <= H + 1 && j < 18; j++) {
      // a_{s-j}: zero before the first step; a step missing from the ring
      // repeats the closest earlier one that is there
      for (int st = step - j; st >= 1; st--)
        if (w->ring_step[st % R] == st) { na.f.slot[j] = st % R; break; }
    }
    if (!net.row_layout(na.m)) { c.err = "ws_predict: network too large for the single-row forward"; return FAST_GPU_EINVAL; }
    na.cur_slot = s1;
    na.params = net.d_params;
    na.ring = w->d_ring;
    na.sigma = w->d_scales;
    na.delta = w->d_scales + 64;
    na.x = net.d_h[0];
    na.y = net.d_h[net.layers()];
    // a_{s-1} = Phi^T u_last into the ring, then the network, in one launch
    WCK(w->project(d_u_last, nullptr, w->d_ring + s1 * 64, &na));
    y = na.y;
  }
  ws_start<<<148, 256, 0, c.stream>>>(n, k, rho, d_u_last, d_u_prev, w->d_phi, tau, y, d_u_pred);
  w->launches++;
  WCK(cudaGetLastError());
  c.end_span(span_net);

  if (w->gal_iters > 0 && c.d_K && c.K_ok) {
    const int64_t span_gal = c.begin_span(FAST_KERNEL_PREDICT_GALERKIN);
    // reduced tangent Phi^T K Phi from the last assembled tangent, its
    // Cholesky factor, and Phi^T f
    const int64_t nrow = 4 * c.nnode;
    const int64_t tot = c.nnode * k;
    ws_block_spmm<<<(unsigned)((tot + 127) / 128), 128, 0, c.stream>>>(c.nnode, k, c.d_rowptr, c.d_col, c.d_K,
                                                                         w->d_phin, w->d_Y);
    w->launches++;
    WCK(w->atb(nrow, k, k, w->d_phin, k, w->d_Y, k, w->d_Er, k));
    ws_chol<<<1, 64, 0, c.stream>>>(k, w->d_Er, w->d_L, w->d_ok);
    w->launches++;
    WCK(w->project(d_f, nullptr, w->d_coef + 64, nullptr));  // Phi^T f
    fast_gpu_ctx *fc = static_cast<fast_gpu_ctx *>(w->c);
    for (int it = 0; it < w->gal_iters; it++) {
      int rc = fast_gpu_set_displacement_device(fc, d_u_pred);
      if (rc == FAST_GPU_OK) rc = fast_gpu_internal_force_device(fc, w->d_g);
      if (rc != FAST_GPU_OK) return rc;
      WCK(w->project(d_f, w->d_g, w->d_coef, nullptr));  // Phi^T (f - g)
      ws_reduced_add<<<148, 256, 0, c.stream>>>(n, k, w->d_L, w->d_ok, w->d_coef, w->d_coef + 64, w->gal_tol,
                                                w->d_phi, d_u_pred, w->d_delta);
      w->launches++;
      w->n_gal++;
    }
    WCK(cudaGetLastError());
    c.end_span(span_gal);
  }
  w->n_pred++;
  c.launches += w->launches - l_start;
  w->pred_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_configure(fast_gpu_ws *w, int32_t use_network, int32_t galerkin_iters,
                                     double galerkin_tol) {
  if (!w || galerkin_iters < 0 || !(galerkin_tol >= 0.0)) return FAST_GPU_EINVAL;
  w->use_network = use_network ? 1 : 0;
  w->gal_iters = galerkin_iters;
  w->gal_tol = galerkin_tol;
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_last_input(fast_gpu_ws *w, float *x) {
  if (!w || !x) return FAST_GPU_EINVAL;
  if (w->n_pred == 0 || !w->use_network) { w->c->err = "ws_last_input: no network prediction yet"; return FAST_GPU_ESTATE; }
  WCK(cudaMemcpyAsync(x, w->net.d_h[0], sizeof(float) * w->in_dim, cudaMemcpyDeviceToHost, w->c->stream));
  WCK(cudaStreamSynchronize(w->c->stream));
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_report(fast_gpu_ws *w, fast_gpu_ws_stats *r) {
  if (!w || !r) return FAST_GPU_EINVAL;
  fast_gpu_ws_stats R{};
  R.trajectories = (int32_t)w->traj.size();
  for (auto &l : w->lam) R.snapshots += (int32_t)l.size();
  R.samples = w->samples;
  R.modes = w->k;
  R.input_dim = w->in_dim;
  R.output_dim = w->o.modes;
  R.epochs = w->epochs;
  R.params = w->net.nparams;
  R.captured_energy = w->energy;
  R.basis_ms = w->basis_ms;
  R.train_ms = w->train_ms;
  R.first_loss = w->first_loss;
  R.last_loss = w->last_loss;
  R.launches = w->launches;
  R.predictions = w->n_pred;
  R.galerkin_iterations = w->n_gal;
  R.predict_ms = w->pred_ms;
  *r = R;
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_get_basis(fast_gpu_ws *w, double *phi) {
  if (!w || !phi) return FAST_GPU_EINVAL;
  if (!w->d_phi) { w->c->err = "ws_get_basis: no basis"; return FAST_GPU_ESTATE; }
  WCK(cudaMemcpyAsync(phi, w->d_phi, sizeof(double) * (size_t)w->n * w->k, cudaMemcpyDeviceToHost, w->c->stream));
  WCK(cudaStreamSynchronize(w->c->stream));
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_ws_get_samples(fast_gpu_ws *w, float *x, float *t) {
  if (!w) return FAST_GPU_EINVAL;
  if (w->samples <= 0) { w->c->err = "ws_get_samples: not trained"; return FAST_GPU_ESTATE; }
  if (x) std::memcpy(x, w->hx.data(), sizeof(float) * w->hx.size());
  if (t) std::memcpy(t, w->ht.data(), sizeof(float) * w->ht.size());
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_mlp_params(fast_gpu_ws *w, float *get, const float *set, int64_t *count) {
  if (!w) return FAST_GPU_EINVAL;
  if (count) *count = w->net.nparams;
  if (set) WCK(cudaMemcpy(w->net.d_params, set, sizeof(float) * w->net.nparams, cudaMemcpyHostToDevice));
  if (get) WCK(cudaMemcpy(get, w->net.d_params, sizeof(float) * w->net.nparams, cudaMemcpyDeviceToHost));
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_mlp_forward(fast_gpu_ws *w, int32_t batch, const float *x, float *y) {
  if (!w || batch <= 0 || !x || !y) return FAST_GPU_EINVAL;
  Ctx &c = *w->c;
  Mlp &net = w->net;
  WCK(net.reserve(batch));
  WCK(cudaMemcpyAsync(net.d_h[0], x, sizeof(float) * (size_t)batch * net.dims[0], cudaMemcpyHostToDevice, c.stream));
  WCK(cudaMemsetAsync(net.d_status, 0, sizeof(int32_t), c.stream));
  const int64_t l0 = net.launches;
  // a single row takes the CUDA-core form the predictor uses
  if (batch == 1) WCK(net.forward_row(c.stream));
  else WCK(net.forward(c.stream, batch));
  int32_t status = 0;
  WCK(cudaMemcpyAsync(y, net.d_h[net.layers()], sizeof(float) * (size_t)batch * net.dims.back(),
                      cudaMemcpyDeviceToHost, c.stream));
  WCK(cudaMemcpyAsync(&status, net.d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
  WCK(cudaStreamSynchronize(c.stream));
  w->launches += net.launches - l0;
  c.launches += net.launches - l0;
  if (status) { c.err = "mlp_forward: a tensor-core wait timed out"; return FAST_GPU_ECUDA; }
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_mlp_loss_grad(fast_gpu_ws *w, int32_t batch, const float *x, const float *t, float *loss,
                                      float *grad) {
  if (!w || batch <= 0 || !x || !t) return FAST_GPU_EINVAL;
  Ctx &c = *w->c;
  Mlp &net = w->net;
  WCK(net.reserve(batch));
  WCK(cudaMemcpyAsync(net.d_h[0], x, sizeof(float) * (size_t)batch * net.dims[0], cudaMemcpyHostToDevice, c.stream));
  WCK(cudaMemcpyAsync(net.d_target, t, sizeof(float) * (size_t)batch * net.dims.back(), cudaMemcpyHostToDevice,
                      c.stream));
  WCK(cudaMemsetAsync(net.d_status, 0, sizeof(int32_t), c.stream));
  const int64_t l0 = net.launches;
  WCK(net.forward(c.stream, batch));
  WCK(net.backward(c.stream, batch));
  int32_t status = 0;
  if (loss) WCK(cudaMemcpyAsync(loss, net.d_loss, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
  if (grad) WCK(cudaMemcpyAsync(grad, net.d_grads, sizeof(float) * net.nparams, cudaMemcpyDeviceToHost, c.stream));
  WCK(cudaMemcpyAsync(&status, net.d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
  WCK(cudaStreamSynchronize(c.stream));
  w->launches += net.launches - l0;
  c.launches += net.launches - l0;
  if (status) { c.err = "mlp_loss_grad: a tensor-core wait timed out"; return FAST_GPU_ECUDA; }
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_mlp_gemm(fast_gpu_ctx *c, int32_t M, int32_t N, int32_t K, const float *A, int32_t ta,
                                 const float *B, int32_t tb, float *C) {
  if (!c || M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return FAST_GPU_EINVAL;
  float *dA = nullptr, *dB = nullptr, *dC = nullptr, *dW = nullptr;
  int32_t *dst = nullptr, status = 0;
  const int sp = gemm_splits(M, N, K, kEpiStore);
  cudaError_t e = cudaMalloc((void **)&dA, sizeof(float) * (size_t)M * K);
  if (e == cudaSuccess && sp > 1) e = cudaMalloc((void **)&dW, sizeof(float) * (size_t)sp * M * N);
  if (e == cudaSuccess) e = cudaMalloc((void **)&dB, sizeof(float) * (size_t)N * K);
  if (e == cudaSuccess) e = cudaMalloc((void **)&dC, sizeof(float) * (size_t)M * N);
  if (e == cudaSuccess) e = cudaMalloc((void **)&dst, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(dst, 0, sizeof(int32_t), c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dA, A, sizeof(float) * (size_t)M * K, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dB, B, sizeof(float) * (size_t)N * K, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = gemm_bf16(c->stream, M, N, K, dA, ta ? M : K, ta != 0, dB, tb ? N : K, tb != 0, dC, N, kEpiStore, nullptr,
                  nullptr, 0, dst, dW);
  c->launches++;
  if (e == cudaSuccess) e = cudaMemcpyAsync(C, dC, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, dst, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  for (void *p : {(void *)dA, (void *)dB, (void *)dC, (void *)dW, (void *)dst})
    if (p) cudaFree(p);
  if (e != cudaSuccess) { c->err = std::string("mlp_gemm: ") + cudaGetErrorString(e); return FAST_GPU_ECUDA; }
  if (status) { c->err = "mlp_gemm: a tensor-core wait timed out"; return FAST_GPU_ECUDA; }
  return FAST_GPU_OK;
}

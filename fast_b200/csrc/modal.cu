// modal.cu - natural frequencies and mode shapes (fast_gpu_modal) and linear
// buckling factors and modes (fast_gpu_buckling) on the device:
// cCtrlModal::Solver (ctrl/ctrlmodal.cpp:48-128) and cCtrlLinStab::Solver
// (ctrl/ctrllinstab.cpp:46-140) with the subspace iteration of
// cGenEigSubSpaces::Solver (mlib/eig.cpp:377-510).
//
//   q = max(2p, p + 8) vectors (at most 32); start: unit vectors at the q
//   smallest K_ii / M_ii, the last one an alternating-sign pseudo-random
//   vector; each iteration
//     K Y_i = M X_i  (X_i itself at the first)      q PCG solves
//     Kp = Y^T K Y,  Mp = Y^T M Y                    2q SpMV + two q x q Gram products
//     Kp phi = lambda Mp phi, phi^T Mp phi = 1       host, q x q
//     X = Y Phi                                      one kernel
//   converged when sqrt(|1 - lambda_i^2 / |phi_i|^2|) <= tol for the p lowest.
//
// The reference factors K once (skyline) and solves each right-hand side
// directly; here each solve is a PCG on the resident K, warm-started from
// X_i / lambda_i (the next Y_i to first order once X spans the modes).  All
// q vectors live in HBM in the node-padded layout [q][4 nnode]; fixed DOFs
// and pads stay 0 (M has no entries there and K an identity row).  The Gram
// products are fixed-order reductions, so the result is the same every run.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

constexpr int kMaxSub = 32;       // subspace vectors (q) at most
constexpr int kGramBlocks = 296;  // 2 x 148 SMs
constexpr int kGramRows = 32;     // rows per shared-memory tile

// K_ii / M_ii of every DOF of the node-padded layout (+inf where M_ii = 0:
// fixed DOFs and pads; M is minus the geometric stiffness for buckling,
// whose diagonal may be negative)
__global__ void modal_ratio(int64_t nnode, const int32_t *__restrict__ diag, const double *__restrict__ K,
                            const double *__restrict__ M, double *__restrict__ out) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const int64_t b = (int64_t)diag[n] * 9;
  for (int i = 0; i < 3; i++) {
    const double m = M[b + 4 * i];
    out[4 * n + i] = m != 0.0 ? K[b + 4 * i] / m : INFINITY;
  }
  out[4 * n + 3] = INFINITY;
}

// per-block partial Gram matrices G[i][j] = sum_r A_i[r] B_j[r] over the
// rows of this block (A, B: q vectors of n rows each, vector-major)
__global__ void __launch_bounds__(256) modal_gram(int q, int64_t n, const double *__restrict__ A,
                                                  const double *__restrict__ B, double *__restrict__ part) {
  // rows padded by one: the threads of a warp read different vectors at the
  // same row, which an unpadded 32-double row would put in one bank
  __shared__ double sA[kMaxSub][kGramRows + 1], sB[kMaxSub][kGramRows + 1];
  const int qq = q * q;
  double acc[kMaxSub * kMaxSub / 256] = {0, 0, 0, 0};
  for (int64_t r0 = (int64_t)blockIdx.x * kGramRows; r0 < n; r0 += (int64_t)gridDim.x * kGramRows) {
    for (int idx = threadIdx.x; idx < q * kGramRows; idx += blockDim.x) {
      const int k = idx / kGramRows, r = idx - k * kGramRows;
      const int64_t row = r0 + r;
      sA[k][r] = row < n ? A[(int64_t)k * n + row] : 0.0;
      sB[k][r] = row < n ? B[(int64_t)k * n + row] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kMaxSub * kMaxSub / 256; s++) {
      const int p = threadIdx.x + 256 * s;
      if (p < qq) {
        const int i = p / q, j = p - i * q;
        double a = acc[s];
#pragma unroll 8
        for (int r = 0; r < kGramRows; r++) a = fma(sA[i][r], sB[j][r], a);
        acc[s] = a;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int s = 0; s < kMaxSub * kMaxSub / 256; s++) {
    const int p = threadIdx.x + 256 * s;
    if (p < qq) part[(int64_t)blockIdx.x * qq + p] = acc[s];
  }
}

// G = sum of the block partials in block order
__global__ void modal_gram_finish(int qq, const double *__restrict__ part, double *__restrict__ G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= qq) return;
  double t = 0.0;
  for (int b = 0; b < kGramBlocks; b++) t += part[(int64_t)b * qq + p];
  G[p] = t;
}

// X_j = sum_k Y_k Phi[k][j] (Phi k-major [q][q])
__global__ void __launch_bounds__(256) modal_combine(int q, int64_t n, const double *__restrict__ Y,
                                                     const double *__restrict__ Phi, double *__restrict__ X) {
  __shared__ double sP[kMaxSub * kMaxSub];
  for (int i = threadIdx.x; i < q * q; i += blockDim.x) sP[i] = Phi[i];
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    double y[kMaxSub];
#pragma unroll
    for (int k = 0; k < kMaxSub; k++) y[k] = k < q ? Y[(int64_t)k * n + r] : 0.0;
    for (int j = 0; j < q; j++) {
      double a = 0.0;
#pragma unroll
      for (int k = 0; k < kMaxSub; k++)
        if (k < q) a = fma(y[k], sP[k * q + j], a);
      X[(int64_t)j * n + r] = a;
    }
  }
}

__global__ void modal_scale(int64_t n, double s, const double *__restrict__ x, double *__restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = s * x[i];
}

// Jacobi eigenvalue sweeps on a symmetric q x q matrix C (row-major); V
// gets the eigenvectors as columns.  Quadratic convergence: a handful of
// sweeps to the round-off level.
bool sym_eigen(int q, std::vector<double> &C, std::vector<double> &V) {
  V.assign((size_t)q * q, 0.0);
  for (int i = 0; i < q; i++) V[(size_t)i * q + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < q; i++)
      for (int j = 0; j < q; j++) {
        const double v = C[(size_t)i * q + j] * C[(size_t)i * q + j];
        tot += v;
        if (i != j) off += v;
      }
    if (off <= 1e-30 * tot) return true;
    for (int p = 0; p < q - 1; p++)
      for (int r = p + 1; r < q; r++) {
        const double apq = C[(size_t)p * q + r];
        if (apq == 0.0) continue;
        const double app = C[(size_t)p * q + p], aqq = C[(size_t)r * q + r];
        const double theta = 0.5 * (aqq - app) / apq;
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < q; k++) {  // columns p, r
          const double ckp = C[(size_t)k * q + p], ckr = C[(size_t)k * q + r];
          C[(size_t)k * q + p] = cs * ckp - sn * ckr;
          C[(size_t)k * q + r] = sn * ckp + cs * ckr;
        }
        for (int k = 0; k < q; k++) {  // rows p, r
          const double cpk = C[(size_t)p * q + k], crk = C[(size_t)r * q + k];
          C[(size_t)p * q + k] = cs * cpk - sn * crk;
          C[(size_t)r * q + k] = sn * cpk + cs * crk;
        }
        for (int k = 0; k < q; k++) {
          const double vkp = V[(size_t)k * q + p], vkr = V[(size_t)k * q + r];
          V[(size_t)k * q + p] = cs * vkp - sn * vkr;
          V[(size_t)k * q + r] = sn * vkp + cs * vkr;
        }
      }
  }
  return false;
}

// Kp phi = lambda Mp phi, ascending, phi^T Mp phi = 1.  Mp definite (modal):
// Mp = L L^T, C = L^-1 Kp L^-T, C z = lambda z, phi = L^-T z.  Swapped (the
// buckling pencil, Mp = -Y^T G Y need not be definite, Kp is): Kp = L L^T,
// C = L^-1 Mp L^-T, C z = mu z, lambda = 1/mu, phi = L^-T z / sqrt(|mu|)
// (so phi^T Mp phi = 1 where mu > 0).  Phi k-major [q][q].
bool projected_eigen(int q, const std::vector<double> &Kp, const std::vector<double> &Mp, std::vector<double> &lam,
                     std::vector<double> &Phi, bool swapped = false) {
  const std::vector<double> &S = swapped ? Kp : Mp, &T = swapped ? Mp : Kp;
  std::vector<double> L((size_t)q * q, 0.0);
  for (int j = 0; j < q; j++) {
    double d = S[(size_t)j * q + j];
    for (int k = 0; k < j; k++) d -= L[(size_t)j * q + k] * L[(size_t)j * q + k];
    if (!(d > 0.0)) return false;
    L[(size_t)j * q + j] = std::sqrt(d);
    for (int i = j + 1; i < q; i++) {
      double s = 0.5 * (S[(size_t)i * q + j] + S[(size_t)j * q + i]);
      for (int k = 0; k < j; k++) s -= L[(size_t)i * q + k] * L[(size_t)j * q + k];
      L[(size_t)i * q + j] = s / L[(size_t)j * q + j];
    }
  }
  // W = L^-1 Ts (Ts the symmetric part of T), then C = W L^-T = L^-1 W^T
  std::vector<double> W((size_t)q * q), C((size_t)q * q);
  for (int col = 0; col < q; col++)
    for (int i = 0; i < q; i++) {
      double s = 0.5 * (T[(size_t)i * q + col] + T[(size_t)col * q + i]);
      for (int k = 0; k < i; k++) s -= L[(size_t)i * q + k] * W[(size_t)k * q + col];
      W[(size_t)i * q + col] = s / L[(size_t)i * q + i];
    }
  for (int col = 0; col < q; col++)
    for (int i = 0; i < q; i++) {
      double s = W[(size_t)col * q + i];
      for (int k = 0; k < i; k++) s -= L[(size_t)i * q + k] * C[(size_t)k * q + col];
      C[(size_t)i * q + col] = s / L[(size_t)i * q + i];
    }
  for (int i = 0; i < q; i++)
    for (int j = i + 1; j < q; j++) {
      const double s = 0.5 * (C[(size_t)i * q + j] + C[(size_t)j * q + i]);
      C[(size_t)i * q + j] = C[(size_t)j * q + i] = s;
    }
  std::vector<double> V;
  if (!sym_eigen(q, C, V)) return false;
  std::vector<double> val(q);
  for (int j = 0; j < q; j++) {
    const double mu = C[(size_t)j * q + j];
    val[j] = swapped ? (mu != 0.0 ? 1.0 / mu : INFINITY) : mu;
  }
  std::vector<int> order(q);
  for (int i = 0; i < q; i++) order[i] = i;
  std::sort(order.begin(), order.end(),
            [&](int a, int b) { return val[a] < val[b] || (val[a] == val[b] && a < b); });
  lam.resize(q);
  Phi.assign((size_t)q * q, 0.0);
  for (int jj = 0; jj < q; jj++) {
    const int j = order[jj];
    lam[jj] = val[j];
    const double mu = C[(size_t)j * q + j];
    const double sc = (swapped && mu != 0.0) ? 1.0 / std::sqrt(std::fabs(mu)) : 1.0;
    // phi = L^-T z: back substitution
    for (int i = q - 1; i >= 0; i--) {
      double s = V[(size_t)i * q + j];
      for (int k = i + 1; k < q; k++) s -= L[(size_t)k * q + i] * Phi[(size_t)k * q + jj];
      Phi[(size_t)i * q + jj] = s / L[(size_t)i * q + i];
    }
    if (sc != 1.0)
      for (int i = 0; i < q; i++) Phi[(size_t)i * q + jj] *= sc;
  }
  return true;
}

// alternating-sign value in (0, 1] for equation j (a fixed hash: the start
// vector is the same every run)
double start_value(int64_t j) {
  uint64_t x = (uint64_t)j * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  x ^= x >> 31;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 29;
  const double u = (double)((x >> 11) + 1) / 9007199254740992.0;
  return (j % 2) ? -u : u;
}

}  // namespace

#define MCK(call)                                                             \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) {                                                  \
      c->err = std::string("modal: ") + #call + ": " + cudaGetErrorString(_e);  \
      rc = FAST_GPU_ECUDA;                                                    \
      goto done;                                                              \
    }                                                                         \
  } while (0)

// The subspace iteration on the pencil (K in the stiffness slot, the
// right-hand matrix in the mass slot), both assembled.
static int subspace_iteration(fast_gpu_ctx *c, const fast_gpu_modal_opts *o, bool swapped, double *lambda,
                              double *modes, fast_gpu_modal_report *rep) {
  const int p = o->num_modes;
  const int q = (int)std::min<int64_t>(std::max(2 * p, p + 8), c->neq);
  const int64_t n4 = 4 * c->nnode;
  const size_t vb = sizeof(double) * n4;
  int rc = FAST_GPU_OK;
  fast_gpu_modal_report R{};
  R.subspace = q;
  double *d_X = nullptr, *d_Y = nullptr, *d_T = nullptr, *d_part = nullptr, *d_G = nullptr, *d_phi = nullptr;
  std::vector<double> Kp((size_t)q * q), Mp((size_t)q * q), lam, Phi, ratio;
  fast_gpu_solve_opts lin = o->lin;
  {
    cudaError_t e = cudaMalloc((void **)&d_X, vb * q);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_Y, vb * q);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_T, vb * q);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_part, sizeof(double) * kGramBlocks * q * q);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_G, sizeof(double) * q * q);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_phi, sizeof(double) * q * q);
    MCK(e);
  }
  MCK(solve_layout(*c, FAST_ASM_MASS, false));
  MCK(solve_layout(*c, FAST_ASM_STIFFNESS, false));

  // start vectors: unit vectors at the q smallest K_ii / M_ii (ties by
  // equation), the last one alternating-sign pseudo-random, unit length
  {
    MCK(cudaMemsetAsync(d_X, 0, vb * q, c->stream));
    modal_ratio<<<(unsigned)((c->nnode + 127) / 128), 128, 0, c->stream>>>(c->nnode, c->d_diag, c->d_K, c->d_M,
                                                                           d_T);
    c->launches++;
    ratio.resize(n4);
    MCK(cudaMemcpyAsync(ratio.data(), d_T, vb, cudaMemcpyDeviceToHost, c->stream));
    MCK(cudaStreamSynchronize(c->stream));
    std::vector<std::pair<double, int64_t>> cand;  // (ratio, equation) of every DOF with an equation
    cand.reserve(c->neq);
    std::vector<int64_t> pos_of_eq(c->neq, -1);
    for (int64_t nd = 0; nd < c->nnode; nd++)
      for (int i = 0; i < 3; i++) {
        const int32_t eq = c->h_eq[3 * nd + i];
        if (eq > 0) {
          pos_of_eq[eq - 1] = 4 * nd + i;
          cand.push_back({ratio[4 * nd + i], (int64_t)eq - 1});
        }
      }
    std::partial_sort(cand.begin(), cand.begin() + q, cand.end());
    std::vector<double> h((size_t)n4, 0.0);
    for (int j = 0; j < q - 1; j++) {
      const double one = 1.0;
      MCK(cudaMemcpyAsync(d_X + (size_t)j * n4 + pos_of_eq[cand[j].second], &one, sizeof(double),
                          cudaMemcpyHostToDevice, c->stream));
      MCK(cudaStreamSynchronize(c->stream));
    }
    double nrm = 0.0;
    for (int64_t k = 0; k < c->neq; k++) {
      const double v = start_value(k);
      h[pos_of_eq[k]] = v;
      nrm += v * v;
    }
    nrm = std::sqrt(nrm);
    for (double &v : h) v /= nrm;
    MCK(cudaMemcpyAsync(d_X + (size_t)(q - 1) * n4, h.data(), vb, cudaMemcpyHostToDevice, c->stream));
    MCK(cudaStreamSynchronize(c->stream));
  }

  for (int it = 0; it < o->max_iter; it++) {
    // K Y_i = M X_i (X_i at the first iteration), warm start X_i / lambda_i
    for (int i = 0; i < q; i++) {
      double *Xi = d_X + (size_t)i * n4;
      if (it == 0) MCK(cudaMemcpyAsync(c->d_f, Xi, vb, cudaMemcpyDeviceToDevice, c->stream));
      else MCK(launch_spmv(*c, c->d_Ms, Xi, c->d_f));
      const bool warm = it > 0 && lam[i] > 0.0;
      if (warm) {
        modal_scale<<<kGramBlocks, 256, 0, c->stream>>>(n4, 1.0 / lam[i], Xi, c->d_u);
        c->launches++;
      } else {
        MCK(cudaMemsetAsync(c->d_u, 0, vb, c->stream));
      }
      fast_gpu_solve_report lr{};
      lin.warm_start = warm ? 1 : 0;
      rc = solve_nodes(*c, &lin, warm, &lr);
      R.linear_iterations += lr.iterations;
      if (rc != FAST_GPU_OK) goto done;
      MCK(cudaMemcpyAsync(d_Y + (size_t)i * n4, c->d_u, vb, cudaMemcpyDeviceToDevice, c->stream));
    }
    // Kp = Y^T K Y, Mp = Y^T M Y
    for (int w = 0; w < 2; w++) {
      for (int i = 0; i < q; i++) MCK(launch_spmv(*c, w == 0 ? c->d_Ks : c->d_Ms, d_Y + (size_t)i * n4,
                                                  d_T + (size_t)i * n4));
      modal_gram<<<kGramBlocks, 256, 0, c->stream>>>(q, n4, d_Y, d_T, d_part);
      modal_gram_finish<<<(q * q + 255) / 256, 256, 0, c->stream>>>(q * q, d_part, d_G);
      c->launches += 2;
      MCK(cudaMemcpyAsync(w == 0 ? Kp.data() : Mp.data(), d_G, sizeof(double) * q * q, cudaMemcpyDeviceToHost,
                          c->stream));
    }
    MCK(cudaStreamSynchronize(c->stream));
    if (!projected_eigen(q, Kp, Mp, lam, Phi, swapped)) {
      c->err = "subspace iteration: projected problem not definite (vectors lost independence)";
      rc = FAST_GPU_ENONCONV;
      goto done;
    }
    MCK(cudaMemcpyAsync(d_phi, Phi.data(), sizeof(double) * q * q, cudaMemcpyHostToDevice, c->stream));
    modal_combine<<<kGramBlocks, 256, 0, c->stream>>>(q, n4, d_Y, d_phi, d_X);
    c->launches++;
    MCK(cudaGetLastError());
    R.iterations = it + 1;
    // the reference's measure: sqrt(|1 - lambda^2 / |phi|^2|) for the p lowest
    double maxerr = 0.0;
    for (int j = 0; j < p; j++) {
      double nn = 0.0;
      for (int k = 0; k < q; k++) nn += Phi[(size_t)k * q + j] * Phi[(size_t)k * q + j];
      maxerr = std::max(maxerr, std::sqrt(std::fabs(1.0 - lam[j] * lam[j] / nn)));
    }
    R.max_err = maxerr;
    if (maxerr <= o->tol) {
      R.converged = 1;
      break;
    }
  }
  if (!R.converged) {
    c->err = "subspace iteration did not converge";
    rc = FAST_GPU_ENONCONV;
  }
  for (int j = 0; j < p && j < (int)lam.size(); j++) lambda[j] = lam[j];
  if (modes && !lam.empty()) {
    for (int j = 0; j < p; j++) {
      MCK(launch_node_to_eq(*c, d_X + (size_t)j * n4, c->d_eq_tmp));
      MCK(cudaMemcpyAsync(modes + (size_t)j * c->neq, c->d_eq_tmp, sizeof(double) * c->neq, cudaMemcpyDeviceToHost,
                          c->stream));
      MCK(cudaStreamSynchronize(c->stream));
    }
  }
done:
  if (rep) *rep = R;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (double *b : {d_X, d_Y, d_T, d_part, d_G, d_phi})
    if (b) cudaFree(b);
  return rc;
}

static int eigen_checks(fast_gpu_ctx *c, const fast_gpu_modal_opts *o, const double *lambda) {
  if (!c || !o || !lambda || o->num_modes <= 0 || o->max_iter <= 0) return FAST_GPU_EINVAL;
  if (c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  if (!c->d_K || c->neq <= 0) { c->err = "eigen solve: no mesh"; return FAST_GPU_ESTATE; }
  const int p = o->num_modes;
  const int q = (int)std::min<int64_t>(std::max(2 * p, p + 8), c->neq);
  if (q > kMaxSub || p > q) {
    c->err = "eigen solve: at most 16 modes (a subspace of 32 vectors)";
    return FAST_GPU_ENOTSUP;
  }
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_modal(fast_gpu_ctx *c, const fast_gpu_modal_opts *o, double *lambda, double *modes,
                              fast_gpu_modal_report *rep) {
  int rc = eigen_checks(c, o, lambda);
  if (rc != FAST_GPU_OK) return rc;
  // cCtrlModal::Solver: M, then K (identity rows on fixed DOFs)
  rc = fast_gpu_assemble(c, FAST_ASM_MASS);
  if (rc == FAST_GPU_OK) rc = fast_gpu_assemble(c, FAST_ASM_STIFFNESS);
  if (rc != FAST_GPU_OK) return rc;
  return subspace_iteration(c, o, false, lambda, modes, rep);
}

// cCtrlLinStab::Solver (ctrl/ctrllinstab.cpp:46-140): K u = f, the geometric
// stiffness G at u, then K v = lambda (-G) v.  -G goes to the mass slot (the
// slot is marked stale afterwards, so a later mass assembly rebuilds M).
extern "C" int fast_gpu_buckling(fast_gpu_ctx *c, const double *f, const fast_gpu_modal_opts *o, double *lambda,
                                 double *modes, double *u, fast_gpu_modal_report *rep) {
  int rc = eigen_checks(c, o, lambda);
  if (rc != FAST_GPU_OK) return rc;
  if (!f) return FAST_GPU_EINVAL;
  for (const Bucket &B : c->buckets)
    if (B.tl || B.type == FAST_ELEM_BSP_SOLID) {
      c->err = "buckling: small-strain hex buckets only";
      return FAST_GPU_ENOTSUP;
    }
  rc = fast_gpu_assemble(c, FAST_ASM_STIFFNESS);
  if (rc != FAST_GPU_OK) return rc;
  fast_gpu_solve_report lr{};
  cudaError_t e = cudaMemcpyAsync(c->d_eq_tmp, f, sizeof(double) * c->neq, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = launch_eq_to_node(*c, c->d_eq_tmp, c->d_f);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_u, 0, sizeof(double) * 4 * c->nnode, c->stream);
  if (e != cudaSuccess) {
    c->err = std::string("buckling: ") + cudaGetErrorString(e);
    return FAST_GPU_ECUDA;
  }
  fast_gpu_solve_opts lin = o->lin;
  lin.warm_start = 0;
  rc = solve_nodes(*c, &lin, false, &lr);
  if (rc != FAST_GPU_OK) return rc;
  e = launch_node_to_eq(*c, c->d_u, c->d_eq_tmp);
  if (e == cudaSuccess && u)
    e = cudaMemcpyAsync(u, c->d_eq_tmp, sizeof(double) * c->neq, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    c->err = std::string("buckling: ") + cudaGetErrorString(e);
    return FAST_GPU_ECUDA;
  }
  rc = fast_gpu_set_displacement_device(c, c->d_eq_tmp);
  if (rc != FAST_GPU_OK) return rc;
  if (!c->d_M) {
    e = cudaMalloc((void **)&c->d_M, sizeof(double) * 9 * c->nnzb);
    if (e != cudaSuccess) {
      c->err = std::string("buckling: ") + cudaGetErrorString(e);
      return FAST_GPU_ENOMEM;
    }
  }
  e = cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_M, 0, sizeof(double) * 9 * c->nnzb, c->stream);
  if (e == cudaSuccess) e = launch_geom_stiffness(*c, c->d_M, -1.0);
  int32_t status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  c->M_ok = false;  // the mass slot holds -G now
  matrix_changed(*c, FAST_ASM_MASS);
  if (e != cudaSuccess) {
    c->err = std::string("buckling: ") + cudaGetErrorString(e);
    return FAST_GPU_ECUDA;
  }
  if (status & 1) {
    c->err = "buckling: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  rc = subspace_iteration(c, o, true, lambda, modes, rep);
  matrix_changed(*c, FAST_ASM_MASS);
  return rc;
}

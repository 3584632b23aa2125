// arclength.cu - path following with the reference's arc-length rules on the
// device (fast_gpu_arclength_solve).
//
// Mirrors cCtrlPath::Solver (ctrl/ctrlpath.cpp:63-265):
//   for each step, for each iteration:
//     K = tangent at u;  K du1 = q;  K du2 = r
//     dlf = IncLoadFac(du1, du2, Du)           (ctrl/ctrlarclen.cpp:95-250)
//     first iteration: Du <- 0 (Du of the last step is kept for the sign)
//     du = dlf du1 - du2;  lambda += dlf;  u += du;  Du += du
//     r = g(u) - lambda q;  converged when |r| / max(1, |q|) < tol
//   after a converged step: the current stiffness parameter
//     CSP = (q . du1 / du1 . du1) / (the same at step 1)
//   which the arc length reset of LoadCoeff = 1 uses.
// Vectors stay on the device; the scalars of the load-increment rule are
// formed on the host from dot products read back once per iteration.  The
// two solves take the unit right-hand sides q/|q| and r/|r| (PCGSolver's
// absolute early exit would otherwise return 0 for a small residual).
#include <cmath>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

constexpr int kArcBlocks = 296;

__global__ void arc_axpby(int32_t n, double a, const double *x, double b, const double *y,
                          double *z) {  // z may alias x or y (same index)
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

struct DotArgs {
  const double *x[6], *y[6];
  int n;
};

// up to six dot products, fixed-order: per-block partials, then one block
__global__ void __launch_bounds__(256) arc_dots(int32_t len, DotArgs a, double *__restrict__ part) {
  __shared__ double sh[6][8];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < a.n; k++) acc[k] += a.x[k][i] * a.y[k][i];
  for (int k = 0; k < a.n; k++) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < a.n) {
    double t = 0.0;
    for (int w = 0; w < 8; w++) t += sh[threadIdx.x][w];
    part[threadIdx.x * kArcBlocks + blockIdx.x] = t;
  }
}

__global__ void arc_dots_finish(int n, const double *__restrict__ part, double *__restrict__ out) {
  if (threadIdx.x < n) {
    double t = 0.0;
    for (int b = 0; b < kArcBlocks; b++) t += part[threadIdx.x * kArcBlocks + b];
    out[threadIdx.x] = t;
  }
}

struct Work {
  double *q = nullptr, *r = nullptr, *u = nullptr, *du1 = nullptr, *du2 = nullptr, *Du = nullptr, *Du0 = nullptr,
         *g = nullptr, *rhs = nullptr, *part = nullptr, *dots = nullptr, *hdots = nullptr;
};

}  // namespace

#define ACK(call)                                                                  \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      c->err = std::string("arclength_solve: ") + cudaGetErrorString(_e);          \
      rc = FAST_GPU_ECUDA;                                                         \
      goto done;                                                                   \
    }                                                                              \
  } while (0)
#define ARC(call)                      \
  do {                                 \
    rc = (call);                       \
    if (rc != FAST_GPU_OK) goto done;  \
  } while (0)

extern "C" int fast_gpu_arclength_solve(fast_gpu_ctx *c, const double *q_host, const fast_gpu_arc_opts *o,
                                        double *u_hist, double *lambda_hist, int32_t *iters,
                                        fast_gpu_arc_report *rep) {
  if (!c || !q_host || !o || o->steps <= 0 || o->max_iter <= 0) return FAST_GPU_EINVAL;
  if (o->method < FAST_ARC_INITIAL_NORMAL || o->method > FAST_ARC_LINEARIZED) return FAST_GPU_EINVAL;
  if (c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  if (!c->d_K || c->neq <= 0) { c->err = "arclength_solve: no mesh"; return FAST_GPU_ESTATE; }
  const int32_t n = c->neq;
  const size_t nb = sizeof(double) * n;
  const unsigned G = 148, T = 256;
  Work w;
  int rc = FAST_GPU_OK;
  fast_gpu_arc_report R{};
  double lam = 0.0, arclen = 0.0, lenq = 0.0, cf = o->load_coeff, sp0 = 1.0, csp1 = 1.0;
  int prev_iter = 0;

  // dot products of up to six pairs, read back (one synchronisation)
  auto dots = [&](std::initializer_list<std::pair<const double *, const double *>> pr, double *out) -> cudaError_t {
    DotArgs a{};
    int k = 0;
    for (auto &p : pr) { a.x[k] = p.first; a.y[k] = p.second; k++; }
    a.n = k;
    arc_dots<<<kArcBlocks, 256, 0, c->stream>>>(n, a, w.part);
    arc_dots_finish<<<1, 32, 0, c->stream>>>(k, w.part, w.dots);
    c->launches += 2;
    cudaError_t e = cudaMemcpyAsync(w.hdots, w.dots, sizeof(double) * k, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    for (int i = 0; i < k; i++) out[i] = w.hdots[i];
    return e;
  };
  auto axpby = [&](double a, const double *x, double b, const double *y, double *z) -> cudaError_t {
    arc_axpby<<<G, T, 0, c->stream>>>(n, a, x, b, y, z);
    c->launches++;
    return cudaGetLastError();
  };
  // x = K^-1 b, solved for b/|b| and scaled back (0 for b = 0)
  auto solve = [&](const double *b, double blen, double *x) -> int {
    if (!(blen > 0.0)) return cudaMemsetAsync(x, 0, nb, c->stream) == cudaSuccess ? FAST_GPU_OK : FAST_GPU_ECUDA;
    if (axpby(1.0 / blen, b, 0.0, b, w.rhs) != cudaSuccess) return FAST_GPU_ECUDA;
    fast_gpu_solve_opts lo = o->lin;
    lo.warm_start = 0;
    fast_gpu_solve_report lr{};
    int s = fast_gpu_solve_device(c, w.rhs, x, &lo, &lr);
    R.linear_iterations += lr.iterations;
    if (s != FAST_GPU_OK && s != FAST_GPU_ENONCONV) return s;
    return axpby(blen, x, 0.0, x, x) == cudaSuccess ? FAST_GPU_OK : FAST_GPU_ECUDA;
  };

  {
    cudaError_t e = cudaSuccess;
    double **bufs[] = {&w.q, &w.r, &w.u, &w.du1, &w.du2, &w.Du, &w.Du0, &w.g, &w.rhs};
    for (double **b : bufs)
      if (e == cudaSuccess) e = cudaMalloc((void **)b, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.part, sizeof(double) * 6 * kArcBlocks);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.dots, sizeof(double) * 6);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&w.hdots, sizeof(double) * 6);
    ACK(e);
  }
  ACK(cudaMemcpyAsync(w.q, q_host, nb, cudaMemcpyHostToDevice, c->stream));
  for (double *v : {w.r, w.u, w.Du, w.Du0}) ACK(cudaMemsetAsync(v, 0, nb, c->stream));
  {
    double h[1];
    ACK(dots({{w.q, w.q}}, h));
    lenq = std::sqrt(h[0]);
  }
  ARC(fast_gpu_set_displacement_device(c, w.u));

  for (int step = 1; step <= o->steps; step++) {
    bool conv = false;
    double Dlf = 0.0, err = 0.0, rlen = 0.0;
    int it;
    {
      double h[1];
      ACK(dots({{w.r, w.r}}, h));
      rlen = std::sqrt(h[0]);
    }
    for (it = 1; it <= o->max_iter; it++) {
      ARC(fast_gpu_assemble(c, FAST_ASM_STIFFNESS));  // tangent at u
      R.iterations++;
      ARC(solve(w.q, lenq, w.du1));
      ARC(solve(w.r, rlen, w.du2));
      // IncLoadFac (ctrl/ctrlarclen.cpp): the Du of the last step decides the
      // sign at the first iteration, the step's own Du the later corrections
      double h[6];
      double dlf;
      if (step == 1 && it == 1) {
        ACK(dots({{w.du1, w.du1}}, h));
        arclen = o->step_factor * (std::sqrt(h[0]) + cf);
        dlf = o->step_factor;
      } else if (it == 1) {
        if (o->target_iter) arclen *= std::sqrt((double)o->target_iter / (double)prev_iter);
        ACK(dots({{w.du1, w.du1}, {w.du1, w.Du}, {w.Du, w.Du}}, h));
        if (cf == 1.0 && (std::fabs(csp1) < 0.3 || std::sqrt(h[2]) > o->tol)) {  // cCtrlArcLength::FirstIncLoadFac
          arclen = std::sqrt(h[2]);
          cf = 0.0;
        }
        dlf = arclen / (std::sqrt(h[0]) + cf);
        if (h[1] < 0.0) dlf = -dlf;
      } else if (o->method == FAST_ARC_INITIAL_NORMAL) {
        ACK(dots({{w.Du0, w.du2}, {w.Du0, w.du1}}, h));
        dlf = h[0] / (h[1] + cf * Dlf);
      } else if (o->method == FAST_ARC_UPDATED_NORMAL) {
        ACK(dots({{w.Du, w.du2}, {w.Du, w.du1}}, h));
        dlf = h[0] / (h[1] + cf * Dlf);
      } else {
        ACK(dots({{w.Du, w.du2}, {w.Du, w.du1}, {w.Du, w.Du}}, h));
        const double r0 = h[2] + cf * Dlf * Dlf - arclen * arclen;
        dlf = (h[0] - 0.5 * r0) / (h[1] + cf * Dlf);
      }
      if (it == 1) {
        if (o->method == FAST_ARC_INITIAL_NORMAL) ACK(axpby(dlf, w.du1, 0.0, w.du1, w.Du0));
        ACK(cudaMemsetAsync(w.Du, 0, nb, c->stream));
        Dlf = 0.0;
      }
      Dlf += dlf;
      lam += dlf;
      // du = dlf du1 - du2 (kept in du2); u += du; Du += du
      ACK(axpby(dlf, w.du1, -1.0, w.du2, w.du2));
      ACK(axpby(1.0, w.u, 1.0, w.du2, w.u));
      ACK(axpby(1.0, w.Du, 1.0, w.du2, w.Du));
      ARC(fast_gpu_set_displacement_device(c, w.u));
      ARC(fast_gpu_internal_force_device(c, w.g));
      ACK(axpby(1.0, w.g, -lam, w.q, w.r));  // r = g - lambda q
      ACK(dots({{w.r, w.r}}, h));
      rlen = std::sqrt(h[0]);
      err = rlen / std::max(1.0, lenq);
      R.last_err = err;
      if (err < o->tol) { conv = true; break; }
      if (!std::isfinite(err)) break;
    }
    if (iters) iters[step - 1] = conv ? it : -1;
    if (!conv) {
      c->err = "arclength_solve: iterations did not converge";
      R.failed_step = step;
      rc = FAST_GPU_ENONCONV;
      goto done;
    }
    {
      double h[2];
      ACK(dots({{w.q, w.du1}, {w.du1, w.du1}}, h));
      const double spv = std::sqrt(h[1]) > 1e-12 ? h[0] / h[1] : 1.0;
      if (step == 1) sp0 = spv; else csp1 = spv / sp0;
    }
    prev_iter = it;
    R.converged_steps = step;
    R.arc_length = arclen;
    if (lambda_hist) lambda_hist[step - 1] = lam;
    if (u_hist) {
      ACK(cudaMemcpyAsync(u_hist + (size_t)(step - 1) * n, w.u, nb, cudaMemcpyDeviceToHost, c->stream));
      ACK(cudaStreamSynchronize(c->stream));
    }
  }
done:
  if (rep) *rep = R;
  if (w.hdots) cudaFreeHost(w.hdots);
  for (double *p : {w.q, w.r, w.u, w.du1, w.du2, w.Du, w.Du0, w.g, w.rhs, w.part, w.dots})
    if (p) cudaFree(p);
  return rc;
}

// nr.cu - load-control Newton-Raphson on the device.
//
// Mirrors cCtrlNR::Solver (ctrl/ctrlnr.cpp:47-270) with proportional loading:
//
//   q = external load, u = 0, g = IntForce(u), lambda = 0
//   for each step: lambda += dlambda; f = lambda q; r = f - g
//     for each iteration: K = tangent at u; solve K du = r; u += du;
//                         g = IntForce(u); r = f - g
//                         converged when |r| / max(1, |f|) < tol
//                         (cControl::Convergence, ctrl/ctrl.cpp:1366-1413)
//
// Everything stays on the device; the host reads two norms per iteration.
// After the first iteration of a solve, every iteration is replayed as one
// captured CUDA graph (tangent assembly, preconditioner, the whole PCG as a
// conditional WHILE node, update, internal force, residual norms): one host
// wait per Newton iteration.
// The reference starts each step from the last converged u; a secant
// predictor (u_k + (u_k - u_{k-1}) for equal steps) and a caller-supplied
// predictor (e.g. a learned one) can start it elsewhere.  A predicted start is
// only taken if its residual is smaller than the residual of the secant
// start; Newton always iterates to the same tolerance.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace fastgpu {

namespace {

constexpr int kNrBlocks = 592;

__global__ void nr_axpby(int32_t n, double a, const double *__restrict__ x, double b, const double *__restrict__ y,
                         double *__restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = a * x[i] + b * y[i];
}

__device__ __forceinline__ double nr_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// fixed-order sums of squares of two vectors: part[0][blk], part[1][blk]
__global__ void __launch_bounds__(256) nr_sumsq2(int32_t n, const double *__restrict__ x, const double *__restrict__ y,
                                                double *__restrict__ part) {
  __shared__ double s0[8], s1[8];
  double a = 0.0, b = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    a += x[i] * x[i];
    if (y) b += y[i] * y[i];
  }
  a = nr_warp_sum(a);
  b = nr_warp_sum(b);
  if ((threadIdx.x & 31) == 0) { s0[threadIdx.x >> 5] = a; s1[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < 8; w++) { ta += s0[w]; tb += s1[w]; }
    part[blockIdx.x] = ta;
    part[kNrBlocks + blockIdx.x] = tb;
  }
}

__global__ void __launch_bounds__(256) nr_finish2(const double *__restrict__ part, double *__restrict__ out) {
  __shared__ double s0[8], s1[8];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < kNrBlocks; i += blockDim.x) { a += part[i]; b += part[kNrBlocks + i]; }
  a = nr_warp_sum(a);
  b = nr_warp_sum(b);
  if ((threadIdx.x & 31) == 0) { s0[threadIdx.x >> 5] = a; s1[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < 8; w++) { ta += s0[w]; tb += s1[w]; }
    out[0] = ta;
    out[1] = tb;
  }
}

// graph-replayed iteration: the linear tolerance (inexact Newton, the same
// formula as the host path) and the right-hand side scaling from the device
// norms; par[0] tolerance, par[1] 1/|r|, par[2] |r| (1 when r = 0)
__global__ void nr_lin_params(const double *__restrict__ sums, double tol, double rel, double tmin, double tmax,
                              double fixed_tol, double *__restrict__ par) {
  const double rlen = sqrt(sums[0]), flen = sqrt(sums[1]);
  double lt = fixed_tol;
  if (rel > 0) {
    const double err = rlen / fmax(1.0, flen);
    const double eta = fmax(rel * err, err > 0 ? 0.5 * tol / err : 1.0);
    lt = fmin(tmax, fmax(tmin, eta));
  }
  par[0] = lt;
  par[1] = rlen > 0 ? 1.0 / rlen : 1.0;
  par[2] = rlen > 0 ? rlen : 1.0;
}

// z = par[k] x (+ y when y is given)
__global__ void nr_scaled(int32_t n, const double *__restrict__ par, int k, const double *__restrict__ x,
                          const double *__restrict__ y, double *__restrict__ z) {
  const double a = par[k];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = y ? 1.0 * y[i] + a * x[i] : a * x[i] + 0.0 * x[i];
}

// what the host reads after a replayed iteration
struct NrIterOut {
  double rlen2, flen2;
  int32_t lin_iters, lin_done, status, pad;
};

__global__ void nr_collect(const double *__restrict__ sums, const PcgState *__restrict__ st,
                           const int32_t *__restrict__ status, NrIterOut *__restrict__ out) {
  out->rlen2 = sums[0];
  out->flen2 = sums[1];
  out->lin_iters = st->iter;
  out->lin_done = st->done;
  out->status = *status;
}

}  // namespace

struct NrWork {
  double *q = nullptr, *f = nullptr, *g = nullptr, *r = nullptr, *u = nullptr, *du = nullptr, *up = nullptr,
         *ucand = nullptr, *gsave = nullptr, *part = nullptr, *sums = nullptr, *hsums = nullptr;
  double *par = nullptr;                 // [3] linear tolerance, 1/|r|, |r|
  NrIterOut *d_out = nullptr, *h_out = nullptr;
  cudaGraphExec_t graph = nullptr;       // one Newton iteration, captured
};

// Records one Newton iteration (after the residual norms of the current u are
// in w.sums) as a graph: tangent at u (zero, every colour, TL buckets), its
// solve copies and preconditioner, the linear tolerance and the scaled
// right-hand side on the device, the whole PCG (conditional WHILE node),
// u += |r| du, the internal force at the new u, r = f - g, its norms, and a
// copy of what the host needs into pinned memory.
static cudaError_t capture_iteration(Ctx &c, NrWork &w, const fast_gpu_nr_opts *o, bool mixed, int64_t *kernels) {
  const fast_gpu_solve_opts &lo = o->lin;
  const int32_t n = c.neq;
  const int maxit = lo.maxit > 0 ? lo.maxit : std::max(20 * c.neq, 100);
  // a mixed solve's FP64 residual every 50 FP32 iterations, the direct
  // solves' chunk (measured on the TL plate's Newton run: 16 -> 133.7, 32 ->
  // 127.2, 50 -> 124.5, 64 -> 122.6 ms; 128 stalls the refinement and doubles
  // the PCG iterations), every 16 for linear tolerances below 1e-10, which
  // need the more frequent corrections
  const int chunk = lo.check_every > 0 ? lo.check_every : (mixed ? (lo.tol > 0 && lo.tol < 1e-10 ? 16 : 50) : 32);
  const double tol = o->tol > 0 ? o->tol : 1e-5;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  const int64_t before = c.launches;
  cudaError_t el = cudaMemsetAsync(c.d_status, 0, sizeof(int32_t), c.stream);
  // tangent at u (c.d_disp already holds u)
  if (el == cudaSuccess) el = launch_zero_matrix(c, c.d_K, true);
  if (el == cudaSuccess) el = launch_assemble(c, FAST_ASM_STIFFNESS, c.d_K);
  if (el == cudaSuccess) el = launch_tl(c, c.d_K, nullptr, true, false);
  if (el == cudaSuccess) el = launch_to_soa(c, c.d_K, c.d_Ks, mixed ? c.d_Ks32 : nullptr);
  if (el == cudaSuccess) el = launch_build_precond(c, c.d_K, lo.precond);
  // K du = r / |r| with the inexact-Newton tolerance
  if (el == cudaSuccess) {
    nr_lin_params<<<1, 1, 0, c.stream>>>(w.sums, tol, o->lin_tol_rel, o->lin_tol_min > 0 ? o->lin_tol_min : 1e-12,
                                         o->lin_tol_max > 0 ? o->lin_tol_max : 1e-2, lo.tol > 0 ? lo.tol : 1e-5,
                                         w.par);
    nr_scaled<<<kNrBlocks, 256, 0, c.stream>>>(n, w.par, 1, w.r, nullptr, w.ucand);
    c.launches += 2;
    el = launch_eq_to_node(c, w.ucand, c.d_f);
  }
  if (el == cudaSuccess) el = record_pcg(c, mixed, false, 1e-5, w.par, maxit, chunk);
  if (el == cudaSuccess) el = launch_node_to_eq(c, c.d_u, w.du);
  if (el == cudaSuccess) {
    nr_scaled<<<kNrBlocks, 256, 0, c.stream>>>(n, w.par, 2, w.du, w.u, w.u);  // u += |r| du
    c.launches++;
    el = launch_eq_to_node(c, w.u, c.d_disp);
  }
  // internal force at the new u, residual and norms
  if (el == cudaSuccess) el = cudaMemsetAsync(c.d_gint, 0, sizeof(double) * 4 * c.nnode, c.stream);
  if (el == cudaSuccess) el = launch_tl(c, nullptr, c.d_gint, false, true);
  if (el == cudaSuccess) el = launch_node_to_eq(c, c.d_gint, w.g);
  if (el == cudaSuccess) {
    nr_axpby<<<kNrBlocks, 256, 0, c.stream>>>(n, 1.0, w.f, -1.0, w.g, w.r);
    nr_sumsq2<<<kNrBlocks, 256, 0, c.stream>>>(n, w.r, w.f, w.part);
    nr_finish2<<<1, 256, 0, c.stream>>>(w.part, w.sums);
    nr_collect<<<1, 1, 0, c.stream>>>(w.sums, c.d_state, c.d_status, w.d_out);
    c.launches += 4;
    el = cudaMemcpyAsync(w.h_out, w.d_out, sizeof(NrIterOut), cudaMemcpyDeviceToHost, c.stream);
  }
  if (el == cudaSuccess) el = cudaGetLastError();
  e = cudaStreamEndCapture(c.stream, &g);
  *kernels = c.launches - before;   // kernels of one replay outside the PCG loop's chunks
  c.launches = before;
  if (el != cudaSuccess) e = el;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&w.graph, g, 0);
  if (g) cudaGraphDestroy(g);
  return e;
}

static cudaError_t axpby(Ctx &c, double a, const double *x, double b, const double *y, double *z) {
  nr_axpby<<<kNrBlocks, 256, 0, c.stream>>>(c.neq, a, x, b, y, z);
  c.launches++;
  return cudaGetLastError();
}

// |x|^2 and |y|^2 read back to the host (y may be null)
static cudaError_t norms2(Ctx &c, NrWork &w, const double *x, const double *y, double *nx, double *ny) {
  nr_sumsq2<<<kNrBlocks, 256, 0, c.stream>>>(c.neq, x, y, w.part);
  nr_finish2<<<1, 256, 0, c.stream>>>(w.part, w.sums);
  c.launches += 2;
  cudaError_t e = cudaMemcpyAsync(w.hsums, w.sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  *nx = w.hsums[0];
  if (ny) *ny = w.hsums[1];
  return e;
}

}  // namespace fastgpu

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

#define NRCK(call)                                                           \
  do {                                                                       \
    cudaError_t _e = (call);                                                 \
    if (_e != cudaSuccess) {                                                 \
      c->err = std::string("nr_solve: ") + cudaGetErrorString(_e);          \
      rc = FAST_GPU_ECUDA;                                                   \
      goto done;                                                             \
    }                                                                        \
  } while (0)
#define NRRC(call)                   \
  do {                               \
    rc = (call);                     \
    if (rc != FAST_GPU_OK) goto done; \
  } while (0)

extern "C" int fast_gpu_nr_solve(fast_gpu_ctx *c, const double *q_host, const fast_gpu_nr_opts *o,
                                 fast_gpu_nr_predictor predictor, void *predictor_user, double *u_hist,
                                 int32_t *iters, fast_gpu_nr_report *rep) {
  if (c && c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  if (!c || !q_host || !o || o->steps <= 0 || o->max_iter <= 0) return FAST_GPU_EINVAL;
  if (!c->d_K) { c->err = "nr_solve: no mesh"; return FAST_GPU_ESTATE; }
  const int32_t n = c->neq;
  const size_t nb = sizeof(double) * n;
  NrWork w;
  int rc = FAST_GPU_OK;
  fast_gpu_nr_report R{};
  double lam = 0.0, flen2 = 0.0, rlen2 = 0.0, glen2 = 0.0, best = 0.0;
  int64_t graph_kernels = 0;
  bool graph_refused = false;
  std::vector<double> hq;
  const double tol = o->tol > 0 ? o->tol : 1e-5;
  if (n <= 0) return FAST_GPU_EINVAL;
  {
    cudaError_t e = cudaSuccess;
    double **bufs[] = {&w.q, &w.f, &w.g, &w.r, &w.u, &w.du, &w.up, &w.ucand, &w.gsave};
    for (double **b : bufs)
      if (e == cudaSuccess) e = cudaMalloc((void **)b, nb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.part, sizeof(double) * 2 * kNrBlocks);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.sums, sizeof(double) * 2);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&w.hsums, sizeof(double) * 2);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.par, sizeof(double) * 3);
    if (e == cudaSuccess) e = cudaMalloc((void **)&w.d_out, sizeof(NrIterOut));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&w.h_out, sizeof(NrIterOut));
    NRCK(e);
  }
  hq.assign(q_host, q_host + n);
  NRCK(cudaMemcpyAsync(w.q, hq.data(), nb, cudaMemcpyHostToDevice, c->stream));
  NRCK(cudaMemsetAsync(w.u, 0, nb, c->stream));
  NRCK(cudaMemsetAsync(w.up, 0, nb, c->stream));
  NRRC(fast_gpu_set_displacement_device(c, w.u));
  NRRC(fast_gpu_internal_force_device(c, w.g));  // initial stresses (zero for these models)

  for (int step = 1; step <= o->steps; step++) {
    lam += o->step_factor;
    NRCK(axpby(*c, lam, w.q, 0.0, w.q, w.f));  // f = lambda q

    // start of the step: the last converged u (the reference), the secant
    // extrapolation 2 u_k - u_{k-1} (equal load steps), or the caller's
    // prediction when its residual is smaller than the secant start's
    // Each candidate start is evaluated once: the chosen one's displacement
    // (set on the device), g, r = f - g and norms (w.sums: |r|^2, |f|^2) are
    // kept for the first iteration instead of being formed again.
    NRCK(cudaMemcpyAsync(w.ucand, w.u, nb, cudaMemcpyDeviceToDevice, c->stream));
    bool have_r = false;
    if (step >= 2 && o->predictor != FAST_NR_PREDICT_NONE) {
      NRCK(axpby(*c, 2.0, w.u, -1.0, w.up, w.ucand));
      NRRC(fast_gpu_set_displacement_device(c, w.ucand));
      NRRC(fast_gpu_internal_force_device(c, w.g));
      NRCK(axpby(*c, 1.0, w.f, -1.0, w.g, w.r));
      NRCK(norms2(*c, w, w.r, w.f, &best, &flen2));
      rlen2 = best;
      have_r = true;
      R.secant_starts++;
      if (o->predictor == FAST_NR_PREDICT_CALLBACK && predictor) {
        // the caller writes its prediction of u at this load level into du
        NRCK(cudaMemcpyAsync(w.gsave, w.g, nb, cudaMemcpyDeviceToDevice, c->stream));
        const int prc = predictor(predictor_user, step, lam, w.u, w.up, w.f, w.du);
        if (prc == 0) {
          NRRC(fast_gpu_set_displacement_device(c, w.du));
          NRRC(fast_gpu_internal_force_device(c, w.g));
          NRCK(axpby(*c, 1.0, w.f, -1.0, w.g, w.r));
          double rl = 0.0;
          NRCK(norms2(*c, w, w.r, w.f, &rl, &flen2));
          R.predictions++;
          if (rl < best) {
            R.predictions_accepted++;
            rlen2 = rl;
            NRCK(cudaMemcpyAsync(w.ucand, w.du, nb, cudaMemcpyDeviceToDevice, c->stream));
          } else {
            // back to the secant start's state
            NRCK(cudaMemcpyAsync(w.g, w.gsave, nb, cudaMemcpyDeviceToDevice, c->stream));
            NRCK(axpby(*c, 1.0, w.f, -1.0, w.g, w.r));
            NRRC(fast_gpu_set_displacement_device(c, w.ucand));
            NRCK(norms2(*c, w, w.r, w.f, &rlen2, &flen2));
          }
        } else {
          // the predictor's own evaluations may have moved the displacement
          NRRC(fast_gpu_set_displacement_device(c, w.ucand));
        }
      }
    }
    NRCK(cudaMemcpyAsync(w.up, w.u, nb, cudaMemcpyDeviceToDevice, c->stream));  // last converged
    NRCK(cudaMemcpyAsync(w.u, w.ucand, nb, cudaMemcpyDeviceToDevice, c->stream));
    if (!have_r) {
      NRRC(fast_gpu_set_displacement_device(c, w.u));
      NRRC(fast_gpu_internal_force_device(c, w.g));
      NRCK(axpby(*c, 1.0, w.f, -1.0, w.g, w.r));  // r = f - g
      NRCK(norms2(*c, w, w.r, w.f, &rlen2, &flen2));
    }

    int conv = 0, it = 0;
    bool start_ok = false;
    if (step >= 2 && o->predictor != FAST_NR_PREDICT_NONE) {
      // a predicted start may already meet the tolerance (never the case for
      // the reference's start, which carries the whole load increment)
      const double flen = std::sqrt(flen2), rlen = std::sqrt(rlen2);
      double err;
      if (flen > tol) {
        err = rlen / std::max(1.0, flen);
      } else {
        NRCK(norms2(*c, w, w.g, nullptr, &glen2, nullptr));
        err = rlen / std::max(1.0, std::sqrt(glen2));
      }
      if (err < tol) {
        conv = 1;
        start_ok = true;
        R.last_err = err;
        R.last_rel_residual = flen > 0 ? rlen / flen : rlen;
      }
    }
    for (it = 1; !conv && it <= o->max_iter; it++) {
      if (w.graph) {
        // the iteration replayed as one graph: one host wait per iteration
        NRCK(cudaGraphLaunch(w.graph, c->stream));
        c->launches += graph_kernels;
        NRCK(cudaStreamSynchronize(c->stream));
        const NrIterOut &io = *w.h_out;
        c->K_ok = true;
        c->K32_current = false;
        c->Ks_ok = true;
        c->precond_built = o->lin.precond;
        if (io.status & 1) {
          c->err = "assemble: non-positive Jacobian determinant in at least one element";
          rc = FAST_GPU_EDETJ;
          goto done;
        }
        R.linear_iterations += io.lin_iters;
        rlen2 = io.rlen2;
        flen2 = io.flen2;
      } else {
      NRRC(fast_gpu_assemble(c, FAST_ASM_STIFFNESS));  // tangent at u
      fast_gpu_solve_opts lo = o->lin;
      if (o->lin_tol_rel > 0) {
        // inexact Newton: the forcing term follows the current residual, but
        // never asks for more than what takes this iteration to the Newton
        // tolerance (eta >= tol / (2 |r|), the safeguard of Kelley, Solving
        // Nonlinear Equations with Newton's Method, SIAM 2003, sec. 3.2.3)
        const double err = std::sqrt(rlen2) / std::max(1.0, std::sqrt(flen2));
        const double eta = std::max(o->lin_tol_rel * err, err > 0 ? 0.5 * tol / err : 1.0);
        lo.tol = std::min(o->lin_tol_max > 0 ? o->lin_tol_max : 1e-2,
                          std::max(o->lin_tol_min > 0 ? o->lin_tol_min : 1e-12, eta));
      }
      fast_gpu_solve_report lr{};
      NRCK(cudaMemsetAsync(w.du, 0, nb, c->stream));
      {
        // K du = r solved for the unit right-hand side r / |r|: PCGSolver's
        // early exit on an absolute |rhs| < tol would otherwise return du = 0
        // once the Newton residual falls below a loose relative tolerance
        const double rn = std::sqrt(rlen2);
        const double sc = rn > 0 ? 1.0 / rn : 1.0;
        NRCK(axpby(*c, sc, w.r, 0.0, w.r, w.ucand));
        rc = fast_gpu_solve_device(c, w.ucand, w.du, &lo, &lr);
        R.linear_iterations += lr.iterations;
        if (rc != FAST_GPU_OK && rc != FAST_GPU_ENONCONV) goto done;
        rc = FAST_GPU_OK;
        NRCK(axpby(*c, 1.0, w.u, rn > 0 ? rn : 1.0, w.du, w.u));  // u += |r| du
      }
      NRRC(fast_gpu_set_displacement_device(c, w.u));
      NRRC(fast_gpu_internal_force_device(c, w.g));
      NRCK(axpby(*c, 1.0, w.f, -1.0, w.g, w.r));  // r = f - g
      NRCK(norms2(*c, w, w.r, w.f, &rlen2, &flen2));
      // every later iteration replays this one as a captured graph (the
      // solve copies and work buffers exist now)
      if (c->graph_steps && !c->timing && !w.graph && !graph_refused &&
          capture_iteration(*c, w, o, o->lin.precision == FAST_PREC_MIXED, &graph_kernels) != cudaSuccess) {
        // capture refused (nothing of it ran): go on kernel by kernel
        (void)cudaGetLastError();
        w.graph = nullptr;
        graph_refused = true;
      }
      }
      R.iterations++;
      const double flen = std::sqrt(flen2), rlen = std::sqrt(rlen2);
      double err;
      if (flen > tol) {
        err = rlen / std::max(1.0, flen);
      } else {
        NRCK(norms2(*c, w, w.g, nullptr, &glen2, nullptr));
        err = rlen / std::max(1.0, std::sqrt(glen2));
      }
      R.last_err = err;
      R.last_rel_residual = flen > 0 ? rlen / flen : rlen;
      if (err < tol) { conv = 1; break; }
      if (!std::isfinite(err)) break;
    }
    if (iters) iters[step - 1] = conv ? (start_ok ? 0 : it) : -1;
    if (!conv) {
      c->err = "nr_solve: Newton iterations did not converge (\"Convergence not achived\")";
      R.failed_step = step;
      rc = FAST_GPU_ENONCONV;
      goto done;
    }
    R.converged_steps = step;
    if (u_hist) {
      NRCK(cudaMemcpyAsync(u_hist + (size_t)(step - 1) * n, w.u, nb, cudaMemcpyDeviceToHost, c->stream));
      NRCK(cudaStreamSynchronize(c->stream));
    }
  }
done:
  if (rep) *rep = R;
  if (w.graph) cudaGraphExecDestroy(w.graph);
  if (w.hsums) cudaFreeHost(w.hsums);
  if (w.h_out) cudaFreeHost(w.h_out);
  if (w.par) cudaFree(w.par);
  if (w.d_out) cudaFree(w.d_out);
  for (double *p : {w.q, w.f, w.g, w.r, w.u, w.du, w.up, w.ucand, w.gsave, w.part, w.sums})
    if (p) cudaFree(p);
  return rc;
}

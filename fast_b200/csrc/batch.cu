// batch.cu - many independent problems in one context (fast_gpu_set_problems,
// fast_gpu_solve_batch).  Each problem is what one FAST run of cLinStat
// (ctrl/ctrllins.cpp:46-99) solves: its own mesh, load and PCGSolver
// (mlib/sysmat.cpp:1061-1125) stopping test.  The meshes are uploaded as one
// mesh with disjoint node ranges, so assembly, the block pattern and the
// solve layout are those of a single system whose matrix is block diagonal;
// the solve runs one CTA per problem in a single launch.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

void free_problems(Ctx &c) {
  for (void *p : {(void *)c.d_noff, (void *)c.d_order, (void *)c.d_piters, (void *)c.d_pdone, (void *)c.d_perr})
    if (p) cudaFree(p);
  c.d_noff = nullptr;
  c.d_order = nullptr;
  c.d_piters = nullptr;
  c.d_pdone = nullptr;
  c.d_perr = nullptr;
  c.nprob = 0;
  c.h_noff.clear();
}

}  // namespace

#define BCK(call)                                                              \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) {                                                   \
      c->err = std::string(#call) + ": " + cudaGetErrorString(_e);            \
      return FAST_GPU_ECUDA;                                                   \
    }                                                                          \
  } while (0)

extern "C" int fast_gpu_set_problems(fast_gpu_ctx *c, int32_t num_problems, const int64_t *node_offsets) {
  if (c && c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  if (!c || num_problems <= 0 || !node_offsets) return FAST_GPU_EINVAL;
  if (c->nnode <= 0) { c->err = "set_problems: no mesh"; return FAST_GPU_ESTATE; }
  std::vector<int64_t> off(node_offsets, node_offsets + num_problems + 1);
  if (off[0] != 0 || off[num_problems] != c->nnode) {
    c->err = "set_problems: node offsets must run from 0 to the number of nodes";
    return FAST_GPU_EINVAL;
  }
  for (int k = 0; k < num_problems; k++)
    if (off[k + 1] < off[k]) { c->err = "set_problems: node offsets must not decrease"; return FAST_GPU_EINVAL; }
  // no block of the pattern may couple two problems
  for (int k = 0; k < num_problems; k++)
    for (int64_t n = off[k]; n < off[k + 1]; n++)
      for (int32_t b = c->h_rowptr[n]; b < c->h_rowptr[n + 1]; b++) {
        const int64_t j = c->h_col[b];
        if (j < off[k] || j >= off[k + 1]) {
          c->err = "set_problems: an element couples node " + std::to_string(n) + " of problem " + std::to_string(k) +
                   " with node " + std::to_string(j) + " of another problem";
          return FAST_GPU_EINVAL;
        }
      }
  free_problems(*c);
  std::vector<int32_t> order(num_problems);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return (off[a + 1] - off[a]) > (off[b + 1] - off[b]);
  });
  BCK(cudaMalloc((void **)&c->d_noff, sizeof(int64_t) * (num_problems + 1)));
  BCK(cudaMalloc((void **)&c->d_order, sizeof(int32_t) * num_problems));
  BCK(cudaMalloc((void **)&c->d_piters, sizeof(int32_t) * num_problems));
  BCK(cudaMalloc((void **)&c->d_pdone, sizeof(int32_t) * num_problems));
  BCK(cudaMalloc((void **)&c->d_perr, sizeof(double) * num_problems));
  BCK(cudaMemcpy(c->d_noff, off.data(), sizeof(int64_t) * (num_problems + 1), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(c->d_order, order.data(), sizeof(int32_t) * num_problems, cudaMemcpyHostToDevice));
  c->nprob = num_problems;
  c->h_noff = off;
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_solve_batch(fast_gpu_ctx *c, const double *f, double *u, const fast_gpu_solve_opts *o,
                                    fast_gpu_problem_report *reps) {
  if (!c || !f || !u) return FAST_GPU_EINVAL;
  if (c->nprob <= 0) { c->err = "solve_batch: call fast_gpu_set_problems first"; return FAST_GPU_ESTATE; }
  if (!c->K_ok) { c->err = "solve_batch: matrix not assembled"; return FAST_GPU_ESTATE; }
  fast_gpu_solve_opts opts{};
  if (o) opts = *o;
  if (opts.precision != FAST_PREC_FP64) {
    c->err = "solve_batch: only FAST_PREC_FP64 (the reference's PCG per problem)";
    return FAST_GPU_ENOTSUP;
  }
  if (opts.precond != FAST_PRECOND_JACOBI && opts.precond != FAST_PRECOND_BLOCK_JACOBI) return FAST_GPU_EINVAL;
  const double tol = opts.tol > 0 ? opts.tol : 1e-5;
  int64_t biggest = 0;
  for (int k = 0; k < c->nprob; k++) biggest = std::max(biggest, c->h_noff[k + 1] - c->h_noff[k]);
  const int maxit = opts.maxit > 0 ? opts.maxit : (int)std::max<int64_t>(60 * biggest, 100);
  if (c->precond_built != opts.precond) BCK(launch_build_precond(*c, c->d_K, opts.precond));
  BCK(solve_layout(*c, FAST_ASM_STIFFNESS, false));
  const size_t nb = sizeof(double) * c->neq;
  BCK(cudaMemcpyAsync(c->d_eq_tmp, f, nb, cudaMemcpyHostToDevice, c->stream));
  BCK(launch_eq_to_node(*c, c->d_eq_tmp, c->d_f));
  const bool warm = opts.warm_start != 0;
  if (warm) {
    BCK(cudaMemcpyAsync(c->d_eq_tmp, u, nb, cudaMemcpyHostToDevice, c->stream));
    BCK(launch_eq_to_node(*c, c->d_eq_tmp, c->d_u));
  }
  const int64_t sp = c->begin_span(FAST_KERNEL_LINEAR_SOLVE);
  BCK(launch_pcg_batch(*c, c->nprob, c->d_order, c->d_noff, tol, maxit, warm, c->d_piters, c->d_perr, c->d_pdone));
  c->end_span(sp);
  BCK(launch_node_to_eq(*c, c->d_u, c->d_eq_tmp));
  BCK(cudaMemcpyAsync(u, c->d_eq_tmp, nb, cudaMemcpyDeviceToHost, c->stream));
  std::vector<int32_t> it(c->nprob), dn(c->nprob);
  std::vector<double> er(c->nprob);
  BCK(cudaMemcpyAsync(it.data(), c->d_piters, sizeof(int32_t) * c->nprob, cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaMemcpyAsync(dn.data(), c->d_pdone, sizeof(int32_t) * c->nprob, cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaMemcpyAsync(er.data(), c->d_perr, sizeof(double) * c->nprob, cudaMemcpyDeviceToHost, c->stream));
  BCK(cudaStreamSynchronize(c->stream));
  c->harvest();
  int bad = 0;
  for (int k = 0; k < c->nprob; k++) {
    if (reps) {
      reps[k].converged = dn[k] == 1;
      reps[k].iterations = it[k];
      reps[k].rel_residual = er[k];
    }
    if (dn[k] != 1) bad++;
  }
  if (bad) {
    c->err = "solve_batch: " + std::to_string(bad) + " problem(s) did not converge";
    return FAST_GPU_ENONCONV;
  }
  return FAST_GPU_OK;
}

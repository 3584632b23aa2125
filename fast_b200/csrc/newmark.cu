// newmark.cu - linear Newmark time integration on the device
// (fast_gpu_newmark), the loop of cCtrlNewmark::Solver
// (ctrl/ctrlnewmark.cpp:79-254), with Rayleigh damping when asked:
//
//   a0 = 1/(beta dt^2), a2 = 1/(beta dt), a3 = 1/(2 beta) - 1,
//   a6 = (1 - gamma) dt, a7 = gamma dt
//   f = ExtLoadVector (a step load: the same f at every time), M a = f
//   K_eff = K + a0 M [+ a1 C],  C = alpha M + beta K (Rayleigh)
//   each step: f_eff = f + M (a0 u + a2 v + a3 a) [+ C (a1 u + a4 v + a5 a)];  K_eff u_new = f_eff
//              du = u_new - u;  a <- -a3 a + a0 du - a2 v;  v <- v + a6 a_old + a7 a
//
// The reference factors K_eff once (skyline Crout); here every step is a PCG
// solve warm-started from the last displacements, with K_eff, M and the
// state vectors resident in HBM and the step's vector work in two fused
// kernels.  The printout's max norms (umax, vmax, amax) are kept on the
// device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

constexpr int kNmBlocks = 592;

// K <- K + s M on the AoS block values
__global__ void nm_axpy(int64_t n, double s, const double *__restrict__ M, double *__restrict__ K) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    K[i] += s * M[i];
}

// w = a0 u + a2 v + a3 a
__global__ void nm_inertia(int64_t n, double a0, double a2, double a3, const double *__restrict__ u,
                           const double *__restrict__ v, const double *__restrict__ a, double *__restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    w[i] = a0 * u[i] + a2 * v[i] + a3 * a[i];
}

// f_eff = q + z; the solver's first iterate = u
__global__ void nm_rhs(int64_t n, const double *__restrict__ q, const double *__restrict__ z,
                       const double *__restrict__ u, double *__restrict__ f, double *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    f[i] = q[i] + z[i];
    x[i] = u[i];
  }
}

// f_eff = (q + z) + z2 (inertia, then damping terms); the solver's first iterate = u
__global__ void nm_rhs2(int64_t n, const double *__restrict__ q, const double *__restrict__ z,
                        const double *__restrict__ z2, const double *__restrict__ u, double *__restrict__ f,
                        double *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    f[i] = q[i] + z[i] + z2[i];
    x[i] = u[i];
  }
}

// C = alpha M + beta K (cCtrlNewmark::DampingMatrix: C = 0, += alpha M, += beta K)
__global__ void nm_rayleigh(int64_t n, double alpha, const double *__restrict__ M, double beta,
                            const double *__restrict__ K, double *__restrict__ C) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    v += alpha * M[i];
    v += beta * K[i];
    C[i] = v;
  }
}

// ordered bits of a non-negative double (max over them is the max of the values)
__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// du = x - u; a_new = -a3 a + a0 du - a2 v; v += a6 a_old + a7 a_new; u = x; running inf-norms
__global__ void nm_update(int64_t n, double a0, double a2, double a3, double a6, double a7, const double *__restrict__ x,
                          double *__restrict__ u, double *__restrict__ v, double *__restrict__ a,
                          unsigned long long *__restrict__ maxes) {
  double mu = 0.0, mv = 0.0, ma = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double un = x[i], du = un - u[i], ao = a[i], vo = v[i];
    double an = -a3 * ao;
    an += a0 * du;
    an += -a2 * vo;
    double vn = vo + a6 * ao;
    vn += a7 * an;
    u[i] = un;
    v[i] = vn;
    a[i] = an;
    mu = fmax(mu, fabs(un));
    mv = fmax(mv, fabs(vn));
    ma = fmax(ma, fabs(an));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(maxes + 0, dbits(mu));
    atomicMax(maxes + 1, dbits(mv));
    atomicMax(maxes + 2, dbits(ma));
  }
}

__global__ void nm_amax0(int64_t n, const double *__restrict__ a, unsigned long long *__restrict__ maxes) {
  double ma = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    ma = fmax(ma, fabs(a[i]));
  for (int o = 16; o > 0; o >>= 1) ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxes + 2, dbits(ma));
}

// probe_hist[step][k] = u at equation probe[k] (node-padded index dof[probe[k]])
__global__ void nm_probe(int nprobe, const int32_t *__restrict__ probe, const int32_t *__restrict__ dof,
                         const double *__restrict__ u, double *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nprobe) out[k] = u[dof[probe[k]]];
}

// graph replays: the step number lives on the device.  stats: [0] steps done,
// [1] PCG iterations, [2] largest step count, [3] first failed step (0: none)
__global__ void nm_step_end(const PcgState *__restrict__ st, int32_t *__restrict__ stats) {
  const int32_t it = st->iter;
  stats[1] += it;
  if (it > stats[2]) stats[2] = it;
  if (st->done != 1 && stats[3] == 0) stats[3] = stats[0] + 1;
  stats[0] += 1;
}

__global__ void nm_probe_step(int nprobe, const int32_t *__restrict__ probe, const int32_t *__restrict__ dof,
                              const double *__restrict__ u, double *__restrict__ hist, const int32_t *__restrict__ stats) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  // written after nm_step_end: the step just done is stats[0] - 1
  if (k < nprobe) hist[(size_t)(stats[0] - 1) * nprobe + k] = u[dof[probe[k]]];
}

}  // namespace

#define NMCK(call)                                                            \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) {                                                  \
      c->err = std::string("newmark: ") + #call + ": " + cudaGetErrorString(_e); \
      rc = FAST_GPU_ECUDA;                                                    \
      goto done;                                                              \
    }                                                                         \
  } while (0)

// Rayleigh damping of cCtrlNewmark (ctrl/ctrlnewmark.cpp:56-59, 150-161,
// 262-278): C = alpha M + beta K with the reference's alpha, beta from
// (omega1, omega2, xi1, xi2); its SoA copy, and the work vectors of C w
struct NmDamp {
  bool on = false;
  double a1 = 0, a4 = 0, a5 = 0;
  double *C = nullptr, *Cs = nullptr, *w2 = nullptr, *z2 = nullptr;
};

// f_eff = q + M (a0 u + a2 v + a3 a) [+ C (a1 u + a4 v + a5 a)], the solver's
// first iterate = u (cCtrlNewmark::Solver, ctrl/ctrlnewmark.cpp:190-207)
static cudaError_t step_rhs(Ctx &c, int64_t n4, double a0, double a2, double a3, const double *d_q, const double *d_u,
                            const double *d_v, const double *d_a, double *d_w, double *d_z, const NmDamp &dm) {
  nm_inertia<<<kNmBlocks, 256, 0, c.stream>>>(n4, a0, a2, a3, d_u, d_v, d_a, d_w);
  c.launches++;
  cudaError_t e = launch_spmv(c, c.d_Ms, d_w, d_z);  // z = M w
  if (e != cudaSuccess) return e;
  if (dm.on) {
    nm_inertia<<<kNmBlocks, 256, 0, c.stream>>>(n4, dm.a1, dm.a4, dm.a5, d_u, d_v, d_a, dm.w2);
    c.launches++;
    if ((e = launch_spmv(c, dm.Cs, dm.w2, dm.z2)) != cudaSuccess) return e;  // z2 = C w2
    nm_rhs2<<<kNmBlocks, 256, 0, c.stream>>>(n4, d_q, d_z, dm.z2, d_u, c.d_f, c.d_u);
  } else {
    nm_rhs<<<kNmBlocks, 256, 0, c.stream>>>(n4, d_q, d_z, d_u, c.d_f, c.d_u);
  }
  c.launches++;
  return cudaGetLastError();
}

// Steps first .. steps-1 as replays of one captured step graph (the first
// step has run directly: the preconditioner and solve copies of K_eff exist).
static int graph_steps(fast_gpu_ctx *c, const fast_gpu_newmark_opts *o, int first, int64_t n4, double a0, double a2,
                       double a3, double a6, double a7, const double *d_q, double *d_u, double *d_v, double *d_a,
                       double *d_w, double *d_z, unsigned long long *d_max, int32_t nprobe, const int32_t *d_probe,
                       double *d_hist, const NmDamp &dm, fast_gpu_newmark_report &R, bool *captured) {
  int rc = FAST_GPU_OK;
  *captured = false;
  int32_t *d_stats = nullptr;
  int32_t h_stats[4] = {first, R.linear_iterations, R.max_step_iterations, 0};
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  const fast_gpu_solve_opts &lo = o->lin;
  const bool mixed = lo.precision == FAST_PREC_MIXED;
  const int maxit = lo.maxit > 0 ? lo.maxit : std::max(20 * c->neq, 100);
  const double tol = lo.tol > 0 ? lo.tol : 1e-5;
  // a mixed solve's FP64 residual every 50 FP32 iterations (the direct
  // solves' chunk: 22.1 -> 20.7 ms per step on the hex20 box at 1e-8), every
  // 16 below 1e-10, where the FP32 iteration needs the more frequent
  // corrections (the damped box to 1e-12 stops converging with 50)
  const int chunk = lo.check_every > 0 ? lo.check_every : (mixed ? (tol < 1e-10 ? 16 : 50) : 32);
  const int64_t before = c->launches;
  int64_t per_step = 0;
  NMCK(cudaMalloc((void **)&d_stats, sizeof(h_stats)));
  NMCK(cudaMemcpyAsync(d_stats, h_stats, sizeof(h_stats), cudaMemcpyHostToDevice, c->stream));
  NMCK(cudaStreamSynchronize(c->stream));
  NMCK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  {
    cudaError_t e = step_rhs(*c, n4, a0, a2, a3, d_q, d_u, d_v, d_a, d_w, d_z, dm);
    if (e == cudaSuccess) e = record_pcg(*c, mixed, lo.warm_start != 0, tol, nullptr, maxit, chunk);
    nm_step_end<<<1, 1, 0, c->stream>>>(c->d_state, d_stats);
    nm_update<<<kNmBlocks, 256, 0, c->stream>>>(n4, a0, a2, a3, a6, a7, c->d_u, d_u, d_v, d_a, d_max);
    if (nprobe > 0)
      nm_probe_step<<<(nprobe + 127) / 128, 128, 0, c->stream>>>(nprobe, d_probe, c->d_dof_of_eq, d_u, d_hist, d_stats);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
    if (e != cudaSuccess) {
      // capture refused (nothing of it ran): the caller goes on kernel by kernel
      (void)cudaGetLastError();
      ge = nullptr;
      c->launches = before;
      goto done;
    }
  }
  *captured = true;
  per_step = c->launches - before + 2 + (nprobe > 0 ? 1 : 0);
  c->launches = before;
  for (int s = first; s < o->steps; s++) {
    NMCK(cudaGraphLaunch(ge, c->stream));
    c->launches += per_step;   // the kernels of the chunks the loop ran are not counted
  }
  NMCK(cudaMemcpyAsync(h_stats, d_stats, sizeof(h_stats), cudaMemcpyDeviceToHost, c->stream));
  NMCK(cudaStreamSynchronize(c->stream));
  R.linear_iterations = h_stats[1];
  R.max_step_iterations = h_stats[2];
  R.steps_done = h_stats[3] ? h_stats[3] - 1 : h_stats[0];
  if (h_stats[3]) {
    R.failed_step = h_stats[3];
    c->err = "newmark: a step's PCG did not converge";
    rc = FAST_GPU_ENONCONV;
  }
done:
  if (ge) cudaGraphExecDestroy(ge);
  if (g) cudaGraphDestroy(g);
  if (d_stats) cudaFree(d_stats);
  return rc;
}

extern "C" int fast_gpu_newmark(fast_gpu_ctx *c, const double *q, const fast_gpu_newmark_opts *o, double *u_out,
                                double *v_out, double *a_out, int32_t nprobe, const int32_t *probe_eq,
                                double *probe_hist, fast_gpu_newmark_report *rep) {
  if (c && c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  if (!c || !q || !o || o->steps <= 0 || !(o->dt > 0) || !(o->beta > 0) || nprobe < 0 ||
      (nprobe > 0 && (!probe_eq || !probe_hist)))
    return FAST_GPU_EINVAL;
  if (!c->d_K) { c->err = "newmark: no mesh"; return FAST_GPU_ESTATE; }
  for (int k = 0; k < nprobe; k++)
    if (probe_eq[k] < 0 || probe_eq[k] >= c->neq) { c->err = "newmark: probe equation out of range"; return FAST_GPU_EINVAL; }
  const int64_t n4 = 4 * c->nnode;
  const double dt = o->dt, gamma = o->gamma, beta = o->beta;
  const double a0 = 1.0 / (beta * dt * dt), a2 = 1.0 / (beta * dt), a3 = 0.5 / beta - 1.0;
  const double a6 = (1.0 - gamma) * dt, a7 = gamma * dt;
  int rc = FAST_GPU_OK;
  fast_gpu_newmark_report R{};
  double *d_q = nullptr, *d_u = nullptr, *d_v = nullptr, *d_a = nullptr, *d_w = nullptr, *d_z = nullptr,
         *d_hist = nullptr;
  int32_t *d_probe = nullptr;
  unsigned long long *d_max = nullptr;
  unsigned long long h_max[3] = {0, 0, 0};
  fast_gpu_solve_report lr{};
  std::vector<double> tmp;
  NmDamp dm;
  dm.on = o->damping != 0;
  dm.a1 = gamma / (beta * dt);
  dm.a4 = gamma / beta - 1.0;
  dm.a5 = (0.5 * gamma / beta - 1.0) * dt;
  {
    cudaError_t e = cudaSuccess;
    for (double **b : {&d_q, &d_u, &d_v, &d_a, &d_w, &d_z})
      if (e == cudaSuccess) e = cudaMalloc((void **)b, sizeof(double) * n4);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_max, sizeof(unsigned long long) * 3);
    if (e == cudaSuccess && nprobe > 0) e = cudaMalloc((void **)&d_probe, sizeof(int32_t) * nprobe);
    if (e == cudaSuccess && nprobe > 0) e = cudaMalloc((void **)&d_hist, sizeof(double) * (size_t)nprobe * o->steps);
    NMCK(e);
  }
  for (double *b : {d_u, d_v, d_a}) NMCK(cudaMemsetAsync(b, 0, sizeof(double) * n4, c->stream));
  NMCK(cudaMemsetAsync(d_max, 0, sizeof(unsigned long long) * 3, c->stream));
  if (nprobe > 0)
    NMCK(cudaMemcpyAsync(d_probe, probe_eq, sizeof(int32_t) * nprobe, cudaMemcpyHostToDevice, c->stream));
  // the load, node-padded
  NMCK(cudaMemcpyAsync(c->d_eq_tmp, q, sizeof(double) * c->neq, cudaMemcpyHostToDevice, c->stream));
  NMCK(launch_eq_to_node(*c, c->d_eq_tmp, d_q));

  // M, then a(0) from M a = f (the solver works on the K slot: M is copied there)
  rc = fast_gpu_assemble(c, FAST_ASM_MASS);
  if (rc != FAST_GPU_OK) goto done;
  NMCK(cudaMemcpyAsync(c->d_K, c->d_M, sizeof(double) * 9 * c->nnzb, cudaMemcpyDeviceToDevice, c->stream));
  NMCK(launch_fixed_identity(*c, c->d_K));  // fixed DOFs: identity rows, as in the stiffness slot
  c->K_ok = true;
  matrix_changed(*c, FAST_ASM_STIFFNESS);
  NMCK(cudaMemcpyAsync(c->d_f, d_q, sizeof(double) * n4, cudaMemcpyDeviceToDevice, c->stream));
  rc = solve_nodes(*c, &o->mass, false, &lr);
  R.mass_iterations = lr.iterations;
  if (rc != FAST_GPU_OK) goto done;
  NMCK(cudaMemcpyAsync(d_a, c->d_u, sizeof(double) * n4, cudaMemcpyDeviceToDevice, c->stream));
  nm_amax0<<<kNmBlocks, 256, 0, c->stream>>>(n4, d_a, d_max);
  c->launches++;

  // K_eff = K + a0 M (+ a1 C)
  rc = fast_gpu_assemble(c, FAST_ASM_STIFFNESS);
  if (rc != FAST_GPU_OK) goto done;
  if (dm.on) {
    const double w1 = o->omega1, w2 = o->omega2, x1 = o->xi1, x2 = o->xi2;
    const double alphar = 2 * w1 * w2 * (x1 * w2 - x2 * w1) / (w2 * w2 - w1 * w1);
    const double betar = 2 * (x2 * w2 - x1 * w1) / (w2 * w2 - w1 * w1);
    const size_t nv = (size_t)9 * c->nnzb_pad;
    NMCK(cudaMalloc((void **)&dm.C, sizeof(double) * 9 * c->nnzb));
    NMCK(cudaMalloc((void **)&dm.Cs, sizeof(double) * nv));
    NMCK(cudaMemsetAsync(dm.Cs, 0, sizeof(double) * nv, c->stream));  // padding stays zero
    NMCK(cudaMalloc((void **)&dm.w2, sizeof(double) * n4));
    NMCK(cudaMalloc((void **)&dm.z2, sizeof(double) * n4));
    nm_rayleigh<<<kNmBlocks, 256, 0, c->stream>>>(9 * c->nnzb, alphar, c->d_M, betar, c->d_K, dm.C);
    c->launches++;
    NMCK(launch_to_soa(*c, dm.C, dm.Cs, nullptr));
  }
  nm_axpy<<<kNmBlocks, 256, 0, c->stream>>>(9 * c->nnzb, a0, c->d_M, c->d_K);
  c->launches++;
  if (dm.on) {
    nm_axpy<<<kNmBlocks, 256, 0, c->stream>>>(9 * c->nnzb, dm.a1, dm.C, c->d_K);
    c->launches++;
  }
  matrix_changed(*c, FAST_ASM_STIFFNESS);
  NMCK(solve_layout(*c, FAST_ASM_MASS, false));

  for (int s = 0; s < o->steps; s++) {
    if (s == 1 && c->graph_steps) {
      // every later step replays one captured graph: right-hand side, the
      // whole PCG (a WHILE node over chunks of iterations), update, probes
      bool captured = false;
      rc = graph_steps(c, o, s, n4, a0, a2, a3, a6, a7, d_q, d_u, d_v, d_a, d_w, d_z, d_max, nprobe, d_probe, d_hist,
                       dm, R, &captured);
      if (rc != FAST_GPU_OK) goto done;
      if (captured) break;
    }
    NMCK(step_rhs(*c, n4, a0, a2, a3, d_q, d_u, d_v, d_a, d_w, d_z, dm));
    rc = solve_nodes(*c, &o->lin, o->lin.warm_start != 0, &lr);
    R.linear_iterations += lr.iterations;
    if (lr.iterations > R.max_step_iterations) R.max_step_iterations = lr.iterations;
    if (lr.escalated) R.escalated_steps++;
    if (rc != FAST_GPU_OK) { R.failed_step = s + 1; goto done; }
    nm_update<<<kNmBlocks, 256, 0, c->stream>>>(n4, a0, a2, a3, a6, a7, c->d_u, d_u, d_v, d_a, d_max);
    c->launches++;
    if (nprobe > 0) {
      nm_probe<<<(nprobe + 127) / 128, 128, 0, c->stream>>>(nprobe, d_probe, c->d_dof_of_eq, d_u,
                                                             d_hist + (size_t)s * nprobe);
      c->launches++;
    }
    R.steps_done = s + 1;
  }
  NMCK(cudaGetLastError());
  tmp.resize(c->neq);
  for (int k = 0; k < 3; k++) {
    double *src = k == 0 ? d_u : (k == 1 ? d_v : d_a);
    double *dst = k == 0 ? u_out : (k == 1 ? v_out : a_out);
    if (!dst) continue;
    NMCK(launch_node_to_eq(*c, src, c->d_eq_tmp));
    NMCK(cudaMemcpyAsync(dst, c->d_eq_tmp, sizeof(double) * c->neq, cudaMemcpyDeviceToHost, c->stream));
    NMCK(cudaStreamSynchronize(c->stream));
  }
  if (nprobe > 0)
    NMCK(cudaMemcpyAsync(probe_hist, d_hist, sizeof(double) * (size_t)nprobe * o->steps, cudaMemcpyDeviceToHost,
                         c->stream));
  NMCK(cudaMemcpyAsync(h_max, d_max, sizeof(h_max), cudaMemcpyDeviceToHost, c->stream));
  NMCK(cudaStreamSynchronize(c->stream));
  {
    double m[3];
    std::memcpy(m, h_max, sizeof(m));
    R.umax = m[0];
    R.vmax = m[1];
    R.amax = m[2];
  }
done:
  if (rep) *rep = R;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (double *b : {d_q, d_u, d_v, d_a, d_w, d_z, d_hist})
    if (b) cudaFree(b);
  if (d_probe) cudaFree(d_probe);
  if (d_max) cudaFree(d_max);
  for (double *b : {dm.C, dm.Cs, dm.w2, dm.z2})
    if (b) cudaFree(b);
  // the K slot now holds K_eff (or M): the next stiffness assembly rebuilds K
  return rc;
}

// solve_kernels.cu - K.u solve on the node-block CSR matrix (sm_100a).
//
// Replaces cSymSprsMatrix::MultVect (mlib/sysmat.cpp:942-963) and PCGSolver
// (mlib/sysmat.cpp:1061-1125).  The iteration is the reference's Jacobi PCG:
//
//   r = f, z = D^-1 r, p = z, dot0 = z.r
//   loop: w = K p; alpha = dot0 / p.w; u += alpha p; r -= alpha w; z = D^-1 r
//         err = |r| / |f|  (|f| > 1e11 replaced by 1);  stop if err < tol
//         dot1 = z.r; beta = dot1/dot0; dot0 = dot1; p = z + beta p
//
// Vectors live in node-DOF space (3 per node); DOFs without an equation
// carry an identity row in K and a zero right-hand side, so they stay zero
// and the iteration is the reference's on the free equations.
//
// Every scalar lives on the device (PcgState) and every reduction uses a
// fixed grid and a fixed combination order, so the host never waits inside
// an iteration and a solve is bit-reproducible.  Kernels check state->done
// first, so iterations launched past convergence cost only their launch.
//
// SpMV: one warp per block-row; a row's 3x3 blocks are contiguous, so the
// warp streams 9*nb values with consecutive lanes on consecutive addresses
// (fully coalesced) and gathers x through L1/L2.  HBM-bound: bytes per call
// = nnzb*(9*sizeof(VT) + 4) + 4*(nnode+1) + vector traffic.
#include <cmath>
#include <cstdint>

#include "internal.h"

namespace fastgpu {

constexpr int kSpmvThreads = 256;
constexpr int kVecThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
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

// y = K x  (MODE 0),  y = b - K x  (MODE 1).  Optional per-block partial of
// x.y (MODE 0) or y.y (MODE 1).
template <typename VT, typename XT, typename AT, int MODE>
__global__ void __launch_bounds__(kSpmvThreads)
spmv_kernel(int64_t nrows, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
            const VT *__restrict__ val, const XT *__restrict__ x, const XT *__restrict__ b,
            XT *__restrict__ y, double *__restrict__ part, const PcgState *__restrict__ st) {
  if (st && st->done) return;
  __shared__ double sbuf[32];
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)kSpmvThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kSpmvThreads) >> 5;
  double pacc = 0.0;
  for (int64_t row = warp; row < nrows; row += nwarps) {
    const int32_t b0 = rowptr[row], b1 = rowptr[row + 1];
    const VT *vrow = val + (int64_t)b0 * 9;
    const int nv = (b1 - b0) * 9;
    AT a0 = 0, a1 = 0, a2 = 0;
    for (int v = lane; v < nv; v += 32) {
      const int blk = v / 9, e = v - 9 * blk, i = e / 3, j = e - 3 * i;
      const int32_t cidx = col[b0 + blk];
      const AT prod = (AT)vrow[v] * (AT)x[3 * (int64_t)cidx + j];
      a0 += (i == 0) ? prod : (AT)0;
      a1 += (i == 1) ? prod : (AT)0;
      a2 += (i == 2) ? prod : (AT)0;
    }
    if (sizeof(AT) == 8) {
      a0 = (AT)warp_sum((double)a0); a1 = (AT)warp_sum((double)a1); a2 = (AT)warp_sum((double)a2);
    } else {
      a0 = (AT)warp_sumf((float)a0); a1 = (AT)warp_sumf((float)a1); a2 = (AT)warp_sumf((float)a2);
    }
    if (lane == 0) {
      XT y0, y1, y2;
      if (MODE == 0) {
        y0 = (XT)a0; y1 = (XT)a1; y2 = (XT)a2;
        if (part) pacc += (double)x[3 * row] * y0 + (double)x[3 * row + 1] * y1 + (double)x[3 * row + 2] * y2;
      } else {
        y0 = b[3 * row] - (XT)a0; y1 = b[3 * row + 1] - (XT)a1; y2 = b[3 * row + 2] - (XT)a2;
        if (part) pacc += (double)y0 * y0 + (double)y1 * y1 + (double)y2 * y2;
      }
      y[3 * row] = y0; y[3 * row + 1] = y1; y[3 * row + 2] = y2;
    }
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

// alpha = dot0 / (p.w)
__global__ void __launch_bounds__(256) pcg_alpha(PcgState *st, const double *part, int n) {
  if (st->done) return;
  __shared__ double sbuf[32];
  const double pw = sum_partials(part, n, sbuf);
  if (threadIdx.x == 0) {
    st->pw = pw;
    if (!(pw > 0.0) || !isfinite(pw)) { st->done = 3; return; }
    st->alpha = st->dot0 / pw;
  }
}

// u += alpha p; r -= alpha w; z = Dinv r (3x3 per node); partials r.r, z.r
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_update(int64_t nnode, T *__restrict__ u, T *__restrict__ r, T *__restrict__ z, const T *__restrict__ p,
           const T *__restrict__ w, const T *__restrict__ dinv, const PcgState *__restrict__ st,
           double *__restrict__ part_rr, double *__restrict__ part_zr) {
  if (st->done) return;
  __shared__ double sbuf[32];
  const T alpha = (T)st->alpha;
  double rr = 0.0, zr = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; n < nnode; n += (int64_t)gridDim.x * kVecThreads) {
    T rv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int64_t i = 3 * n + k;
      u[i] = u[i] + alpha * p[i];
      rv[k] = r[i] + (-alpha) * w[i];
      r[i] = rv[k];
    }
    const T *D = dinv + 9 * n;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const T zk = D[3 * k] * rv[0] + D[3 * k + 1] * rv[1] + D[3 * k + 2] * rv[2];
      z[3 * n + k] = zk;
      rr += (double)rv[k] * (double)rv[k];
      zr += (double)zk * (double)rv[k];
    }
  }
  const double t1 = block_sum<kVecThreads>(rr, sbuf);
  if (threadIdx.x == 0) part_rr[blockIdx.x] = t1;
  const double t2 = block_sum<kVecThreads>(zr, sbuf);
  if (threadIdx.x == 0) part_zr[blockIdx.x] = t2;
}

// err, convergence, beta
__global__ void __launch_bounds__(256) pcg_beta(PcgState *st, const double *part_rr, const double *part_zr, int n) {
  if (st->done) return;
  __shared__ double sbuf[32];
  const double rr = sum_partials(part_rr, n, sbuf);
  const double zr = sum_partials(part_zr, n, sbuf);
  if (threadIdx.x == 0) {
    st->iter += 1;
    st->rr = rr;
    st->err = sqrt(rr) / st->lenf;
    if (st->err < st->tol) { st->done = 1; return; }
    if (!isfinite(st->err)) { st->done = 3; return; }
    if (st->iter >= st->maxit) { st->done = 2; return; }
    st->beta = zr / st->dot0;
    st->dot0 = zr;
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_pupdate(int64_t n3, T *__restrict__ p, const T *__restrict__ z, const PcgState *__restrict__ st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (int64_t i = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; i < n3; i += (int64_t)gridDim.x * kVecThreads)
    p[i] = z[i] + beta * p[i];
}

// z = Dinv r, p = z; partials z.r and rhs.rhs
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
pcg_init_vec(int64_t nnode, const T *__restrict__ r, T *__restrict__ z, T *__restrict__ p,
             const T *__restrict__ dinv, const T *__restrict__ rhs, double *part_zr, double *part_ff) {
  __shared__ double sbuf[32];
  double zr = 0.0, ff = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)kVecThreads + threadIdx.x; n < nnode; n += (int64_t)gridDim.x * kVecThreads) {
    const T r0 = r[3 * n], r1 = r[3 * n + 1], r2 = r[3 * n + 2];
    const T *D = dinv + 9 * n;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const T zk = D[3 * k] * r0 + D[3 * k + 1] * r1 + D[3 * k + 2] * r2;
      z[3 * n + k] = zk;
      p[3 * n + k] = zk;
      const T rk = (k == 0) ? r0 : (k == 1) ? r1 : r2;
      zr += (double)zk * (double)rk;
      const double fk = (double)rhs[3 * n + k];
      ff += fk * fk;
    }
  }
  const double t1 = block_sum<kVecThreads>(zr, sbuf);
  if (threadIdx.x == 0) part_zr[blockIdx.x] = t1;
  const double t2 = block_sum<kVecThreads>(ff, sbuf);
  if (threadIdx.x == 0) part_ff[blockIdx.x] = t2;
}

__global__ void __launch_bounds__(256) pcg_init_scalar(PcgState *st, const double *part_zr, const double *part_ff,
                                                       const double *part_rr0, int n, double tol, int maxit) {
  __shared__ double sbuf[32];
  const double zr = sum_partials(part_zr, n, sbuf);
  const double ff = sum_partials(part_ff, n, sbuf);
  double rr0 = ff;
  if (part_rr0) rr0 = sum_partials(part_rr0, n, sbuf);
  if (threadIdx.x == 0) {
    PcgState s{};
    s.dot0 = zr;
    double lenf = sqrt(ff);
    s.tol = tol;
    s.maxit = maxit;
    s.iter = 0;
    s.done = 0;
    if (lenf < tol) s.done = 1;        // PCGSolver returns at once for a null load
    if (lenf > 10e+10) lenf = 1.0;     // PCGSolver's large-load normaliser
    s.lenf = lenf;
    s.rr = rr0;
    s.err = sqrt(rr0) / lenf;
    if (!s.done && s.err < tol) s.done = 1;
    *st = s;
  }
}

// x = 0 copy helpers
template <typename S, typename D>
__global__ void convert_scale(int64_t n, const S *__restrict__ s, D *__restrict__ d, double scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (D)((double)s[i] * scale);
}

// Jacobi / block-Jacobi inverse per node from the diagonal block
template <typename T>
__global__ void build_dinv(int64_t nnode, const int32_t *__restrict__ diag, const double *__restrict__ K,
                           T *__restrict__ dinv, int block) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  T *D = dinv + 9 * n;
  const int32_t d = diag[n];
  double a[9];
  for (int k = 0; k < 9; k++) a[k] = (d >= 0) ? K[(int64_t)d * 9 + k] : (k % 4 == 0 ? 1.0 : 0.0);
  if (!block) {
    for (int k = 0; k < 9; k++) D[k] = (T)0;
    D[0] = (T)(1.0 / a[0]);
    D[4] = (T)(1.0 / a[4]);
    D[8] = (T)(1.0 / a[8]);
    return;
  }
  const double c00 = a[4] * a[8] - a[5] * a[7], c01 = -(a[3] * a[8] - a[5] * a[6]), c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  const double id = 1.0 / det;
  D[0] = (T)(c00 * id);
  D[1] = (T)(-(a[1] * a[8] - a[2] * a[7]) * id);
  D[2] = (T)((a[1] * a[5] - a[2] * a[4]) * id);
  D[3] = (T)(c01 * id);
  D[4] = (T)((a[0] * a[8] - a[2] * a[6]) * id);
  D[5] = (T)(-(a[0] * a[5] - a[2] * a[3]) * id);
  D[6] = (T)(c02 * id);
  D[7] = (T)(-(a[0] * a[7] - a[1] * a[6]) * id);
  D[8] = (T)((a[0] * a[4] - a[1] * a[3]) * id);
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

__global__ void scale_kernel(int64_t n, double *__restrict__ x, double a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void axpy_kernel(int64_t n, double *__restrict__ y, const double *__restrict__ x, double a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// ---------------------------------------------------------------------------
// host side

cudaError_t scale_inplace(Ctx &c, double *x, int64_t n, double a) {
  scale_kernel<<<kRedBlocks, 256, 0, c.stream>>>(n, x, a);
  c.launches++;
  return cudaGetLastError();
}
cudaError_t axpy_inplace(Ctx &c, double *y, const double *x, int64_t n, double a) {
  axpy_kernel<<<kRedBlocks, 256, 0, c.stream>>>(n, y, x, a);
  c.launches++;
  return cudaGetLastError();
}

static int spmv_grid(const Ctx &c) { return c.sm_count * 8; }

cudaError_t launch_spmv(Ctx &c, const double *K, const double *x, double *y) {
  spmv_kernel<double, double, double, 0><<<spmv_grid(c), kSpmvThreads, 0, c.stream>>>(
      c.nnode, c.d_rowptr, c.d_col, K, x, nullptr, y, nullptr, nullptr);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_spmv32(Ctx &c, const float *K, const float *x, float *y) {
  spmv_kernel<float, float, float, 0><<<spmv_grid(c), kSpmvThreads, 0, c.stream>>>(
      c.nnode, c.d_rowptr, c.d_col, K, x, nullptr, y, nullptr, nullptr);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_residual(Ctx &c, const double *K, const double *f, const double *u, double *r, double *rr_out) {
  double *part = c.d_partials;
  spmv_kernel<double, double, double, 1><<<spmv_grid(c), kSpmvThreads, 0, c.stream>>>(
      c.nnode, c.d_rowptr, c.d_col, K, u, f, r, part, nullptr);
  c.launches++;
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
  cudaError_t e = cudaMemsetAsync(nodev, 0, sizeof(double) * 3 * (size_t)c.nnode, c.stream);
  if (e != cudaSuccess) return e;
  if (c.neq > 0) scatter_eq_to_node<<<(c.neq + 255) / 256, 256, 0, c.stream>>>(c.neq, c.d_dof_of_eq, eqv, nodev);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_node_to_eq(Ctx &c, const double *nodev, double *eqv) {
  if (c.neq > 0) gather_node_to_eq<<<(c.neq + 255) / 256, 256, 0, c.stream>>>(c.neq, c.d_dof_of_eq, nodev, eqv);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_build_precond(Ctx &c, const double *K, int precond) {
  const int bs = 256;
  const unsigned g = (unsigned)((c.nnode + bs - 1) / bs);
  build_dinv<double><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K, c.d_dinv, precond);
  c.launches++;
  build_dinv<float><<<g, bs, 0, c.stream>>>(c.nnode, c.d_diag, K, c.s_dinv, precond);
  c.launches++;
  c.precond_built = precond;
  return cudaGetLastError();
}

// Runs PCG on K (FP64) or K32 (FP32).  rhs and x are FP64 node-DOF vectors;
// in FP32 mode they are converted at entry/exit (x returned = FP32 solution).
cudaError_t pcg_solve_device(Ctx &c, bool fp32, const double *d_rhs, double *d_x, bool warm, double tol,
                             int maxit, int check_every, int precond, int *iters, double *err, int *done) {
  (void)precond;
  const int64_t nn = c.nnode, n3 = 3 * nn;
  const int G = spmv_grid(c);
  const int R = kRedBlocks;
  double *pA = c.d_partials;            // [G]  p.w
  double *pB = c.d_partials + 2048;     // [R]  r.r
  double *pC = c.d_partials + 4096;     // [R]  z.r
  double *pD = c.d_partials + 6144;     // [R]  rhs.rhs
  double *pE = c.d_partials + 8192;     // [G]  initial r.r
  PcgState *st = c.d_state;
  cudaError_t e;
  if (!fp32) {
    if (warm) {
      spmv_kernel<double, double, double, 1><<<G, kSpmvThreads, 0, c.stream>>>(
          nn, c.d_rowptr, c.d_col, c.d_K, d_x, d_rhs, c.d_r, pE, nullptr);
      c.launches++;
    } else {
      cudaMemsetAsync(d_x, 0, sizeof(double) * n3, c.stream);
      cudaMemcpyAsync(c.d_r, d_rhs, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c.stream);
    }
    pcg_init_vec<double><<<R, kVecThreads, 0, c.stream>>>(nn, c.d_r, c.d_z, c.d_p, c.d_dinv, d_rhs, pC, pD);
    c.launches++;
    pcg_init_scalar<<<1, 256, 0, c.stream>>>(st, pC, pD, warm ? pE : nullptr, warm ? G : R, tol, maxit);
    c.launches++;
  } else {
    // FP32: rhs converted, x starts at 0
    convert_scale<double, float><<<R, 256, 0, c.stream>>>(n3, d_rhs, c.s_r, 1.0);
    c.launches++;
    cudaMemsetAsync(c.s_u, 0, sizeof(float) * n3, c.stream);
    pcg_init_vec<float><<<R, kVecThreads, 0, c.stream>>>(nn, c.s_r, c.s_z, c.s_p, c.s_dinv, c.s_r, pC, pD);
    c.launches++;
    pcg_init_scalar<<<1, 256, 0, c.stream>>>(st, pC, pD, nullptr, R, tol, maxit);
    c.launches++;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;

  if (check_every <= 0) check_every = 32;
  cudaEvent_t ev;
  if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
  int launched = 0;
  bool pending = false;
  while (true) {
    // launch one chunk
    for (int k = 0; k < check_every && launched < maxit; k++, launched++) {
      if (!fp32) {
        spmv_kernel<double, double, double, 0><<<G, kSpmvThreads, 0, c.stream>>>(
            nn, c.d_rowptr, c.d_col, c.d_K, c.d_p, nullptr, c.d_w, pA, st);
        c.launches++;
        pcg_alpha<<<1, 256, 0, c.stream>>>(st, pA, G);
        c.launches++;
        pcg_update<double><<<R, kVecThreads, 0, c.stream>>>(nn, d_x, c.d_r, c.d_z, c.d_p, c.d_w, c.d_dinv, st, pB, pC);
        c.launches++;
        pcg_beta<<<1, 256, 0, c.stream>>>(st, pB, pC, R);
        c.launches++;
        pcg_pupdate<double><<<R, kVecThreads, 0, c.stream>>>(n3, c.d_p, c.d_z, st);
        c.launches++;
      } else {
        spmv_kernel<float, float, float, 0><<<G, kSpmvThreads, 0, c.stream>>>(
            nn, c.d_rowptr, c.d_col, c.d_K32, c.s_p, nullptr, c.s_w, pA, st);
        c.launches++;
        pcg_alpha<<<1, 256, 0, c.stream>>>(st, pA, G);
        c.launches++;
        pcg_update<float><<<R, kVecThreads, 0, c.stream>>>(nn, c.s_u, c.s_r, c.s_z, c.s_p, c.s_w, c.s_dinv, st, pB, pC);
        c.launches++;
        pcg_beta<<<1, 256, 0, c.stream>>>(st, pB, pC, R);
        c.launches++;
        pcg_pupdate<float><<<R, kVecThreads, 0, c.stream>>>(n3, c.s_p, c.s_z, st);
        c.launches++;
      }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    // check the state of the previous chunk while this one runs
    if (pending) {
      if ((e = cudaEventSynchronize(ev)) != cudaSuccess) break;
      if (c.h_state->done) break;
    }
    if ((e = cudaMemcpyAsync(c.h_state, st, sizeof(PcgState), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess) break;
    if ((e = cudaEventRecord(ev, c.stream)) != cudaSuccess) break;
    pending = true;
    if (launched >= maxit) {
      if ((e = cudaEventSynchronize(ev)) != cudaSuccess) break;
      break;
    }
  }
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return e;
  // final state
  if ((e = cudaMemcpyAsync(c.h_state, st, sizeof(PcgState), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(c.stream)) != cudaSuccess) return e;
  *iters = c.h_state->iter;
  *err = c.h_state->err;
  *done = c.h_state->done;
  if (fp32) {
    // return the FP32 solution in d_x
    convert_scale<float, double><<<R, 256, 0, c.stream>>>(n3, c.s_u, d_x, 1.0);
    c.launches++;
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace fastgpu

// noalloc.cu - a K.u solve that allocates no device memory.
//
// Some callers cannot let a library allocate device memory: applications
// that hand the whole device to their own memory pool (a framework's caching
// allocator, a solver that budgets HBM up front) and loops that must not
// stall, since cudaMalloc/cudaFree synchronise the device and so block every
// other stream of the process.  fast_gpu_pcg_solve_noalloc serves them: the
// caller passes the matrix, the load and the solution buffer in device
// memory; every work vector and reduction buffer of the solve lives in one
// file-scope __device__ array below.
//
// When that array gets its memory: it belongs to this file's module of the
// library.  Under CUDA's lazy module loading (the default of the CUDA 12
// runtime unless CUDA_MODULE_LOADING=EAGER is set) the module, and with it the
// array, is loaded onto a device the first time anything in this file is used
// there, i.e. inside the first call made on that device.  That first call may
// therefore take device memory for the array (and fail with FAST_GPU_ECUDA if
// the device has none left) and may synchronise the device.  A caller whose
// own pool takes the device should make the first call, for instance the
// set-up-only call with num_eq = 0, before the pool is created, and before any
// stream capture; every later call allocates nothing and does not synchronise
// the device (it synchronises only its own stream, to read the convergence
// state).
//
// The solve is the same FP64 Jacobi PCG as fast_gpu_solve with
// FAST_PREC_FP64 / FAST_PRECOND_JACOBI (same iteration, same stopping test
// |r|/|f| < tol with |f| > 1e11 replaced by 1), here on a scalar CSR matrix in
// equation space (full symmetric storage, both triangles), so its iterates
// and result agree with that entry point to rounding.
//
// Limits and sharing: at most kNoAllocMaxEq equations (the array holds five
// vectors of that length, 20 MB in all, on every device that has loaded it,
// until the process exits).  Every call uses the same array and it keeps the
// previous call's contents; everything a solve needs is re-initialised at the
// start of each call.  Two calls whose work overlaps on the GPU (different
// streams, or different host threads) race on the array and must not be
// issued.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "internal.h"

namespace {

constexpr int64_t kNoAllocMaxEq = 500000;
constexpr int kNoAllocBlocks = 592;      // fixed reduction grid (4 x 148 SMs)
constexpr int kNoAllocThreads = 256;
// scratch layout (doubles): r, z, p, w, dinv [kNoAllocMaxEq each];
// partials [4][kNoAllocBlocks]; solver state
constexpr size_t kOffR = 0, kOffZ = kNoAllocMaxEq, kOffP = 2 * kNoAllocMaxEq, kOffW = 3 * kNoAllocMaxEq,
                 kOffD = 4 * kNoAllocMaxEq, kOffPart = 5 * kNoAllocMaxEq,
                 kOffState = kOffPart + 4 * kNoAllocBlocks;
constexpr size_t kScratchDoubles = kOffState + 32;

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// done: 0 running, 1 converged, 2 maxit reached, 3 breakdown (p.Kp not
// positive, or a non-finite value), 4 a row without a usable diagonal
struct NaState {
  double dot0, alpha, beta, lenf, rr, err, tol;
  int32_t iter, done, maxit, pad;
};
static_assert(sizeof(NaState) <= 32 * sizeof(double), "state fits its slot");

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double na_block_sum(double v, double *sbuf) {
  v = na_warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sbuf[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) t = na_warp_sum(lane < kNoAllocThreads / 32 ? sbuf[lane] : 0.0);
  return t;
}

__device__ __forceinline__ double na_sum_partials(const double *p, double *sbuf) {
  double v = 0.0;
  for (int i = threadIdx.x; i < kNoAllocBlocks; i += blockDim.x) v += p[i];
  return na_block_sum(v, sbuf);
}

// r = f, u = 0, dinv = 1/diag(K), z = dinv r, p = z; partials z.r, f.f and
// the number of rows whose diagonal is not stored, zero or not finite (Jacobi
// is undefined there; such a row gets dinv = 0 and the solve is rejected)
__global__ void __launch_bounds__(kNoAllocThreads)
na_init(int32_t n, const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col,
        const double *__restrict__ val, const double *__restrict__ f, double *__restrict__ u, double *S) {
  __shared__ double sbuf[32];
  double *r = S + kOffR, *z = S + kOffZ, *p = S + kOffP, *dinv = S + kOffD, *part = S + kOffPart;
  double zr = 0.0, ff = 0.0, bad = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++)
      if (col[k] == i) d = val[k];
    const bool usable = d != 0.0 && isfinite(d);
    bad += usable ? 0.0 : 1.0;
    const double di = usable ? 1.0 / d : 0.0;
    const double fi = f[i];
    dinv[i] = di;
    u[i] = 0.0;
    r[i] = fi;
    z[i] = di * fi;
    p[i] = di * fi;
    zr += di * fi * fi;
    ff += fi * fi;
  }
  const double t1 = na_block_sum(zr, sbuf);
  if (threadIdx.x == 0) part[blockIdx.x] = t1;
  const double t2 = na_block_sum(ff, sbuf);
  if (threadIdx.x == 0) part[kNoAllocBlocks + blockIdx.x] = t2;
  const double t3 = na_block_sum(bad, sbuf);
  if (threadIdx.x == 0) part[2 * kNoAllocBlocks + blockIdx.x] = t3;
}

__global__ void __launch_bounds__(kNoAllocThreads) na_init_scalar(double *S, double tol, int maxit) {
  __shared__ double sbuf[32];
  const double *part = S + kOffPart;
  const double zr = na_sum_partials(part, sbuf);
  const double ff = na_sum_partials(part + kNoAllocBlocks, sbuf);
  const double bad = na_sum_partials(part + 2 * kNoAllocBlocks, sbuf);
  if (threadIdx.x == 0) {
    NaState s{};
    double lenf = sqrt(ff);
    s.dot0 = zr;
    s.tol = tol;
    s.maxit = maxit;
    if (lenf < tol) s.done = 1;       // PCGSolver returns at once for a null load
    if (lenf > 10e+10) lenf = 1.0;    // PCGSolver's large-load normaliser
    s.lenf = lenf;
    s.rr = ff;
    s.err = sqrt(ff) / (lenf > 0 ? lenf : 1.0);
    if (bad > 0.0) s.done = 4;
    *reinterpret_cast<NaState *>(S + kOffState) = s;
  }
}

// w = K p (one warp per row), partial p.w
__global__ void __launch_bounds__(kNoAllocThreads)
na_spmv(int32_t n, const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col,
        const double *__restrict__ val, double *S) {
  const NaState *st = reinterpret_cast<const NaState *>(S + kOffState);
  if (st->done) return;
  __shared__ double sbuf[32];
  const double *p = S + kOffP;
  double *w = S + kOffW, *part = S + kOffPart;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double pw = 0.0;
  for (int64_t i = warp; i < n; i += nwarps) {
    double s = 0.0;
    for (int64_t k = rowptr[i] + lane; k < rowptr[i + 1]; k += 32) s += val[k] * p[col[k]];
    s = na_warp_sum(s);
    if (lane == 0) {
      w[i] = s;
      pw += p[i] * s;
    }
  }
  const double t = na_block_sum(pw, sbuf);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kNoAllocThreads) na_alpha(double *S) {
  NaState *st = reinterpret_cast<NaState *>(S + kOffState);
  if (st->done) return;
  __shared__ double sbuf[32];
  const double pw = na_sum_partials(S + kOffPart, sbuf);
  if (threadIdx.x == 0) {
    const double al = st->dot0 / pw;
    if (!(al > 0.0) || !isfinite(pw) || !isfinite(al)) { st->done = 3; return; }
    st->alpha = al;
  }
}

// u += alpha p; r -= alpha w; z = dinv r; partials r.r, z.r
__global__ void __launch_bounds__(kNoAllocThreads) na_update(int32_t n, double *__restrict__ u, double *S) {
  const NaState *st = reinterpret_cast<const NaState *>(S + kOffState);
  if (st->done) return;
  __shared__ double sbuf[32];
  double *r = S + kOffR, *z = S + kOffZ, *part = S + kOffPart;
  const double *p = S + kOffP, *w = S + kOffW, *dinv = S + kOffD;
  const double alpha = st->alpha;
  double rr = 0.0, zr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    u[i] = u[i] + alpha * p[i];
    const double ri = r[i] + (-alpha) * w[i];
    r[i] = ri;
    const double zi = dinv[i] * ri;
    z[i] = zi;
    rr += ri * ri;
    zr += zi * ri;
  }
  const double t1 = na_block_sum(rr, sbuf);
  if (threadIdx.x == 0) part[2 * kNoAllocBlocks + blockIdx.x] = t1;
  const double t2 = na_block_sum(zr, sbuf);
  if (threadIdx.x == 0) part[3 * kNoAllocBlocks + blockIdx.x] = t2;
}

__global__ void __launch_bounds__(kNoAllocThreads) na_beta(double *S) {
  NaState *st = reinterpret_cast<NaState *>(S + kOffState);
  if (st->done) return;
  __shared__ double sbuf[32];
  const double rr = na_sum_partials(S + kOffPart + 2 * kNoAllocBlocks, sbuf);
  const double zr = na_sum_partials(S + kOffPart + 3 * kNoAllocBlocks, sbuf);
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

__global__ void __launch_bounds__(kNoAllocThreads) na_pupdate(int32_t n, double *S) {
  const NaState *st = reinterpret_cast<const NaState *>(S + kOffState);
  if (st->done) return;
  double *p = S + kOffP;
  const double *z = S + kOffZ;
  const double beta = st->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

}  // namespace

extern "C" int fast_gpu_pcg_solve_noalloc(int32_t num_eq, const int64_t *d_rowptr, const int32_t *d_col,
                                          const double *d_val, const double *d_f, double *d_u, double tol,
                                          int32_t maxit, void *cuda_stream, fast_gpu_solve_report *rep) {
  // the size limit is checked first, before any CUDA call
  if (num_eq > kNoAllocMaxEq) return FAST_GPU_ETOOBIG;
  if (num_eq < 0) return FAST_GPU_EINVAL;
  if (num_eq > 0 && (!d_rowptr || !d_col || !d_val || !d_f || !d_u)) return FAST_GPU_EINVAL;
  if (!(tol > 0)) tol = 1e-5;           // cSysMatrix's default tolerance
  if (maxit <= 0) maxit = num_eq;       // cSysMatrix(n) sets maxit = n
  // The device address of the scratch array, looked up on every call with
  // the caller's device current: the array's host-side name is not a device
  // address, and the address can change if the context is torn down and
  // re-created (cudaDeviceReset), so it is never cached.  On the first call
  // on a device this lookup is what loads this file's module there.
  double *S = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&S, g_noalloc_scratch);
  if (e != cudaSuccess || !S) return FAST_GPU_ECUDA;
  if (num_eq == 0) return FAST_GPU_OK;  // set-up only
  cudaStream_t s = (cudaStream_t)cuda_stream;
  const int G = kNoAllocBlocks, T = kNoAllocThreads;
  na_init<<<G, T, 0, s>>>(num_eq, d_rowptr, d_col, d_val, d_f, d_u, S);
  na_init_scalar<<<1, T, 0, s>>>(S, tol, maxit);
  if ((e = cudaGetLastError()) != cudaSuccess) return FAST_GPU_ECUDA;
  NaState h{};
  const int chunk = 32;
  for (int launched = 0; launched < maxit;) {
    const int k = (maxit - launched < chunk) ? (maxit - launched) : chunk;
    for (int i = 0; i < k; i++) {
      na_spmv<<<G, T, 0, s>>>(num_eq, d_rowptr, d_col, d_val, S);
      na_alpha<<<1, T, 0, s>>>(S);
      na_update<<<G, T, 0, s>>>(num_eq, d_u, S);
      na_beta<<<1, T, 0, s>>>(S);
      na_pupdate<<<G, T, 0, s>>>(num_eq, S);
    }
    launched += k;
    if ((e = cudaGetLastError()) != cudaSuccess) return FAST_GPU_ECUDA;
    if ((e = cudaMemcpyAsync(&h, S + kOffState, sizeof(NaState), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return FAST_GPU_ECUDA;
    if (h.done) break;
  }
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->converged = h.done == 1;
    rep->iterations = h.iter;
    rep->outer = 1;
    rep->rel_residual = h.err;
    rep->true_rel_residual = -1.0;  // not recomputed here
  }
  if (h.done == 4) return FAST_GPU_EINVAL;  // a row without a usable diagonal
  if (h.done != 1) return FAST_GPU_ENONCONV;  // maxit reached (2) or breakdown (3)
  return FAST_GPU_OK;
}

// autotune.cu - launch shapes chosen by measurement on the system at hand
// (fast_gpu_autotune; no reference counterpart).
//
// What is tuned, and why it is worth measuring:
//   * the launch shape of the element kernels, bucket by bucket: resident
//     CTAs per SM (fewer CTAs leave each more L1 and shared-memory bandwidth,
//     more hide the latency of the gathers and the scatter) and, for B-spline
//     buckets, how many CTAs share one element's node pairs (more CTAs per
//     element fill the GPU on short colours but repeat the element's
//     geometry work); the best point depends on the element type, its Gauss
//     rule and the colour sizes of the mesh, so each is timed on the mesh;
//   * lanes per block-row of the FP32 and FP64 SpMV (and for FP32 the
//     bulk-staged and the cache-streaming forms): the best split of a row's
//     blocks over lanes depends on the row length (27 blocks for hex8 meshes,
//     ~57 for hex20, ~125 for degree-3 B-spline patches) and on how many rows a
//     warp then covers;
//   * the PCG iteration path: one persistent cooperative kernel per chunk
//     (latency-bound small systems) or a CUDA graph of kernels (bandwidth-
//     bound large ones).  The crossover depends on the system, so both are
//     timed on the same 64 FP64 iterations.
// The choices become the context's options (fast_gpu_set_option); the caller
// may cache them per device and mesh type.
#include <algorithm>
#include <functional>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

// median over `reps` launches, each bracketed by events on the context stream
cudaError_t median_ms(Ctx &c, const std::function<cudaError_t()> &launch, int reps, double &ms) {
  cudaEvent_t a, b;
  cudaError_t e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  std::vector<double> t;
  for (int r = 0; r < reps + 1 && e == cudaSuccess; r++) {  // the first launch warms up
    e = cudaEventRecord(a, c.stream);
    if (e == cudaSuccess) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(b, c.stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float f = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, a, b);
    if (e == cudaSuccess && r > 0) t.push_back(f);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return e;
  std::sort(t.begin(), t.end());
  ms = t[t.size() / 2];
  return cudaSuccess;
}

}  // namespace

#define ATK(call)                                                                     \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess) {                                                          \
      c->err = std::string("autotune: ") + #call + ": " + cudaGetErrorString(_e);    \
      return FAST_GPU_ECUDA;                                                          \
    }                                                                                 \
  } while (0)

namespace {

// Times one bucket's assembly under every launch shape the kernels admit and
// keeps the fastest (a shape replaces the default only when it is at least
// 2 % faster).  `tc`: the tensor-core kernels (resident CTAs per SM only).
cudaError_t tune_bucket(Ctx &c, size_t b, bool tc, double &ms_default, double &ms_best) {
  Bucket &B = c.buckets[b];
  auto launch = [&] {
    return tc ? launch_assemble_tc_bucket(c, b, c.d_K32) : launch_assemble_bucket(c, b, c.d_K);
  };
  constexpr int kReps = 3;
  int &ctas = tc ? B.tune_tc_ctas : B.tune_ctas;
  ctas = 0;
  if (!tc) B.tune_split = 0;
  if (!tc) B.tune_kernel = 0;
  c.elem_occ = c.elem_split_max = 0;
  cudaError_t e = median_ms(c, launch, kReps, ms_default);
  if (e != cudaSuccess) return e;
  int best_c = 0, best_s = 0, best_k = 0;
  ms_best = ms_default;
  // FP64 hex buckets: both kernels (CTA per element, warp per element)
  const int kernels = (!tc && warp_supported(B)) ? 2 : 1;
  for (int kern = 0; kern < kernels; kern++) {
    if (!tc) B.tune_kernel = kern;
    int occ = 0;
    if (kern == 0) {
      occ = c.elem_occ;
    } else {
      // the warp kernel's own occupancy from a run at its default shape
      ctas = 0;
      c.elem_occ = 0;
      double ms = 0.0;
      e = median_ms(c, launch, kReps, ms);
      if (e != cudaSuccess) return e;
      if (ms < 0.98 * ms_best) { ms_best = ms; best_c = 0; best_s = 0; best_k = kern; }
      occ = c.elem_occ;
    }
    occ = std::min(occ, 16);
    const int smax = (tc || B.type != FAST_ELEM_BSP_SOLID) ? 0 : std::min(c.elem_split_max, 16);
    for (int k = 1; k <= occ; k++)
      for (int sp = 0; sp <= smax; sp++) {
        if (k == occ && sp == 0) continue;  // the kernel's default
        ctas = k;
        if (!tc) B.tune_split = sp;
        double ms = 0.0;
        e = median_ms(c, launch, kReps, ms);
        if (e != cudaSuccess) return e;
        if (ms < 0.98 * ms_best) { ms_best = ms; best_c = k; best_s = sp; best_k = kern; }
      }
  }
  ctas = best_c;
  if (!tc) {
    B.tune_split = best_s;
    B.tune_kernel = best_k;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" int fast_gpu_autotune(fast_gpu_ctx *c, fast_gpu_tune_report *rep) {
  if (!c || !rep) return FAST_GPU_EINVAL;
  if (!c->K_ok) { c->err = "autotune: matrix not assembled"; return FAST_GPU_ESTATE; }
  fast_gpu_tune_report R{};

  // element launch shapes (the timed assemblies add into K; it is rebuilt below)
  bool all_tc = !c->buckets.empty();
  for (const Bucket &B : c->buckets) all_tc = all_tc && tc_supported(B);
  if (all_tc && !c->d_K32) {
    ATK(cudaMalloc((void **)&c->d_K32, sizeof(float) * 9 * (size_t)c->nnzb));
    ATK(cudaMemsetAsync(c->d_K32, 0, sizeof(float) * 9 * (size_t)c->nnzb, c->stream));
  }
  R.elem_tc = all_tc ? 1 : 0;
  for (size_t b = 0; b < c->buckets.size(); b++) {
    if (c->buckets[b].tl) continue;  // tangent kernels: not tuned
    double d64 = 0.0, t64 = 0.0, dtc = 0.0, ttc = 0.0;
    ATK(tune_bucket(*c, b, false, d64, t64));
    if (all_tc) ATK(tune_bucket(*c, b, true, dtc, ttc));
    if (b < 8) {
      const Bucket &B = c->buckets[b];
      R.elem_buckets = (int32_t)b + 1;
      R.elem_ctas[b] = B.tune_ctas;
      R.elem_split[b] = B.tune_split;
      R.elem_tc_ctas[b] = B.tune_tc_ctas;
      R.elem_kernel[b] = B.tune_kernel;
      R.elem_ms_default[b] = d64;
      R.elem_ms_tuned[b] = t64;
      R.elem_tc_ms_default[b] = dtc;
      R.elem_tc_ms_tuned[b] = ttc;
    }
  }
  ATK(cudaStreamSynchronize(c->stream));
  {
    const int rc = fast_gpu_assemble(c, FAST_ASM_STIFFNESS);
    if (rc != FAST_GPU_OK) return rc;
  }
  ATK(solve_layout(*c, FAST_ASM_STIFFNESS, true));
  const size_t n4 = 4 * (size_t)c->nnode;
  ATK(cudaMemsetAsync(c->d_p, 0x3F, sizeof(double) * n4, c->stream));  // any finite vector
  ATK(cudaMemsetAsync(c->s_p, 0x3F, sizeof(float) * n4, c->stream));
  const int lanes[4] = {4, 8, 16, 32};
  c->spmv32_bulk = c->spmv32_stream = c->spmv32_c16 = false;   // the plain kernels first
  int best32 = c->lpr32, best64 = c->lpr64;
  double b32 = 1e300, b64 = 1e300;
  for (int i = 0; i < 4; i++) {
    c->lpr32 = c->lpr64 = lanes[i];
    ATK(median_ms(*c, [&] { return launch_spmv32(*c, c->d_Ks32, c->s_p, c->s_w); }, 9, R.ms_fp32[i]));
    ATK(median_ms(*c, [&] { return launch_spmv(*c, c->d_Ks, c->d_p, c->d_w); }, 9, R.ms_fp64[i]));
    if (R.ms_fp32[i] < b32) { b32 = R.ms_fp32[i]; best32 = lanes[i]; }
    if (R.ms_fp64[i] < b64) { b64 = R.ms_fp64[i]; best64 = lanes[i]; }
  }
  // the bulk-staged FP32 SpMV (matrix through shared memory), 8 and 16 lanes
  bool bulk = false;
  const bool tiles = ensure_bulk_tiles(*c) == cudaSuccess;  // rows too long for shared memory: not offered
  (void)cudaGetLastError();
  c->spmv32_bulk = tiles;
  for (int i = 0; i < 2 && tiles; i++) {
    c->lpr32 = i == 0 ? 8 : 16;
    ATK(median_ms(*c, [&] { return launch_spmv32(*c, c->d_Ks32, c->s_p, c->s_w); }, 9, R.ms_fp32_bulk[i]));
    if (R.ms_fp32_bulk[i] < b32) { b32 = R.ms_fp32_bulk[i]; best32 = c->lpr32; bulk = true; }
  }
  c->spmv32_bulk = false;
  // cache-streaming matrix loads, 8 and 16 lanes (timed alone for the report)
  bool stream = false;
  c->spmv32_stream = true;
  for (int i = 0; i < 2; i++) {
    c->lpr32 = i == 0 ? 8 : 16;
    ATK(median_ms(*c, [&] { return launch_spmv32(*c, c->d_Ks32, c->s_p, c->s_w); }, 9, R.ms_fp32_stream[i]));
    if (R.ms_fp32_stream[i] < b32) { b32 = R.ms_fp32_stream[i]; best32 = c->lpr32; stream = true; bulk = false; }
  }
  (void)stream;
  // The FP32 form is chosen inside the iteration, not in isolation: 64 mixed
  // PCG iterations (kernel per step) with each form.  Between two products
  // the vector kernels run, and the cache-streaming loads measured 3 % faster
  // alone but 45 % slower there on the hex20 box.
  c->lpr64 = best64;
  {
    if (c->precond_built != FAST_PRECOND_JACOBI) ATK(launch_build_precond(*c, c->d_K, FAST_PRECOND_JACOBI));
    c->precond_built = FAST_PRECOND_JACOBI;
    ATK(cudaMemsetAsync(c->d_f, 0x3F, sizeof(double) * n4, c->stream));
    const int64_t saved_p = c->persist_max_nodes;
    c->persist_max_nodes = 0;
    struct Form { int lanes; bool stream, bulk, c16; };
    const Form forms[8] = {{8, false, false, false}, {16, false, false, false}, {8, true, false, false},
                           {16, true, false, false}, {8, false, true, false},  {16, false, true, false},
                           {8, false, false, true},  {16, false, false, true}};
    const bool c16 = ensure_col16(*c) == cudaSuccess;   // rows spanning 65,536 nodes or more: not offered
    (void)cudaGetLastError();
    constexpr int kIt = 64;
    double best = 1e300;
    Form pick{best32, false, bulk, false};
    for (int f = 0; f < 8; f++) {
      if ((forms[f].bulk && !tiles) || (forms[f].c16 && !c16)) continue;
      c->lpr32 = forms[f].lanes;
      c->spmv32_stream = forms[f].stream;
      c->spmv32_bulk = forms[f].bulk;
      c->spmv32_c16 = forms[f].c16;
      c->drop_graphs();
      double ms = 0.0;
      ATK(median_ms(*c, [&] { return pcg_mixed(*c, false, 0.0, kIt, kIt); }, 3, ms));
      (f < 6 ? R.us_iter_mixed[f] : R.us_iter_mixed_col16[f - 6]) = ms * 1e3 / kIt;
      if (ms < best) { best = ms; pick = forms[f]; }
    }
    c->persist_max_nodes = saved_p;
    best32 = pick.lanes;
    stream = pick.stream;
    bulk = pick.bulk;
    c->spmv32_c16 = pick.c16;
    R.col16_fp32 = pick.c16 ? 1 : 0;
  }
  c->spmv32_stream = stream;
  c->spmv32_bulk = bulk;
  R.bulk_fp32 = bulk ? 1 : 0;
  R.stream_fp32 = stream ? 1 : 0;
  c->lpr32 = best32;
  c->drop_graphs();
  R.lanes_fp32 = best32;
  R.lanes_fp64 = best64;

  // PCG path: both timed on 64 FP64 iterations with a dummy load (tol 0 never
  // stops early), for systems within reach of one co-resident grid
  R.persistent_max_nodes = c->persist_max_nodes;
  const int64_t saved = c->persist_max_nodes;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
  if (coop && c->nnode <= (int64_t)1 << 20) {
    if (c->precond_built != FAST_PRECOND_JACOBI) ATK(launch_build_precond(*c, c->d_K, FAST_PRECOND_JACOBI));
    ATK(cudaMemsetAsync(c->d_f, 0x3F, sizeof(double) * n4, c->stream));
    constexpr int kIt = 64;
    double ms_p = 0.0, ms_k = 0.0;
    c->persist_max_nodes = (int64_t)1 << 40;
    ATK(median_ms(*c, [&] { return pcg_fp64(*c, false, 0.0, kIt, kIt); }, 3, ms_p));
    c->persist_max_nodes = 0;
    ATK(median_ms(*c, [&] { return pcg_fp64(*c, false, 0.0, kIt, kIt); }, 3, ms_k));
    R.us_iter_persistent = ms_p * 1e3 / kIt;
    R.us_iter_kernels = ms_k * 1e3 / kIt;
    c->persist_max_nodes = (ms_p < ms_k) ? std::max<int64_t>(saved, c->nnode) : std::min<int64_t>(saved, c->nnode - 1);
    R.persistent_max_nodes = c->persist_max_nodes;
    c->drop_graphs();
  }
  ATK(cudaMemsetAsync(c->d_p, 0, sizeof(double) * n4, c->stream));
  ATK(cudaMemsetAsync(c->s_p, 0, sizeof(float) * n4, c->stream));
  ATK(cudaStreamSynchronize(c->stream));
  *rep = R;
  return FAST_GPU_OK;
}

// elem_persist.cu - the tensor-core stiffness of every bucket (hex8, hex20,
// B-spline solids, whatever their Gauss rules) in one persistent launch.
//
// The per-colour path (elem_tc.cu, bsp_tc.cu) launches one kernel per
// bucket and colour: the tied four-block column of hex8, hex20 and B-spline
// p=2 / p=3 blocks takes 8 + 8 + 27 + 64 launches, most of them on colours
// far too small to fill the GPU.  Here one cooperative launch of one CTA per
// SM (or as many as fit) walks a device work list:
//
//   * phases: colour k of every bucket forms phase k, since elements of
//     different buckets that share no node can never write the same block;
//     buckets that do share nodes are put one after the other, in bucket
//     order (the order the first-touch flags assume).  Phases are separated
//     by a grid barrier (bounded wait; a time-out sets status bit 2 and every
//     CTA leaves at its next barrier);
//   * within a phase the CTAs take elements one at a time from an atomic
//     counter, the segments of the heaviest element kinds first, so a CTA
//     that drew a degree-3 B-spline element does not hold up the phase while
//     others idle; an element of two 128-row tiles (degree 3) is two work
//     items, one per tile;
//   * a CTA keeps its tensor memory (the widest kind's columns), its two
//     mbarriers and its shared memory across elements; when the next element
//     is of another bucket it sets that bucket up (operands zeroed, Gauss
//     tables brought in) and goes on with the same element functions as the
//     per-colour kernels (tc_hex_body.cuh, tc_bsp_body.cuh).
//
// The elements touching a tied node follow in the tied-interface kernels, as
// on the per-colour path.  Elements run colour by colour without atomics on
// K, so K is the same bits as the per-colour path's.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "elem_common.cuh"
#include "internal.h"
#include "tc_bsp_body.cuh"
#include "tc_hex_body.cuh"

namespace fastgpu {

bool tc_supported(const Bucket &B);

namespace {

using tcb::kThreads;

// the element kinds of the tensor-core path (bucket type x Gauss rule)
enum TcKind {
  kHex8G1, kHex8G8, kHex8G27, kHex20G8, kHex20G27, kHex20G64,
  kBsp222G3, kBsp222G4, kBsp333G4, kBsp332G4, kNumKinds
};

// relative cost of one element of each kind (the segments of a phase are
// handed out heaviest first)
constexpr int kKindWeight[kNumKinds] = {1, 2, 4, 6, 12, 24, 30, 60, 400, 300};

int kind_of(const Bucket &B) {
  if (B.type == FAST_ELEM_HEX8) return B.ng == 1 ? kHex8G1 : B.ng == 8 ? kHex8G8 : B.ng == 27 ? kHex8G27 : -1;
  if (B.type == FAST_ELEM_HEX20) return B.ng == 8 ? kHex20G8 : B.ng == 27 ? kHex20G27 : B.ng == 64 ? kHex20G64 : -1;
  if (B.type == FAST_ELEM_BSP_SOLID) {
    const int *p = B.pd, ng = B.ngp[0];
    if (p[0] == 2 && p[1] == 2 && p[2] == 2) return ng == 3 ? kBsp222G3 : ng == 4 ? kBsp222G4 : -1;
    if (p[0] == 3 && p[1] == 3 && p[2] == 3 && ng == 4) return kBsp333G4;
    if (p[0] == 3 && p[1] == 3 && p[2] == 2 && ng == 4) return kBsp332G4;
  }
  return -1;
}

// shared-memory bytes and tensor-memory columns of a kind (the same template
// arguments as the per-colour launchers)
void kind_shape(int k, int &bytes, int &cols) {
  switch (k) {
#define HEX(K, NN, NG)                        \
  case K:                                     \
    bytes = tcb::TcHex<NN, NG>::bytes;        \
    cols = tcb::TcHex<NN, NG>::TCOLS;         \
    return;
#define BSP(K, A, B, C, G, L)                     \
  case K:                                         \
    bytes = tcb::BspTc<A, B, C, G, L>::bytes;     \
    cols = tcb::BspTc<A, B, C, G, L>::TCOLS;      \
    return;
    HEX(kHex8G1, 8, 1) HEX(kHex8G8, 8, 8) HEX(kHex8G27, 8, 27)
    HEX(kHex20G8, 20, 8) HEX(kHex20G27, 20, 27) HEX(kHex20G64, 20, 64)
    BSP(kBsp222G3, 2, 2, 2, 3, 3) BSP(kBsp222G4, 2, 2, 2, 4, 2) BSP(kBsp333G4, 3, 3, 3, 4, 1)
    BSP(kBsp332G4, 3, 3, 2, 4, 1)
#undef HEX
#undef BSP
    default: bytes = 0; cols = 0; return;
  }
}

__device__ bool kind_setup(int k, const ElemArgs &A, uint8_t *sm, tcb::Cta &c) {
  switch (k) {
    case kHex8G1: return tcb::tc_hex_setup<8, 1>(A, sm, c);
    case kHex8G8: return tcb::tc_hex_setup<8, 8>(A, sm, c);
    case kHex8G27: return tcb::tc_hex_setup<8, 27>(A, sm, c);
    case kHex20G8: return tcb::tc_hex_setup<20, 8>(A, sm, c);
    case kHex20G27: return tcb::tc_hex_setup<20, 27>(A, sm, c);
    case kHex20G64: return tcb::tc_hex_setup<20, 64>(A, sm, c);
    case kBsp222G3: tcb::tc_bsp_setup<2, 2, 2, 3, 3>(sm); return true;
    case kBsp222G4: tcb::tc_bsp_setup<2, 2, 2, 4, 2>(sm); return true;
    case kBsp333G4: tcb::tc_bsp_setup<3, 3, 3, 4, 1>(sm); return true;
    case kBsp332G4: tcb::tc_bsp_setup<3, 3, 2, 4, 1>(sm); return true;
    default: return false;
  }
}

// CTAs that share one element of a kind: the two-tile B-spline kinds are
// split by tile (each part forms and scatters one 128-row tile)
__host__ __device__ constexpr int kind_parts(int k) { return (k == 8 || k == 9) ? 2 : 1; }
static_assert(kind_parts(kBsp333G4) == 2 && kind_parts(kBsp332G4) == 2 && kind_parts(kBsp222G4) == 1, "parts");

__device__ bool kind_element(int k, const ElemArgs &A, float *K32, uint8_t *sm, tcb::Cta &c, int64_t e, int part) {
  switch (k) {
    case kHex8G1: return tcb::tc_hex_element<8, 1>(A, K32, sm, c, 0, e);
    case kHex8G8: return tcb::tc_hex_element<8, 8>(A, K32, sm, c, 0, e);
    case kHex8G27: return tcb::tc_hex_element<8, 27>(A, K32, sm, c, 0, e);
    case kHex20G8: return tcb::tc_hex_element<20, 8>(A, K32, sm, c, 0, e);
    case kHex20G27: return tcb::tc_hex_element<20, 27>(A, K32, sm, c, 0, e);
    case kHex20G64: return tcb::tc_hex_element<20, 64>(A, K32, sm, c, 0, e);
    case kBsp222G3: return tcb::tc_bsp_element<2, 2, 2, 3, 3>(A, K32, sm, c, 0, e);
    case kBsp222G4: return tcb::tc_bsp_element<2, 2, 2, 4, 2>(A, K32, sm, c, 0, e);
    case kBsp333G4: return tcb::tc_bsp_element<3, 3, 3, 4, 1>(A, K32, sm, c, 0, e, part, 2);
    case kBsp332G4: return tcb::tc_bsp_element<3, 3, 2, 4, 1>(A, K32, sm, c, 0, e, part, 2);
    default: return false;
  }
}

struct PersistBucket {
  ElemArgs a;   // the bucket's arguments (first-touch flags, B-spline tables)
  int kind;
  int parts;    // CTAs per element (kind_parts)
};

struct Barrier {
  unsigned int count;
  unsigned int gen;
  int32_t err;
  int32_t pad;
};

constexpr uint64_t kPhaseWaitNs = 1000000000ull;

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barrier of the cooperative launch (arrival counter, generation word);
// every wait is bounded, a time-out or an error posted by another CTA makes
// every CTA return false here.
__device__ bool phase_barrier(Barrier *b, int *ok_sh) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *vgen = &b->gen;
    volatile int32_t *verr = &b->err;
    int ok = *verr == 0;
    if (ok) {
      const unsigned int g = *vgen;
      __threadfence();
      if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
        atomicExch(&b->count, 0u);
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        const uint64_t t0 = now_ns();
        while (*vgen == g) {
          if (*verr != 0) { ok = 0; break; }
          if (now_ns() - t0 > kPhaseWaitNs) { atomicExch(&b->err, 1); ok = 0; break; }
        }
      }
      __threadfence();
    }
    *ok_sh = ok;
  }
  __syncthreads();
  return *ok_sh != 0;
}

struct Plan {
  int nphase;
  const int32_t *phase_seg;        // [nphase + 1] segment ranges of the phases
  const int32_t *seg_bucket;       // [nseg]
  const int64_t *seg_first;        // [nseg] first colour-sorted element
  const int64_t *seg_count;        // [nseg] work items: elements x parts
  const PersistBucket *buckets;    // [nbucket]
  unsigned int *counters;          // [nphase] elements handed out (zero at launch)
  Barrier *bar;                    // (zero at launch)
  float *K32;
  int32_t *status;
};

__global__ void __launch_bounds__(kThreads, 1) elem_persist_kernel(Plan P, uint32_t cols) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh, ok_sh;
  __shared__ long long item_sh;
  __shared__ ElemArgs args_sh;
  __shared__ int kind_sh, parts_sh;
  tcb::Cta c = tcb::cta_begin(cols, bars, &tmem_sh, &fail_sh);
  const int tid = threadIdx.x;
  int cur = -1;   // bucket set up in shared memory
  bool ok = true;
  for (int p = 0; ok && p < P.nphase; p++) {
    const int s0 = P.phase_seg[p], s1 = P.phase_seg[p + 1];
    int64_t total = 0;
    for (int s = s0; s < s1; s++) total += P.seg_count[s];
    while (true) {
      if (tid == 0) item_sh = (long long)atomicAdd(&P.counters[p], 1u);
      __syncthreads();
      int64_t item = (int64_t)item_sh;
      if (item >= total) break;   // (uniform: every thread read the same item)
      int s = s0;
      while (item >= P.seg_count[s]) item -= P.seg_count[s++];
      const int b = P.seg_bucket[s];
      if (b != cur) {
        __syncthreads();
        if (tid == 0) {
          args_sh = P.buckets[b].a;
          kind_sh = P.buckets[b].kind;
          parts_sh = P.buckets[b].parts;
        }
        __syncthreads();
        cur = b;
        if (!kind_setup(kind_sh, args_sh, sm, c)) { ok = false; break; }
      }
      const int64_t el = item / parts_sh;
      if (!kind_element(kind_sh, args_sh, P.K32, sm, c, P.seg_first[s] + el, (int)(item - el * parts_sh))) {
        ok = false;
        break;
      }
    }
    if (!ok) {
      if (tid == 0) atomicExch(&P.bar->err, 1);
      break;
    }
    if (!phase_barrier(P.bar, &ok_sh)) {
      if (tid == 0) atomicExch(c.fail, 1);
      ok = false;
    }
  }
  tcb::cta_end(c, cols, P.status);
}

}  // namespace

// The plan of one mesh (built once per upload, kept in Ctx::persist).
struct PersistPlanHost {
  int nphase = 0;
  int bytes = 0, cols = 0;
  void *d_mem = nullptr;     // every device array of the plan in one allocation
  Plan plan{};
};

void free_persist_plan(Ctx &c) {
  if (!c.persist) return;
  if (c.persist->d_mem) cudaFree(c.persist->d_mem);
  delete c.persist;
  c.persist = nullptr;
}

namespace {

cudaError_t build_plan(Ctx &c, PersistPlanHost &H) {
  const int nb = (int)c.buckets.size();
  if (nb == 0 || nb > 64) return cudaErrorNotSupported;
  std::vector<int> kind(nb);
  for (int b = 0; b < nb; b++) {
    if (!tc_supported(c.buckets[b]) || (kind[b] = kind_of(c.buckets[b])) < 0) return cudaErrorNotSupported;
    int by, co;
    kind_shape(kind[b], by, co);
    H.bytes = std::max(H.bytes, by);
    H.cols = std::max(H.cols, co);
  }
  // buckets whose regular elements share a node are phased one after the other
  std::vector<uint64_t> node_mask((size_t)c.nnode, 0);
  for (int b = 0; b < nb; b++) {
    const Bucket &B = c.buckets[b];
    for (size_t i = 0; i < (size_t)B.ne_regular * B.nn; i++) node_mask[B.h_conn[i]] |= 1ull << b;
  }
  std::vector<uint64_t> conflict(nb, 0);
  for (uint64_t m : node_mask)
    for (int b = 0; b < nb; b++)
      if ((m >> b) & 1) conflict[b] |= m & ~(1ull << b);
  std::vector<int> offset(nb, 0), ncol(nb);
  int nphase = 0;
  for (int b = 0; b < nb; b++) {
    ncol[b] = (int)c.buckets[b].color_off.size() - 1;
    for (int q = 0; q < b; q++)
      if ((conflict[b] >> q) & 1) offset[b] = std::max(offset[b], offset[q] + ncol[q]);
    nphase = std::max(nphase, offset[b] + ncol[b]);
  }
  // segments of each phase, heaviest kind first
  std::vector<int32_t> phase_seg(nphase + 1, 0), seg_bucket;
  std::vector<int64_t> seg_first, seg_count;
  std::vector<int> order(nb);
  for (int b = 0; b < nb; b++) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return kKindWeight[kind[x]] > kKindWeight[kind[y]]; });
  for (int p = 0; p < nphase; p++) {
    for (int b : order) {
      const int k = p - offset[b];
      if (k < 0 || k >= ncol[b]) continue;
      const Bucket &B = c.buckets[b];
      const int64_t cnt = B.color_off[k + 1] - B.color_off[k];
      if (cnt <= 0) continue;
      seg_bucket.push_back(b);
      seg_first.push_back(B.color_off[k]);
      seg_count.push_back(cnt * kind_parts(kind[b]));
    }
    phase_seg[p + 1] = (int32_t)seg_bucket.size();
  }
  std::vector<PersistBucket> pb(nb);
  for (int b = 0; b < nb; b++) {
    const Bucket &B = c.buckets[b];
    ElemArgs a{};
    a.conn = B.d_conn;
    a.E = B.d_E;
    a.nu = B.d_nu;
    a.slot = B.d_slot;
    a.X = c.d_X;
    a.fix = c.d_fix;
    a.dN = B.d_dN;
    a.w = B.d_w;
    a.status = c.d_status;
    a.span = B.d_span;
    for (int d = 0; d < 3; d++) a.bas[d] = B.d_bas ? B.d_bas + B.bas_off[d] : nullptr;
    a.wt = B.d_wt;
    a.rational = B.rational;
    pb[b].a = a;   // first-touch flags are set per launch
    pb[b].kind = kind[b];
    pb[b].parts = kind_parts(kind[b]);
  }
  // one allocation: buckets, counters + barrier, then the index arrays
  const size_t nseg = seg_bucket.size();
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
  const size_t o_b = take(sizeof(PersistBucket) * nb), o_cnt = take(sizeof(unsigned int) * nphase + sizeof(Barrier));
  const size_t o_ps = take(sizeof(int32_t) * (nphase + 1)), o_sb = take(sizeof(int32_t) * std::max<size_t>(nseg, 1));
  const size_t o_sf = take(sizeof(int64_t) * std::max<size_t>(nseg, 1)), o_sc = take(sizeof(int64_t) * std::max<size_t>(nseg, 1));
  cudaError_t e = cudaMalloc(&H.d_mem, off);
  if (e != cudaSuccess) return e;
  uint8_t *m = static_cast<uint8_t *>(H.d_mem);
  e = cudaMemcpy(m + o_b, pb.data(), sizeof(PersistBucket) * nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m + o_ps, phase_seg.data(), sizeof(int32_t) * (nphase + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nseg) e = cudaMemcpy(m + o_sb, seg_bucket.data(), sizeof(int32_t) * nseg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nseg) e = cudaMemcpy(m + o_sf, seg_first.data(), sizeof(int64_t) * nseg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nseg) e = cudaMemcpy(m + o_sc, seg_count.data(), sizeof(int64_t) * nseg, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  H.nphase = nphase;
  Plan &P = H.plan;
  P.nphase = nphase;
  P.phase_seg = reinterpret_cast<const int32_t *>(m + o_ps);
  P.seg_bucket = reinterpret_cast<const int32_t *>(m + o_sb);
  P.seg_first = reinterpret_cast<const int64_t *>(m + o_sf);
  P.seg_count = reinterpret_cast<const int64_t *>(m + o_sc);
  P.buckets = reinterpret_cast<const PersistBucket *>(m + o_b);
  P.counters = reinterpret_cast<unsigned int *>(m + o_cnt);
  P.bar = reinterpret_cast<Barrier *>(m + o_cnt + sizeof(unsigned int) * nphase);
  P.status = c.d_status;
  return cudaSuccess;
}

}  // namespace

// Whether the mesh's tensor-core stiffness can take the persistent launch
// (every bucket of a kind it knows, at most 64 buckets)
bool persist_supported(const Ctx &c) {
  if (c.buckets.empty() || c.buckets.size() > 64) return false;
  for (const Bucket &B : c.buckets)
    if (!tc_supported(B) || kind_of(B) < 0) return false;
  return true;
}

// The regular elements of every bucket into K32 in one cooperative launch
// (K32 zero-filled beforehand unless the first-touch flags are in use).
cudaError_t launch_persist_elements(Ctx &c, float *K32) {
  if (!c.persist) {
    c.persist = new PersistPlanHost();
    cudaError_t e = build_plan(c, *c.persist);
    if (e != cudaSuccess) {
      free_persist_plan(c);
      return e;
    }
  }
  PersistPlanHost &H = *c.persist;
  if (H.nphase == 0) return cudaSuccess;
  // first-touch flags of this launch, per bucket
  const bool ft = c.use_first_touch();
  if (ft != c.persist_first) {
    std::vector<PersistBucket> pb(c.buckets.size());
    cudaError_t e = cudaStreamSynchronize(c.stream);   // no launch of the old arguments still reads them
    if (e == cudaSuccess) e = cudaMemcpy(pb.data(), H.plan.buckets, sizeof(PersistBucket) * pb.size(), cudaMemcpyDeviceToHost);
    for (size_t b = 0; b < pb.size() && e == cudaSuccess; b++) {
      pb[b].a.first = ft ? c.buckets[b].d_first : nullptr;
      pb[b].a.fw = first_words(c.buckets[b].nn);
    }
    if (e == cudaSuccess)
      e = cudaMemcpy(const_cast<PersistBucket *>(H.plan.buckets), pb.data(), sizeof(PersistBucket) * pb.size(),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    c.persist_first = ft;
  }
  auto kern = elem_persist_kernel;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, H.bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, H.bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm * H.cols > 512) per_sm = 512 / H.cols;   // tensor memory of the resident CTAs
  const unsigned grid = (unsigned)(per_sm * c.sm_count);
  e = cudaMemsetAsync(H.plan.counters, 0, sizeof(unsigned int) * H.nphase + sizeof(Barrier), c.stream);
  if (e != cudaSuccess) return e;
  Plan P = H.plan;
  P.K32 = K32;
  uint32_t cols = (uint32_t)H.cols;
  void *args[] = {&P, &cols};
  e = cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(kThreads), args, (size_t)H.bytes, c.stream);
  c.launches++;
  return e;
}

}  // namespace fastgpu

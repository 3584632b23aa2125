// tc_hex_body.cuh - one hex element's stiffness on the tensor cores
// (tcgen05.mma.kind::tf32, TF32 operands split in three, FP32 accumulators in
// tensor memory), as device functions shared by the per-colour kernel
// (elem_tc.cu) and the persistent multi-bucket kernel (elem_persist.cu).
// Private to libfastgpu.
//
// Computes what cElmParam::StiffMat (elc/elmparam.cpp:539-597) computes for
// an isotropic solid element, K_e = sum_g w_g detJ_g B_g^T C B_g, in the
// factored form used by elem_kernels.cu: with D[(i,a)][g] = sqrt(c_g)
// dN_a/dx_i(g) (c_g = w_g detJ_g, detJ > 0 required), the Gauss-point
// contraction
//     H = D D^T,   H[(i,a),(j,b)] = sum_g c_g dN_a/dx_i dN_b/dx_j ,
// is the one dense product of the element (the MatTripBtCB of
// mlib/matvec.cpp:372-388, regrouped), and the 3x3 block (a, b) of K_e follows
// from H and the isotropic C (cSolid::QMatrix, elc/anmodel.cpp:1286-1298):
//     i == j : C00 H_ii + G (tr - H_ii),   i != j : C01 H_ij + G H_ji .
//
// The product serves the mixed-precision path, whose stiffness has to be as
// accurate as its FP32 storage: the iteration's FP32 operator and the FP64
// residual it is corrected by may differ by little more than FP32 rounding,
// or the corrections stall on ill-conditioned systems.  H is formed on the
// tensor cores from TF32 operands split in three, D = D_hi + D_lo + D_mid,
// as the six partial products down to 2^-22 of the product (D_lo D_lo^T,
// D_hi D_mid^T, D_mid D_hi^T, D_hi D_lo^T, D_lo D_hi^T, D_hi D_hi^T, smallest
// first) accumulated in FP32; the dropped terms are below 2^-32 of it.  (The
// two-part "3xTF32" product leaves about 2^-21, some 8x the FP32 rounding of
// the entries, which stalled the corrections on slender and large models.)
// The blocks are added into an FP32 block matrix.  Geometry (Jacobian,
// determinant, inverse, dN/dx) stays in FP64.
//
// Per element (one CTA, 256 threads):
//   1. one thread starts bulk copies (cp.async.bulk, completion on mbarrier
//      0) of the elements' incidence rows, NN x NN slot rows and first-touch
//      flags; the natural-derivative table is read through L1;
//   2. coordinates are gathered, the element's current FP32 K blocks are
//      requested with cp.async (they arrive while the element is computed);
//   3. Jacobians, inverses and D in FP64; D is split and written as three
//      K-major TF32 operands (rows (i, a), K = Gauss points padded to 8);
//   4. one elected thread issues 6 x KP/8 tcgen05.mma (M = 128 rows, N = the
//      rows rounded up to 16; A and B are operands in shared memory) and
//      commits them to mbarrier 1;
//   5. the accumulator is read back with tcgen05.ld (one thread per row),
//      staged as H in shared memory, turned into 3x3 blocks by one thread per
//      node pair and added to the old blocks; the write-back is coalesced and
//      skips DOFs without an equation (a block's first write stores it).
// Elements of a colour share no node, so the scatter needs no atomics and K
// is bit-identical from run to run.  Every mbarrier wait is bounded (1 s): a
// wait that runs out sets the CTA's failure flag; the element function waits
// once more (bounded) for its work in flight and returns false.
#pragma once

#include <cstdint>

#include "elem_common.cuh"
#include "tc_common.cuh"

namespace fastgpu {
namespace tcb {

constexpr uint64_t kWaitNs = 1000000000ull;
constexpr int kThreads = 256;

__host__ __device__ constexpr int pow2_cols(int n) {
  return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : (n <= 256 ? 256 : 512)));
}

// Per-CTA state of the tensor-core element functions: two mbarriers in shared
// memory with the parity each waits for next, the tensor-memory base and the
// CTA's failure flag.  Every element function leaves both barriers idle.
struct Cta {
  uint64_t *bars;
  uint32_t phase[2];
  uint32_t tmem;
  int *fail;
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(tc::smem_u32(smem)), "l"(gmem));
}

// One CTA's start: `cols` columns of tensor memory, both barriers, the flag.
__device__ __forceinline__ Cta cta_begin(uint32_t cols, uint64_t *bars, uint32_t *tmem_sh, int *fail_sh) {
  const int tid = threadIdx.x;
  if ((tid >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_sh)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *fail_sh = 0;
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  Cta c;
  c.bars = bars;
  c.phase[0] = c.phase[1] = 0;
  c.tmem = *tmem_sh;
  c.fail = fail_sh;
  return c;
}

// The CTA's end: status bit 2 on a failed wait, tensor memory freed.
__device__ __forceinline__ void cta_end(const Cta &c, uint32_t cols, int32_t *status) {
  __syncthreads();
  if (*c.fail && threadIdx.x == 0) atomicOr(status, 4);
  tc::fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(cols) : "memory");
}

// bounded wait on barrier b of the CTA for its next phase; false on time-out
// (the flag is set)
__device__ __forceinline__ bool wait_bar(Cta &c, int b) {
  const bool ok = tc::mbar_wait(&c.bars[b], c.phase[b], kWaitNs);
  c.phase[b] ^= 1;
  if (!ok) atomicExch(c.fail, 1);
  return ok;
}

// the same, and after a time-out one more bounded wait for the work still
// in flight on that barrier (bulk copies or MMAs must not land in the shared
// memory of a CTA that has moved on or exited)
__device__ __forceinline__ bool wait_bar_drain(Cta &c, int b) {
  if (wait_bar(c, b)) return true;
  tc::mbar_wait(&c.bars[b], c.phase[b] ^ 1, kWaitNs);
  return false;
}

// EPT elements share one 128-row operand tile: rows j*R .. j*R+R-1 hold
// element j (hex8: five elements, hex20: two), and the MMA forms all their
// products at once (the off-diagonal blocks between elements are not read),
// so every phase of a pass works on EPT elements between the same barriers.
template <int NN, int NG, int EPT = 1>
struct TcHex {
  static constexpr int R = 3 * NN;                 // operand rows (i, a) of one element, i-major
  static constexpr int KP = (NG + 7) / 8 * 8;      // Gauss points padded to the MMA K
  static constexpr int N = (EPT * R + 15) / 16 * 16;  // accumulator columns (M = 128 needs N % 16 == 0)
  static constexpr int RP = 128;                   // operand rows held (one M tile)
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int OPB = RP * KP * 4;          // bytes of one operand part (hi, lo or mid)
  static constexpr int TCOLS = pow2_cols(N);
  static_assert(EPT * R <= 128, "the elements of a pass share one M tile");
  static_assert(NP <= kThreads, "one thread per node pair");
  static_assert((NN * NN * 4) % 16 == 0 && (NN * 4) % 16 == 0 && (NG * NN * 3 * 8) % 16 == 0,
                "bulk-copy sizes are multiples of 16 bytes");
  // shared memory carve-up (bytes from a 1024-aligned base, every piece on a
  // 16-byte boundary); per-element pieces repeat EPT times at stride s*
  static constexpr int al(int x) { return (x + 15) / 16 * 16; }
  // (new blocks staged as V by one thread per node pair and old blocks by
  // cp.async measured faster than forming each entry in the write-back, with
  // or without the old-block staging: 8.3 against 10.0 ms on the hex20 box)
  static constexpr int sH = al(R * R * 4), sKo = al(NN * NN * 9 * 4), sV = al(NP * 9 * 4);
  static constexpr int sX = al(NN * 3 * 8), sJ = al(NG * 9 * 8), sC = al(NG * 8);
  static constexpr int FW = (NN * NN + 127) / 128 * 4;        // first-touch flag words (first_words)
  static constexpr int sSlot = al(NN * NN * 4), sConn = al(NN * 4), sFirst = FW * 4, sFix = al(NN);
  static constexpr int oHi = 0, oLo = oHi + OPB, oMid = oLo + OPB;
  // H is staged over the operands (dead once the MMAs completed); the next
  // pass rewrites the operand rows it uses and zeroes their K padding
  static constexpr int oH = 0;                                // float [EPT][R][R]
  static constexpr int sOpH = 3 * OPB > EPT * sH ? 3 * OPB : EPT * sH;
  static constexpr int oKo = sOpH;                            // float [EPT][NN*NN][9] old blocks
  static constexpr int oV = oKo + EPT * sKo;                  // float [EPT][NP][9] new blocks
  static constexpr int ow = oV + EPT * sV;                    // double [NG] (the natural derivatives stay in global memory, read through L1)
  static constexpr int oX = ow + al(NG * 8);                  // double [EPT][NN][3]
  static constexpr int oJ = oX + EPT * sX;                    // double [EPT][NG][9]
  static constexpr int oc = oJ + EPT * sJ;                    // double [EPT][NG]
  static constexpr int oSlot = oc + EPT * sC;                 // int32 [EPT][NN][NN] (bulk-copy targets)
  static constexpr int oConn = oSlot + EPT * sSlot;           // int32 [EPT][NN] (bulk-copy targets)
  static constexpr int oFirst = oConn + EPT * sConn;          // uint32 [EPT][FW] (bulk-copy targets)
  static constexpr int oCst = oFirst + EPT * sFirst;          // double [EPT][3] C00, C01, G
  static constexpr int oFix = oCst + EPT * 32;                // uint8 [EPT][NN]
  static constexpr int used = oFix + EPT * sFix;
  static_assert(oSlot % 16 == 0 && oConn % 16 == 0 && oFirst % 16 == 0 && OPB % 16 == 0 &&
                    sFirst % 16 == 0 && sSlot % 16 == 0 && sConn % 16 == 0,
                "bulk-copy targets on 16-byte boundaries");
  static constexpr int bytes = used + 1024;                   // + alignment slack of the base
  static_assert(bytes <= 232448, "shared memory of one CTA");
};

// A hex bucket's set-up in a CTA: operands zeroed, the Gauss weights in
// shared memory.  False on a failed wait.
template <int NN, int NG, int EPT = 1>
__device__ bool tc_hex_setup(const ElemArgs &A, uint8_t *sm, Cta &c) {
  using S = TcHex<NN, NG, EPT>;
  const int tid = threadIdx.x;
  for (int i = tid; i < 3 * S::OPB / 16; i += kThreads) reinterpret_cast<uint4 *>(sm + S::oHi)[i] = make_uint4(0, 0, 0, 0);
  double *sw = reinterpret_cast<double *>(sm + S::ow);
  for (int g = tid; g < NG; g += kThreads) sw[g] = A.w[g];
  __syncthreads();
  return *c.fail == 0;
}

// One pass over nv <= EPT elements: element j is launch item its[j] at
// colour-sorted position es[j] (the same values in every thread).  Their
// blocks go into K32 (null: only the dense FP64 element matrices into
// A.Ke_out, at the items' positions).  False on a failed wait, after the
// work in flight has finished (bounded).
template <int NN, int NG, int EPT>
__device__ bool tc_hex_elements(const ElemArgs &A, float *__restrict__ K32, uint8_t *sm, Cta &c,
                                const int64_t (&its)[EPT], const int64_t (&es)[EPT], int nv) {
  using S = TcHex<NN, NG, EPT>;
  constexpr int R = S::R, KP = S::KP, N = S::N, NP = S::NP;
  uint8_t *opHi = sm + S::oHi, *opLo = sm + S::oLo, *opMid = sm + S::oMid;
  const double *__restrict__ sdN = A.dN;   // [NG][NN][3], read through L1
  double *sw = reinterpret_cast<double *>(sm + S::ow);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t kLBO = 128, kSBO = (KP / 4) * 128;
  constexpr uint32_t kId = tc::idesc(128, N, tc::kTypeTF32);
  auto H = [&](int j) { return reinterpret_cast<float *>(sm + S::oH + j * S::sH); };
  auto Ko = [&](int j) { return reinterpret_cast<float *>(sm + S::oKo + j * S::sKo); };
  auto V = [&](int j) { return reinterpret_cast<float *>(sm + S::oV + j * S::sV); };
  auto X = [&](int j) { return reinterpret_cast<double *>(sm + S::oX + j * S::sX); };
  auto Jm = [&](int j) { return reinterpret_cast<double *>(sm + S::oJ + j * S::sJ); };
  auto Cg = [&](int j) { return reinterpret_cast<double *>(sm + S::oc + j * S::sC); };
  auto Slot = [&](int j) { return reinterpret_cast<int32_t *>(sm + S::oSlot + j * S::sSlot); };
  auto Conn = [&](int j) { return reinterpret_cast<int32_t *>(sm + S::oConn + j * S::sConn); };
  auto First = [&](int j) { return reinterpret_cast<uint32_t *>(sm + S::oFirst + j * S::sFirst); };
  auto Fix = [&](int j) { return sm + S::oFix + j * S::sFix; };
  auto Cst = [&](int j) { return reinterpret_cast<double *>(sm + S::oCst + j * 32); };

  __syncthreads();
  if (tid == 0) {
    tc::mbar_arrive_tx(&c.bars[0], nv * (NN * NN * 4 + NN * 4 + (A.first ? S::FW * 4 : 0)));
    for (int j = 0; j < nv; j++) {
      tc::bulk_g2s(Slot(j), A.slot + es[j] * NN * NN, NN * NN * 4, &c.bars[0]);
      tc::bulk_g2s(Conn(j), A.conn + es[j] * NN, NN * 4, &c.bars[0]);
      if (A.first) tc::bulk_g2s(First(j), A.first + es[j] * S::FW, S::FW * 4, &c.bars[0]);
    }
  }
  wait_bar_drain(c, 0);
  __syncthreads();
  if (*c.fail) return false;
  for (int t = tid; t < nv * NN * 3; t += kThreads) {
    const int j = t / (NN * 3), i = t - j * NN * 3;
    X(j)[i] = A.X[3 * (int64_t)Conn(j)[i / 3] + (i % 3)];
  }
  for (int t = tid; t < nv * NN; t += kThreads) {
    const int j = t / NN, i = t - j * NN;
    Fix(j)[i] = A.fix[Conn(j)[i]];
  }
  if (K32) {
    if (BlockWalk<NN, kThreads>::takes(tid))
      for (BlockWalk<NN, kThreads> w(tid); w.j < nv; w.next()) {
        const int q = w.qq();
        // a block this element writes first is not read
        if (!(A.first && ((First(w.j)[q >> 5] >> (q & 31)) & 1u)))
          cp_async4(Ko(w.j) + 9 * q + w.k, K32 + (int64_t)Slot(w.j)[q] * 9 + w.k);
      }
    asm volatile("cp.async.commit_group;\n" ::);
  }
  __syncthreads();
  // the isotropic constants of each element (cSolid::QMatrix, elc/anmodel.cpp:1286-1298)
  if (tid < nv) {
    const double E = A.E[es[tid]], nu = A.nu[es[tid]];
    const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
    double *cs = Cst(tid);
    cs[0] = E * (1.0 - nu) / dd;
    cs[1] = E * nu / dd;
    cs[2] = 0.5 * E / (1.0 + nu);
  }
  // Jacobians J[g][p][q] = sum_a dN_a/dxi_p X_a,q (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126)
  for (int t = tid; t < nv * NG * 9; t += kThreads) {
    const int j = t / (NG * 9), tt = t - j * NG * 9;
    const int g = tt / 9, pq = tt - 9 * g, p = pq / 3, q = pq - 3 * p;
    const double *d = sdN + g * NN * 3 + p;
    const double *x = X(j);
    double s = 0.0;
#pragma unroll 4
    for (int a = 0; a < NN; a++) s += d[3 * a] * x[3 * a + q];
    Jm(j)[tt] = s;
  }
  __syncthreads();
  // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
  for (int t = tid; t < nv * NG; t += kThreads) {
    const int j = t / NG, g = t - j * NG;
    double *J = Jm(j) + 9 * g;
    const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                 j21 = J[7], j22 = J[8];
    const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
    if (!(det > 0.0)) atomicOr(A.status, 1);
    const double id = 1.0 / ((det != 0.0) ? det : 1.0);
    J[0] = (j11 * j22 - j12 * j21) * id;
    J[1] = -(j01 * j22 - j02 * j21) * id;
    J[2] = (j01 * j12 - j02 * j11) * id;
    J[3] = -(j10 * j22 - j12 * j20) * id;
    J[4] = (j00 * j22 - j02 * j20) * id;
    J[5] = -(j00 * j12 - j02 * j10) * id;
    J[6] = (j10 * j21 - j11 * j20) * id;
    J[7] = -(j00 * j21 - j01 * j20) * id;
    J[8] = (j00 * j11 - j01 * j10) * id;
    Cg(j)[g] = sqrt(fmax(sw[g] * det, 0.0));
  }
  __syncthreads();
  // the K padding (Gauss points NG..KP-1) of the rows in use: zero (the last
  // pass staged H over it)
  if (KP > NG)
    for (int t = tid; t < nv * R * (KP - NG); t += kThreads) {
      const int r = t / (KP - NG), g = NG + (t - r * (KP - NG));
      const uint32_t off = tc::kmajor_off4(r, g, KP);
      *reinterpret_cast<uint32_t *>(opHi + off) = 0u;
      *reinterpret_cast<uint32_t *>(opLo + off) = 0u;
      *reinterpret_cast<uint32_t *>(opMid + off) = 0u;
    }
  // D[(i,a)][g] = sqrt(c_g) dN_a/dx_i, split into three TF32 operands; element
  // j on rows j*R .. j*R+R-1
  for (int t = tid; t < nv * NG * NN; t += kThreads) {
    const int j = t / (NG * NN), tt = t - j * NG * NN;
    const int g = tt / NN, a = tt - NN * g;
    const double *J = Jm(j) + 9 * g;
    const double *dn = sdN + (g * NN + a) * 3;
    const double d0 = dn[0], d1 = dn[1], d2 = dn[2], sq = Cg(j)[g];
    const double x[3] = {sq * (J[0] * d0 + J[1] * d1 + J[2] * d2), sq * (J[3] * d0 + J[4] * d1 + J[5] * d2),
                         sq * (J[6] * d0 + J[7] * d1 + J[8] * d2)};
#pragma unroll
    for (int i = 0; i < 3; i++) {
      uint32_t hi, lo, mid;
      tc::split3_tf32(x[i], hi, lo, mid);
      const uint32_t off = tc::kmajor_off4(j * R + i * NN + a, g, KP);
      *reinterpret_cast<uint32_t *>(opHi + off) = hi;
      *reinterpret_cast<uint32_t *>(opLo + off) = lo;
      *reinterpret_cast<uint32_t *>(opMid + off) = mid;
    }
  }
  tc::fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tc::fence_after();
    const uint32_t part[3] = {tc::smem_u32(opHi), tc::smem_u32(opLo), tc::smem_u32(opMid)};
#pragma unroll
    for (int tm = 0; tm < tc::kSplitTerms; tm++) {
      int pa_, pb_;
      tc::split_term(tm, pa_, pb_);
#pragma unroll
      for (int kk = 0; kk < KP / 8; kk++)
        tc::mma_tf32(c.tmem, tc::smem_desc(part[pa_] + kk * 256, kLBO, kSBO),
                     tc::smem_desc(part[pb_] + kk * 256, kLBO, kSBO), kId, (tm > 0 || kk > 0) ? 1u : 0u);
    }
    tc::commit(&c.bars[1]);
  }
  wait_bar_drain(c, 1);
  __syncthreads();
  if (*c.fail) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    return false;
  }
  tc::fence_after();
  // accumulator -> H_j (lane = row j*R + (i, a), columns j*R + (j', b) of its own element)
  if (warp < 4 && warp * 32 < nv * R) {
    const int r = warp * 32 + lane;
    const int j = r / R, rr = r - j * R;
    const uint32_t tb = c.tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < N; c0 += 8) {
      float v[8];
      tc::ld_32x32b_x8(tb + c0, v);
      if (r < nv * R) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int col = c0 + k - j * R;
          if (col >= 0 && col < R) H(j)[rr * R + col] = v[k];
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  // block (a, b), entry (i, jj) of element j from H, in FP64: for a > b the
  // transpose of block (b, a) (K_e stays exactly symmetric)
  auto block_value = [&](int j, int a, int b, int i, int jj) -> double {
    const float *Hj = H(j);
    const bool up = a <= b;
    const int pa = up ? a : b, pb = up ? b : a, ii = up ? i : jj, j2 = up ? jj : i;
    const double *cs = Cst(j);
    if (ii == j2) {
      const double h0 = Hj[pa * R + pb], h1 = Hj[(NN + pa) * R + NN + pb], h2 = Hj[(2 * NN + pa) * R + 2 * NN + pb];
      const double tr = h0 + h1 + h2;
      const double hd = ii == 0 ? h0 : (ii == 1 ? h1 : h2);
      return cs[0] * hd + cs[2] * (tr - hd);
    }
    return cs[1] * (double)Hj[(ii * NN + pa) * R + j2 * NN + pb] + cs[2] * (double)Hj[(j2 * NN + pa) * R + ii * NN + pb];
  };
  for (int t = tid; t < nv * NP; t += kThreads) {
    const int j = t / NP, pp = t - j * NP;
    int pa, pb;
    pair_of(pp, NN, pa, pb);
    double v[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) v[3 * i + jj] = block_value(j, pa, pb, i, jj);
    if (A.Ke_out) {
      constexpr int ND = 3 * NN;
      double *Kout = A.Ke_out + its[j] * ND * ND;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          Kout[(3 * pa + i) * ND + 3 * pb + jj] = v[3 * i + jj];
          Kout[(3 * pb + jj) * ND + 3 * pa + i] = v[3 * i + jj];
        }
    }
    float *Vj = V(j);
#pragma unroll
    for (int k = 0; k < 9; k++) Vj[9 * pp + k] = (float)v[k];
  }
  if (K32) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // old + new for every entry whose two DOFs have equations (block (b, a)
    // is the transpose of (a, b)); first writes store new, fixed entries too
    if (BlockWalk<NN, kThreads>::takes(tid)) {
      BlockWalk<NN, kThreads> w(tid);
      const int k = w.k, i = k / 3, jj = k - 3 * i, kt = 3 * jj + i;
      for (; w.j < nv; w.next()) {
        const int j = w.j, a = w.a, b = w.b, q = w.qq();
        const bool fst = A.first && ((First(j)[q >> 5] >> (q & 31)) & 1u);
        const uint8_t *fx = Fix(j);
        const bool fixed = ((fx[a] >> i) & 1) || ((fx[b] >> jj) & 1);
        const float add = V(j)[upper_entry<NN>(a, b, k, kt)];
        float out;
        if (entry_value(fst, fixed, a == b && i == jj, fst ? 0.f : Ko(j)[9 * q + k], add, out))
          K32[(int64_t)Slot(j)[q] * 9 + k] = out;
      }
    }
  }
  return true;
}

// One element (the persistent kernel's unit of work)
template <int NN, int NG>
__device__ bool tc_hex_element(const ElemArgs &A, float *__restrict__ K32, uint8_t *sm, Cta &c, int64_t it,
                               int64_t e) {
  const int64_t its[1] = {it}, es[1] = {e};
  return tc_hex_elements<NN, NG, 1>(A, K32, sm, c, its, es, 1);
}

}  // namespace tcb
}  // namespace fastgpu

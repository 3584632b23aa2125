// tc_bsp_body.cuh - one B-spline / NURBS solid element's stiffness on the
// tensor cores, as device functions shared by the per-colour kernel
// (bsp_tc.cu) and the persistent multi-bucket kernel (elem_persist.cu).
// Private to libfastgpu.
//
// The element is that of bsp_kernels.cu (cElmParam::StiffMat,
// elc/elmparam.cpp:539-597, on the basis of cShapeBspSolid,
// shp/shpbsp.cpp:928-1067): geometry in FP64 from the Bezier-extracted span
// tables, then the Gauss-point contraction
//     H[(a,i),(b,j)] = sum_g c_g dN_a/dx_i(g) dN_b/dx_j(g),   c_g = w_g detJ_g,
// and the isotropic 3x3 block of each node pair (cSolid::QMatrix,
// elc/anmodel.cpp:1286-1298).  c_g keeps its sign (a left-handed patch has
// detJ < 0, as in the reference), so the two factors differ: A rows
// (a, i) hold c_g dN_a/dx_i, B rows (b, j) hold dN_b/dx_j, and H = A B^T is
// formed from TF32 parts A = A_hi + A_lo + A_mid, B likewise, as the six
// partial products down to 2^-22 of the product, smallest first (FP32
// accumulation: FP32-accurate entries, as the mixed-precision path whose
// stiffness is FP32 needs; see tc_hex_body.cuh).
//
// Layout.  A rows are node-major in quads, row 4a + i (i < 3; row 4a + 3 is
// zero), so the three rows of a node sit in one warp's tensor-memory lanes;
// B rows are 3b + j.  The Gauss points are taken in chunks of whole t-layers
// (the degree-3 element's 64 points as four chunks of 16), each chunk's
// geometry computed into shared memory, its operands written into one of two
// buffers, and its MMAs issued while the next chunk's geometry is computed;
// all chunks accumulate into the same tensor memory (two 128-row tiles when
// 4 NN > 128).  Epilogue: one thread per row reads its accumulator row with
// tcgen05.ld; the 3x3 block (a, b) is gathered across the quad of node a with
// warp shuffles; thread (a, i) writes row i of block (a, b) and column i of
// block (b, a) for b >= a, so K stays exactly symmetric.  Elements run one
// colour at a time, no atomics: K is bit-identical run to run.  Every
// mbarrier wait is bounded (1 s): on a time-out the CTA's failure flag is set
// and the element function waits once more (bounded) for the MMAs in flight
// and returns false.
#pragma once

#include <cstdint>

#include "elem_common.cuh"
#include "tc_common.cuh"
#include "tc_hex_body.cuh"

namespace fastgpu {
namespace tcb {

template <int PR, int PS, int PT, int NG1, int LPC>
struct BspTc {
  static constexpr int QR = PR + 1, QS = PS + 1, QT = PT + 1;
  static constexpr int NN = QR * QS * QT;
  static constexpr int NG = NG1 * NG1 * NG1;
  static constexpr int GCH = LPC * NG1 * NG1;          // Gauss points per chunk
  static constexpr int NCH = NG1 / LPC;                 // chunks per element
  static constexpr int KC = (GCH + 7) / 8 * 8;          // chunk K padded to the MMA K
  static constexpr int MT = (4 * NN + 127) / 128;       // 128-row tiles of A
  static constexpr int RA = MT * 128;                   // A rows held
  static constexpr int NGRP = (NN + 7) / 8;             // epilogue column groups of 8 nodes (24 columns)
  static constexpr int NB = ((3 * NN > NGRP * 24 ? 3 * NN : NGRP * 24) + 15) / 16 * 16;  // B rows = N
  static constexpr int TSTRIDE = 256;                   // tensor-memory column offset of tile 1
  static constexpr int TCOLS = MT == 1 ? (NB <= 32 ? 32 : NB <= 64 ? 64 : NB <= 128 ? 128 : 256) : 512;
  static constexpr int NBUF = NCH > 1 ? 2 : 1;
  static constexpr int OA = RA * KC * 4, OB = NB * KC * 4;
  static constexpr int OBUF = 3 * OA + 3 * OB;          // A_hi, A_lo, A_mid, B_hi, B_lo, B_mid
  static_assert(NG1 % LPC == 0, "whole chunks");
  static_assert(MT <= 2 && NB <= 256, "at most two M tiles, N <= 256");
  static constexpr int al(int x) { return (x + 15) / 16 * 16; }
  static constexpr int oOp = 0;                                  // NBUF operand buffers
  static constexpr int oD = oOp + NBUF * OBUF;                   // double [GCH][3][NN]
  static constexpr int oB = oD + al(GCH * 3 * NN * 8);           // double [GCH][NN] rational numerators
  static constexpr int oJ = oB + al(GCH * NN * 8);               // double [GCH][9]
  static constexpr int oc = oJ + al(GCH * 9 * 8);                // double [GCH]
  static constexpr int oWg = oc + al(GCH * 8);                   // double [GCH][4]
  static constexpr int oX = oWg + al(GCH * 4 * 8);               // double [NN][3]
  static constexpr int oW = oX + al(NN * 3 * 8);                 // double [NN]
  static constexpr int oFix = oW + al(NN * 8);                   // uint8 [NN]
  static constexpr int bytes = oFix + al(NN) + 1024;             // + alignment slack of the base
  static_assert(OA % 16 == 0 && OB % 16 == 0, "operand sections on 16-byte boundaries");
  static_assert(bytes <= 232448, "shared memory of one CTA");
};

// A B-spline bucket's set-up in a CTA: the operand buffers zeroed (K padding
// columns and pad rows stay zero for every element).
template <int PR, int PS, int PT, int NG1, int LPC>
__device__ void tc_bsp_setup(uint8_t *sm) {
  using S = BspTc<PR, PS, PT, NG1, LPC>;
  __syncthreads();
  for (int i = threadIdx.x; i < S::NBUF * S::OBUF / 16; i += kThreads)
    reinterpret_cast<uint4 *>(sm + S::oOp)[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
}

// Element `it` of the launch (colour-sorted position e): its blocks into K32
// (null: only the dense FP64 element matrix into A.Ke_out).  The chunks' MMAs
// complete on barriers 0 and 1 (one per operand buffer).  With nparts = MT
// (two 128-row tiles) the element is shared by two CTAs: part p forms and
// scatters tile p only (the node pairs whose first node is in it), both
// compute the element's geometry.  False on a failed wait, after the MMAs in
// flight have finished (bounded).
template <int PR, int PS, int PT, int NG1, int LPC>
__device__ bool tc_bsp_element(const ElemArgs &A, float *__restrict__ K32, uint8_t *sm, Cta &c, int64_t it,
                               int64_t e, int part = 0, int nparts = 1) {
  using S = BspTc<PR, PS, PT, NG1, LPC>;
  constexpr int QR = S::QR, QS = S::QS, NN = S::NN, GCH = S::GCH, KC = S::KC, MT = S::MT, NB = S::NB;
  constexpr int ND = 3 * NN;
  double *sD = reinterpret_cast<double *>(sm + S::oD);
  double *sB = reinterpret_cast<double *>(sm + S::oB);
  double *sJ = reinterpret_cast<double *>(sm + S::oJ);
  double *sc = reinterpret_cast<double *>(sm + S::oc);
  double *sWg = reinterpret_cast<double *>(sm + S::oWg);
  double *sX = reinterpret_cast<double *>(sm + S::oX);
  double *sW = reinterpret_cast<double *>(sm + S::oW);
  uint8_t *sfix = sm + S::oFix;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NW = kThreads / 32;
  const bool rat = A.rational != 0;
  constexpr uint32_t kLBO = 128, kSBO = (KC / 4) * 128;
  constexpr uint32_t kId = tc::idesc(128, NB, tc::kTypeTF32);
  bool pending[2] = {false, false};
  __syncthreads();
  const int32_t *en = A.conn + e * NN;
  for (int i = tid; i < NN * 3; i += kThreads) sX[i] = A.X[3 * (int64_t)en[i / 3] + (i % 3)];
  for (int i = tid; i < NN; i += kThreads) {
    sfix[i] = A.fix[en[i]];
    sW[i] = (rat && A.wt) ? A.wt[en[i]] : 1.0;
  }
  // the element's slot row and its current K blocks, prefetched into L2 while
  // the geometry is computed: the epilogue's read-modify-writes then wait on
  // L2, not on DRAM
  if (K32) {
    const int32_t *es = A.slot + e * NN * NN;
#pragma unroll 4
    for (int q = tid; q < NN * NN; q += kThreads) tc::prefetch_l2(K32 + (int64_t)es[q] * 9);
  }
  const int sr = A.span[4 * e], ss = A.span[4 * e + 1], st = A.span[4 * e + 2];
  const double *br = A.bas[0] + (size_t)sr * NG1 * QR * 2;
  const double *bs = A.bas[1] + (size_t)ss * NG1 * QS * 2;
  const double *bt = A.bas[2] + (size_t)st * NG1 * S::QT * 2;
  __syncthreads();

  for (int ch = 0; ch < S::NCH; ch++) {
    // tensor-product basis of the chunk's points (cShapeBspSolid::DrvShpRST,
    // shp/shpbsp.cpp:985-1067); point g = ch*GCH + gl, r fastest, t slowest
    for (int t = tid; t < GCH * NN; t += kThreads) {
      const int gl = t / NN, a = t - NN * gl, g = ch * GCH + gl;
      const int g0 = g % NG1, g1 = (g / NG1) % NG1, g2 = g / (NG1 * NG1);
      const int ia = a % QR, ja = (a / QR) % QS, ka = a / (QR * QS);
      const double *fr = br + (g0 * QR + ia) * 2, *fs = bs + (g1 * QS + ja) * 2, *ft = bt + (g2 * S::QT + ka) * 2;
      double *D = sD + gl * ND;
      const double w = rat ? sW[a] : 1.0;
      if (rat) sB[gl * NN + a] = fr[0] * fs[0] * ft[0] * w;
      D[a] = fr[1] * fs[0] * ft[0] * w;
      D[NN + a] = fr[0] * fs[1] * ft[0] * w;
      D[2 * NN + a] = fr[0] * fs[0] * ft[1] * w;
    }
    if (rat) {
      __syncthreads();
      // W and dW/dxi per point: one warp per point, then the quotient rule
      for (int gl = warp; gl < GCH; gl += NW) {
        const double *D = sD + gl * ND;
        double w = 0.0, wr = 0.0, ws = 0.0, wt = 0.0;
        for (int a = lane; a < NN; a += 32) {
          w += sB[gl * NN + a];
          wr += D[a];
          ws += D[NN + a];
          wt += D[2 * NN + a];
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) {
          w += __shfl_xor_sync(0xffffffffu, w, m);
          wr += __shfl_xor_sync(0xffffffffu, wr, m);
          ws += __shfl_xor_sync(0xffffffffu, ws, m);
          wt += __shfl_xor_sync(0xffffffffu, wt, m);
        }
        if (lane == 0) {
          sWg[4 * gl] = w;
          sWg[4 * gl + 1] = wr;
          sWg[4 * gl + 2] = ws;
          sWg[4 * gl + 3] = wt;
        }
      }
      __syncthreads();
      for (int t = tid; t < GCH * NN; t += kThreads) {
        const int gl = t / NN, a = t - NN * gl;
        const double *Wg = sWg + 4 * gl;
        const double n = sB[gl * NN + a] / Wg[0];
        double *D = sD + gl * ND;
        D[a] = (D[a] - n * Wg[1]) / Wg[0];
        D[NN + a] = (D[NN + a] - n * Wg[2]) / Wg[0];
        D[2 * NN + a] = (D[2 * NN + a] - n * Wg[3]) / Wg[0];
      }
    }
    __syncthreads();
    // Jacobians (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126): one warp per point
    for (int gl = warp; gl < GCH; gl += NW) {
      const double *D = sD + gl * ND;
      double j[9];
#pragma unroll
      for (int k = 0; k < 9; k++) j[k] = 0.0;
      for (int a = lane; a < NN; a += 32) {
        const double x0 = sX[3 * a], x1 = sX[3 * a + 1], x2 = sX[3 * a + 2];
#pragma unroll
        for (int p = 0; p < 3; p++) {
          const double d = D[p * NN + a];
          j[3 * p] = fma(d, x0, j[3 * p]);
          j[3 * p + 1] = fma(d, x1, j[3 * p + 1]);
          j[3 * p + 2] = fma(d, x2, j[3 * p + 2]);
        }
      }
#pragma unroll
      for (int k = 0; k < 9; k++)
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) j[k] += __shfl_xor_sync(0xffffffffu, j[k], m);
      if (lane < 9) {
        double v = j[0];
#pragma unroll
        for (int k = 1; k < 9; k++)
          if (lane == k) v = j[k];
        sJ[9 * gl + lane] = v;
      }
    }
    __syncthreads();
    // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
    for (int gl = tid; gl < GCH; gl += kThreads) {
      double *J = sJ + 9 * gl;
      const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                   j21 = J[7], j22 = J[8];
      const double det =
          j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
      if (!(fabs(det) > 0.0) || !isfinite(det)) atomicOr(A.status, 1);
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
      sc[gl] = A.w[ch * GCH + gl] * det;
    }
    // the operand buffer of this chunk: wait for the MMAs that last read it
    const int buf = ch % S::NBUF;
    if (pending[buf]) {
      tcb::wait_bar_drain(c, buf);
      pending[buf] = false;
    }
    __syncthreads();
    if (*c.fail) break;
    uint8_t *op = sm + S::oOp + buf * S::OBUF;
    uint8_t *aPart[3] = {op, op + S::OA, op + 2 * S::OA};
    uint8_t *bPart[3] = {op + 3 * S::OA, op + 3 * S::OA + S::OB, op + 3 * S::OA + 2 * S::OB};
    // dN/dx, split into the TF32 operands: A row 4a+i = c_g dN_a/dx_i, B row 3b+j = dN_b/dx_j
    for (int t = tid; t < GCH * NN; t += kThreads) {
      const int gl = t / NN, a = t - NN * gl;
      const double *J = sJ + 9 * gl;
      const double *D = sD + gl * ND;
      const double d0 = D[a], d1 = D[NN + a], d2 = D[2 * NN + a], cg = sc[gl];
      const double x[3] = {J[0] * d0 + J[1] * d1 + J[2] * d2, J[3] * d0 + J[4] * d1 + J[5] * d2,
                           J[6] * d0 + J[7] * d1 + J[8] * d2};
      const bool mine = nparts == 1 || ((4 * a) >> 7) == part;   // this part's A tile
#pragma unroll
      for (int i = 0; i < 3; i++) {
        uint32_t pt[3];
        if (mine) {
          tc::split3_tf32(cg * x[i], pt[0], pt[1], pt[2]);
          const uint32_t oa = tc::kmajor_off4(4 * a + i, gl, KC);
#pragma unroll
          for (int k = 0; k < 3; k++) *reinterpret_cast<uint32_t *>(aPart[k] + oa) = pt[k];
        }
        tc::split3_tf32(x[i], pt[0], pt[1], pt[2]);
        const uint32_t ob = tc::kmajor_off4(3 * a + i, gl, KC);
#pragma unroll
        for (int k = 0; k < 3; k++) *reinterpret_cast<uint32_t *>(bPart[k] + ob) = pt[k];
      }
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      const uint32_t ua[3] = {tc::smem_u32(aPart[0]), tc::smem_u32(aPart[1]), tc::smem_u32(aPart[2])};
      const uint32_t ub[3] = {tc::smem_u32(bPart[0]), tc::smem_u32(bPart[1]), tc::smem_u32(bPart[2])};
#pragma unroll
      for (int t = 0; t < MT; t++) {
        if (nparts > 1 && t != part) continue;
        const uint32_t d = c.tmem + t * S::TSTRIDE;
        const uint32_t toff = t * 16 * kSBO;   // 128 rows = 16 row groups
#pragma unroll
        for (int tm = 0; tm < tc::kSplitTerms; tm++) {
          int pa_, pb_;
          tc::split_term(tm, pa_, pb_);
#pragma unroll
          for (int kk = 0; kk < KC / 8; kk++)
            tc::mma_tf32(d, tc::smem_desc(ua[pa_] + toff + kk * 256, kLBO, kSBO),
                         tc::smem_desc(ub[pb_] + kk * 256, kLBO, kSBO), kId,
                         (ch > 0 || tm > 0 || kk > 0) ? 1u : 0u);
        }
      }
      tc::commit(&c.bars[buf]);
    }
    pending[buf] = true;
  }
  // every chunk's MMAs complete before the accumulator is read (after a
  // failed wait: once more, bounded, before giving up)
  for (int b = 0; b < S::NBUF; b++)
    if (pending[b]) {
      tcb::wait_bar_drain(c, b);
      pending[b] = false;
    }
  __syncthreads();
  if (*c.fail) return false;
  tc::fence_after();

  // epilogue: warp w reads tile w / 4, lanes 32 (w % 4) ..; row 4a + i
  // (split: both warp quartets read the part's tile, even / odd column groups)
  const int tile = nparts > 1 ? part : (warp >> 2), sub = warp & 3;
  const int grp0 = nparts > 1 ? (warp >> 2) : 0, gstep = nparts > 1 ? 2 : 1;
  if (tile < MT) {
    const int row = tile * 128 + sub * 32 + lane;
    const int a = row >> 2, i = row & 3;
    const int qbase = lane & ~3;
    const bool own = a < NN && i < 3;
    const uint32_t taddr = c.tmem + tile * S::TSTRIDE + ((uint32_t)(sub * 32) << 16);
    const double E = A.E[e], nu = A.nu[e];
    const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
    const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
    const uint8_t fa = own ? sfix[a] : 0;
#pragma unroll 1
    for (int grp = grp0; grp < S::NGRP; grp += gstep) {
      float h[24];
      tc::ld_32x32b_x8(taddr + grp * 24, h);
      tc::ld_32x32b_x8(taddr + grp * 24 + 8, h + 8);
      tc::ld_32x32b_x8(taddr + grp * 24 + 16, h + 16);
      // the current values of the group's blocks (row i of (a, b), column i
      // of (b, a)), every load issued before any store, so their latencies
      // overlap; a block this element writes first is not read
      // (four blocks at a time: the registers of eight cost the SM a CTA)
#pragma unroll
      for (int half = 0; half < 2; half++) {
      float oab[4][3], oba[4][3];
      float *pab[4], *pba[4];
      bool f1[4], f2[4];
#pragma unroll
      for (int bl = 0; bl < 4; bl++) {
        const int b = grp * 8 + half * 4 + bl;
        pab[bl] = pba[bl] = nullptr;
        f1[bl] = f2[bl] = false;
        if (!K32 || !own || b >= NN || b < a) continue;
        pab[bl] = K32 + (int64_t)A.slot[(e * NN + a) * NN + b] * 9 + 3 * i;
        f1[bl] = first_touch(A, e, a * NN + b);
        if (!f1[bl]) {
#pragma unroll
          for (int j = 0; j < 3; j++) oab[bl][j] = pab[bl][j];
        }
        if (b != a) {
          pba[bl] = K32 + (int64_t)A.slot[(e * NN + b) * NN + a] * 9 + i;
          f2[bl] = first_touch(A, e, b * NN + a);
          if (!f2[bl]) {
#pragma unroll
            for (int j = 0; j < 3; j++) oba[bl][j] = pba[bl][3 * j];
          }
        }
      }
#pragma unroll
      for (int bl = 0; bl < 4; bl++) {
        const int b = grp * 8 + half * 4 + bl;
        // the 3x3 block M[s][j] = H[(a,s),(b,j)] from the quad of node a
        double M[9];
#pragma unroll
        for (int s2 = 0; s2 < 3; s2++)
#pragma unroll
          for (int j = 0; j < 3; j++) M[3 * s2 + j] = (double)__shfl_sync(0xffffffffu, h[3 * (half * 4 + bl) + j], qbase + s2);
        if (!own || b >= NN || b < a) continue;
        const double tr = M[0] + M[4] + M[8];
        double v[3];
#pragma unroll
        for (int j = 0; j < 3; j++)
          v[j] = (i == j) ? C00 * M[4 * i] + G * (tr - M[4 * i]) : C01 * M[3 * i + j] + G * M[3 * j + i];
        if (A.Ke_out) {
          double *Ko = A.Ke_out + it * ND * ND;
#pragma unroll
          for (int j = 0; j < 3; j++) {
            Ko[(3 * a + i) * ND + 3 * b + j] = v[j];
            Ko[(3 * b + j) * ND + 3 * a + i] = v[j];
          }
        }
        if (pab[bl]) {
          // add where both DOFs have equations; a first write (first-touch
          // flags) stores the entry instead, 1 / 0 where a DOF is fixed
          const uint8_t fb = sfix[b];
          const bool fai = (fa >> i) & 1;
#pragma unroll
          for (int j = 0; j < 3; j++) {
            const bool fixed = fai || ((fb >> j) & 1);
            if (f1[bl]) pab[bl][j] = fixed ? ((a == b && i == j) ? 1.f : 0.f) : (float)v[j];
            else if (!fixed) pab[bl][j] = oab[bl][j] + (float)v[j];
          }
          if (pba[bl]) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
              const bool fixed = fai || ((fb >> j) & 1);
              if (f2[bl]) pba[bl][3 * j] = fixed ? 0.f : (float)v[j];
              else if (!fixed) pba[bl][3 * j] = oba[bl][j] + (float)v[j];
            }
          }
        }
      }
      }
    }
  }
  tc::fence_before();
  return true;
}

}  // namespace tcb
}  // namespace fastgpu

// elem_common.cuh - shared by the element kernels (private to libfastgpu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace fastgpu {

struct ElemArgs {
  int64_t ne;                 // elements in this launch
  const int32_t *index;       // optional: colour-sorted positions to process (else 0..ne-1 + offset)
  int64_t offset;             // first colour-sorted element of this launch
  const int32_t *conn;        // [*][NN]
  const double *E, *nu, *rho;
  const int32_t *slot;        // [*][NN][NN]
  const double *X;            // [nnode][3]
  const uint8_t *fix;         // [nnode]
  const double *dN;           // [NG][NN][3]
  const double *N;            // [NG][NN]
  const double *w;            // [NG]
  double *K;                  // block values [nnzb][3][3] or null
  double *Ke_out;             // [ne][3NN][3NN] or null (unmasked element matrices)
  int32_t *status;            // bit 0: non-positive Jacobian determinant
  const double *U;            // [nnode][4] nodal displacements (total-Lagrangian / internal force)
  double *G;                  // [nnode][4] internal force, added to (colour-safe) or null
  const int32_t *skip;        // optional device flag: the launch does nothing when it is non-zero
  // B-spline solids
  const int32_t *span;        // [*][4] colour-sorted knot spans (r, s, t, unused)
  const double *bas[3];       // per direction [nspan][ngp][p+1][2] {N, dN/dt}
  const double *wt;           // [nnode] control-point weights (rational patches)
  int rational;
  // launch shape (0: default)
  int ctas_per_sm;            // resident CTAs per SM at most
  int split;                  // B-spline kernels: CTAs sharing one element at most
  // first-touch flags (stiffness assembly without a zero fill) or null:
  // [*][fw] words, bit a*NN+b set when this element writes block (a, b) first
  const uint32_t *first;
  int fw;
};

// Whether colour-sorted element e writes the block of its node pair q =
// a*NN+b first (then it stores the block outright instead of adding to it)
__device__ __forceinline__ bool first_touch(const ElemArgs &A, int64_t e, int q) {
  return A.first && ((__ldg(A.first + e * A.fw + (q >> 5)) >> (q & 31)) & 1u);
}

// The value a block entry (i, j) of node pair (a, b) takes: old + add where
// both DOFs have equations; where one is fixed the entry is left alone,
// unless this is the block's first write, which stores 1 on the diagonal of a
// fixed DOF and 0 elsewhere.  Returns false when the entry is left alone.
template <typename T>
__device__ __forceinline__ bool entry_value(bool first, bool fixed, bool diag, T old, double add, T &out) {
  if (fixed) {
    if (!first) return false;
    out = diag ? T(1) : T(0);
    return true;
  }
  out = first ? T(add) : T(old + T(add));
  return true;
}

struct Ctx;
struct Bucket;
// B-spline solid buckets (bsp_kernels.cu): stiffness (or, with mass, the
// consistent mass; degrees up to 3) scatter or element matrices
cudaError_t launch_bsp_elements(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, bool mass = false);
// B-spline solid buckets (bsp_tl.cu): total-Lagrangian tangent and / or
// internal force (mode 0 both, 1 tangent, 2 force), small-strain internal force
cudaError_t launch_bsp_tl(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, int mode);

// The entries (element j, block q = a NN + b of its NN x NN node-pair grid,
// entry k of the 3x3 block) of a CTA's elements, walked with k fixed per
// thread: thread t < 9 QS takes entry k = t % 9 of the blocks t / 9,
// t / 9 + QS, ... (q counted over all elements, element-major).  Consecutive
// threads take consecutive entries, as a plain t, t + NT, ... walk over 9 q +
// k would, but the block, element and node indices advance by additions
// instead of divisions per entry.
template <int NN, int NT>
struct BlockWalk {
  static constexpr int QS = NT / 9;  // blocks per trip
  static_assert(QS / NN + 1 <= NN, "one carry per step");
  int k, q, j, a, b;
  __device__ __forceinline__ explicit BlockWalk(int t) {
    k = t % 9;
    q = t / 9;
    j = q / (NN * NN);
    const int qq = q - j * NN * NN;
    a = qq / NN;
    b = qq - NN * a;
  }
  __device__ __forceinline__ static bool takes(int t) { return t < 9 * QS; }
  __device__ __forceinline__ int qq() const { return a * NN + b; }
  __device__ __forceinline__ void next() {
    q += QS;
    b += QS % NN;
    a += QS / NN;
    if (b >= NN) { b -= NN; a++; }
    if (a >= NN) { a -= NN; j++; }
  }
};

// 9 x the index of the upper-triangle pair (min(a,b), max(a,b)) plus the
// entry k (a <= b) or its transpose kt (a > b): where a node-pair block of
// the element sits among the blocks stored for a <= b
template <int NN>
__device__ __forceinline__ int upper_entry(int a, int b, int k, int kt) {
  return a <= b ? 9 * (a * NN - a * (a - 1) / 2 + (b - a)) + k : 9 * (b * NN - b * (b - 1) / 2 + (a - b)) + kt;
}

// (a, b) pair index -> a <= b, row-major over the upper triangle
__device__ __forceinline__ void pair_of(int p, int n, int &a, int &b) {
  int r = 0;
  while (p >= n - r) { p -= n - r; r++; }
  a = r;
  b = r + p;
}

}  // namespace fastgpu

// ties.cu - tied interfaces by elimination of the slave DOFs (sm_100a).
//
// A tie makes slave node s follow its master nodes:  u_s = sum_k w_k u_(m_k)
// (three equations per slave, one per direction; in the reference these are
// %NODE.MULTI-POINT.CONSTRAINT rows, node/node.cpp:459-509, which
// cSysMatrix::SolveMPC, mlib/sysmat.cpp:72-143, enforces with dense Lagrange
// multipliers: one full solve per constraint).  With u = T u~ the constrained
// problem is K~ u~ = T^T f, K~ = T^T K T, and the slave DOFs leave the system.
// K~ is assembled directly:
//   * an element without slave nodes scatters as usual;
//   * an element with slave nodes ("tied element") first writes its dense
//     K_e to a scratch buffer (the element kernels' inspection path), then
//     tied_scatter adds T_e^T K_e T_e onto its expanded node list (non-slave
//     nodes plus the slaves' masters).  Block (A, B) of the expanded matrix is
//         sum_{(a,ta) -> A} sum_{(b,tb) -> B} ta tb K_e(a, b)
//     over the pre-images of A and B.  Tied elements are coloured on their
//     expanded lists, one launch per colour: no atomics, fixed order, K~ is
//     bit-identical from run to run.
// Slave rows keep an identity diagonal block (their DOFs are flagged like
// fixed ones), the load restriction and the displacement prolongation are
// gathers over precomputed maps.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

namespace {

constexpr int kTiedThreads = 1024;

// STAGE: the element matrix is first copied to shared memory (when it fits)
template <bool STAGE, typename KT>
__global__ void __launch_bounds__(kTiedThreads) tied_scatter(int64_t first, int64_t count, const int64_t *__restrict__ nptr,
                             const int32_t *__restrict__ nodes, const int64_t *__restrict__ sptr,
                             const int32_t *__restrict__ slot, const int64_t *__restrict__ pptr,
                             const int32_t *__restrict__ pa, const double *__restrict__ pt,
                             const int64_t *__restrict__ keoff, const int32_t *__restrict__ nn_of,
                             const double *__restrict__ ke, const uint8_t *__restrict__ fix, KT *__restrict__ K) {
  extern __shared__ double sKe[];
  for (int64_t it = blockIdx.x; it < count; it += gridDim.x) {
    const int64_t x = first + it;
    const int64_t n0 = nptr[x];
    const int m = (int)(nptr[x + 1] - n0);
    const int nd = 3 * nn_of[x];
    const double *Ke = ke + keoff[x];
    if (STAGE) {
      for (int i = threadIdx.x; i < nd * nd; i += blockDim.x) sKe[i] = Ke[i];
      __syncthreads();
      Ke = sKe;
    }
    const int32_t *sl = slot + sptr[x];
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int A = q / m, B = q - A * m;
      double v[9];
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = 0.0;
      for (int64_t ia = pptr[n0 + A]; ia < pptr[n0 + A + 1]; ia++) {
        const int a = pa[ia];
        const double ta = pt[ia];
        for (int64_t ib = pptr[n0 + B]; ib < pptr[n0 + B + 1]; ib++) {
          const int b = pa[ib];
          const double t = ta * pt[ib];
          const double *r = Ke + (int64_t)(3 * a) * nd + 3 * b;
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) v[3 * i + j] = fma(t, r[(int64_t)i * nd + j], v[3 * i + j]);
        }
      }
      const uint8_t fa = fix[nodes[n0 + A]], fb = fix[nodes[n0 + B]];
      KT *Kb = K + (int64_t)sl[q] * 9;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          if (!((fa >> i) & 1) && !((fb >> j) & 1)) Kb[3 * i + j] += (KT)v[3 * i + j];
    }
    __syncthreads();
  }
}

// f[m] += sum w f[s] over the slaves of each master (DOFs without an equation
// take nothing), then f[s] = 0
__global__ void tie_restrict(int64_t nmaster, const int32_t *__restrict__ master, const int64_t *__restrict__ mptr,
                             const int32_t *__restrict__ mslave, const double *__restrict__ mw,
                             const uint8_t *__restrict__ fix, double *__restrict__ f) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nmaster) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t k = mptr[j]; k < mptr[j + 1]; k++) {
    const double *fs = f + 4 * (int64_t)mslave[k];
    a0 = fma(mw[k], fs[0], a0);
    a1 = fma(mw[k], fs[1], a1);
    a2 = fma(mw[k], fs[2], a2);
  }
  double *fm = f + 4 * (int64_t)master[j];
  const uint8_t fx = fix[master[j]];
  if (!(fx & 1)) fm[0] += a0;
  if (!(fx & 2)) fm[1] += a1;
  if (!(fx & 4)) fm[2] += a2;
}

__global__ void tie_zero(int64_t nslave, const int32_t *__restrict__ slave, double *__restrict__ v) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= nslave) return;
  double *p = v + 4 * (int64_t)slave[s];
  p[0] = 0.0;
  p[1] = 0.0;
  p[2] = 0.0;
}

// u[s] = sum w u[m]
__global__ void tie_prolong(int64_t nslave, const int32_t *__restrict__ slave, const int64_t *__restrict__ sptr,
                            const int32_t *__restrict__ smaster, const double *__restrict__ sw, double *__restrict__ u) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= nslave) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t k = sptr[s]; k < sptr[s + 1]; k++) {
    const double *um = u + 4 * (int64_t)smaster[k];
    a0 = fma(sw[k], um[0], a0);
    a1 = fma(sw[k], um[1], a1);
    a2 = fma(sw[k], um[2], a2);
  }
  double *us = u + 4 * (int64_t)slave[s];
  us[0] = a0;
  us[1] = a1;
  us[2] = a2;
}

template <class T>
cudaError_t upload(T **d, const std::vector<T> &h) {
  *d = nullptr;
  cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(1, h.size()));
  if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return e;
}

template <class T>
void release(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

}  // namespace

cudaError_t upload_ties(Ctx &c) {
  TiedSet &T = c.tied;
  cudaError_t e = cudaSuccess;
  if (T.n > 0) {
    std::vector<int32_t> nn(T.h_nn.begin(), T.h_nn.end());
    if (e == cudaSuccess) e = upload(&T.d_nptr, T.h_nptr);
    if (e == cudaSuccess) e = upload(&T.d_nodes, T.h_nodes);
    if (e == cudaSuccess) e = upload(&T.d_sptr, T.h_sptr);
    if (e == cudaSuccess) e = upload(&T.d_slot, T.h_slot);
    if (e == cudaSuccess) e = upload(&T.d_pptr, T.h_pptr);
    if (e == cudaSuccess) e = upload(&T.d_pa, T.h_pa);
    if (e == cudaSuccess) e = upload(&T.d_pt, T.h_pt);
    if (e == cudaSuccess) e = upload(&T.d_keoff, T.h_keoff);
    if (e == cudaSuccess) e = upload(&T.d_nn, nn);
    if (e == cudaSuccess) e = upload(&T.d_eptr, T.h_eptr);
    if (e == cudaSuccess) e = upload(&T.d_econn, T.h_econn);
    if (e == cudaSuccess) e = cudaMalloc((void **)&T.d_ke, sizeof(double) * std::max<int64_t>(1, T.ke_total));
    T.d_bucket_pos.assign(T.bucket_pos.size(), nullptr);
    for (size_t b = 0; b < T.bucket_pos.size() && e == cudaSuccess; b++)
      if (!T.bucket_pos[b].empty()) e = upload(&T.d_bucket_pos[b], T.bucket_pos[b]);
  }
  if (c.has_ties() && e == cudaSuccess) {
    TieMaps &M = c.tmaps;
    const int64_t ns = (int64_t)c.h_tslave.size();
    M.nslave = ns;
    std::vector<int32_t> sl(ns), sm(c.h_tmaster.size());
    for (int64_t s = 0; s < ns; s++) sl[s] = (int32_t)c.h_tslave[s];
    for (size_t k = 0; k < sm.size(); k++) sm[k] = (int32_t)c.h_tmaster[k];
    // transpose: distinct masters, each with its (slave, weight) list in slave order
    std::vector<int64_t> cnt(c.nnode + 1, 0);
    for (int32_t m : sm) cnt[m + 1]++;
    std::vector<int32_t> mlist;
    std::vector<int64_t> mptr(1, 0), pos(c.nnode, -1);
    for (int64_t n = 0; n < c.nnode; n++)
      if (cnt[n + 1]) { pos[n] = (int64_t)mlist.size(); mlist.push_back((int32_t)n); mptr.push_back(cnt[n + 1]); }
    for (size_t j = 0; j + 1 < mptr.size(); j++) mptr[j + 1] += mptr[j];
    std::vector<int32_t> mslave(sm.size());
    std::vector<double> mw(sm.size());
    std::vector<int64_t> fill(mptr.begin(), mptr.end() - 1);
    for (int64_t s = 0; s < ns; s++)
      for (int64_t k = c.h_tptr[s]; k < c.h_tptr[s + 1]; k++) {
        const int64_t j = pos[sm[k]];
        mslave[fill[j]] = sl[s];
        mw[fill[j]++] = c.h_tweight[k];
      }
    M.nmaster = (int64_t)mlist.size();
    if (e == cudaSuccess) e = upload(&M.d_slave, sl);
    if (e == cudaSuccess) e = upload(&M.d_sptr, c.h_tptr);
    if (e == cudaSuccess) e = upload(&M.d_smaster, sm);
    if (e == cudaSuccess) e = upload(&M.d_sw, c.h_tweight);
    if (e == cudaSuccess) e = upload(&M.d_master, mlist);
    if (e == cudaSuccess) e = upload(&M.d_mptr, mptr);
    if (e == cudaSuccess) e = upload(&M.d_mslave, mslave);
    if (e == cudaSuccess) e = upload(&M.d_mw, mw);
  }
  return e;
}

void free_ties(Ctx &c) {
  TiedSet &T = c.tied;
  release(T.d_nptr); release(T.d_nodes); release(T.d_sptr); release(T.d_slot); release(T.d_pptr);
  release(T.d_pa); release(T.d_pt); release(T.d_keoff); release(T.d_nn); release(T.d_ke);
  release(T.d_eptr); release(T.d_econn);
  for (int32_t *&p : T.d_bucket_pos) release(p);
  T = TiedSet();
  TieMaps &M = c.tmaps;
  release(M.d_slave); release(M.d_sptr); release(M.d_smaster); release(M.d_sw);
  release(M.d_master); release(M.d_mptr); release(M.d_mslave); release(M.d_mw);
  M = TieMaps();
  c.h_tslave.clear(); c.h_tptr.clear(); c.h_tmaster.clear(); c.h_tweight.clear(); c.h_slave_of.clear();
}

// the tied scatter of every tied colour into K (element matrices already in
// the scratch buffer)
template <typename KT>
static cudaError_t tied_scatter_all(Ctx &c, KT *K) {
  TiedSet &T = c.tied;
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k + 1 < T.color_off.size(); k++) {
    const int64_t first = T.color_off[k], cnt = T.color_off[k + 1] - first;
    if (cnt <= 0) continue;
    // one element per CTA; 1024 threads share its expanded pairs, whose K
    // read-modify-writes are latency-bound
    const unsigned grid = (unsigned)std::min<int64_t>(cnt, 2LL * c.sm_count);
    int maxnn = 0;
    for (int32_t v : T.h_nn) maxnn = std::max(maxnn, v);
    const size_t smem = sizeof(double) * 9 * maxnn * maxnn;
    if (smem <= 96 * 1024) {
      e = cudaFuncSetAttribute(tied_scatter<true, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      tied_scatter<true, KT><<<grid, kTiedThreads, smem, c.stream>>>(first, cnt, T.d_nptr, T.d_nodes, T.d_sptr,
                                                                      T.d_slot, T.d_pptr, T.d_pa, T.d_pt, T.d_keoff,
                                                                      T.d_nn, T.d_ke, c.d_fix, K);
    } else {
      tied_scatter<false, KT><<<grid, kTiedThreads, 0, c.stream>>>(first, cnt, T.d_nptr, T.d_nodes, T.d_sptr, T.d_slot,
                                                                    T.d_pptr, T.d_pa, T.d_pt, T.d_keoff, T.d_nn,
                                                                    T.d_ke, c.d_fix, K);
    }
    c.launches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_tied_assemble(Ctx &c, double *K) {
  TiedSet &T = c.tied;
  if (T.n == 0) return cudaSuccess;
  cudaError_t e = launch_tied_element_matrices(c);
  if (e != cudaSuccess) return e;
  return tied_scatter_all<double>(c, K);
}

cudaError_t launch_tied_assemble32(Ctx &c, float *K32) {
  TiedSet &T = c.tied;
  if (T.n == 0) return cudaSuccess;
  cudaError_t e = launch_tied_element_matrices(c);
  if (e != cudaSuccess) return e;
  return tied_scatter_all<float>(c, K32);
}

// G += K_e u_e per tied element, one CTA per element of one colour: the
// element's displacements gathered to shared memory, one thread per row of
// K_e, the node sums written by the rows of that node (colour-safe)
__global__ void __launch_bounds__(256) tied_matvec(int64_t first, int64_t count, const int64_t *__restrict__ eptr,
                                                   const int32_t *__restrict__ econn,
                                                   const int64_t *__restrict__ keoff, const int32_t *__restrict__ nn_of,
                                                   const double *__restrict__ ke, const double *__restrict__ u,
                                                   double *__restrict__ G, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double su[3 * 64];
  for (int64_t it = blockIdx.x; it < count; it += gridDim.x) {
    const int64_t x = first + it;
    const int nn = nn_of[x], nd = 3 * nn;
    const int32_t *en = econn + eptr[x];
    const double *Ke = ke + keoff[x];
    __syncthreads();
    for (int i = threadIdx.x; i < nd; i += blockDim.x) su[i] = u[4 * (int64_t)en[i / 3] + (i % 3)];
    __syncthreads();
    // every row, slave DOFs included (they carry the element's force to the
    // masters in the restriction that follows; the caller zeroes fixed DOFs)
    for (int r = threadIdx.x; r < nd; r += blockDim.x) {
      const int a = r / 3, i = r - 3 * a;
      const double *row = Ke + (int64_t)r * nd;
      double g = 0.0;
      for (int k = 0; k < nd; k++) g = fma(row[k], su[k], g);
      G[4 * (int64_t)en[a] + i] += g;
    }
  }
}

cudaError_t launch_tied_matvec(Ctx &c, const double *u, double *G, const int32_t *skip) {
  TiedSet &T = c.tied;
  for (size_t k = 0; k + 1 < T.color_off.size(); k++) {
    const int64_t first = T.color_off[k], cnt = T.color_off[k + 1] - first;
    if (cnt <= 0) continue;
    const unsigned grid = (unsigned)std::min<int64_t>(cnt, 4LL * c.sm_count);
    tied_matvec<<<grid, 256, 0, c.stream>>>(first, cnt, T.d_eptr, T.d_econn, T.d_keoff, T.d_nn, T.d_ke, u, G, skip);
    c.launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// v[DOF] = 0 for every DOF without an equation (supports and tied slaves)
__global__ void zero_fixed_dofs(int64_t nnode, const uint8_t *__restrict__ fix, double *__restrict__ v,
                                const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const uint8_t f = fix[n];
  if (!f) return;
  for (int i = 0; i < 3; i++)
    if ((f >> i) & 1) v[4 * n + i] = 0.0;
}

cudaError_t launch_zero_fixed(Ctx &c, double *v, const int32_t *skip) {
  zero_fixed_dofs<<<(unsigned)((c.nnode + 255) / 256), 256, 0, c.stream>>>(c.nnode, c.d_fix, v, skip);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_tie_restrict(Ctx &c, double *f) {
  const TieMaps &M = c.tmaps;
  if (M.nslave == 0) return cudaSuccess;
  tie_restrict<<<(unsigned)((M.nmaster + 255) / 256), 256, 0, c.stream>>>(M.nmaster, M.d_master, M.d_mptr,
                                                                           M.d_mslave, M.d_mw, c.d_fix, f);
  tie_zero<<<(unsigned)((M.nslave + 255) / 256), 256, 0, c.stream>>>(M.nslave, M.d_slave, f);
  c.launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_tie_zero(Ctx &c, double *v) {
  const TieMaps &M = c.tmaps;
  if (M.nslave == 0) return cudaSuccess;
  tie_zero<<<(unsigned)((M.nslave + 255) / 256), 256, 0, c.stream>>>(M.nslave, M.d_slave, v);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_tie_prolong(Ctx &c, double *u) {
  const TieMaps &M = c.tmaps;
  if (M.nslave == 0) return cudaSuccess;
  tie_prolong<<<(unsigned)((M.nslave + 255) / 256), 256, 0, c.stream>>>(M.nslave, M.d_slave, M.d_sptr, M.d_smaster,
                                                                         M.d_sw, u);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace fastgpu

// pattern.cpp - host-side structural set-up of the device matrix.
//
// FAST builds its global-matrix structure on the fly: the skyline profile in
// cControl::CompProf (ctrl/ctrl.cpp:2112-2157) or a sorted linked list per
// row grown by every cSysMatrix::Add (mlib/sysmat.cpp:722-765).  Here the
// structure is fixed once per mesh topology:
//
//   1. node adjacency -> node-block CSR (one 3x3 block per pair of nodes that
//      share an element; full, both triangles, columns sorted);
//   2. element slot map: for element e and local nodes (a, b), the index of
//      block (node_a, node_b) in that CSR;
//   3. greedy element colouring on the "shares a node" conflict graph.  Two
//      elements of one colour write disjoint blocks, so one colour is one
//      race-free launch and the summation order per entry is the fixed colour
//      order: the assembled matrix is bit-identical from run to run.
//
// Elements are then stored colour-sorted, so each colour is a contiguous
// range in device memory.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace fastgpu {

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

bool build_pattern(Ctx &c, const fast_gpu_mesh &m) {
  const double t0 = now_s();
  const int64_t nnode = m.num_nodes;

  // node -> elements (over all buckets), as CSR
  std::vector<int64_t> ecount(nnode + 1, 0);
  for (int b = 0; b < m.num_buckets; b++) {
    const fast_gpu_bucket &bk = m.buckets[b];
    const int nn = bucket_nodes(bk);
    for (int64_t e = 0; e < bk.num_elems; e++)
      for (int a = 0; a < nn; a++) {
        int32_t n = bk.conn[e * nn + a];
        if (n < 0 || n >= nnode) return c.set_error("element incidence out of range");
        ecount[n + 1]++;
      }
  }
  for (int64_t i = 0; i < nnode; i++) ecount[i + 1] += ecount[i];
  std::vector<int64_t> eptr(ecount);
  std::vector<int64_t> elist(ecount[nnode]);  // packed (bucket << 40) | element
  {
    std::vector<int64_t> fill(ecount.begin(), ecount.end() - 1);
    for (int b = 0; b < m.num_buckets; b++) {
      const fast_gpu_bucket &bk = m.buckets[b];
      const int nn = bucket_nodes(bk);
      for (int64_t e = 0; e < bk.num_elems; e++)
        for (int a = 0; a < nn; a++) elist[fill[bk.conn[e * nn + a]]++] = ((int64_t)b << 40) | e;
    }
  }

  // 1. node-block CSR: rows in parallel, a marker per thread
  c.h_rowptr.assign(nnode + 1, 0);
  {
    std::vector<int32_t> deg(nnode, 0);
#pragma omp parallel
    {
      std::vector<int64_t> mark(nnode, -1);
#pragma omp for schedule(dynamic, 1024)
      for (int64_t i = 0; i < nnode; i++) {
        int cnt = 0;
        for (int64_t k = eptr[i]; k < eptr[i + 1]; k++) {
          const int b = (int)(elist[k] >> 40);
          const int64_t e = elist[k] & ((1LL << 40) - 1);
          const fast_gpu_bucket &bk = m.buckets[b];
          const int nn = bucket_nodes(bk);
          for (int a = 0; a < nn; a++) {
            int32_t n = bk.conn[e * nn + a];
            if (mark[n] != i) { mark[n] = i; cnt++; }
          }
        }
        deg[i] = cnt;
      }
    }
    int64_t acc = 0;
    for (int64_t i = 0; i < nnode; i++) {
      acc += deg[i];
      if (acc > INT32_MAX) return c.set_error("pattern too large for 32-bit block indices");
      c.h_rowptr[i + 1] = (int32_t)acc;
    }
    c.nnzb = acc;
    c.h_col.assign(c.nnzb, 0);
#pragma omp parallel
    {
      std::vector<int64_t> mark(nnode, -1);
#pragma omp for schedule(dynamic, 1024)
      for (int64_t i = 0; i < nnode; i++) {
        int32_t *out = c.h_col.data() + c.h_rowptr[i];
        int cnt = 0;
        for (int64_t k = eptr[i]; k < eptr[i + 1]; k++) {
          const int b = (int)(elist[k] >> 40);
          const int64_t e = elist[k] & ((1LL << 40) - 1);
          const fast_gpu_bucket &bk = m.buckets[b];
          const int nn = bucket_nodes(bk);
          for (int a = 0; a < nn; a++) {
            int32_t n = bk.conn[e * nn + a];
            if (mark[n] != i) { mark[n] = i; out[cnt++] = n; }
          }
        }
        std::sort(out, out + cnt);
      }
    }
  }
  c.h_diag.assign(nnode, -1);
  for (int64_t i = 0; i < nnode; i++) {
    const int32_t *b0 = c.h_col.data() + c.h_rowptr[i], *b1 = c.h_col.data() + c.h_rowptr[i + 1];
    const int32_t *p = std::lower_bound(b0, b1, (int32_t)i);
    if (p != b1 && *p == i) c.h_diag[i] = (int32_t)(p - c.h_col.data());
  }

  // padded solve layout: rows rounded up to 4 blocks; padding columns point at
  // the row itself and carry zero values
  c.h_srow.assign(nnode + 1, 0);
  {
    int64_t acc = 0;
    for (int64_t i = 0; i < nnode; i++) {
      const int64_t nb = c.h_rowptr[i + 1] - c.h_rowptr[i];
      acc += (nb + 3) & ~int64_t(3);
      if (9 * acc > INT32_MAX) return c.set_error("padded pattern too large for 32-bit value indices");
      c.h_srow[i + 1] = (int32_t)acc;
    }
    c.nnzb_pad = acc;
    c.h_scol.assign(acc, 0);
    for (int64_t i = 0; i < nnode; i++) {
      const int32_t nb = c.h_rowptr[i + 1] - c.h_rowptr[i];
      const int32_t nbp = c.h_srow[i + 1] - c.h_srow[i];
      for (int32_t p = 0; p < nbp; p++) c.h_scol[c.h_srow[i] + p] = p < nb ? c.h_col[c.h_rowptr[i] + p] : (int32_t)i;
    }
  }

  // equation-space lower-triangle count (what the reference stores)
  {
    int64_t cnt = 0;
    for (int64_t i = 0; i < nnode; i++)
      for (int64_t k = c.h_rowptr[i]; k < c.h_rowptr[i + 1]; k++) {
        const int64_t j = c.h_col[k];
        for (int p = 0; p < 3; p++) {
          const int32_t ei = c.h_eq[i * 3 + p];
          if (!ei) continue;
          for (int q = 0; q < 3; q++) {
            const int32_t ej = c.h_eq[j * 3 + q];
            if (ej && ej <= ei) cnt++;
          }
        }
      }
    c.nnz_lower_eq = cnt;
  }

  // 2./3. per bucket: greedy colouring (element order), colour sort, slot map
  // Buckets are assembled one after another, so colours are per bucket.
  c.ncolors = 0;
  for (int b = 0; b < m.num_buckets; b++) {
    const fast_gpu_bucket &bk = m.buckets[b];
    Bucket &B = c.buckets[b];
    // bit k of a node's mask: a colour-k element uses the node.  B-spline
    // solids of degree p need at least (p+1)^3 colours (64 for p = 3).
    constexpr int kWords = 4;  // up to 256 colours
    std::vector<uint64_t> node_colors((size_t)nnode * kWords, 0);
    const int nn = B.nn;
    std::vector<int32_t> color(bk.num_elems);
    int ncol = 0;
    for (int64_t e = 0; e < bk.num_elems; e++) {
      uint64_t used[kWords] = {0, 0, 0, 0};
      for (int a = 0; a < nn; a++)
        for (int w = 0; w < kWords; w++) used[w] |= node_colors[(size_t)bk.conn[e * nn + a] * kWords + w];
      int col = -1;
      for (int w = 0; w < kWords && col < 0; w++)
        if (~used[w] != 0) col = 64 * w + __builtin_ctzll(~used[w]);
      if (col < 0) return c.set_error("element colouring needs more than 256 colours");
      color[e] = col;
      ncol = std::max(ncol, col + 1);
      for (int a = 0; a < nn; a++) node_colors[(size_t)bk.conn[e * nn + a] * kWords + col / 64] |= (1ULL << (col % 64));
    }
    c.ncolors = std::max(c.ncolors, ncol);
    // stable counting sort by colour
    B.color_off.assign(ncol + 1, 0);
    for (int64_t e = 0; e < bk.num_elems; e++) B.color_off[color[e] + 1]++;
    for (int k = 0; k < ncol; k++) B.color_off[k + 1] += B.color_off[k];
    B.perm.assign(bk.num_elems, 0);
    B.inv.assign(bk.num_elems, 0);
    {
      std::vector<int64_t> fill(B.color_off.begin(), B.color_off.end() - 1);
      for (int64_t e = 0; e < bk.num_elems; e++) {
        int64_t pos = fill[color[e]]++;
        B.perm[pos] = (int32_t)e;
        B.inv[e] = (int32_t)pos;
      }
    }
    B.h_conn.assign(bk.num_elems * nn, 0);
    for (int64_t s = 0; s < bk.num_elems; s++)
      std::memcpy(&B.h_conn[s * nn], &bk.conn[(int64_t)B.perm[s] * nn], sizeof(int32_t) * nn);
    // slot map, colour-sorted element order
    B.h_slot.assign(bk.num_elems * nn * nn, -1);
    bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
    for (int64_t s = 0; s < bk.num_elems; s++) {
      const int32_t *en = &B.h_conn[s * nn];
      for (int a = 0; a < nn; a++) {
        const int32_t *r0 = c.h_col.data() + c.h_rowptr[en[a]];
        const int32_t *r1 = c.h_col.data() + c.h_rowptr[en[a] + 1];
        for (int q = 0; q < nn; q++) {
          const int32_t *p = std::lower_bound(r0, r1, en[q]);
          if (p == r1 || *p != en[q]) { bad = true; continue; }
          B.h_slot[(s * nn + a) * nn + q] = (int32_t)(p - c.h_col.data());
        }
      }
    }
    if (bad) return c.set_error("internal: element node pair missing from the pattern");
  }
  c.pattern_seconds = now_s() - t0;
  return true;
}

}  // namespace fastgpu

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
#include <cmath>
#include <chrono>
#include <cstring>
#include <numeric>
#include <string>

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

  // ties: slave -> (masters, weights)
  c.h_slave_of.assign(nnode, -1);
  c.h_tslave.clear(); c.h_tptr.clear(); c.h_tmaster.clear(); c.h_tweight.clear();
  if (m.ties && m.ties->num_slaves > 0) {
    const fast_gpu_ties &T = *m.ties;
    if (!T.slave || !T.ptr || !T.master || !T.weight) return c.set_error("ties: missing arrays");
    c.h_tslave.assign(T.slave, T.slave + T.num_slaves);
    c.h_tptr.assign(T.ptr, T.ptr + T.num_slaves + 1);
    if (c.h_tptr[0] != 0) return c.set_error("ties: ptr must start at 0");
    for (int64_t s = 0; s < T.num_slaves; s++)
      if (c.h_tptr[s + 1] <= c.h_tptr[s]) return c.set_error("ties: every slave needs at least one master");
    c.h_tmaster.assign(T.master, T.master + c.h_tptr.back());
    c.h_tweight.assign(T.weight, T.weight + c.h_tptr.back());
    for (int64_t s = 0; s < T.num_slaves; s++) {
      const int64_t n = c.h_tslave[s];
      if (n < 0 || n >= nnode) return c.set_error("ties: slave node out of range");
      if (c.h_slave_of[n] >= 0) return c.set_error("ties: node " + std::to_string(n) + " is tied twice");
      c.h_slave_of[n] = (int32_t)s;
    }
    for (int64_t k = 0; k < (int64_t)c.h_tmaster.size(); k++) {
      const int64_t n = c.h_tmaster[k];
      if (n < 0 || n >= nnode) return c.set_error("ties: master node out of range");
      if (c.h_slave_of[n] >= 0) return c.set_error("ties: node " + std::to_string(n) + " is both slave and master");
      if (!std::isfinite(c.h_tweight[k])) return c.set_error("ties: weight is not finite");
    }
  }

  // expanded incidence of every element (global id gofs[b] + e): its nodes, a
  // slave node replaced by its masters (first appearance order, no repeats)
  std::vector<int64_t> gofs(m.num_buckets + 1, 0);
  for (int b = 0; b < m.num_buckets; b++) gofs[b + 1] = gofs[b] + m.buckets[b].num_elems;
  const int64_t nel = gofs[m.num_buckets];
  std::vector<uint8_t> tied(nel, 0);
  std::vector<int64_t> iptr(nel + 1, 0);
  std::vector<int32_t> inc;
  {
    std::vector<int32_t> tmp;
    for (int b = 0; b < m.num_buckets; b++) {
      const fast_gpu_bucket &bk = m.buckets[b];
      const int nn = bucket_nodes(bk);
      for (int64_t e = 0; e < bk.num_elems; e++) {
        const int64_t g = gofs[b] + e;
        tmp.clear();
        bool t = false;
        for (int a = 0; a < nn; a++) {
          const int32_t n = bk.conn[e * nn + a];
          if (n < 0 || n >= nnode) return c.set_error("element incidence out of range");
          const int32_t s = c.h_slave_of[n];
          if (s < 0) {
            tmp.push_back(n);
          } else {
            t = true;
            for (int64_t k = c.h_tptr[s]; k < c.h_tptr[s + 1]; k++) tmp.push_back((int32_t)c.h_tmaster[k]);
          }
        }
        if (t) {  // remove repeats, keep first appearance
          std::vector<int32_t> u;
          for (int32_t n : tmp)
            if (std::find(u.begin(), u.end(), n) == u.end()) u.push_back(n);
          tmp.swap(u);
          tied[g] = 1;
        }
        inc.insert(inc.end(), tmp.begin(), tmp.end());
        iptr[g + 1] = (int64_t)inc.size();
      }
    }
  }

  // node -> elements (expanded incidence), as CSR
  std::vector<int64_t> ecount(nnode + 1, 0);
  for (int64_t k = 0; k < (int64_t)inc.size(); k++) ecount[inc[k] + 1]++;
  for (int64_t i = 0; i < nnode; i++) ecount[i + 1] += ecount[i];
  std::vector<int64_t> eptr(ecount);
  std::vector<int64_t> elist(ecount[nnode]);
  {
    std::vector<int64_t> fill(ecount.begin(), ecount.end() - 1);
    for (int64_t g = 0; g < nel; g++)
      for (int64_t k = iptr[g]; k < iptr[g + 1]; k++) elist[fill[inc[k]]++] = g;
  }

  // 1. node-block CSR: rows in parallel, a marker per thread.  A slave row
  //    keeps only its diagonal block (identity on its eliminated DOFs).
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
          const int64_t g = elist[k];
          for (int64_t q = iptr[g]; q < iptr[g + 1]; q++) {
            const int32_t n = inc[q];
            if (mark[n] != i) { mark[n] = i; cnt++; }
          }
        }
        if (c.h_slave_of[i] >= 0) cnt = 1;
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
        if (c.h_slave_of[i] >= 0) { out[0] = (int32_t)i; continue; }
        int cnt = 0;
        for (int64_t k = eptr[i]; k < eptr[i + 1]; k++) {
          const int64_t g = elist[k];
          for (int64_t q = iptr[g]; q < iptr[g + 1]; q++) {
            const int32_t n = inc[q];
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

  // 2./3. per bucket: greedy colouring (element order) of the elements that
  // touch no slave node, colour sort, slot map.  Buckets are assembled one
  // after another, so colours are per bucket.  Tied elements follow the
  // coloured ones in the bucket's element order.
  constexpr int kWords = 4;  // up to 256 colours; B-spline solids of degree p need (p+1)^3
  auto colour = [&](const std::vector<int64_t> &ids, std::vector<int32_t> &color, int &ncol) -> bool {
    std::vector<uint64_t> node_colors((size_t)nnode * kWords, 0);  // bit k: a colour-k element uses the node
    color.assign(ids.size(), 0);
    ncol = 0;
    for (size_t x = 0; x < ids.size(); x++) {
      const int64_t g = ids[x];
      uint64_t used[kWords] = {0, 0, 0, 0};
      for (int64_t q = iptr[g]; q < iptr[g + 1]; q++)
        for (int w = 0; w < kWords; w++) used[w] |= node_colors[(size_t)inc[q] * kWords + w];
      int col = -1;
      for (int w = 0; w < kWords && col < 0; w++)
        if (~used[w] != 0) col = 64 * w + __builtin_ctzll(~used[w]);
      if (col < 0) return false;
      color[x] = col;
      ncol = std::max(ncol, col + 1);
      for (int64_t q = iptr[g]; q < iptr[g + 1]; q++)
        node_colors[(size_t)inc[q] * kWords + col / 64] |= (1ULL << (col % 64));
    }
    return true;
  };
  c.ncolors = 0;
  for (int b = 0; b < m.num_buckets; b++) {
    const fast_gpu_bucket &bk = m.buckets[b];
    Bucket &B = c.buckets[b];
    const int nn = B.nn;
    std::vector<int64_t> ids, tids;
    for (int64_t e = 0; e < bk.num_elems; e++) (tied[gofs[b] + e] ? tids : ids).push_back(gofs[b] + e);
    std::vector<int32_t> color;
    int ncol = 0;
    if (!colour(ids, color, ncol)) return c.set_error("element colouring needs more than 256 colours");
    c.ncolors = std::max(c.ncolors, ncol);
    // stable counting sort by colour, tied elements last
    B.ne_regular = (int64_t)ids.size();
    B.color_off.assign(ncol + 1, 0);
    for (size_t x = 0; x < ids.size(); x++) B.color_off[color[x] + 1]++;
    for (int k = 0; k < ncol; k++) B.color_off[k + 1] += B.color_off[k];
    B.perm.assign(bk.num_elems, 0);
    B.inv.assign(bk.num_elems, 0);
    {
      std::vector<int64_t> fill(B.color_off.begin(), B.color_off.end() - 1);
      for (size_t x = 0; x < ids.size(); x++) {
        const int64_t pos = fill[color[x]]++;
        const int32_t e = (int32_t)(ids[x] - gofs[b]);
        B.perm[pos] = e;
        B.inv[e] = (int32_t)pos;
      }
      int64_t pos = B.ne_regular;
      for (int64_t g : tids) {
        const int32_t e = (int32_t)(g - gofs[b]);
        B.perm[pos] = e;
        B.inv[e] = (int32_t)pos;
        pos++;
      }
    }
    B.h_conn.assign(bk.num_elems * nn, 0);
    for (int64_t s = 0; s < bk.num_elems; s++)
      std::memcpy(&B.h_conn[s * nn], &bk.conn[(int64_t)B.perm[s] * nn], sizeof(int32_t) * nn);
    // slot map of the coloured elements, colour-sorted element order
    B.h_slot.assign(bk.num_elems * nn * nn, -1);
    bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
    for (int64_t s = 0; s < B.ne_regular; s++) {
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

  // tied elements of all buckets: coloured together on their expanded lists
  TiedSet &T = c.tied;
  T = TiedSet();
  T.bucket_pos.assign(m.num_buckets, {});
  T.bucket_keoff.assign(m.num_buckets, 0);
  {
    std::vector<int64_t> tids;
    for (int64_t g = 0; g < nel; g++)
      if (tied[g]) tids.push_back(g);
    T.n = (int64_t)tids.size();
    if (T.n > 0) {
      // scratch layout: per bucket, its tied elements in perm order
      std::vector<int64_t> keoff_of(nel, -1);
      int64_t ke = 0;
      for (int b = 0; b < m.num_buckets; b++) {
        Bucket &B = c.buckets[b];
        const int64_t nd = 3 * B.nn;
        T.bucket_keoff[b] = ke;
        for (int64_t pos = B.ne_regular; pos < B.ne; pos++) {
          T.bucket_pos[b].push_back((int32_t)pos);
          keoff_of[gofs[b] + B.perm[pos]] = ke;
          ke += nd * nd;
        }
      }
      T.ke_total = ke;
      std::vector<int32_t> color;
      int ncol = 0;
      if (!colour(tids, color, ncol)) return c.set_error("tied element colouring needs more than 256 colours");
      c.ncolors = std::max(c.ncolors, ncol);
      T.color_off.assign(ncol + 1, 0);
      for (size_t x = 0; x < tids.size(); x++) T.color_off[color[x] + 1]++;
      for (int k = 0; k < ncol; k++) T.color_off[k + 1] += T.color_off[k];
      std::vector<int64_t> order(tids.size());
      {
        std::vector<int64_t> fill(T.color_off.begin(), T.color_off.end() - 1);
        for (size_t x = 0; x < tids.size(); x++) order[fill[color[x]]++] = tids[x];
      }
      T.h_nptr.assign(T.n + 1, 0);
      T.h_eptr.assign(1, 0);
      T.h_econn.clear();
      T.h_sptr.assign(T.n + 1, 0);
      T.h_pptr.assign(1, 0);
      for (int64_t x = 0; x < T.n; x++) {
        const int64_t g = order[x];
        const int b = (int)(std::upper_bound(gofs.begin(), gofs.end(), g) - gofs.begin()) - 1;
        const int64_t e = g - gofs[b];
        const fast_gpu_bucket &bk = m.buckets[b];
        const int nn = c.buckets[b].nn;
        const int64_t m0 = iptr[g], me = iptr[g + 1] - iptr[g];
        T.h_nodes.insert(T.h_nodes.end(), inc.begin() + m0, inc.begin() + m0 + me);
        T.h_nptr[x + 1] = T.h_nptr[x] + me;
        // pre-image of each expanded node: (local node, weight)
        for (int64_t A = 0; A < me; A++) {
          const int32_t N = inc[m0 + A];
          for (int a = 0; a < nn; a++) {
            const int32_t n = bk.conn[e * nn + a];
            const int32_t s = c.h_slave_of[n];
            if (s < 0) {
              if (n == N) { T.h_pa.push_back(a); T.h_pt.push_back(1.0); }
            } else {
              for (int64_t k = c.h_tptr[s]; k < c.h_tptr[s + 1]; k++)
                if (c.h_tmaster[k] == N) { T.h_pa.push_back(a); T.h_pt.push_back(c.h_tweight[k]); }
            }
          }
          T.h_pptr.push_back((int64_t)T.h_pa.size());
        }
        // block slots of the expanded pairs, row-major
        for (int64_t A = 0; A < me; A++) {
          const int32_t na = inc[m0 + A];
          const int32_t *r0 = c.h_col.data() + c.h_rowptr[na];
          const int32_t *r1 = c.h_col.data() + c.h_rowptr[na + 1];
          for (int64_t Bq = 0; Bq < me; Bq++) {
            const int32_t *p = std::lower_bound(r0, r1, inc[m0 + Bq]);
            if (p == r1 || *p != inc[m0 + Bq]) return c.set_error("internal: tied pair missing from the pattern");
            T.h_slot.push_back((int32_t)(p - c.h_col.data()));
          }
        }
        T.h_sptr[x + 1] = (int64_t)T.h_slot.size();
        T.h_keoff.push_back(keoff_of[g]);
        T.h_nn.push_back(nn);
        // its own nodes, in the element's local order (node-space products)
        T.h_econn.insert(T.h_econn.end(), bk.conn + e * nn, bk.conn + (e + 1) * nn);
        T.h_eptr.push_back((int64_t)T.h_econn.size());
      }
    }
  }
  // 4. first-touch flags: the stiffness assembly visits buckets, then
  // colours, in order; the first element to reach a block writes it outright
  // (no read; fixed entries zero, 1 on the diagonal of a fixed DOF), so K
  // needs no zero fill.  Only where every block is reached that way: no tied
  // interfaces (their blocks come from the tied scatter), no total-Lagrangian
  // buckets (their tangent is added by other kernels), no block left over.
  c.first_touch = false;
  bool eligible = c.tied.n == 0;
  for (const Bucket &B : c.buckets) eligible = eligible && !B.tl && B.ne_regular == B.ne;
  if (eligible) {
    const int64_t nnzb = c.h_rowptr[nnode];
    std::vector<uint8_t> touched((size_t)nnzb, 0);
    for (Bucket &B : c.buckets) {
      const int nn = B.nn;
      const int fw = first_words(nn);
      B.h_first.assign((size_t)B.ne * fw, 0u);
      for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
        // elements of one colour share no node, hence no block
#pragma omp parallel for schedule(static)
        for (int64_t s = B.color_off[k]; s < B.color_off[k + 1]; s++) {
          const int32_t *sl = &B.h_slot[(size_t)s * nn * nn];
          uint32_t *f = &B.h_first[(size_t)s * fw];
          for (int q = 0; q < nn * nn; q++)
            if (!touched[sl[q]]) {
              touched[sl[q]] = 1;
              f[q >> 5] |= 1u << (q & 31);
            }
        }
      }
    }
    bool all = true;
    for (int64_t q = 0; q < nnzb && all; q++) all = touched[q] != 0;
    c.first_touch = all;
    if (!all)
      for (Bucket &B : c.buckets) std::vector<uint32_t>().swap(B.h_first);
  }
  c.pattern_seconds = now_s() - t0;
  return true;
}

}  // namespace fastgpu

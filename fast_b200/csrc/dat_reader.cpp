// dat_reader.cpp - the solid subset of FAST's .dat input, read on all host
// cores (include/fast_dat.h).
//
// The reference reads its deck as one istream: Utl::NextLabel skips to the
// next '%', reads the label, and the label's reader extracts the tokens it
// needs (main/input.cpp:355-401, main/utl.cpp:125-133).  Here the file is
// mapped once, the '%' positions split it into blocks, and each large block
// (coordinates, supports, elements, loads) is tokenised in parallel: a
// counting pass per chunk (chunk edges moved to whitespace so no token is
// split), a prefix sum, then a parsing pass that writes every number to its
// global token index.  Records are fixed-length token groups, so the line
// layout does not matter, as for the reference's stream extraction.
// Numbers are parsed with std::from_chars (correctly rounded, as strtod is
// for istream >> double); a token that is not wholly a number is an error.
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fast_dat.h"

namespace {

constexpr int64_t kMaxLabel = int64_t(1) << 31;  // labels are int in the reference

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

struct Block {
  std::string label;
  const char *b, *e;  // data: after the label up to the next '%'
};

// face tables of cShapeBrick8/20::GetFace (shp/shpsolid.cpp:264-276, 459-471):
// corner nodes, then the face nodes in face-shape order
const int kHex8Corner[6][4] = {{0, 1, 2, 3}, {3, 2, 6, 7}, {1, 5, 6, 2}, {0, 4, 5, 1}, {0, 3, 7, 4}, {4, 7, 6, 5}};
const int kHex20Corner[6][4] = {{0, 2, 4, 6},    {2, 0, 12, 14}, {4, 2, 14, 16},
                                {6, 4, 16, 18}, {12, 18, 16, 14}, {18, 6, 0, 12}};
const int kHex20Face[6][8] = {{0, 1, 2, 3, 4, 5, 6, 7},       {2, 1, 0, 8, 12, 13, 14, 9},
                              {4, 3, 2, 9, 14, 15, 16, 10},   {6, 5, 4, 10, 16, 17, 18, 11},
                              {12, 19, 18, 17, 16, 15, 14, 13}, {18, 11, 6, 7, 0, 8, 12, 19}};

}  // namespace

struct fast_dat {
  std::string err;
  const char *base = nullptr;  // the mapped file (for line numbers in messages)
  size_t size = 0;
  fast_dat_info info{};
  std::vector<double> coords, nodal_f, E, nu, rho, face_q;
  std::vector<uint8_t> fixed;
  std::vector<int64_t> solver_rank;
  std::vector<int32_t> conn, face_elem, face_corner, face_nodes, face_local;
  // B-spline solid decks: the patch (knots expanded) and the element spans
  std::vector<double> knots[3], weights;
  std::vector<int32_t> span;  // [ne][3]
  std::vector<int32_t> cps;   // node index of each patch control point, r fastest
  fast_gpu_patch patch{};
};

namespace {

struct Reader {
  fast_dat &d;
  int threads;
  std::vector<Block> blocks;

  int line_of(const char *p) const {
    if (!d.base || p < d.base || p > d.base + d.size) return 0;
    return 1 + (int)std::count(d.base, p, '\n');
  }
  int fail(const std::string &what, const char *where) {
    d.err = what;
    if (where) d.err += " (line " + std::to_string(line_of(where)) + ")";
    return FAST_GPU_EINVAL;
  }

  // Utl::NextLabel: every '%' starts a label (the next whitespace-delimited
  // word); %END ends the input
  void split() {
    const char *p = d.base, *end = d.base + d.size;
    while (p < end) {
      const char *q = (const char *)memchr(p, '%', end - p);
      if (!q) break;
      q++;
      while (q < end && is_ws(*q)) q++;
      const char *l = q;
      while (q < end && !is_ws(*q) && *q != '%') q++;
      std::string label(l, q);
      if (label == "END") break;
      const char *nx = (const char *)memchr(q, '%', end - q);
      blocks.push_back({label, q, nx ? nx : end});
      p = nx ? nx : end;
    }
  }
  std::vector<const Block *> find_all(const char *label) const {
    std::vector<const Block *> v;
    for (auto &b : blocks)
      if (b.label == label) v.push_back(&b);
    return v;
  }
  const Block *find(const char *label) const {  // a repeated block: the last one counts
    const Block *r = nullptr;
    for (auto &b : blocks)
      if (b.label == label) r = &b;
    return r;
  }

  template <class T>
  static bool parse_one(const char *s, const char *e, T &v) {
    if (s < e && *s == '+') s++;  // istream >> accepts a leading '+', from_chars does not
    auto r = std::from_chars(s, e, v);
    return r.ec == std::errc() && r.ptr == e;
  }

  // the first `need` tokens of [b, e) as T; need < 0: the first token is a
  // count n and the block holds 1 + n * (-need) tokens
  template <class T>
  int tokens(const Block &blk, int64_t need, std::vector<T> &out, const char *what) {
    const char *b = blk.b, *e = blk.e;
    if (need < 0) {  // read the count first
      const char *s = b;
      while (s < e && is_ws(*s)) s++;
      const char *t = s;
      while (t < e && !is_ws(*t)) t++;
      int64_t n;
      if (s == t || !parse_one(s, t, n) || n < 0 || n > (int64_t)(e - b))
        return fail(std::string("error in the number of ") + what, s);
      need = 1 + n * (-need);
    }
    const size_t bytes = e - b;
    int nt = (int)std::min<size_t>(threads, std::max<size_t>(1, bytes >> 20));
    std::vector<const char *> edge(nt + 1);
    edge[0] = b;
    edge[nt] = e;
    for (int t = 1; t < nt; t++) {
      const char *p = b + bytes * t / nt;
      if (p < edge[t - 1]) p = edge[t - 1];
      while (p < e && !is_ws(*p)) p++;
      edge[t] = p;
    }
    std::vector<int64_t> cnt(nt + 1, 0);
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; t++) {
      int64_t c = 0;
      const char *p = edge[t], *pe = edge[t + 1];
      while (p < pe) {
        while (p < pe && is_ws(*p)) p++;
        if (p >= pe) break;
        c++;
        while (p < pe && !is_ws(*p)) p++;
      }
      cnt[t + 1] = c;
    }
    for (int t = 0; t < nt; t++) cnt[t + 1] += cnt[t];
    if (cnt[nt] < need)
      return fail(std::string("error in the input of ") + what + ": " + std::to_string(need) + " numbers expected, " +
                      std::to_string(cnt[nt]) + " found",
                  b);
    out.resize(need);
    std::atomic<const char *> bad{nullptr};
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; t++) {
      int64_t k = cnt[t];
      const char *p = edge[t], *pe = edge[t + 1];
      while (p < pe && k < need) {
        while (p < pe && is_ws(*p)) p++;
        if (p >= pe) break;
        const char *s = p;
        while (p < pe && !is_ws(*p)) p++;
        if (!parse_one(s, p, out[k])) {
          const char *cur = bad.load();
          while ((!cur || s < cur) && !bad.compare_exchange_weak(cur, s)) {
          }
        }
        k++;
      }
    }
    if (bad.load()) return fail(std::string("error in the input of ") + what + ": not a number", bad.load());
    return FAST_GPU_OK;
  }

  // a quoted string (Utl::ReadString) or the first word
  std::string word(const Block &blk) const {
    const char *p = blk.b, *e = blk.e;
    while (p < e && is_ws(*p)) p++;
    if (p < e && *p == '\'') {
      const char *q = (const char *)memchr(p + 1, '\'', e - p - 1);
      return q ? std::string(p + 1, q) : std::string(p + 1, e);
    }
    const char *s = p;
    while (p < e && !is_ws(*p)) p++;
    return std::string(s, p);
  }
  template <class T>
  int scalar(const char *label, T &v) {
    const Block *b = find(label);
    if (!b) return FAST_GPU_OK;
    std::vector<T> t;
    int rc = tokens(*b, 1, t, label);
    if (rc == FAST_GPU_OK) v = t[0];
    return rc;
  }

  int header() {
    fast_dat_info &I = d.info;
    I.max_steps = 1;
    I.target_iter = -1;
    I.print_step = 1;
    I.tol = 1e-5;
    I.step_factor = 1.0;
    I.newmark[0] = 0.5;
    I.newmark[1] = 0.25;
    if (const Block *b = find("HEADER")) {
      const char *p = b->b, *e = b->e;
      while (p < e && (*p == '\n' || *p == '\r' || *p == ' ' || *p == '\t')) p++;
      const char *q = p;
      while (q < e && *q != '\n' && *q != '\r') q++;
      snprintf(I.title, sizeof I.title, "%.*s", (int)(q - p), p);
    }
    if (const Block *b = find("HEADER.ANALYSIS.ALGORITHM"))
      snprintf(I.algorithm, sizeof I.algorithm, "%s", word(*b).c_str());
    if (const Block *b = find("HEADER.ANALYSIS.MATRIX.TYPE"))
      snprintf(I.matrix_type, sizeof I.matrix_type, "%s", word(*b).c_str());
    int rc;
    int64_t iv;
    if ((rc = scalar("HEADER.ANALYSIS.TOLERANCE", I.tol))) return rc;
    if ((rc = scalar("HEADER.ANALYSIS.STEP.FACTOR", I.step_factor))) return rc;
    if ((rc = scalar("HEADER.ANALYSIS.TIME.STEP", I.time_step))) return rc;
    iv = I.max_iter;
    if ((rc = scalar("HEADER.ANALYSIS.MAXIMUM.ITERATIONS", iv))) return rc;
    I.max_iter = (int32_t)iv;
    iv = I.max_steps;
    if ((rc = scalar("HEADER.ANALYSIS.MAXIMUM.STEPS", iv))) return rc;
    I.max_steps = (int32_t)iv;
    iv = I.target_iter;
    if ((rc = scalar("HEADER.ANALYSIS.TARGET.ITERATIONS", iv))) return rc;
    I.target_iter = (int32_t)iv;
    iv = I.print_step;
    if ((rc = scalar("HEADER.ANALYSIS.PRINT.STEPS", iv))) return rc;
    I.print_step = (int32_t)iv;
    if (const Block *b = find("HEADER.ANALYSIS.ARC-LENGTH")) {
      std::vector<double> t;
      if ((rc = tokens(*b, 1, t, "ARC-LENGTH"))) return rc;
      I.has_arc_length = 1;
      I.arc_load_coeff = t[0];
    }
    if (const Block *b = find("HEADER.ANALYSIS.NEWMARK.PARAMETERS")) {
      std::vector<double> t;
      if ((rc = tokens(*b, 2, t, "NEWMARK.PARAMETERS"))) return rc;
      I.newmark[0] = t[0];
      I.newmark[1] = t[1];
    }
    return FAST_GPU_OK;
  }

  // %PATCH (cBspPat::Read, geom/patch.cpp:1459-1484): one 'bspsol' patch:
  // id, type, rational flag, per direction degree 'General' #knots values
  // multiplicities (cKnotVector::ReadKnot / ReadMult, geom/knotvec.cpp:91-170),
  // then the control-point node labels, r fastest.  Quoted words are tokens.
  int read_patch(int64_t nnode, int deg[3], int64_t nbas[3], std::vector<int32_t> &cps) {
    const Block *b = find("PATCH");
    if (!b) return fail("B-spline elements without %PATCH", nullptr);
    std::vector<std::string> tok;
    for (const char *p = b->b; p < b->e;) {
      while (p < b->e && is_ws(*p)) p++;
      if (p >= b->e) break;
      const char *q = p;
      if (*p == '\'') {
        q = (const char *)memchr(p + 1, '\'', b->e - p - 1);
        q = q ? q + 1 : b->e;
      } else {
        while (q < b->e && !is_ws(*q)) q++;
      }
      tok.emplace_back(p, q);
      p = q;
    }
    size_t pos = 0;
    auto num = [&](double &v) -> bool { return pos < tok.size() && parse_one(tok[pos].data(), tok[pos].data() + tok[pos].size(), v) && ++pos; };
    double v;
    if (!num(v) || v != 1.0) {
      d.err = "one B-spline patch per deck is read here";
      return FAST_GPU_ENOTSUP;
    }
    if (!num(v) || pos >= tok.size() || tok[pos] != "'bspsol'") {
      d.err = "the patch must be a 'bspsol' B-spline solid";
      return FAST_GPU_ENOTSUP;
    }
    pos++;
    double rat;
    if (!num(rat)) return fail("error in the input of the patch rational flag", b->b);
    d.patch.rational = rat != 0.0;
    for (int k = 0; k < 3; k++) {
      double p_, nk;
      if (!num(p_) || pos >= tok.size()) return fail("error in the input of the patch degrees", b->b);
      if (tok[pos] != "'General'") {
        d.err = "knot vector format " + tok[pos] + " is not read here";
        return FAST_GPU_ENOTSUP;
      }
      pos++;
      if (!num(nk) || nk < 1) return fail("error in the input of the knot vector", b->b);
      std::vector<double> vals((size_t)nk), mult((size_t)nk);
      for (auto &x : vals)
        if (!num(x)) return fail("error in the input of the knot values", b->b);
      for (auto &x : mult)
        if (!num(x) || x < 1) return fail("error in the input of the knot multiplicities", b->b);
      deg[k] = (int)p_;
      d.knots[k].clear();
      for (size_t i = 0; i < vals.size(); i++)
        for (int m = 0; m < (int)mult[i]; m++) d.knots[k].push_back(vals[i]);
      nbas[k] = (int64_t)d.knots[k].size() - deg[k] - 1;
      if (deg[k] < 1 || nbas[k] < 1) return fail("invalid knot vector / degree in the patch", b->b);
    }
    const int64_t ncp = nbas[0] * nbas[1] * nbas[2];
    cps.resize(ncp);
    for (int64_t i = 0; i < ncp; i++) {
      if (!num(v) || v < 1 || v > nnode) return fail("invalid control point in the patch", b->b);
      cps[i] = (int32_t)v - 1;
    }
    d.weights.clear();
    if (const Block *w = find("CONTROL.POINT.WEIGHT")) {
      std::vector<double> t;
      int rc;
      if ((rc = tokens(*w, -2, t, "control point weights"))) return rc;
      d.weights.assign(nnode, 1.0);
      for (int64_t r = 0; r < (int64_t)t[0]; r++) {
        const double id = t[1 + 2 * r];
        if (!(id >= 1 && id <= (double)nnode)) return fail("weight of an invalid control point", w->b);
        d.weights[(int64_t)id - 1] = t[2 + 2 * r];
      }
    }
    return FAST_GPU_OK;
  }

  int run() {
    split();
    int rc = header();
    if (rc) return rc;
    fast_dat_info &I = d.info;
    for (const char *unsup : {"NODE.MULTI-POINT.CONSTRAINT"})
      if (find(unsup)) {
        d.err = std::string("%") + unsup + " decks are not read here";
        return FAST_GPU_ENOTSUP;
      }

    // nodes: the i-th record is node i+1 (cNode::ReadCoord)
    const Block *bc = find("NODE.COORD");
    if (!bc) return fail("no %NODE.COORD", nullptr);
    std::vector<double> tc;
    if ((rc = tokens(*bc, -4, tc, "nodal coordinates"))) return rc;
    const int64_t nnode = (int64_t)tc[0];
    if (const Block *bn = find("NODE")) {
      std::vector<int64_t> t;
      if ((rc = tokens(*bn, 1, t, "number of nodes"))) return rc;
      if (t[0] != nnode) return fail("error in the input of the number of nodal coordinates", bc->b);
    }
    if (nnode <= 0) return fail("no nodes", bc->b);
    I.num_nodes = nnode;
    d.coords.resize(3 * nnode);
#pragma omp parallel for num_threads(threads)
    for (int64_t i = 0; i < nnode; i++)
      for (int k = 0; k < 3; k++) d.coords[3 * i + k] = tc[1 + 4 * i + 1 + k];
    std::vector<double>().swap(tc);

    d.fixed.assign(3 * nnode, 0);
    for (const Block *b : find_all("NODE.SUPPORT")) {
      std::vector<int64_t> t;
      if ((rc = tokens(*b, -7, t, "supports"))) return rc;
      for (int64_t r = 0; r < t[0]; r++) {
        const int64_t *row = &t[1 + 7 * r];
        if (row[0] < 1 || row[0] > nnode) return fail("support on an invalid node", b->b);
        for (int k = 0; k < 3; k++)
          if (row[1 + k]) d.fixed[3 * (row[0] - 1) + k] = 1;
      }
    }
    if (const Block *b = find("NODE.SOLVER.ORDER")) {
      std::vector<int64_t> t;
      if ((rc = tokens(*b, -1, t, "nodes in solver order"))) return rc;
      if (t[0] != nnode) return fail("error in the input of the number of nodes in solver order", b->b);
      d.solver_rank.assign(t.begin() + 1, t.end());
      for (int64_t v : d.solver_rank)
        if (v < 1 || v > nnode) return fail("invalid node number in solver order", b->b);
      I.has_solver_order = 1;
    }

    // materials and sections, by label (VecMat[id-1], VecSec[id-1]): dense
    // tables indexed by label, label 0 unused
    struct Mat { double E = 0, nu = 0, rho = 0; bool def = false; };
    std::vector<Mat> mat;
    std::vector<int64_t> sec;  // material label of each section label, 0 = undefined
    auto grow = [](auto &v, int64_t id) {
      if ((int64_t)v.size() <= id) v.resize(id + 1);
    };
    for (const Block *b : find_all("MATERIAL.ISOTROPIC")) {
      std::vector<double> t;
      if ((rc = tokens(*b, -3, t, "isotropic materials"))) return rc;
      for (int64_t r = 0; r < (int64_t)t[0]; r++) {
        const double id = t[1 + 3 * r];
        if (!(id >= 1 && id <= (double)kMaxLabel)) return fail("error in the input of elastic isotropic material", b->b);
        grow(mat, (int64_t)id);
        Mat &m = mat[(int64_t)id];
        m.E = t[2 + 3 * r];
        m.nu = t[3 + 3 * r];
        m.def = true;
      }
    }
    for (const Block *b : find_all("MATERIAL.DENSITY")) {
      std::vector<double> t;
      if ((rc = tokens(*b, -2, t, "densities"))) return rc;
      for (int64_t r = 0; r < (int64_t)t[0]; r++) {
        const double id = t[1 + 2 * r];
        if (!(id >= 1 && id <= (double)kMaxLabel)) return fail("error in the input of densities", b->b);
        grow(mat, (int64_t)id);
        mat[(int64_t)id].rho = t[2 + 2 * r];
      }
      I.has_density = 1;
    }
    for (const Block *b : find_all("SECTION.HOMOGENEOUS.ISOTROPIC.3D")) {
      std::vector<int64_t> t;
      if ((rc = tokens(*b, -2, t, "3D homogeneous sections"))) return rc;
      for (int64_t r = 0; r < t[0]; r++) {
        const int64_t id = t[1 + 2 * r];
        if (id < 1 || id > kMaxLabel) return fail("error in the input of 3D homogeneous section", b->b);
        grow(sec, id);
        sec[id] = t[2 + 2 * r];
      }
    }
    std::vector<int64_t> ord;
    if (const Block *b = find("INTEGRATION.ORDER")) {
      if ((rc = tokens(*b, -7, ord, "integration orders"))) return rc;
    }

    // elements: one solid type, addressed by label
    struct Kind { const char *label; int type, nn, form; };
    const Kind kinds[] = {{"ELEMENT.BRICK8", FAST_ELEM_HEX8, 8, FAST_FORM_SMALL_STRAIN},
                          {"ELEMENT.BRICK20", FAST_ELEM_HEX20, 20, FAST_FORM_SMALL_STRAIN},
                          {"ELEMENT.BRICK8TL", FAST_ELEM_HEX8, 8, FAST_FORM_TOTAL_LAGRANGIAN},
                          {"ELEMENT.BRICK20TL", FAST_ELEM_HEX20, 20, FAST_FORM_TOTAL_LAGRANGIAN},
                          {"ELEMENT.BSPLINE.SOLID", FAST_ELEM_BSP_SOLID, 0, FAST_FORM_SMALL_STRAIN},
                          {"ELEMENT.BSPLINE.SOLIDTL", FAST_ELEM_BSP_SOLID, 0, FAST_FORM_TOTAL_LAGRANGIAN}};
    const Kind *kind = nullptr;
    for (auto &k : kinds)
      if (find(k.label)) {
        if (kind) {
          d.err = "decks with more than one solid element type are not read here";
          return FAST_GPU_ENOTSUP;
        }
        kind = &k;
      }
    if (!kind) {
      d.err = "no %ELEMENT.BRICK8 / BRICK20 (TL) or BSPLINE.SOLID (TL) block";
      return FAST_GPU_ENOTSUP;
    }
    const bool bsp = kind->type == FAST_ELEM_BSP_SOLID;
    int deg[3] = {0, 0, 0};
    int64_t nbas[3] = {0, 0, 0};
    std::vector<int32_t> cps;
    std::vector<int64_t> first[3];  // first basis function of each non-zero span
    if (bsp) {
      if ((rc = read_patch(nnode, deg, nbas, cps))) return rc;
      // cBSplineBasis::getBasInd (geom/bspbasis.cpp:59-62): spans with a gap above 1e-5
      for (int k = 0; k < 3; k++) {
        const std::vector<double> &U = d.knots[k];
        for (size_t i = 1; i < U.size(); i++)
          if (U[i] - U[i - 1] > 1e-5) first[k].push_back((int64_t)i - 1 - deg[k]);
      }
      if (find("LOAD.CASE.AREA.UNIFORM")) {
        d.err = "area loads on B-spline solids are not read here";
        return FAST_GPU_ENOTSUP;
      }
    }
    const int nn = bsp ? (deg[0] + 1) * (deg[1] + 1) * (deg[2] + 1) : kind->nn;
    // cShapeBsp::ReadIGA (shp/shpbsp.cpp:57-116): id section order patch span_r span_s span_t
    const int rec = bsp ? 7 : 3 + nn;
    std::vector<std::vector<int64_t>> eblk;
    int64_t nrec = 0;
    for (const Block *b : find_all(kind->label)) {
      eblk.emplace_back();
      if ((rc = tokens(*b, -rec, eblk.back(), kind->label + 8))) return rc;
      if (eblk.back()[0] < 1) return fail(std::string("error in the number of ") + (kind->label + 8) + " elements", b->b);
      nrec += eblk.back()[0];
    }
    int64_t nelem = nrec;
    if (const Block *b = find("ELEMENT")) {
      std::vector<int64_t> t;
      if ((rc = tokens(*b, 1, t, "number of elements"))) return rc;
      nelem = t[0];
    }
    if (nrec != nelem) return fail("the element blocks do not define every element exactly once", nullptr);
    I.num_elems = nelem;
    I.elem_type = kind->type;
    I.nodes_per_elem = nn;
    I.formulation = kind->form;
    I.nodes_per_face = bsp ? 0 : (nn == 8 ? 4 : 8);
    d.conn.assign((size_t)nelem * nn, -1);
    if (bsp) d.span.assign((size_t)nelem * 3, 0);
    d.E.assign(nelem, 0.0);
    d.nu.assign(nelem, 0.0);
    if (I.has_density) d.rho.assign(nelem, 0.0);
    std::vector<uint8_t> seen(nelem, 0);
    std::vector<int64_t> elem_sec(nelem), elem_ord(nelem);
    std::atomic<int> bad{0};  // 1 label, 2 node, 3 twice
    for (auto &t : eblk) {
      const int64_t n = t[0];
#pragma omp parallel for num_threads(threads)
      for (int64_t r = 0; r < n; r++) {
        const int64_t *row = &t[1 + rec * r];
        const int64_t id = row[0];
        if (id < 1 || id > nelem) { bad = 1; continue; }
        const int64_t e = id - 1;
        if (seen[e]) bad = 3;
        seen[e] = 1;
        elem_sec[e] = row[1];
        elem_ord[e] = row[2];
        if (bsp) {
          // the element's control points, r fastest (cShapeBspSolid::Init, shp/shpbsp.cpp:873-902)
          int64_t b0[3];
          bool ok = true;
          for (int k = 0; k < 3; k++) {
            const int64_t sp = row[4 + k] - 1;
            if (sp < 0 || sp >= (int64_t)first[k].size()) { ok = false; break; }
            d.span[3 * e + k] = (int32_t)sp;
            b0[k] = first[k][sp];
          }
          if (!ok) { bad = 2; continue; }
          int loc = 0;
          for (int kk = 0; kk <= deg[2]; kk++)
            for (int jj = 0; jj <= deg[1]; jj++)
              for (int ii = 0; ii <= deg[0]; ii++, loc++) {
                const int64_t cp = (b0[0] + ii) + nbas[0] * (b0[1] + jj) + nbas[0] * nbas[1] * (b0[2] + kk);
                d.conn[(size_t)e * nn + loc] = (cp >= 0 && cp < (int64_t)cps.size()) ? cps[cp] : (bad = 2, 0);
              }
          continue;
        }
        for (int k = 0; k < nn; k++) {
          const int64_t v = row[3 + k];
          if (v < 1 || v > nnode) bad = 2;
          d.conn[(size_t)e * nn + k] = (int32_t)(v - 1);
        }
      }
    }
    if (bad == 1) return fail(std::string("error in the input of ") + (kind->label + 8) + " elements (label)", nullptr);
    if (bad == 2) return fail(bsp ? "element knot span outside the patch" : "element incidence names an invalid node",
                              nullptr);
    if (bad == 3 || std::count(seen.begin(), seen.end(), 0))
      return fail("the element blocks do not define every element exactly once", nullptr);
    // cElmParam::Read: section by label, integration order by position
    if (ord.empty()) return fail("no %INTEGRATION.ORDER", nullptr);
    const int64_t nord = ord[0];
    const int64_t ord0 = elem_ord[0];
    if (ord0 < 1 || ord0 > nord) return fail("invalid integration order for element 1", nullptr);
    std::atomic<int64_t> bad_sec{0}, bad_ord{0};
    std::atomic<int> mixed{0};
    const int64_t *o0 = &ord[1 + 7 * (ord0 - 1)];
#pragma omp parallel for num_threads(threads)
    for (int64_t e = 0; e < nelem; e++) {
      const int64_t s = elem_sec[e];
      const int64_t m = (s >= 1 && s < (int64_t)sec.size()) ? sec[s] : 0;
      if (m < 1 || m >= (int64_t)mat.size() || !mat[m].def) {
        int64_t cur = bad_sec.load();
        while ((cur == 0 || e + 1 < cur) && !bad_sec.compare_exchange_weak(cur, e + 1)) {
        }
        continue;
      }
      d.E[e] = mat[m].E;
      d.nu[e] = mat[m].nu;
      if (I.has_density) d.rho[e] = mat[m].rho;
      const int64_t o = elem_ord[e];
      if (o < 1 || o > nord) {
        bad_ord = e + 1;
        continue;
      }
      const int64_t *oa = &ord[1 + 7 * (o - 1)];
      if (oa[1] != o0[1] || oa[2] != o0[2] || oa[3] != o0[3]) mixed = 1;
    }
    if (bad_sec) return fail("invalid element section or material for element " + std::to_string(bad_sec.load()), nullptr);
    if (bad_ord) return fail("invalid integration order for element " + std::to_string(bad_ord.load()), nullptr);
    if (mixed) {
      d.err = "one integration order per deck is read here";
      return FAST_GPU_ENOTSUP;
    }
    for (int k = 0; k < 3; k++) I.ngp[k] = (int32_t)ord[1 + 7 * (ord0 - 1) + 1 + k];

    // loads
    for (const Block *b : find_all("LOAD.CASE.NODAL.FORCE")) {
      std::vector<double> t;
      if ((rc = tokens(*b, -7, t, "nodal loads"))) return rc;
      if (d.nodal_f.empty()) d.nodal_f.assign(3 * nnode, 0.0);
      for (int64_t r = 0; r < (int64_t)t[0]; r++) {
        const double *row = &t[1 + 7 * r];
        const int64_t id = (int64_t)row[0];
        if (id < 1 || id > nnode) return fail("nodal load on an invalid node", b->b);
        for (int k = 0; k < 3; k++) d.nodal_f[3 * (id - 1) + k] += row[1 + k];
      }
      I.has_nodal_forces = 1;
    }
    for (const Block *b : find_all("LOAD.CASE.AREA.UNIFORM")) {
      std::vector<double> t;
      if ((rc = tokens(*b, -8, t, "uniform face loads"))) return rc;
      const int64_t n = (int64_t)t[0], off = (int64_t)d.face_elem.size();
      const int nf = I.nodes_per_face;
      d.face_elem.resize(off + n);
      d.face_corner.resize(3 * (off + n));
      d.face_nodes.resize(nf * (off + n));
      d.face_local.resize(off + n);
      d.face_q.resize(3 * (off + n));
      std::atomic<int> fbad{0};
#pragma omp parallel for num_threads(threads)
      for (int64_t r = 0; r < n; r++) {
        const double *row = &t[1 + 8 * r];
        const int64_t f = off + r, id = (int64_t)row[0];
        if (id < 1 || id > nelem) { fbad = 1; continue; }
        const int32_t *en = &d.conn[(size_t)(id - 1) * nn];
        d.face_elem[f] = (int32_t)(id - 1);
        for (int k = 0; k < 3; k++) d.face_corner[3 * f + k] = (int32_t)((int64_t)row[1 + k] - 1);
        d.face_local[f] = (int32_t)row[4];
        for (int k = 0; k < 3; k++) d.face_q[3 * f + k] = row[5 + k];
        // cShape::GetShapeFace: the first face whose corners hold all three
        int hit = -1;
        for (int fc = 0; fc < 6 && hit < 0; fc++) {
          int found = 0;
          for (int c = 0; c < 3; c++)
            for (int j = 0; j < 4; j++)
              if (d.face_corner[3 * f + c] == en[nn == 8 ? kHex8Corner[fc][j] : kHex20Corner[fc][j]]) {
                found++;
                break;
              }
          if (found == 3) hit = fc;
        }
        if (hit < 0) { fbad = 2; continue; }
        for (int k = 0; k < nf; k++) d.face_nodes[(size_t)nf * f + k] = en[nn == 8 ? kHex8Corner[hit][k] : kHex20Face[hit][k]];
      }
      if (fbad == 1) return fail("uniform area load on an invalid element", b->b);
      if (fbad == 2) return fail("error in the input of uniform face (area) loads: corners match no face", b->b);
    }
    I.num_faces = (int64_t)d.face_elem.size();
    if (bsp) {
      for (int k = 0; k < 3; k++) {
        I.patch_degree[k] = deg[k];
        I.patch_num_knots[k] = (int32_t)d.knots[k].size();
        d.patch.degree[k] = deg[k];
        d.patch.num_knots[k] = (int32_t)d.knots[k].size();
        d.patch.knots[k] = d.knots[k].data();
      }
      d.patch.span = d.span.data();
      d.cps = cps;
      I.patch_num_cps = (int64_t)cps.size();
      d.patch.weights = d.weights.empty() ? nullptr : d.weights.data();
      I.patch_rational = d.patch.rational;
      I.has_weights = !d.weights.empty();
    }
    return FAST_GPU_OK;
  }
};

}  // namespace

extern "C" int fast_dat_read(const char *path, int32_t threads, fast_dat **out) {
  if (!out) return FAST_GPU_EINVAL;
  *out = nullptr;
  fast_dat *d = new (std::nothrow) fast_dat;
  if (!d) return FAST_GPU_ENOMEM;
  *out = d;
  if (!path) { d->err = "no path"; return FAST_GPU_EINVAL; }
  const int fd = open(path, O_RDONLY);
  if (fd < 0) { d->err = std::string("cannot open ") + path; return FAST_GPU_EINVAL; }
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size == 0) {
    close(fd);
    d->err = std::string("empty or unreadable file ") + path;
    return FAST_GPU_EINVAL;
  }
  void *m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (m == MAP_FAILED) { d->err = std::string("cannot map ") + path; return FAST_GPU_ENOMEM; }
  d->base = (const char *)m;
  d->size = (size_t)st.st_size;
  int rc;
  try {
    Reader r{*d, threads > 0 ? threads : omp_get_num_procs(), {}};
    rc = r.run();
  } catch (const std::bad_alloc &) {
    d->err = "out of host memory";
    rc = FAST_GPU_ENOMEM;
  }
  munmap(m, d->size);
  d->base = nullptr;
  return rc;
}

extern "C" const char *fast_dat_error(const fast_dat *d) { return d ? d->err.c_str() : "no deck"; }

extern "C" void fast_dat_free(fast_dat *d) { delete d; }

extern "C" int fast_dat_get_info(const fast_dat *d, fast_dat_info *info) {
  if (!d || !info || !d->err.empty()) return FAST_GPU_EINVAL;
  *info = d->info;
  return FAST_GPU_OK;
}

extern "C" int fast_dat_get_nodes(const fast_dat *d, double *coords, uint8_t *fixed, int64_t *solver_rank,
                                  double *nodal_f) {
  if (!d || !d->err.empty()) return FAST_GPU_EINVAL;
  const size_t n = (size_t)d->info.num_nodes;
  if (coords) memcpy(coords, d->coords.data(), 3 * n * sizeof(double));
  if (fixed) memcpy(fixed, d->fixed.data(), 3 * n);
  if (solver_rank && !d->solver_rank.empty()) memcpy(solver_rank, d->solver_rank.data(), n * sizeof(int64_t));
  if (nodal_f) {
    if (d->nodal_f.empty()) memset(nodal_f, 0, 3 * n * sizeof(double));
    else memcpy(nodal_f, d->nodal_f.data(), 3 * n * sizeof(double));
  }
  return FAST_GPU_OK;
}

extern "C" int fast_dat_get_elements(const fast_dat *d, int32_t *conn, double *E, double *nu, double *rho) {
  if (!d || !d->err.empty()) return FAST_GPU_EINVAL;
  const size_t ne = (size_t)d->info.num_elems;
  if (conn) memcpy(conn, d->conn.data(), d->conn.size() * sizeof(int32_t));
  if (E) memcpy(E, d->E.data(), ne * sizeof(double));
  if (nu) memcpy(nu, d->nu.data(), ne * sizeof(double));
  if (rho) {
    if (d->rho.empty()) memset(rho, 0, ne * sizeof(double));
    else memcpy(rho, d->rho.data(), ne * sizeof(double));
  }
  return FAST_GPU_OK;
}

extern "C" int fast_dat_get_faces(const fast_dat *d, int32_t *elem, int32_t *corners, int32_t *face_nodes,
                                  int32_t *local, double *q) {
  if (!d || !d->err.empty()) return FAST_GPU_EINVAL;
  const size_t nf = d->face_elem.size();
  if (elem) memcpy(elem, d->face_elem.data(), nf * sizeof(int32_t));
  if (corners) memcpy(corners, d->face_corner.data(), 3 * nf * sizeof(int32_t));
  if (face_nodes) memcpy(face_nodes, d->face_nodes.data(), d->face_nodes.size() * sizeof(int32_t));
  if (local) memcpy(local, d->face_local.data(), nf * sizeof(int32_t));
  if (q) memcpy(q, d->face_q.data(), 3 * nf * sizeof(double));
  return FAST_GPU_OK;
}

extern "C" int fast_dat_get_patch(const fast_dat *d, double *knots, int32_t *span, double *weights, int32_t *cps) {
  if (!d || !d->err.empty() || d->info.elem_type != FAST_ELEM_BSP_SOLID) return FAST_GPU_EINVAL;
  if (knots)
    for (int k = 0; k < 3; k++) {
      memcpy(knots, d->knots[k].data(), d->knots[k].size() * sizeof(double));
      knots += d->knots[k].size();
    }
  if (span) memcpy(span, d->span.data(), d->span.size() * sizeof(int32_t));
  if (weights) {
    if (d->weights.empty())
      for (int64_t i = 0; i < d->info.num_nodes; i++) weights[i] = 1.0;
    else memcpy(weights, d->weights.data(), d->weights.size() * sizeof(double));
  }
  if (cps) memcpy(cps, d->cps.data(), d->cps.size() * sizeof(int32_t));
  return FAST_GPU_OK;
}

extern "C" int fast_dat_bucket(const fast_dat *d, fast_gpu_bucket *b) {
  if (!d || !b || !d->err.empty()) return FAST_GPU_EINVAL;
  memset(b, 0, sizeof *b);
  b->elem_type = d->info.elem_type;
  for (int k = 0; k < 3; k++) b->ngp[k] = d->info.ngp[k];
  b->num_elems = d->info.num_elems;
  b->conn = d->conn.data();
  b->E = d->E.data();
  b->nu = d->nu.data();
  b->rho = d->rho.empty() ? nullptr : d->rho.data();
  b->formulation = d->info.formulation;
  b->patch = d->info.elem_type == FAST_ELEM_BSP_SOLID ? &d->patch : nullptr;
  return FAST_GPU_OK;
}

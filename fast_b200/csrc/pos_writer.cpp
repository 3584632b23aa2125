// pos_writer.cpp - FAST's .pos result file for solid decks, formatted on all
// host cores (include/fast_pos.h).
//
// The reference streams every number through iostream (scientific, showpos,
// setprecision(OutPrec)) one node or element at a time.  Here each block is
// cut into row ranges, every thread formats its rows into its own buffer with
// std::to_chars (the same correctly rounded digits as the printf conversion
// iostream uses), and the buffers are written in order.  The step list that
// the reference writes at the end over a blank area reserved after
// "%RESULT.CASE" (cControl::End, ctrl/ctrl.cpp:597-622) is written the same
// way: seek back, overwrite.
#include <omp.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fast_pos.h"

struct fast_pos {
  std::string err;
  FILE *fp = nullptr;
  int prec = 5, max_steps = 1, avg = 0, threads = 1;
  int steps = 0;
  long case_pos = 0;
  bool left = false;                // the stream's adjustfield after the last block
  std::vector<int64_t> reac_nodes;  // staged for the next step
  std::vector<double> reac_vals;
};

namespace {

const char *kLabels = "'STRESS_XX'  'STRESS_YY'  'STRESS_ZZ'  'STRESS_XY'  'STRESS_XZ'  'STRESS_YZ'  \n";

// iostream's scientific output of v at precision p ('+' first when showpos)
// at o; returns the end.  At most p + 9 characters.
inline char *put_num(char *o, double v, int p, bool plus) {
  if (plus && !std::signbit(v)) *o++ = '+';
  return std::to_chars(o, o + p + 16, v, std::chars_format::scientific, p).ptr;
}

inline char *put_int(char *o, int64_t v) { return std::to_chars(o, o + 24, v).ptr; }

// left << setw(5) << label << " "
inline char *put_label(char *o, int64_t label) {
  char *b = o;
  o = put_int(o, label);
  while (o - b < 5) *o++ = ' ';
  *o++ = ' ';
  return o;
}

bool put(fast_pos &p, const char *s, size_t n) {
  if (n && fwrite(s, 1, n, p.fp) != n) {
    p.err = "write error";
    return false;
  }
  return true;
}
bool put(fast_pos &p, const std::string &s) { return put(p, s.data(), s.size()); }

// rows [0, n) formatted by fmt(row, char *) -> end in parallel, each row at
// most row_max characters, written in order
template <class F>
bool rows(fast_pos &p, int64_t n, size_t row_max, F fmt) {
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(p.threads, n / 1024));
  // rounds of at most 64 MB of text per thread keep the buffers bounded
  const int64_t per_round = std::max<int64_t>(1, (int64_t)(((size_t)64 << 20) / row_max)) * nt;
  std::vector<std::vector<char>> buf(nt);
  std::vector<size_t> used(nt);
  for (int64_t r0 = 0; r0 < n; r0 += per_round) {
    const int64_t r1 = std::min(n, r0 + per_round), m = r1 - r0;
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; t++) {
      const int64_t a = r0 + m * t / nt, b = r0 + m * (t + 1) / nt;
      std::vector<char> &v = buf[t];
      if (v.size() < (size_t)(b - a) * row_max) v.resize((size_t)(b - a) * row_max);
      char *o = v.data();
      for (int64_t i = a; i < b; i++) o = fmt(i, o);
      used[t] = (size_t)(o - v.data());
    }
    for (int t = 0; t < nt; t++)
      if (!put(p, buf[t].data(), used[t])) return false;
  }
  return true;
}

}  // namespace

extern "C" int fast_pos_open(const char *pos_path, const char *dat_path, const fast_pos_opts *o, fast_pos **out) {
  if (!out) return FAST_GPU_EINVAL;
  *out = new (std::nothrow) fast_pos;
  if (!*out) return FAST_GPU_ENOMEM;
  fast_pos &p = **out;
  if (!pos_path || !dat_path || !o || o->precision < 0 || o->precision > 40 || o->max_steps < 0) {
    p.err = "bad arguments";
    return FAST_GPU_EINVAL;
  }
  p.prec = o->precision;
  p.max_steps = o->max_steps;
  p.avg = o->print_average;
  p.threads = o->threads > 0 ? o->threads : omp_get_num_procs();
  FILE *in = fopen(dat_path, "rb");
  if (!in) {
    p.err = std::string("cannot open ") + dat_path;
    return FAST_GPU_EINVAL;
  }
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = fread(buf, 1, sizeof buf, in)) > 0) text.append(buf, got);
  fclose(in);
  p.fp = fopen(pos_path, "wb");
  if (!p.fp) {
    p.err = std::string("cannot create ") + pos_path;
    return FAST_GPU_EINVAL;
  }
  // main/main.cpp:113-114, then InpCopyData (main/input.cpp:405-420): the
  // first line skipped, then every line up to one that is exactly "%END"; a
  // last line without its newline is still copied, and reading past a final
  // newline yields one more empty line
  std::string s = "%HEADER\n";
  s += o->header_line ? o->header_line : "Output file generated by the B200 solid path of libfastgpu.";
  s += "\n";
  size_t pos = text.find('\n');
  if (pos != std::string::npos) {
    pos++;
    while (true) {
      const size_t nl = text.find('\n', pos);
      const std::string line = text.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos);
      if (line == "%END") break;
      s += line;
      s += "\n";
      if (nl == std::string::npos) break;
      pos = nl + 1;
    }
  }
  return put(p, s) ? FAST_GPU_OK : FAST_GPU_EINVAL;
}

extern "C" int fast_pos_step(fast_pos *pp, double factor, int64_t nnode, const double *displ, int64_t ne,
                             int32_t points, const double *gs, int32_t nn, const double *en, const double *avg) {
  if (!pp || !pp->fp) return FAST_GPU_EINVAL;
  fast_pos &p = *pp;
  if (nnode <= 0 || !displ || (gs && (ne <= 0 || points <= 0)) || (en && (ne <= 0 || nn <= 0)) ||
      (p.avg && !avg)) {
    p.err = "bad arguments";
    return FAST_GPU_EINVAL;
  }
  const int prec = p.prec;
  const size_t num = (size_t)prec + 11;  // one number with its separators
  std::string s;
  if (++p.steps == 1) {  // cControl::PrintResult, first printed step
    s += "%RESULT\n1\n1  'result1'\n\n%RESULT.CASE\n";
    if (!put(p, s)) return FAST_GPU_EINVAL;
    s.clear();
    p.case_pos = ftell(p.fp);
    for (int i = 0; i <= 1.1 * p.max_steps; i++) s += "             \n";
  }
  char fb[64];
  s += "%RESULT.CASE.STEP\n" + std::to_string(p.steps) + "\n\n%RESULT.CASE.STEP.FACTOR\n";
  s.append(fb, put_num(fb, factor, prec, false));
  s += "\n\n%RESULT.CASE.STEP.NODAL.DISPLACEMENT\n" + std::to_string(nnode) + "  'displacement'\n";
  if (!put(p, s)) return FAST_GPU_EINVAL;
  bool ok = rows(p, nnode, 6 * num + 32, [&](int64_t i, char *o) {
    o = put_label(o, i + 1);
    for (int j = 0; j < 6; j++) {
      o = put_num(o, j < 3 ? displ[3 * i + j] : 0.0, prec, true);
      *o++ = ' ';
      *o++ = ' ';
    }
    *o++ = '\n';
    return o;
  });
  if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
  p.left = true;
  if (!p.reac_nodes.empty()) {
    // left << setw(4) << label << " ", then scientific << right <<
    // setprecision(5) << setw(13) << value << " " for the six components
    s = "%RESULT.CASE.STEP.NODAL.REACTIONS\n" + std::to_string(p.reac_nodes.size()) + "\n";
    if (!put(p, s)) return FAST_GPU_EINVAL;
    ok = rows(p, (int64_t)p.reac_nodes.size(), 6 * 24 + 32, [&](int64_t r, char *o) {
      char *b = o;
      o = put_int(o, p.reac_nodes[r] + 1);
      while (o - b < 4) *o++ = ' ';
      *o++ = ' ';
      for (int j = 0; j < 6; j++) {
        char nb[40];
        const int len = (int)(put_num(nb, j < 3 ? p.reac_vals[3 * r + j] : 0.0, 5, false) - nb);
        for (int k = len; k < 13; k++) *o++ = ' ';
        memcpy(o, nb, len);
        o += len;
        *o++ = ' ';
      }
      *o++ = '\n';
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
    p.left = false;
    p.reac_nodes.clear();
    p.reac_vals.clear();
  }
  if (gs) {
    s = std::string("%RESULT.CASE.STEP.ELEMENT.GAUSS.SCALAR\n6\n") + kLabels +
        "\n%RESULT.CASE.STEP.ELEMENT.GAUSS.SCALAR.DATA\n" + std::to_string(ne) + "\n";
    if (!put(p, s)) return FAST_GPU_EINVAL;
    ok = rows(p, ne, (size_t)points * (6 * num + 1) + 64, [&](int64_t k, char *o) {
      o = put_int(o, k + 1);
      *o++ = '\n';
      o = put_int(o, points);
      *o++ = '\n';
      const double *v = gs + (size_t)k * points * 6;
      for (int g = 0; g < points; g++) {
        for (int c = 0; c < 6; c++) {
          o = put_num(o, v[6 * g + c], prec, true);
          *o++ = ' ';
        }
        *o++ = '\n';
      }
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
  }
  if (en) {
    s = std::string("%RESULT.CASE.STEP.ELEMENT.NODAL.SCALAR\n6\n") + kLabels +
        "\n%RESULT.CASE.STEP.ELEMENT.NODAL.SCALAR.DATA\n" + std::to_string(ne) + "\n";
    if (!put(p, s)) return FAST_GPU_EINVAL;
    ok = rows(p, ne, (size_t)nn * (6 * num + 1) + 32, [&](int64_t k, char *o) {
      o = put_int(o, k + 1);
      *o++ = '\n';
      const double *v = en + (size_t)k * nn * 6;
      for (int a = 0; a < nn; a++) {
        for (int c = 0; c < 6; c++) {
          o = put_num(o, v[6 * a + c], prec, true);
          *o++ = ' ';
        }
        *o++ = '\n';
      }
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
  }
  if (p.avg) {
    s = std::string("%RESULT.CASE.STEP.NODAL.SCALAR\n6\n") + kLabels + "\n%RESULT.CASE.STEP.NODAL.SCALAR.DATA\n" +
        std::to_string(nnode) + "\n";
    if (!put(p, s)) return FAST_GPU_EINVAL;
    ok = rows(p, nnode, 6 * num + 32, [&](int64_t i, char *o) {
      o = put_label(o, i + 1);
      for (int c = 0; c < 6; c++) {
        o = put_num(o, avg[6 * i + c], prec, true);
        *o++ = ' ';
        *o++ = ' ';
      }
      *o++ = '\n';
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
    p.left = true;
  }
  return FAST_GPU_OK;
}

extern "C" int fast_pos_reactions(fast_pos *pp, int64_t count, const int64_t *nodes, const double *R) {
  if (!pp || !pp->fp || count < 0 || (count > 0 && (!nodes || !R))) return FAST_GPU_EINVAL;
  pp->reac_nodes.assign(nodes, nodes + count);
  pp->reac_vals.assign(R, R + 3 * count);
  return FAST_GPU_OK;
}

extern "C" int fast_pos_velacc(fast_pos *pp, int64_t nnode, const double *v, const double *a) {
  if (!pp || !pp->fp) return FAST_GPU_EINVAL;
  fast_pos &p = *pp;
  if (nnode <= 0 || !v || !a) {
    p.err = "bad arguments";
    return FAST_GPU_EINVAL;
  }
  const int prec = p.prec;
  const size_t num = (size_t)prec + 11;
  for (int k = 0; k < 2; k++) {
    const double *x = k == 0 ? v : a;
    const std::string s = std::string(k == 0 ? "%RESULT.CASE.STEP.VELOCITY\n" : "%RESULT.CASE.STEP.ACCELERATION\n") +
                          std::to_string(nnode) + (k == 0 ? "  'velocity'\n" : "  'acceleration'\n");
    if (!put(p, s)) return FAST_GPU_EINVAL;
    const bool ok = rows(p, nnode, 6 * num + 32, [&](int64_t i, char *o) {
      o = put_label(o, i + 1);
      for (int j = 0; j < 6; j++) {
        o = put_num(o, j < 3 ? x[3 * i + j] : 0.0, prec, true);
        *o++ = ' ';
        *o++ = ' ';
      }
      *o++ = '\n';
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
  }
  p.left = true;
  return FAST_GPU_OK;
}

extern "C" int fast_pos_modes(fast_pos *pp, int32_t kind, int32_t nmodes, const double *values, int64_t nnode,
                              const double *modes) {
  if (!pp || !pp->fp) return FAST_GPU_EINVAL;
  fast_pos &p = *pp;
  if ((kind != FAST_POS_VIBRATION && kind != FAST_POS_BUCKLING) || nmodes < 0 || nnode <= 0 ||
      (nmodes > 0 && (!values || !modes))) {
    p.err = "bad arguments";
    return FAST_GPU_EINVAL;
  }
  const bool vib = kind == FAST_POS_VIBRATION;
  const int prec = p.prec;
  const size_t num = (size_t)prec + 11;
  std::string s = std::string("\n%RESULT.CASE.STEP.") + (vib ? "VIBRATION" : "BUCKLING") + ".MODES\n" +
                  std::to_string(nmodes) + "\n";
  if (!put(p, s)) return FAST_GPU_EINVAL;
  for (int m = 0; m < nmodes; m++) {
    // mode + 1 << "  " << showpos << right << scientific << setw(14) << value
    char fb[64];
    const int len = (int)(put_num(fb, values[m], prec, true) - fb);
    s = std::string("\n%RESULT.CASE.STEP.") + (vib ? "NATURAL.FREQUENCY" : "BUCKLING.FACTOR") + "\n" +
        std::to_string(m + 1) + "  ";
    for (int k = len; k < 14; k++) s += ' ';
    s.append(fb, len);
    s += "\n\n%RESULT.CASE.STEP.NODAL.EIGENVECTOR\n" + std::to_string(nnode) +
         (vib ? "  'Vibration mode'\n" : "  'Buckling mode'\n");
    if (!put(p, s)) return FAST_GPU_EINVAL;
    const double *v = modes + (size_t)m * nnode * 3;
    // left << setw(4) << label << " ", then " " before each of the six values
    const bool ok = rows(p, nnode, 6 * num + 32, [&](int64_t i, char *o) {
      char *b = o;
      o = put_int(o, i + 1);
      while (o - b < 4) *o++ = ' ';
      *o++ = ' ';
      for (int j = 0; j < 6; j++) {
        *o++ = ' ';
        o = put_num(o, j < 3 ? v[3 * i + j] : 0.0, prec, true);
      }
      *o++ = '\n';
      return o;
    });
    if (!ok || !put(p, "\n", 1)) return FAST_GPU_EINVAL;
    p.left = true;
  }
  return FAST_GPU_OK;
}

extern "C" int fast_pos_finish(fast_pos *pp) {
  if (!pp || !pp->fp) return FAST_GPU_EINVAL;
  fast_pos &p = *pp;
  // cControl::End: "%END", then the step list over the reserved area;
  // setw(2) pads under the adjustfield the last block left behind ("1 "
  // after displacement rows, " 1" after support reactions)
  bool ok = put(p, "\n%END\n", 6);
  if (ok && p.case_pos != 0 && fseek(p.fp, p.case_pos, SEEK_SET) != 0) {
    p.err = "seek error";
    ok = false;
  }
  if (ok) {
    std::string s = "1   " + std::to_string(p.steps) + "\n";
    for (int i = 1; i <= p.steps; i++) {
      std::string n = std::to_string(i);
      if (n.size() < 2) n = p.left ? n + " " : " " + n;  // setw(2) under the stream's adjustfield
      s += n + "  'step" + std::to_string(i) + "'\n";
    }
    ok = put(p, s);
  }
  if (fclose(p.fp) != 0 && ok) {
    p.err = "close error";
    ok = false;
  }
  p.fp = nullptr;
  return ok ? FAST_GPU_OK : FAST_GPU_EINVAL;
}

extern "C" const char *fast_pos_error(const fast_pos *p) { return p ? p->err.c_str() : "no file"; }

extern "C" void fast_pos_free(fast_pos *p) {
  if (!p) return;
  if (p->fp) fclose(p->fp);
  delete p;
}

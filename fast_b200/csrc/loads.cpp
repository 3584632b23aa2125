// loads.cpp - external load vector from uniform face tractions, on the host.
//
// Restates cControl::ExtLoadVector (ctrl/ctrl.cpp:668-715) for
// %LOAD.CASE.AREA.UNIFORM loads: cElemLoad::ExtForce (load/load.cpp:618-706)
// integrates N^T q over the loaded face with the element's Gauss order
// (cElmParam::GetIntOrd, elc/elmparam.cpp:349-361) on the Q4/Q8 surface shape
// (shp/shpplane.cpp:353-488), |J| = |dx/dr x dx/ds| (cShapeSurf::DrvShpXYZ,
// shp/shpsurf.cpp:58-117); with Local = 1 the traction is rotated from the
// face's local frame (cShapeSurf::LocalSys, shp/shpsurf.cpp:121-160).  The
// load vector is an input of the solve, computed once per load case, so it
// stays on the host.
#include <cmath>
#include <cstring>

#include "internal.h"

namespace {

void q4(double r, double s, double *N, double *dN) {
  const int rn[4] = {-1, 1, 1, -1}, sn[4] = {-1, -1, 1, 1};
  for (int a = 0; a < 4; a++) {
    N[a] = 0.25 * (1 + rn[a] * r) * (1 + sn[a] * s);
    dN[2 * a] = 0.25 * rn[a] * (1 + sn[a] * s);
    dN[2 * a + 1] = 0.25 * sn[a] * (1 + rn[a] * r);
  }
}

void q8(double r, double s, double *N, double *dN) {
  // serendipity quadrilateral, nodes: corners at 0,2,4,6, mid-sides at 1,3,5,7
  const int rn[8] = {-1, 0, 1, 1, 1, 0, -1, -1}, sn[8] = {-1, -1, -1, 0, 1, 1, 1, 0};
  for (int a = 0; a < 8; a++) {
    const double ri = rn[a], si = sn[a];
    if (ri != 0 && si != 0) {
      const double fr = 1 + ri * r, fs = 1 + si * s, g = ri * r + si * s - 1;
      N[a] = 0.25 * fr * fs * g;
      dN[2 * a] = 0.25 * ri * fs * (g + fr);
      dN[2 * a + 1] = 0.25 * si * fr * (g + fs);
    } else if (ri == 0) {
      const double fs = 1 + si * s;
      N[a] = 0.5 * (1 - r * r) * fs;
      dN[2 * a] = -r * fs;
      dN[2 * a + 1] = 0.5 * (1 - r * r) * si;
    } else {
      const double fr = 1 + ri * r;
      N[a] = 0.5 * fr * (1 - s * s);
      dN[2 * a] = 0.5 * ri * (1 - s * s);
      dN[2 * a + 1] = -s * fr;
    }
  }
}

}  // namespace

extern "C" int fast_gpu_face_load_vector(int64_t num_nodes, const double *coords, const int32_t *node_eq,
                                         int32_t num_eq, int32_t num_faces, int32_t nodes_per_face,
                                         const int32_t *face_nodes, const double *q, const int32_t *local,
                                         int32_t ngp1d, double *f) {
  if (!coords || !node_eq || !f || num_eq < 0 || (num_faces > 0 && (!face_nodes || !q))) return FAST_GPU_EINVAL;
  if (nodes_per_face != 4 && nodes_per_face != 8) return FAST_GPU_ENOTSUP;
  double gr[6], gw[6];
  if (!fastgpu::gauss_rule(ngp1d, gr, gw)) return FAST_GPU_EINVAL;
  std::memset(f, 0, sizeof(double) * num_eq);
  const int nf = nodes_per_face;
  double N[8], dN[16], X[24], fe[24];
  for (int32_t k = 0; k < num_faces; k++) {
    for (int a = 0; a < nf; a++) {
      const int32_t n = face_nodes[(int64_t)k * nf + a];
      if (n < 0 || n >= num_nodes) return FAST_GPU_EINVAL;
      for (int d = 0; d < 3; d++) X[3 * a + d] = coords[3 * (int64_t)n + d];
    }
    std::memset(fe, 0, sizeof(fe));
    const double *qk = q + 3 * (int64_t)k;
    for (int i = 0; i < ngp1d; i++)
      for (int j = 0; j < ngp1d; j++) {
        const double r = gr[j], s = gr[i], wgt = gw[j] * gw[i];
        if (nf == 4) q4(r, s, N, dN); else q8(r, s, N, dN);
        double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
        for (int a = 0; a < nf; a++)
          for (int d = 0; d < 3; d++) {
            tr[d] += dN[2 * a] * X[3 * a + d];
            ts[d] += dN[2 * a + 1] * X[3 * a + d];
          }
        const double nv[3] = {tr[1] * ts[2] - tr[2] * ts[1], tr[2] * ts[0] - tr[0] * ts[2], tr[0] * ts[1] - tr[1] * ts[0]};
        const double detJ = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
        double val[3] = {qk[0], qk[1], qk[2]};
        if (local && local[k]) {
          const double lu = std::sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
          const double lv = std::sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
          double u[3] = {tr[0] / lu, tr[1] / lu, tr[2] / lu}, v[3] = {ts[0] / lv, ts[1] / lv, ts[2] / lv};
          const double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
          const double v2[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
          for (int d = 0; d < 3; d++) val[d] = u[d] * qk[0] + v2[d] * qk[1] + w[d] * qk[2];
        }
        const double coeff = wgt * detJ;
        for (int a = 0; a < nf; a++)
          for (int d = 0; d < 3; d++) fe[3 * a + d] += N[a] * (coeff * val[d]);
      }
    for (int a = 0; a < nf; a++) {
      const int32_t n = face_nodes[(int64_t)k * nf + a];
      for (int d = 0; d < 3; d++) {
        const int32_t e = node_eq[3 * (int64_t)n + d];
        if (e > 0 && e <= num_eq) f[e - 1] += fe[3 * a + d];
      }
    }
  }
  return FAST_GPU_OK;
}

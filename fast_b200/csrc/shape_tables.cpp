// shape_tables.cpp - Gauss rules and shape-function tables at the Gauss
// points, computed once on the host and uploaded per bucket.
//
// Gauss abscissae/weights: FAST tabulates them to 15 significant digits
// (elc/intpoint.cpp:742-800) and FP64 parity with it depends on using the
// same numbers, so the table is reproduced as data.  Points are ordered r
// fastest, then s, then t (cIntPoint::CreateBrickPoints, elc/intpoint.cpp:579-618).
//
// Shapes: trilinear hex8 (cShapeBrick8, shp/shpsolid.cpp:188-238) and the
// 20-node serendipity hex20 (cShapeBrick20, shp/shpsolid.cpp:301-433), both in
// FAST's local node order, written here from the standard closed forms
//   corner  N = 1/8 (1+r ri)(1+s si)(1+t ti)(r ri + s si + t ti - 2)
//   edge    N = 1/4 (1-r^2)(1+s si)(1+t ti)   (and permutations).
#include <cmath>
#include <vector>

#include "internal.h"

namespace fastgpu {

namespace {

const double kGaussR[6][6] = {
    {0.000000000000000},
    {-0.577350269189626, 0.577350269189626},
    {-0.774596669241483, 0.000000000000000, 0.774596669241483},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
    {-0.906179845938664, -0.538469310105683, 0.000000000000000, 0.538469310105683, 0.906179845938664},
    {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466264,
     0.932469514203152}};
const double kGaussW[6][6] = {
    {2.000000000000000},
    {1.000000000000000, 1.000000000000000},
    {0.555555555555556, 0.888888888888889, 0.555555555555556},
    {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454},
    {0.236926885056189, 0.478628670499367, 0.568888888888889, 0.478628670499367, 0.236926885056189},
    {0.171324492379170, 0.360761573048139, 0.467913934572691, 0.467913934572691, 0.360761573048139,
     0.171324492379170}};

// natural coordinates of the local nodes, FAST order
const int kHex8Nat[8][3] = {{-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
                            {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}};
const int kHex20Nat[20][3] = {{-1, -1, 1}, {0, -1, 1}, {1, -1, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}, {-1, 1, 1},
                              {-1, 0, 1}, {-1, -1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, 1, 0}, {-1, -1, -1},
                              {0, -1, -1}, {1, -1, -1}, {1, 0, -1}, {1, 1, -1}, {0, 1, -1}, {-1, 1, -1},
                              {-1, 0, -1}};

void hex8(double r, double s, double t, double *N, double *dN) {
  for (int a = 0; a < 8; a++) {
    const double ri = kHex8Nat[a][0], si = kHex8Nat[a][1], ti = kHex8Nat[a][2];
    const double fr = 1.0 + ri * r, fs = 1.0 + si * s, ft = 1.0 + ti * t;
    N[a] = 0.125 * fr * fs * ft;
    dN[3 * a] = 0.125 * ri * fs * ft;
    dN[3 * a + 1] = 0.125 * si * fr * ft;
    dN[3 * a + 2] = 0.125 * ti * fr * fs;
  }
}

void hex20(double r, double s, double t, double *N, double *dN) {
  for (int a = 0; a < 20; a++) {
    const double ri = kHex20Nat[a][0], si = kHex20Nat[a][1], ti = kHex20Nat[a][2];
    double *d = dN + 3 * a;
    if (ri != 0 && si != 0 && ti != 0) {
      const double fr = 1 + ri * r, fs = 1 + si * s, ft = 1 + ti * t;
      const double g = ri * r + si * s + ti * t - 2.0;
      N[a] = 0.125 * fr * fs * ft * g;
      d[0] = 0.125 * ri * fs * ft * (g + fr);
      d[1] = 0.125 * si * fr * ft * (g + fs);
      d[2] = 0.125 * ti * fr * fs * (g + ft);
    } else if (ri == 0) {
      const double fs = 1 + si * s, ft = 1 + ti * t, q = 1 - r * r;
      N[a] = 0.25 * q * fs * ft;
      d[0] = -0.5 * r * fs * ft;
      d[1] = 0.25 * q * si * ft;
      d[2] = 0.25 * q * fs * ti;
    } else if (si == 0) {
      const double fr = 1 + ri * r, ft = 1 + ti * t, q = 1 - s * s;
      N[a] = 0.25 * fr * q * ft;
      d[0] = 0.25 * ri * q * ft;
      d[1] = -0.5 * s * fr * ft;
      d[2] = 0.25 * fr * q * ti;
    } else {
      const double fr = 1 + ri * r, fs = 1 + si * s, q = 1 - t * t;
      N[a] = 0.25 * fr * fs * q;
      d[0] = 0.25 * ri * fs * q;
      d[1] = 0.25 * fr * si * q;
      d[2] = -0.5 * t * fr * fs;
    }
  }
}

}  // namespace

int nodes_of(int type) {
  switch (type) {
    case FAST_ELEM_HEX8: return 8;
    case FAST_ELEM_HEX20: return 20;
    default: return 0;
  }
}

bool gauss_rule(int n, double *r, double *w) {
  if (n < 1 || n > 6) return false;
  for (int i = 0; i < n; i++) {
    r[i] = kGaussR[n - 1][i];
    w[i] = kGaussW[n - 1][i];
  }
  return true;
}

void gauss_point_tables(int type, const int ngp[3], std::vector<double> &N, std::vector<double> &dN,
                        std::vector<double> &w) {
  const int nn = nodes_of(type);
  const int ng = ngp[0] * ngp[1] * ngp[2];
  N.assign((size_t)ng * nn, 0.0);
  dN.assign((size_t)ng * nn * 3, 0.0);
  w.assign(ng, 0.0);
  int k = 0;
  for (int i = 0; i < ngp[2]; i++)
    for (int j = 0; j < ngp[1]; j++)
      for (int l = 0; l < ngp[0]; l++, k++) {
        const double r = kGaussR[ngp[0] - 1][l], s = kGaussR[ngp[1] - 1][j], t = kGaussR[ngp[2] - 1][i];
        w[k] = kGaussW[ngp[0] - 1][l] * kGaussW[ngp[1] - 1][j] * kGaussW[ngp[2] - 1][i];
        if (type == FAST_ELEM_HEX8)
          hex8(r, s, t, &N[(size_t)k * nn], &dN[(size_t)k * nn * 3]);
        else
          hex20(r, s, t, &N[(size_t)k * nn], &dN[(size_t)k * nn * 3]);
      }
}

}  // namespace fastgpu

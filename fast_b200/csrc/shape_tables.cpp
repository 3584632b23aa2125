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
#include <algorithm>
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

int bucket_nodes(const fast_gpu_bucket &bk) {
  if (bk.elem_type != FAST_ELEM_BSP_SOLID) return nodes_of(bk.elem_type);
  if (!bk.patch) return 0;
  int nn = 1;
  for (int d = 0; d < 3; d++) {
    const int p = bk.patch->degree[d];
    if (p < 2 || p > 5) return 0;
    nn *= p + 1;
  }
  return nn;
}

namespace {

// The p+1 B-splines of degree p that are non-zero on knot span [U[k], U[k+1]),
// evaluated at u by the Cox-de Boor recurrence, built up one degree at a time:
//   N_{i,q}(u) = (u - U_i)/(U_{i+q} - U_i) N_{i,q-1} + (U_{i+q+1} - u)/(U_{i+q+1} - U_{i+1}) N_{i+1,q-1}
// (de Boor 1972; 0/0 := 0).  out[i] = N_{k-p+i,p}(u).  The span is given, so u
// may sit on its right end and the value is that of the span's polynomial piece.
void span_basis(int p, const double *U, int k, double u, double *out) {
  double N[8] = {0.0};
  N[p] = 1.0;  // degree 0: only N_{k,0} = 1 on the span
  for (int q = 1; q <= p; q++) {
    // degree q functions N_{k-q..k, q} stored at N[p-q .. p]
    for (int t = p - q; t <= p; t++) {
      const int i = k - p + t;  // global index of the function at slot t
      double v = 0.0;
      const double dl = U[i + q] - U[i];
      if (t >= p - q + 1 && dl > 0.0) v += (u - U[i]) / dl * N[t];
      const double dr = U[i + q + 1] - U[i + 1];
      if (t + 1 <= p && dr > 0.0) v += (U[i + q + 1] - u) / dr * N[t + 1];
      N[t] = v;
    }
  }
  for (int i = 0; i <= p; i++) out[i] = N[i];
}

double binom(int n, int k) {
  double r = 1.0;
  for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
  return r;
}

// Bernstein polynomials of degree p on [0, 1] and their derivatives
void bernstein(int p, double x, double *B, double *dB) {
  for (int j = 0; j <= p; j++) B[j] = binom(p, j) * std::pow(x, j) * std::pow(1.0 - x, p - j);
  if (!dB) return;
  double lo[8];
  for (int j = 0; j < p; j++) lo[j] = binom(p - 1, j) * std::pow(x, j) * std::pow(1.0 - x, p - 1 - j);
  for (int j = 0; j <= p; j++) dB[j] = p * ((j > 0 ? lo[j - 1] : 0.0) - (j < p ? lo[j] : 0.0));
}

// Solve A x = b (n <= 8) by Gaussian elimination with partial pivoting
bool small_solve(int n, double A[8][8], double *b) {
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
    if (A[piv][c] == 0.0) return false;
    if (piv != c) {
      for (int k = 0; k < n; k++) std::swap(A[c][k], A[piv][k]);
      std::swap(b[c], b[piv]);
    }
    for (int r = c + 1; r < n; r++) {
      const double f = A[r][c] / A[c][c];
      for (int k = c; k < n; k++) A[r][k] -= f * A[c][k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; c--) {
    double v = b[c];
    for (int k = c + 1; k < n; k++) v -= A[c][k] * b[k];
    b[c] = v / A[c][c];
  }
  return true;
}

}  // namespace

// Bezier extraction of one knot span: the span's B-splines as combinations of
// the degree-p Bernstein polynomials in xi = (u - U_k)/(U_{k+1} - U_k),
//   N_{k-p+i}(u) = sum_j C[i][j] B_j(xi)
// (the operator cKnotVector::CompBezExtMat builds by knot insertion,
// geom/knotvec.cpp:415-493).  Here it is found by collocation instead: both
// sides are degree-p polynomials on the span, so matching them at the p+1
// points xi_c = c/p determines C.  Then the Gauss-point tables follow the
// reference's evaluation (cShapeBsp::EvalBspBas/EvalBspBasDerv,
// shp/shpbsp.cpp:254-300): xi = (t+1)/2, and dN/dt takes the Bernstein
// derivative halved.
bool bspline_gauss_tables(int p, int nknots, const double *U, int ng, int &nspan, std::vector<double> &out) {
  nspan = 0;
  out.clear();
  if (p < 1 || p > 7 || ng < 1 || ng > 6 || !U || nknots < 2 * (p + 1)) return false;
  for (int i = 1; i < nknots; i++)
    if (!(U[i] >= U[i - 1])) return false;
  // non-zero spans as the reference counts them (knot gap above 1e-5,
  // cKnotVector::FindSpan(int), geom/knotvec.cpp:303-313)
  std::vector<int> left;
  for (int i = 1; i < nknots; i++)
    if (U[i] - U[i - 1] > 1e-5) left.push_back(i - 1);
  if (left.empty()) return false;
  for (int k : left)
    if (k < p || k > nknots - p - 2) return false;  // needs p functions on each side
  nspan = (int)left.size();
  double tr[6], tw[6];
  gauss_rule(ng, tr, tw);
  out.assign((size_t)nspan * ng * (p + 1) * 2, 0.0);
  for (int s = 0; s < nspan; s++) {
    const int k = left[s];
    const double u0 = U[k], h = U[k + 1] - U[k];
    // collocation: V[c][j] = B_j(xi_c), rhs columns N_i(u_c)
    double V[8][8], Nc[8][8];
    for (int c = 0; c <= p; c++) {
      const double xi = (double)c / p;
      bernstein(p, xi, V[c], nullptr);
      double nb[8];
      span_basis(p, U, k, u0 + xi * h, nb);
      for (int i = 0; i <= p; i++) Nc[i][c] = nb[i];
    }
    double C[8][8];
    for (int i = 0; i <= p; i++) {
      double A[8][8], x[8];
      for (int r = 0; r <= p; r++) {
        for (int cc = 0; cc <= p; cc++) A[r][cc] = V[r][cc];
        x[r] = Nc[i][r];
      }
      if (!small_solve(p + 1, A, x)) return false;
      for (int j = 0; j <= p; j++) C[i][j] = x[j];
    }
    for (int g = 0; g < ng; g++) {
      const double xi = 0.5 * (tr[g] + 1.0);
      double B[8], dB[8];
      bernstein(p, xi, B, dB);
      for (int j = 0; j <= p; j++) dB[j] /= 2.0;
      for (int i = 0; i <= p; i++) {
        double n = 0.0, d = 0.0;
        for (int j = 0; j <= p; j++) {
          n += C[i][j] * B[j];
          d += C[i][j] * dB[j];
        }
        double *o = &out[(((size_t)s * ng + g) * (p + 1) + i) * 2];
        o[0] = n;
        o[1] = d;
      }
    }
  }
  return true;
}

// Stress extrapolation to the nodes (cElmParam::CompTRMatrix,
// elc/elmparam.cpp:1444-1535): the linear field a0 + a1 r + a2 s + a3 t that
// fits the Gauss-point values in the least-squares sense, evaluated at the
// node: TR[a][g] = c_a^T A^-1 u_g with A = sum_g u_g u_g^T, u = (1, r, s, t),
// c_a the node's (1, r, s, t).  A is symmetric, so each row is one 4x4 solve
// A y = c_a followed by y . u_g.  A one-point first order gives the average.
bool extrapolation_matrix(int type, const int ngp[3], std::vector<double> &TR, const int *pd) {
  // B-spline solids: the control points' natural coordinates are the uniform
  // grid of (p+1) points per direction over [-1, 1], r fastest
  // (cShapeBspSolid::NodeNatCoord, shp/shpbsp.cpp:906-923)
  const bool bsp = type == FAST_ELEM_BSP_SOLID;
  if (bsp && (!pd || pd[0] < 1 || pd[1] < 1 || pd[2] < 1)) return false;
  const int nn = bsp ? (pd[0] + 1) * (pd[1] + 1) * (pd[2] + 1) : nodes_of(type);
  const int ng = ngp[0] * ngp[1] * ngp[2];
  if (nn <= 0 || ng <= 0) return false;
  TR.assign((size_t)nn * ng, 0.0);
  if (ngp[0] == 1) {
    for (double &v : TR) v = 1.0 / ng;
    return true;
  }
  std::vector<double> u((size_t)ng * 4);
  int k = 0;
  for (int i = 0; i < ngp[2]; i++)
    for (int j = 0; j < ngp[1]; j++)
      for (int l = 0; l < ngp[0]; l++, k++) {
        u[4 * k] = 1.0;
        u[4 * k + 1] = kGaussR[ngp[0] - 1][l];
        u[4 * k + 2] = kGaussR[ngp[1] - 1][j];
        u[4 * k + 3] = kGaussR[ngp[2] - 1][i];
      }
  double A0[4][4] = {};
  for (int g = 0; g < ng; g++)
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < 4; q++) A0[p][q] += u[4 * g + p] * u[4 * g + q];
  for (int a = 0; a < nn; a++) {
    double nat[3];
    if (bsp) {
      const int k = a % (pd[0] + 1), j = (a / (pd[0] + 1)) % (pd[1] + 1), i = a / ((pd[0] + 1) * (pd[1] + 1));
      nat[0] = -1.0 + (2.0 / pd[0]) * k;
      nat[1] = -1.0 + (2.0 / pd[1]) * j;
      nat[2] = -1.0 + (2.0 / pd[2]) * i;
    } else {
      const int *h = type == FAST_ELEM_HEX8 ? kHex8Nat[a] : kHex20Nat[a];
      for (int d = 0; d < 3; d++) nat[d] = (double)h[d];
    }
    double A[8][8] = {};
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < 4; q++) A[p][q] = A0[p][q];
    double y[8] = {1.0, nat[0], nat[1], nat[2]};
    if (!small_solve(4, A, y)) return false;
    for (int g = 0; g < ng; g++)
      TR[(size_t)a * ng + g] = y[0] * u[4 * g] + y[1] * u[4 * g + 1] + y[2] * u[4 * g + 2] + y[3] * u[4 * g + 3];
  }
  return true;
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

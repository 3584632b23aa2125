/* fem_oracle.c - CPU restatement of FAST's solid element, load and PCG
 * arithmetic.  TEST INFRASTRUCTURE ONLY: the tests, smoke() and the CPU
 * baseline of bench.py call it as the checker; the product never does.
 *
 * Each function follows the reference routine cited beside it, including
 * loop and summation order, so that FP64 results agree with the reference
 * to rounding.  Parity pinned against golden dumps of the reference program
 * (tests/golden, made by tests/golden/make_golden.py).
 */
#include "fem_oracle.h"

#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>

/* ---- Gauss data: the reference's 15-significant-digit table
 * (elc/intpoint.cpp:742-800), kept as numbers because parity depends on
 * the exact abscissae and weights. */
static const double GR[6][6] = {
  { 0.000000000000000 },
  {-0.577350269189626, 0.577350269189626},
  {-0.774596669241483, 0.000000000000000, 0.774596669241483},
  {-0.861136311594053,-0.339981043584856, 0.339981043584856, 0.861136311594053},
  {-0.906179845938664,-0.538469310105683, 0.000000000000000, 0.538469310105683, 0.906179845938664},
  {-0.932469514203152,-0.661209386466264,-0.238619186083197, 0.238619186083197, 0.661209386466264, 0.932469514203152}};
static const double GW[6][6] = {
  { 2.000000000000000 },
  { 1.000000000000000, 1.000000000000000},
  { 0.555555555555556, 0.888888888888889, 0.555555555555556},
  { 0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454},
  { 0.236926885056189, 0.478628670499367, 0.568888888888889, 0.478628670499367, 0.236926885056189},
  { 0.171324492379170, 0.360761573048139, 0.467913934572691, 0.467913934572691, 0.360761573048139, 0.171324492379170}};

int fo_gauss(int n, double *r, double *w)
{
  if (n < 1 || n > 6) return -1;
  for (int i = 0; i < n; i++) { r[i] = GR[n - 1][i]; w[i] = GW[n - 1][i]; }
  return 0;
}

/* ---- shapes: cShapeBrick8 (shp/shpsolid.cpp:188-238) */
void fo_shape_hex8(double r, double s, double t, double *N, double *dN)
{
  static const int sr[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  static const int ss[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  static const int st[8] = { 1, 1, 1, 1, -1, -1, -1, -1};
  for (int a = 0; a < 8; a++)
  {
    double fr = 1.0 + sr[a] * r, fs = 1.0 + ss[a] * s, ft = 1.0 + st[a] * t;
    if (N) N[a] = 0.125 * fr * fs * ft;
    dN[3 * a + 0] = 0.125 * sr[a] * fs * ft;
    dN[3 * a + 1] = 0.125 * ss[a] * fr * ft;
    dN[3 * a + 2] = 0.125 * st[a] * fr * fs;
  }
}

/* cShapeBrick20 (shp/shpsolid.cpp:301-433): serendipity 20-node brick, node
 * natural coordinates in FAST's order. */
static const int H20[20][3] = {
  {-1,-1, 1},{ 0,-1, 1},{ 1,-1, 1},{ 1, 0, 1},{ 1, 1, 1},{ 0, 1, 1},{-1, 1, 1},{-1, 0, 1},
  {-1,-1, 0},{ 1,-1, 0},{ 1, 1, 0},{-1, 1, 0},
  {-1,-1,-1},{ 0,-1,-1},{ 1,-1,-1},{ 1, 0,-1},{ 1, 1,-1},{ 0, 1,-1},{-1, 1,-1},{-1, 0,-1}};

void fo_shape_hex20(double r, double s, double t, double *N, double *dN)
{
  for (int a = 0; a < 20; a++)
  {
    double ri = H20[a][0], si = H20[a][1], ti = H20[a][2];
    double *d = dN + 3 * a;
    if (ri != 0 && si != 0 && ti != 0)
    {
      /* corner: 1/8 (1+r ri)(1+s si)(1+t ti)(r ri + s si + t ti - 2) */
      double fr = 1 + r * ri, fs = 1 + s * si, ft = 1 + t * ti, g = r * ri + s * si + t * ti - 2.0;
      if (N) N[a] = 0.125 * fr * fs * ft * g;
      d[0] = 0.125 * ri * fs * ft * (g + fr);
      d[1] = 0.125 * si * fr * ft * (g + fs);
      d[2] = 0.125 * ti * fr * fs * (g + ft);
    }
    else if (ri == 0)
    {
      double fs = 1 + s * si, ft = 1 + t * ti;
      if (N) N[a] = 0.25 * (1 - r * r) * fs * ft;
      d[0] = -0.5 * r * fs * ft; d[1] = 0.25 * (1 - r * r) * si * ft; d[2] = 0.25 * (1 - r * r) * fs * ti;
    }
    else if (si == 0)
    {
      double fr = 1 + r * ri, ft = 1 + t * ti;
      if (N) N[a] = 0.25 * fr * (1 - s * s) * ft;
      d[0] = 0.25 * ri * (1 - s * s) * ft; d[1] = -0.5 * s * fr * ft; d[2] = 0.25 * fr * (1 - s * s) * ti;
    }
    else
    {
      double fr = 1 + r * ri, fs = 1 + s * si;
      if (N) N[a] = 0.25 * fr * fs * (1 - t * t);
      d[0] = 0.25 * ri * fs * (1 - t * t); d[1] = 0.25 * fr * si * (1 - t * t); d[2] = -0.5 * t * fr * fs;
    }
  }
}

static void shape(int nn, double r, double s, double t, double *N, double *dN)
{
  if (nn == 8) fo_shape_hex8(r, s, t, N, dN); else fo_shape_hex20(r, s, t, N, dN);
}

/* cShapeSolid::DrvShpXYZ (shp/shpsolid.cpp:58-126) + cShape::ShpMatInv (shp/shape.cpp:360-393). */
static int drv_xyz(int nn, const double *dN, const double *X, double *detJ, double *dX)
{
  double J[3][3] = {{0}}, B[3][3];
  for (int i = 0; i < nn; i++)
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) J[p][q] += dN[3 * i + p] * X[3 * i + q];
  double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  *detJ = det;
  if (fabs(det) == 0.0) return -1;
  B[0][0] =  (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  B[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) / det;
  B[0][2] =  (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  B[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) / det;
  B[1][1] =  (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  B[1][2] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) / det;
  B[2][0] =  (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  B[2][1] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) / det;
  B[2][2] =  (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  for (int i = 0; i < nn; i++)
    for (int p = 0; p < 3; p++)
      dX[3 * i + p] = B[p][0] * dN[3 * i] + B[p][1] * dN[3 * i + 1] + B[p][2] * dN[3 * i + 2];
  return det > 0 ? 0 : -1;
}

/* cSolid::BMatrix (elc/anmodel.cpp:1418-1447); B is [6][nd], Voigt xx yy zz xy xz yz. */
static void bmatrix(int nn, const double *dX, double *B)
{
  int nd = 3 * nn;
  memset(B, 0, sizeof(double) * 6 * nd);
  for (int i = 0; i < nn; i++)
  {
    double x = dX[3 * i], y = dX[3 * i + 1], z = dX[3 * i + 2];
    B[0 * nd + 3 * i] = x;
    B[1 * nd + 3 * i + 1] = y;
    B[2 * nd + 3 * i + 2] = z;
    B[3 * nd + 3 * i] = y; B[3 * nd + 3 * i + 1] = x;
    B[4 * nd + 3 * i] = z; B[4 * nd + 3 * i + 2] = x;
    B[5 * nd + 3 * i + 1] = z; B[5 * nd + 3 * i + 2] = y;
  }
}

/* cSolid::QMatrix (elc/anmodel.cpp:1286-1298). */
static void qmatrix(double E, double nu, double *C)
{
  double d = (1.0 + nu) * (1.0 - 2.0 * nu);
  memset(C, 0, sizeof(double) * 36);
  C[0] = C[7] = C[14] = E * (1.0 - nu) / d;
  C[1] = C[6] = C[2] = C[12] = C[8] = C[13] = E * nu / d;
  C[21] = C[28] = C[35] = 0.5 * E / (1.0 + nu);
}

/* MatTripBtCB (mlib/matvec.cpp:372-388): K[i][j] += w B[k][i] C[k][l] B[l][j] with zero skipping. */
static void trip_btcb(int m, int n, const double *B, const double *C, double w, double *K)
{
  for (int i = 0; i < n; i++)
    for (int k = 0; k < m; k++)
      if (B[k * n + i] != 0.0)
      {
        double a1 = w * B[k * n + i];
        for (int l = 0; l < m; l++)
          if (C[k * m + l] != 0.0)
          {
            double a2 = a1 * C[k * m + l];
            const double *Bl = B + l * n;
            double *Ki = K + i * n;
            for (int j = 0; j < n; j++) Ki[j] += a2 * Bl[j];
          }
      }
}

/* cIntPoint::CreateBrickPoints (elc/intpoint.cpp:579-618): r fastest, then s, then t. */
static int gauss_pts(const int *ngp, double *pts, double *wts)
{
  int k = 0;
  for (int i = 0; i < ngp[2]; i++)
    for (int j = 0; j < ngp[1]; j++)
      for (int l = 0; l < ngp[0]; l++)
      {
        pts[3 * k] = GR[ngp[0] - 1][l];
        pts[3 * k + 1] = GR[ngp[1] - 1][j];
        pts[3 * k + 2] = GR[ngp[2] - 1][i];
        wts[k] = GW[ngp[0] - 1][l] * GW[ngp[1] - 1][j] * GW[ngp[2] - 1][i];
        k++;
      }
  return k;
}

int fo_elem_stiff(int nn, const int *ngp, const double *X, double E, double nu, double *Ke)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], B[6 * 60], C[36];
  int np = gauss_pts(ngp, pts, wts);
  memset(Ke, 0, sizeof(double) * nd * nd);
  qmatrix(E, nu, C);
  for (int g = 0; g < np; g++)
  {
    double detJ;
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    bmatrix(nn, dX, B);
    trip_btcb(6, nd, B, C, wts[g] * detJ, Ke);
  }
  return bad;
}

int fo_elem_intforce(int nn, const int *ngp, const double *X, double E, double nu,
                     const double *ue, double *ge)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], B[6 * 60], C[36], e[6], s[6];
  int np = gauss_pts(ngp, pts, wts);
  memset(ge, 0, sizeof(double) * nd);
  qmatrix(E, nu, C);
  for (int g = 0; g < np; g++)
  {
    double detJ;
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    bmatrix(nn, dX, B);
    for (int k = 0; k < 6; k++) { e[k] = 0; for (int j = 0; j < nd; j++) e[k] += B[k * nd + j] * ue[j]; }
    for (int k = 0; k < 6; k++) { s[k] = 0; for (int j = 0; j < 6; j++) s[k] += C[k * 6 + j] * e[j]; }
    double w = wts[g] * detJ;
    /* MatVecMultTAcc (mlib/matvec.cpp:359): v[i] += A[j][i]*(a*u[j]) */
    for (int k = 0; k < 6; k++) { double aj = w * s[k]; for (int i = 0; i < nd; i++) ge[i] += B[k * nd + i] * aj; }
  }
  return bad;
}

/* Gauss-point strains e = B u_e and stresses s = C e, point by point in the
 * rule's order (cElmParam::IntPntStress, elc/elmparam.cpp:859-935; the
 * isotropic section's Stress, sec/secanalysis.cpp:219-224). */
int fo_elem_stress(int nn, const int *ngp, const double *X, double E, double nu,
                   const double *ue, double *strain, double *stress)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], B[6 * 60], C[36];
  int np = gauss_pts(ngp, pts, wts);
  qmatrix(E, nu, C);
  for (int g = 0; g < np; g++)
  {
    double detJ, *e = strain + 6 * g, *s = stress + 6 * g;
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    bmatrix(nn, dX, B);
    for (int k = 0; k < 6; k++) { e[k] = 0; for (int j = 0; j < nd; j++) e[k] += B[k * nd + j] * ue[j]; }
    for (int k = 0; k < 6; k++) { s[k] = 0; for (int j = 0; j < 6; j++) s[k] += C[k * 6 + j] * e[j]; }
  }
  return bad;
}

/* Geometric stiffness at the displacements ue (cElmParam::GeomStiff,
 * elc/elmparam.cpp:743-830, with cSolid::BnlMatrix / SMatrix,
 * elc/anmodel.cpp:1514-1560): G = sum_g w detJ Bnl^T S Bnl, Bnl the 9 x 3nn
 * gradient operator and S three copies of the stress tensor of s = C B ue,
 * i.e. G[3a+i][3b+j] = delta_ij sum_g w detJ dN_a^T sigma dN_b. */
int fo_elem_geom(int nn, const int *ngp, const double *X, double E, double nu, const double *ue, double *Ge)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], B[6 * 60], C[36];
  int np = gauss_pts(ngp, pts, wts);
  qmatrix(E, nu, C);
  for (int i = 0; i < nd * nd; i++) Ge[i] = 0.0;
  for (int g = 0; g < np; g++)
  {
    double detJ, e[6], s[6];
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    bmatrix(nn, dX, B);
    for (int k = 0; k < 6; k++) { e[k] = 0; for (int j = 0; j < nd; j++) e[k] += B[k * nd + j] * ue[j]; }
    for (int k = 0; k < 6; k++) { s[k] = 0; for (int j = 0; j < 6; j++) s[k] += C[k * 6 + j] * e[j]; }
    const double S[3][3] = {{s[0], s[3], s[4]}, {s[3], s[1], s[5]}, {s[4], s[5], s[2]}};
    const double c = wts[g] * detJ;
    for (int a = 0; a < nn; a++)
      for (int b = 0; b < nn; b++)
      {
        double v = 0.0;
        for (int p = 0; p < 3; p++)
          for (int q = 0; q < 3; q++) v += dX[3 * a + p] * S[p][q] * dX[3 * b + q];
        for (int i = 0; i < 3; i++) Ge[(3 * a + i) * nd + 3 * b + i] += c * v;
      }
  }
  return bad;
}

/* Extrapolation matrix TR [nn][ng] (cElmParam::CompTRMatrix,
 * elc/elmparam.cpp:1444-1535): a linear field a0 + a1 r + a2 s + a3 t fitted
 * by least squares to the Gauss-point values and evaluated at the nodes,
 * TR = CN A^-1 CI with A = sum_i u_i u_i^T, u = (1, r, s, t); a one-point
 * rule (first order 1) gives the average.  The 4x4 system is solved by
 * Gaussian elimination with partial pivoting. */
int fo_extrap_matrix(int nn, const int *ngp, double *TR)
{
  double pts[216 * 3], wts[216];
  int np = gauss_pts(ngp, pts, wts);
  if (ngp[0] == 1)
  {
    for (int i = 0; i < nn * np; i++) TR[i] = 1.0 / np;
    return 0;
  }
  double A[4][4] = {{0}};
  for (int g = 0; g < np; g++)
  {
    double u[4] = {1.0, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2]};
    for (int k = 0; k < 4; k++)
      for (int l = 0; l < 4; l++) A[k][l] += u[k] * u[l];
  }
  /* Q = A^-1 CI, one Gauss point (column) at a time */
  double Q[4][216];
  for (int g = 0; g < np; g++)
  {
    double M[4][5];
    double u[4] = {1.0, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2]};
    for (int k = 0; k < 4; k++)
    {
      for (int l = 0; l < 4; l++) M[k][l] = A[k][l];
      M[k][4] = u[k];
    }
    for (int c = 0; c < 4; c++)
    {
      int piv = c;
      for (int r = c + 1; r < 4; r++)
        if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
      if (M[piv][c] == 0.0) return -1;
      for (int l = 0; l < 5; l++) { double t = M[c][l]; M[c][l] = M[piv][l]; M[piv][l] = t; }
      for (int r = c + 1; r < 4; r++)
      {
        double f = M[r][c] / M[c][c];
        for (int l = c; l < 5; l++) M[r][l] -= f * M[c][l];
      }
    }
    for (int c = 3; c >= 0; c--)
    {
      double v = M[c][4];
      for (int l = c + 1; l < 4; l++) v -= M[c][l] * Q[l][g];
      Q[c][g] = v / M[c][c];
    }
  }
  for (int a = 0; a < nn; a++)
  {
    double r, s, t;
    if (nn == 8)
    {
      static const int sr[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
      static const int ss[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
      static const int st[8] = { 1, 1, 1, 1, -1, -1, -1, -1};
      r = sr[a]; s = ss[a]; t = st[a];
    }
    else { r = H20[a][0]; s = H20[a][1]; t = H20[a][2]; }
    double cn[4] = {1.0, r, s, t};
    for (int g = 0; g < np; g++)
    {
      double v = 0.0;
      for (int k = 0; k < 4; k++) v += cn[k] * Q[k][g];
      TR[a * np + g] = v;
    }
  }
  return 0;
}

int fo_elem_mass(int nn, const int *ngp, const double *X, double rho, double *Me)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], Nm[3 * 60], Mb[9];
  int np = gauss_pts(ngp, pts, wts);
  memset(Me, 0, sizeof(double) * nd * nd);
  memset(Mb, 0, sizeof(Mb));
  Mb[0] = Mb[4] = Mb[8] = rho;
  for (int g = 0; g < np; g++)
  {
    double detJ;
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    memset(Nm, 0, sizeof(double) * 3 * nd);
    for (int i = 0; i < 3; i++) for (int a = 0; a < nn; a++) Nm[i * nd + 3 * a + i] = N[a];
    trip_btcb(3, nd, Nm, Mb, wts[g] * detJ, Me);
  }
  return bad;
}

int fo_elem_tl(int nn, const int *ngp, const double *X, double E, double nu,
               const double *ue, double *Kt, double *ge)
{
  int nd = 3 * nn, bad = 0;
  double pts[216 * 3], wts[216], N[20], dN[60], dX[60], B[6 * 60], Bl[6 * 60], Bnl[9 * 60];
  double C[36], S[81], e[6], s[6];
  int np = gauss_pts(ngp, pts, wts);
  if (Kt) memset(Kt, 0, sizeof(double) * nd * nd);
  if (ge) memset(ge, 0, sizeof(double) * nd);
  qmatrix(E, nu, C);
  for (int g = 0; g < np; g++)
  {
    double detJ;
    shape(nn, pts[3 * g], pts[3 * g + 1], pts[3 * g + 2], N, dN);
    if (drv_xyz(nn, dN, X, &detJ, dX)) bad = -1;
    bmatrix(nn, dX, B);
    /* cSolid::BlMatrix (elc/anmodel.cpp:1451-1510) */
    double l[3][3] = {{0}};
    for (int i = 0; i < nn; i++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) l[a][b] += ue[3 * i + a] * dX[3 * i + b];
    memset(Bl, 0, sizeof(double) * 6 * nd);
    for (int i = 0; i < nn; i++)
    {
      double x = dX[3 * i], y = dX[3 * i + 1], z = dX[3 * i + 2];
      for (int a = 0; a < 3; a++)
      {
        Bl[0 * nd + 3 * i + a] = l[a][0] * x;
        Bl[1 * nd + 3 * i + a] = l[a][1] * y;
        Bl[2 * nd + 3 * i + a] = l[a][2] * z;
        Bl[3 * nd + 3 * i + a] = l[a][0] * y + l[a][1] * x;
        Bl[4 * nd + 3 * i + a] = l[a][0] * z + l[a][2] * x;
        Bl[5 * nd + 3 * i + a] = l[a][1] * z + l[a][2] * y;
      }
    }
    /* cSolid::BnlMatrix (elc/anmodel.cpp:1514-1532) */
    memset(Bnl, 0, sizeof(double) * 9 * nd);
    for (int i = 0; i < nn; i++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Bnl[(3 * a + b) * nd + 3 * i + a] = dX[3 * i + b];
    /* cElmParamTL::GreenStrain (elc/elmparam.cpp:1899-1919): e = B u + 0.5 (Bl u) */
    for (int k = 0; k < 6; k++)
    {
      double s1 = 0, s2 = 0;
      for (int j = 0; j < nd; j++) s1 += B[k * nd + j] * ue[j];
      for (int j = 0; j < nd; j++) s2 += Bl[k * nd + j] * ue[j];
      s2 *= 0.5;
      e[k] = s1 + s2;
    }
    for (int k = 0; k < 6; k++) { s[k] = 0; for (int j = 0; j < 6; j++) s[k] += C[k * 6 + j] * e[j]; }
    /* cSolid::SMatrix (elc/anmodel.cpp:1536-1568): three copies of the 3x3 stress tensor */
    memset(S, 0, sizeof(S));
    double T[3][3] = {{s[0], s[3], s[4]}, {s[3], s[1], s[5]}, {s[4], s[5], s[2]}};
    for (int blk = 0; blk < 3; blk++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) S[(3 * blk + a) * 9 + 3 * blk + b] = T[a][b];
    for (int k = 0; k < 6 * nd; k++) B[k] += Bl[k];
    double w = wts[g] * detJ;
    if (Kt) { trip_btcb(6, nd, B, C, w, Kt); trip_btcb(9, nd, Bnl, S, w, Kt); }
    if (ge) for (int k = 0; k < 6; k++) { double aj = w * s[k]; for (int i = 0; i < nd; i++) ge[i] += B[k * nd + i] * aj; }
  }
  return bad;
}

/* Q4 / Q8 surface shapes (shp/shpplane.cpp:353-488), used on faces. */
static void face_shape(int nf, double r, double s, double *N, double *dN)
{
  if (nf == 4)
  {
    N[0] = 0.25 * (1 - r) * (1 - s); N[1] = 0.25 * (1 + r) * (1 - s);
    N[2] = 0.25 * (1 + r) * (1 + s); N[3] = 0.25 * (1 - r) * (1 + s);
    dN[0] = -0.25 * (1 - s); dN[2] = 0.25 * (1 - s); dN[4] = 0.25 * (1 + s); dN[6] = -0.25 * (1 + s);
    dN[1] = -0.25 * (1 - r); dN[3] = -0.25 * (1 + r); dN[5] = 0.25 * (1 + r); dN[7] = 0.25 * (1 - r);
  }
  else
  {
    N[0] = 0.25 * (1 - r) * (1 - s) - 0.25 * (1 - r) * (1 - s * s) - 0.25 * (1 - r * r) * (1 - s);
    N[1] = 0.50 * (1 - r * r) * (1 - s);
    N[2] = 0.25 * (1 + r) * (1 - s) - 0.25 * (1 - r * r) * (1 - s) - 0.25 * (1 - s * s) * (1 + r);
    N[3] = 0.50 * (1 - s * s) * (1 + r);
    N[4] = 0.25 * (1 + r) * (1 + s) - 0.25 * (1 - s * s) * (1 + r) - 0.25 * (1 + s) * (1 - r * r);
    N[5] = 0.50 * (1 - r * r) * (1 + s);
    N[6] = 0.25 * (1 - r) * (1 + s) - 0.25 * (1 - r * r) * (1 + s) - 0.25 * (1 - s * s) * (1 - r);
    N[7] = 0.50 * (1 - s * s) * (1 - r);
    dN[0] = (2 * r - 2 * r * s - s * s + s) / 4.0;  dN[1] = (2 * s - r * r - 2 * r * s + r) / 4.0;
    dN[2] = r * s - r;                              dN[3] = (r * r - 1) / 2.0;
    dN[4] = (2 * r - 2 * r * s + s * s - s) / 4.0;  dN[5] = (2 * s - r * r + 2 * r * s - r) / 4.0;
    dN[6] = (1 - s * s) / 2.0;                      dN[7] = -s - r * s;
    dN[8] = (2 * r + 2 * r * s + s * s + s) / 4.0;  dN[9] = (2 * s + r * r + 2 * r * s + r) / 4.0;
    dN[10] = -r - r * s;                            dN[11] = (1 - r * r) / 2.0;
    dN[12] = (2 * r + 2 * r * s - s * s - s) / 4.0; dN[13] = (2 * s + r * r - 2 * r * s - r) / 4.0;
    dN[14] = (s * s - 1) / 2.0;                     dN[15] = r * s - s;
  }
}

int fo_face_load(int nf, int ngp1d, const double *Xf, const double *q, int local, double *fe)
{
  double N[8], dN[16];
  memset(fe, 0, sizeof(double) * 3 * nf);
  /* cIntPoint::CreateQuadPoints (elc/intpoint.cpp:266-300): r fastest */
  for (int i = 0; i < ngp1d; i++)
    for (int j = 0; j < ngp1d; j++)
    {
      double r = GR[ngp1d - 1][j], s = GR[ngp1d - 1][i];
      double wgt = GW[ngp1d - 1][j] * GW[ngp1d - 1][i];
      face_shape(nf, r, s, N, dN);
      double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
      for (int a = 0; a < nf; a++)
        for (int k = 0; k < 3; k++) { tr[k] += dN[2 * a] * Xf[3 * a + k]; ts[k] += dN[2 * a + 1] * Xf[3 * a + k]; }
      double n[3] = {tr[1] * ts[2] - tr[2] * ts[1], tr[2] * ts[0] - tr[0] * ts[2], tr[0] * ts[1] - tr[1] * ts[0]};
      double detJ = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      double val[3] = {q[0], q[1], q[2]};
      if (local)
      {
        /* cShapeSurf::LocalSys (shp/shpsurf.cpp:121-160): u = tr/|tr|, v = ts/|ts|, w = u x v, v = w x u */
        double lu = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
        double lv = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
        double u[3] = {tr[0] / lu, tr[1] / lu, tr[2] / lu}, v[3] = {ts[0] / lv, ts[1] / lv, ts[2] / lv};
        double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        v[0] = w[1] * u[2] - w[2] * u[1]; v[1] = w[2] * u[0] - w[0] * u[2]; v[2] = w[0] * u[1] - w[1] * u[0];
        for (int k = 0; k < 3; k++) val[k] = u[k] * q[0] + v[k] * q[1] + w[k] * q[2];
      }
      double coeff = wgt * detJ;
      for (int a = 0; a < nf; a++)
        for (int k = 0; k < 3; k++) fe[3 * a + k] += N[a] * (coeff * val[k]);
    }
  return 0;
}

void fo_spmv(int n, const int64_t *rowptr, const int32_t *col, const double *val,
             const double *x, double *y)
{
  for (int i = 0; i < n; i++)
  {
    double s = 0.0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++) s += val[k] * x[col[k]];
    y[i] = s;
  }
}

static double dot(int n, const double *a, const double *b)
{
  double s = 0.0;
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

int fo_pcg(int n, const int64_t *rowptr, const int32_t *col, const double *val,
           const double *f, double *u, int maxit, double tol, int *iters, double *err_out)
{
  double lenf = sqrt(dot(n, f, f));
  memset(u, 0, sizeof(double) * n);
  *iters = 0;
  *err_out = 0.0;
  if (lenf < tol) return 1;
  if (lenf > 10e+10) lenf = 1.0;
  double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
  double *d = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
  for (int i = 0; i < n; i++)
  {
    d[i] = 0.0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++) if (col[k] == i) d[i] = val[k];
  }
  for (int i = 0; i < n; i++) { r[i] = f[i]; z[i] = r[i] / d[i]; p[i] = z[i]; }
  double dot0 = dot(n, z, r), err = 0.0;
  int conv = 0, k;
  for (k = 1; k <= maxit; k++)
  {
    fo_spmv(n, rowptr, col, val, p, w);
    double alpha = dot0 / dot(n, p, w);
    for (int i = 0; i < n; i++) u[i] = u[i] + alpha * p[i];
    for (int i = 0; i < n; i++) r[i] = r[i] + (-alpha) * w[i];
    for (int i = 0; i < n; i++) z[i] = r[i] / d[i];
    err = sqrt(dot(n, r, r)) / lenf;
    if (err < tol) { conv = 1; break; }
    double dot1 = dot(n, z, r);
    double beta = dot1 / dot0;
    dot0 = dot1;
    for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
  }
  *iters = conv ? k : maxit;
  *err_out = err;
  free(r); free(p); free(d); free(w); free(z);
  return conv;
}

/* The same iteration with every vector operation and the SpMV split over the
 * host threads (pthreads, one static range of rows per thread): a
 * large-system checker, not a restatement of the reference's loop order.
 * Sums are per-thread partials combined in thread order, so a run is
 * reproducible for a fixed thread count. */
enum { PT_SPMV_DOT, PT_UPDATE, PT_PUPDATE, PT_INIT };
typedef struct {
  int op, n, t, nt;
  const int64_t *rowptr; const int32_t *col; const double *val;
  const double *f; double *u, *r, *p, *d, *w, *z;
  double alpha, beta, s1, s2;
} pt_job;

static void *pt_run(void *arg)
{
  pt_job *j = (pt_job *)arg;
  const int i0 = (int)((int64_t)j->n * j->t / j->nt), i1 = (int)((int64_t)j->n * (j->t + 1) / j->nt);
  double s1 = 0.0, s2 = 0.0;
  switch (j->op)
  {
    case PT_INIT:
      for (int i = i0; i < i1; i++)
      {
        j->d[i] = 0.0;
        for (int64_t k = j->rowptr[i]; k < j->rowptr[i + 1]; k++) if (j->col[k] == i) j->d[i] = j->val[k];
        j->r[i] = j->f[i]; j->z[i] = j->r[i] / j->d[i]; j->p[i] = j->z[i];
        s1 += j->z[i] * j->r[i];
        s2 += j->f[i] * j->f[i];
      }
      break;
    case PT_SPMV_DOT:   /* w = K p, p.w */
      for (int i = i0; i < i1; i++)
      {
        double s = 0.0;
        for (int64_t k = j->rowptr[i]; k < j->rowptr[i + 1]; k++) s += j->val[k] * j->p[j->col[k]];
        j->w[i] = s;
        s1 += j->p[i] * s;
      }
      break;
    case PT_UPDATE:     /* u += a p; r -= a w; z = r / d; r.r, z.r */
      for (int i = i0; i < i1; i++)
      {
        j->u[i] = j->u[i] + j->alpha * j->p[i];
        j->r[i] = j->r[i] + (-j->alpha) * j->w[i];
        j->z[i] = j->r[i] / j->d[i];
        s1 += j->r[i] * j->r[i];
        s2 += j->z[i] * j->r[i];
      }
      break;
    case PT_PUPDATE:    /* p = z + b p */
      for (int i = i0; i < i1; i++) j->p[i] = j->z[i] + j->beta * j->p[i];
      break;
  }
  j->s1 = s1;
  j->s2 = s2;
  return NULL;
}

/* run one operation on nt threads; *s1, *s2 = partial sums combined in thread order */
static void pt_parallel(pt_job *jobs, int nt, int op, double alpha, double beta, double *s1, double *s2)
{
  pthread_t th[64];
  for (int t = 0; t < nt; t++)
  {
    jobs[t].op = op; jobs[t].alpha = alpha; jobs[t].beta = beta;
    if (t > 0) pthread_create(&th[t], NULL, pt_run, &jobs[t]);
  }
  pt_run(&jobs[0]);
  for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
  double a = 0.0, b = 0.0;
  for (int t = 0; t < nt; t++) { a += jobs[t].s1; b += jobs[t].s2; }
  if (s1) *s1 = a;
  if (s2) *s2 = b;
}

int fo_pcg_threaded(int n, const int64_t *rowptr, const int32_t *col, const double *val,
                    const double *f, double *u, int maxit, double tol, int *iters, double *err_out)
{
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  int nt = ncpu < 1 ? 1 : (ncpu > 64 ? 64 : (int)ncpu);
  memset(u, 0, sizeof(double) * n);
  *iters = 0;
  *err_out = 0.0;
  double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
  double *d = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
  pt_job jobs[64];
  for (int t = 0; t < nt; t++)
  {
    pt_job j = {0, n, t, nt, rowptr, col, val, f, u, r, p, d, w, z, 0.0, 0.0, 0.0, 0.0};
    jobs[t] = j;
  }
  double dot0 = 0.0, ff = 0.0, err = 0.0;
  pt_parallel(jobs, nt, PT_INIT, 0.0, 0.0, &dot0, &ff);
  double lenf = sqrt(ff);
  int conv = 0, k = 0;
  if (lenf < tol) { conv = 1; goto out; }
  if (lenf > 10e+10) lenf = 1.0;
  for (k = 1; k <= maxit; k++)
  {
    double pw = 0.0, rr = 0.0, zr = 0.0;
    pt_parallel(jobs, nt, PT_SPMV_DOT, 0.0, 0.0, &pw, NULL);
    double alpha = dot0 / pw;
    pt_parallel(jobs, nt, PT_UPDATE, alpha, 0.0, &rr, &zr);
    err = sqrt(rr) / lenf;
    if (err < tol) { conv = 1; break; }
    double beta = zr / dot0;
    dot0 = zr;
    pt_parallel(jobs, nt, PT_PUPDATE, 0.0, beta, NULL, NULL);
  }
  *iters = conv ? k : maxit;
  *err_out = err;
out:
  free(r); free(p); free(d); free(w); free(z);
  return conv;
}

int fo_elems_stiff(int nn, const int *ngp, int64_t ne, const int32_t *conn, const double *Xn,
                   const double *E, const double *nu, double *Ke)
{
  int nd = 3 * nn, bad = 0;
  double X[60];
  for (int64_t e = 0; e < ne; e++)
  {
    for (int a = 0; a < nn; a++)
      for (int k = 0; k < 3; k++) X[3 * a + k] = Xn[3 * (int64_t)conn[e * nn + a] + k];
    if (fo_elem_stiff(nn, ngp, X, E[e], nu[e], Ke + e * nd * nd)) bad = -1;
  }
  return bad;
}

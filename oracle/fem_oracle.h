/* fem_oracle.h - CPU restatement of FAST's solid element / assembly / solve
 * path, used ONLY as a checker by the tests, by __graft_entry__.smoke() and by
 * the CPU-baseline leg of bench.py.  Never linked into the product.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function below
 * against golden vectors dumped from the reference FAST program itself
 * (oracle/ref_harness.cpp linked against the reference objects).
 */
#ifndef FEM_ORACLE_H
#define FEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss points/weights as tabulated by FAST (elc/intpoint.cpp:742-790), n = 1..6. */
int fo_gauss(int n, double *r, double *w);

/* Shape functions and natural derivatives; dN is [nn][3] (r, s, t). */
void fo_shape_hex8(double r, double s, double t, double *N, double *dN);
void fo_shape_hex20(double r, double s, double t, double *N, double *dN);

/* Element stiffness K = sum_g w_g detJ_g B^T C B (cElmParam::StiffMat,
 * elc/elmparam.cpp:539-597) with MatTripBtCB's loop order and zero skipping
 * (mlib/matvec.cpp:372-388).  nn = 8 or 20.  X is [nn][3]; Ke is
 * [3nn][3nn] row-major.  Returns 0 on success, -1 if a Jacobian
 * determinant is <= 0. */
int fo_elem_stiff(int nn, const int *ngp, const double *X, double E, double nu, double *Ke);

/* Batched fo_elem_stiff over ne elements: conn [ne][nn] 0-based node
 * indices into Xn [nnode][3]; Ke [ne][3nn][3nn]. */
int fo_elems_stiff(int nn, const int *ngp, int64_t ne, const int32_t *conn, const double *Xn,
                   const double *E, const double *nu, double *Ke);

/* Internal force g = sum_g w detJ B^T C B u (cElmParam::IntForce,
 * elc/elmparam.cpp:449-535). */
int fo_elem_intforce(int nn, const int *ngp, const double *X, double E, double nu,
                     const double *ue, double *ge);
int fo_elem_stress(int nn, const int *ngp, const double *X, double E, double nu,
                   const double *ue, double *strain, double *stress);

/* Geometric stiffness Ge [3nn][3nn] at element displacements ue
 * (cElmParam::GeomStiff, elc/elmparam.cpp:743-830). */
int fo_elem_geom(int nn, const int *ngp, const double *X, double E, double nu, const double *ue, double *Ge);

/* Stress extrapolation matrix TR [nn][ng] of cElmParam::CompTRMatrix
 * (elc/elmparam.cpp:1444-1535): element-nodal stresses = TR x Gauss-point
 * stresses (cElmParam::NodalStress, :1304-1312). */
int fo_extrap_matrix(int nn, const int *ngp, double *TR);

/* Consistent mass M = sum_g w detJ rho N^T N (cElmParam::MassMat, elc/elmparam.cpp:672-739). */
int fo_elem_mass(int nn, const int *ngp, const double *X, double rho, double *Me);

/* Total-Lagrangian St. Venant-Kirchhoff element (cElmParamTL::StiffMat / IntForce,
 * elc/elmparam.cpp:1615-1807; cSolid::BlMatrix/BnlMatrix/SMatrix,
 * elc/anmodel.cpp:1451-1568).  ue are the element nodal displacements. */
int fo_elem_tl(int nn, const int *ngp, const double *X, double E, double nu,
               const double *ue, double *Kt, double *ge);

/* Uniform traction on a Q4 (nf=4) or Q8 (nf=8) face with ngp1d^2 Gauss points
 * (cElemLoad::ExtForce, load/load.cpp:618-706; cShapeSurf::DrvShpXYZ,
 * shp/shpsurf.cpp:58-117; LocalSys :121-160).  Xf [nf][3]; fe [nf][3]. */
int fo_face_load(int nf, int ngp1d, const double *Xf, const double *q, int local, double *fe);

/* Jacobi PCG exactly as FAST's PCGSolver (mlib/sysmat.cpp:1061-1125) on a full
 * symmetric CSR matrix: u starts at 0, z = r/diag, err = |r|/|f| (|f| > 1e11
 * is replaced by 1).  Returns 1 on convergence, 0 otherwise; *iters and *err
 * report the last iteration. */
int fo_pcg(int n, const int64_t *rowptr, const int32_t *col, const double *val,
           const double *f, double *u, int maxit, double tol, int *iters, double *err);

/* The same PCG with its vector operations and SpMV on all host threads
 * (pthreads): a checker for systems of millions of equations. */
int fo_pcg_threaded(int n, const int64_t *rowptr, const int32_t *col, const double *val,
                    const double *f, double *u, int maxit, double tol, int *iters, double *err);

/* y = A x for a full CSR matrix. */
void fo_spmv(int n, const int64_t *rowptr, const int32_t *col, const double *val,
             const double *x, double *y);

#ifdef __cplusplus
}
#endif
#endif

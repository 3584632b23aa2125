// fast_shim.cpp - the FAST-side binding of libfastgpu.so.
//
// A FAST build links this file (against FAST's own headers) and
// libfastgpu.so, and the unmodified controllers (cLinStat::Solver,
// ctrl/ctrllins.cpp:46-99, and the others that go through
// cSysMatrix::CreateMatrix and cControl::StiffnessMatrix) run on the device
// for a deck that says
//
//     %HEADER.ANALYSIS.MATRIX.TYPE
//     'gpu'
//
// What it supplies:
//   * cGpuSysMatrix, a cSysMatrix (mlib/sysmat.h:60-99) whose virtuals forward
//     to the C ABI of include/fast_gpu.h: Zero, Add, Get, MultVect, AddMat and
//     Solve (Jacobi PCG with the controller's SetParam(maxit, tol), as
//     cSymSprsMatrix::Solve -> PCGSolver, mlib/sysmat.cpp:966-970, 1061-1125);
//   * a batched cControl::StiffnessMatrix (ctrl/ctrl.cpp:886-975) for that
//     matrix: the whole mesh is uploaded once and every element is
//     integrated and scattered on the device in one call; spring supports,
//     spring connections and the prescribed-DOF penalty still go through
//     K->Add exactly as in the reference;
//   * the label 'gpu' for cControl::ReadMatrixType (ctrl/ctrl.cpp:213-238).
//
// How it hooks in without editing FAST's sources: the reader table
// (main/input.cpp:205) and the controllers reference ReadMatrixType,
// CreateMatrix and StiffnessMatrix from other object files, so the linker's
// --wrap option routes those references here:
//
//   -Wl,--wrap=_ZN8cControl14ReadMatrixTypeEv
//   -Wl,--wrap=_ZN10cSysMatrix12CreateMatrixE7eSMTypeiPi
//   -Wl,--wrap=_ZN8cControl15StiffnessMatrixEP10cSysMatrix
//
// Each wrapper hands every case that is not the device matrix to the
// reference's own function (__real_...), so decks with other matrix types run
// exactly as before.  A maintainer who prefers source edits adds the three
// lines instead (an eSMType value, the label, the CreateMatrix case) and calls
// the functions below.
//
// Device options (environment, read once): FAST_GPU_DEVICE (default 0),
// FAST_GPU_PRECISION = fp64 (default: the reference's iteration) | mixed.
// Elements the device path does not integrate (anything but small-strain
// %ELEMENT.BRICK8 / BRICK20 solids with an isotropic elastic material) stop
// the run with a message: there is no CPU fallback for the device matrix.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

using namespace std;

#include "ctrl.h"
#include "element.h"
#include "elmparam.h"
#include "gbldef.h"
#include "material.h"
#include "node.h"
#include "prescdof.h"
#include "section.h"
#include "shape.h"
#include "spring.h"
#include "sysmat.h"
#include "utl.h"
#include "vec.h"

#include "fast_gpu.h"

extern ifstream in;   // the deck stream owned by main/main.cpp

namespace {

// An eSMType value outside the reference's enumeration (mlib/sysmat.h:41-48)
const eSMType kSymGpu = static_cast<eSMType>(1000);

[[noreturn]] void die(const char *what, int rc, fast_gpu_ctx *ctx) {
  fprintf(stderr, "fast_shim: %s failed (%d): %s\n", what, rc, ctx ? fast_gpu_last_error(ctx) : "");
  exit(1);
}

void check(int rc, const char *what, fast_gpu_ctx *ctx) {
  if (rc != FAST_GPU_OK) die(what, rc, ctx);
}

// access to the controller's protected statics
struct Ctrl : public cControl {
  static eSMType &MatType() { return SysMatType; }
  static int NEq() { return NumEq; }
};

int env_int(const char *name, int def) {
  const char *v = getenv(name);
  return v && *v ? atoi(v) : def;
}

}  // namespace

// ---------------------------------------------------------------------------
// The device matrix
class cGpuSysMatrix : public cSysMatrix {
 public:
  static fast_gpu_ctx *ctx;      // one device context per FAST process
  static bool mesh_uploaded;

  explicit cGpuSysMatrix(int n) : cSysMatrix(n) {
    if (!ctx) check(fast_gpu_create(env_int("FAST_GPU_DEVICE", 0), &ctx), "fast_gpu_create", nullptr);
  }
  int Symmetric(void) { return 1; }
  void Zero(void) {
    if (mesh_uploaded) check(fast_gpu_zero(ctx, FAST_ASM_STIFFNESS), "fast_gpu_zero", ctx);
  }
  // symmetric storage: the reference's symmetric matrices ignore i < j
  void Add(int i, int j, double v) {
    if (i >= j) check(fast_gpu_add(ctx, FAST_ASM_STIFFNESS, i, j, v), "fast_gpu_add", ctx);
  }
  double Get(int i, int j) {
    double v = 0.0;
    check(fast_gpu_get(ctx, FAST_ASM_STIFFNESS, i, j, &v), "fast_gpu_get", ctx);
    return v;
  }
  void Print(void) {}
  void MultVect(double *x, double *y) {
    check(fast_gpu_mult_vect(ctx, FAST_ASM_STIFFNESS, x, y), "fast_gpu_mult_vect", ctx);
  }
  // K += a M where M is the device mass slot (cCtrlNewmark's K_eff)
  void AddMat(double a, cSysMatrix *) {
    check(fast_gpu_add_mat(ctx, FAST_ASM_STIFFNESS, a, FAST_ASM_MASS), "fast_gpu_add_mat", ctx);
  }
  int Solve(cVector &b, cVector &x) {
    fast_gpu_solve_opts o;
    memset(&o, 0, sizeof(o));
    const char *p = getenv("FAST_GPU_PRECISION");
    o.precision = (p && string(p) == "mixed") ? FAST_PREC_MIXED : FAST_PREC_FP64;
    o.precond = FAST_PRECOND_JACOBI;
    o.tol = tol;          // SetParam(MaxIter, Tol) of the controller
    o.maxit = maxit;
    fast_gpu_solve_report r;
    const int rc = fast_gpu_solve(ctx, b.Val(), x.Val(), &o, &r);
    if (rc != FAST_GPU_OK && rc != FAST_GPU_ENONCONV) die("fast_gpu_solve", rc, ctx);
    return r.converged ? 1 : 0;   // 1 = ok, as cSysMatrix::Solve
  }
};

fast_gpu_ctx *cGpuSysMatrix::ctx = nullptr;
bool cGpuSysMatrix::mesh_uploaded = false;

namespace {

// Gauss points per direction of an element: the distinct natural
// coordinates of its integration points along r, s and t
void gauss_counts(cElement *elm, int ngp[3]) {
  const int np = elm->GetNumIntPnt();
  vector<double> c[3];
  for (int i = 0; i < np; i++) {
    sNatCoord q;
    double w;
    elm->GetIntPnt(i, q, w);
    const double v[3] = {q.r, q.s, q.t};
    for (int k = 0; k < 3; k++) {
      bool seen = false;
      for (double x : c[k]) seen = seen || fabs(x - v[k]) < 1e-12;
      if (!seen) c[k].push_back(v[k]);
    }
  }
  for (int k = 0; k < 3; k++) ngp[k] = (int)c[k].size();
}

struct BucketData {
  int type = 0, ngp[3] = {0, 0, 0};
  vector<int32_t> conn;
  vector<double> E, nu;
};

// Gather FAST's mesh (cNode / cElement registries) into the ABI's
// description and upload it: node coordinates and equation numbers as
// cControl::CompEqs left them, one bucket per (shape, Gauss rule).
void upload_mesh(fast_gpu_ctx *ctx) {
  const int nnode = cNode::GetNumNode();
  unordered_map<const cNode *, int32_t> index;
  index.reserve((size_t)nnode * 2);
  vector<double> X((size_t)nnode * 3);
  vector<int32_t> eq((size_t)nnode * 3);
  for (int i = 0; i < nnode; i++) {
    cNode *nd = cNode::GetNode(i);
    index[nd] = i;
    const sNodeCoord c = nd->GetCoord();
    X[3 * (size_t)i] = c.x;
    X[3 * (size_t)i + 1] = c.y;
    X[3 * (size_t)i + 2] = c.z;
    for (int j = 0; j < 3; j++) eq[3 * (size_t)i + j] = nd->GetDof(j);
  }
  map<vector<int>, BucketData> buckets;  // key: type, ngp
  const int ne = cElement::GetNumElm();
  for (int e = 0; e < ne; e++) {
    cElement *elm = cElement::GetElm(e);
    cShape *shp = elm->GetShape();
    int type = 0;
    if (shp->GetType() == SHAPE_BRICK8) type = FAST_ELEM_HEX8;
    if (shp->GetType() == SHAPE_BRICK20) type = FAST_ELEM_HEX20;
    cMaterial *m = elm->GetSection() ? elm->GetSection()->GetMaterial() : nullptr;
    cMatElastIso *mat = m ? dynamic_cast<cMatElastIso *>(m->GetMecProp()) : nullptr;
    if (!type || elm->GetType() != PARAMETRIC || !mat) {
      fprintf(stderr, "fast_shim: element %d is not a small-strain hex8/hex20 solid with an isotropic elastic "
                      "material; the 'gpu' matrix type cannot take this deck\n", elm->GetLabel());
      exit(1);
    }
    int ngp[3];
    gauss_counts(elm, ngp);
    BucketData &b = buckets[{type, ngp[0], ngp[1], ngp[2]}];
    b.type = type;
    memcpy(b.ngp, ngp, sizeof(ngp));
    for (int a = 0; a < shp->GetNumNode(); a++) b.conn.push_back(index.at(shp->GetNode(a)));
    double prm[3];
    mat->GetParam(prm);
    b.E.push_back(prm[0]);
    b.nu.push_back(prm[1]);
  }
  vector<fast_gpu_bucket> bk;
  for (auto &kv : buckets) {
    fast_gpu_bucket d;
    memset(&d, 0, sizeof(d));
    d.elem_type = kv.second.type;
    memcpy(d.ngp, kv.second.ngp, sizeof(d.ngp));
    d.num_elems = (int64_t)kv.second.E.size();
    d.conn = kv.second.conn.data();
    d.E = kv.second.E.data();
    d.nu = kv.second.nu.data();
    d.formulation = FAST_FORM_SMALL_STRAIN;
    bk.push_back(d);
  }
  fast_gpu_mesh m;
  memset(&m, 0, sizeof(m));
  m.num_nodes = nnode;
  m.coords = X.data();
  m.node_eq = eq.data();
  m.num_eq = Ctrl::NEq();
  m.num_buckets = (int32_t)bk.size();
  m.buckets = bk.data();
  check(fast_gpu_upload_mesh(ctx, &m), "fast_gpu_upload_mesh", ctx);
  cGpuSysMatrix::mesh_uploaded = true;
}

// the device-matrix branch of cControl::StiffnessMatrix
void gpu_stiffness_matrix(cGpuSysMatrix *K) {
  if (!cGpuSysMatrix::mesh_uploaded) upload_mesh(cGpuSysMatrix::ctx);
  // zero + every element, colour by colour (deterministic)
  check(fast_gpu_assemble(cGpuSysMatrix::ctx, FAST_ASM_STIFFNESS), "fast_gpu_assemble", cGpuSysMatrix::ctx);
  // spring supports and connections, through K->Add as in the reference
  cMatrix Ks(cSpring::GetMaxDof(), cSpring::GetMaxDof());
  for (int i = 0; i < cSpringSupp::GetNumSpring(); i++) {
    cSpringSupp *s = cSpringSupp::GetSpring(i);
    s->StiffMat(Ks);
    s->AddGlobMat(Ks, K);
  }
  for (int i = 0; i < cSpringConn::GetNumSpring(); i++) {
    cSpringConn *s = cSpringConn::GetSpring(i);
    s->StiffMat(Ks);
    s->AddGlobMat(Ks, K);
  }
  // prescribed DOFs: the penalty on the diagonal
  const int npd = cPrescDof::GetNumPrescDofs();
  if (npd > 0) {
    vector<int> pd(npd);
    cPrescDof::GetPrescDofs(pd.data());
    for (int d : pd) K->Add(d - 1, d - 1, PENALTY_STIFFNESS);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Link-level hooks (-Wl,--wrap=...): the reference's functions stay the
// fallback for every other matrix type.
extern "C" {

void __real__ZN8cControl14ReadMatrixTypeEv(void);
cSysMatrix *__real__ZN10cSysMatrix12CreateMatrixE7eSMTypeiPi(eSMType, int, int *);
void __real__ZN8cControl15StiffnessMatrixEP10cSysMatrix(cSysMatrix *);

// cControl::ReadMatrixType: 'gpu' selects the device matrix; any other label
// is re-read by the reference's reader
void __wrap__ZN8cControl14ReadMatrixTypeEv(void) {
  const streampos at = in.tellg();
  char label[100];
  if (Utl::ReadString(in, label) && string(label) == "gpu") {
    Ctrl::MatType() = kSymGpu;
    return;
  }
  in.clear();
  in.seekg(at);
  __real__ZN8cControl14ReadMatrixTypeEv();
}

// cSysMatrix::CreateMatrix
cSysMatrix *__wrap__ZN10cSysMatrix12CreateMatrixE7eSMTypeiPi(eSMType type, int n, int *profile) {
  if (type == kSymGpu) return new cGpuSysMatrix(n);
  return __real__ZN10cSysMatrix12CreateMatrixE7eSMTypeiPi(type, n, profile);
}

// cControl::StiffnessMatrix
void __wrap__ZN8cControl15StiffnessMatrixEP10cSysMatrix(cSysMatrix *K) {
  if (cGpuSysMatrix *G = dynamic_cast<cGpuSysMatrix *>(K)) {
    gpu_stiffness_matrix(G);
    return;
  }
  __real__ZN8cControl15StiffnessMatrixEP10cSysMatrix(K);
}

}  // extern "C"

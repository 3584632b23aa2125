// ref_harness.cpp - test-infrastructure harness around the reference FAST
// program.  It is linked against the reference's own object files (every
// translation unit except main/main.cpp, which it replaces) and is used only
// by the golden-fixture generator, the tests and the CPU-baseline leg of the
// benchmark.  Nothing in the product links or runs it.
//
// Modes
//   fastref dump  <deck> <out.bin> [--no-triplets] [--no-solve] [--mass]
//                                  [--u <u.f8>] [--solver-tol <t>]
//       Reads <deck>.dat with the reference reader (main/input.cpp:355
//       InpReadData), runs cControl::Init (ctrl/ctrl.cpp:536) and writes, in
//       FP64:
//         neq                      number of equations (ctrl/ctrl.cpp:2056 CompEqs)
//         node_eq   [nnode][3]     1-based equation of each translational DOF, 0 = fixed
//         elm_dofs  [ne][ndof]     cElement::GetElmDofs (elc/element.cpp:2907)
//         elm_K     [ne][ndof][ndof] cElement::StiffMat (elc/elmparam.cpp:539)
//         elm_g     [ne][ndof]     cElement::IntForce  (elc/elmparam.cpp:449)
//         elm_M     [ne][ndof][ndof] cElement::MassMat (elc/elmparam.cpp:672), --mass
//         f         [neq]          cControl::ExtLoadVector (ctrl/ctrl.cpp:668)
//         K_i,K_j,K_v              every cSysMatrix::Add(i,j,v) issued by
//                                  cControl::StiffnessMatrix (ctrl/ctrl.cpp:886),
//                                  in call order, through a recording matrix
//         u         [neq]          K->Solve(f,u) with the deck's own matrix type
//                                  and MAXIMUM.ITERATIONS / TOLERANCE, as
//                                  cLinStat::Solver does (ctrl/ctrllins.cpp:46-70)
//         g_of_u    [neq]          cControl::IntForceVector after AssignDispl(u)
//       With --u the element quantities are evaluated at the given nodal state
//       (for total-Lagrangian elements).  With --stress, at the solved (or the
//       --u) state:
//         elm_strain, elm_stress [ne][nip][6]  cElement::IntPntStress
//                                  (elc/elmparam.cpp:859-935), Voigt xx yy zz xy xz yz
//         elm_nodal_stress [ne][nn][6]  (with --nodal) cElmParam::NodalStress with extrapolation
//                                  (elc/elmparam.cpp:1304-1312, CompTRMatrix :1444-1535)
//       With --reactions, at the same state:
//         reactions [nnode][6]     cControl::SuppReactions (ctrl/ctrl.cpp:844-882)
//       With --geom, at the same state:
//         elm_G [ne][ndof][ndof]   cElmParam::GeomStiff (elc/elmparam.cpp:743-830)
//
//   fastref bench <deck> <pcg_iters> [reps] [pcg_iters2]
//       Times the reference CPU path on one host thread: StiffnessMatrix into
//       the deck's sparse matrix (cSymSprsMatrix, mlib/sysmat.cpp:889) once,
//       then [reps] (default 1) runs of <pcg_iters> iterations of PCGSolver
//       (mlib/sysmat.cpp:1061), each timed, each followed (when given) by a
//       run of <pcg_iters2> iterations.  Prints one JSON line.

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace std;

#include "input.h"
#include "ctrl.h"
#include "element.h"
#include "node.h"
#include "shape.h"
#include "shpiga.h"
#include "sysmat.h"
#include "vec.h"
#include "mat.h"
#include "gblvar.h"

// Globals owned by main/main.cpp in the reference program (main/main.cpp:37-42).
ifstream in;
ofstream out, outem;
string   fname;
bool     Feedback = false;
bool     Printing = false;

// Access to the protected controller statics.
struct CtrlAccess : public cControl
{
  static int     NEq(void)     { return NumEq; }
  static eSMType MatType(void) { return SysMatType; }
  static int*    Prof(void)    { return Profile; }
  static int     MaxIt(void)   { return MaxIter; }
  static double  Tolerance(void) { return Tol; }
};

// Matrix that records every Add in call order.
class cRecMatrix : public cSysMatrix
{
 public:
  vector<int> I, J;
  vector<double> V;
  explicit cRecMatrix(int n) : cSysMatrix(n) { }
  int    Symmetric(void) { return 1; }
  double Get(int, int) { return 0.0; }
  void   Add(int i, int j, double v) { I.push_back(i); J.push_back(j); V.push_back(v); }
  void   Print(void) { }
  void   MultVect(double *, double *) { }
};

// ------------------------------------------------------------------------
// Minimal tagged binary writer: "FREF" then records
//   u32 namelen, name, char dtype[4], u32 ndim, i64 shape[ndim], raw data.
class RecWriter
{
  FILE *fp;
 public:
  explicit RecWriter(const char *path) { fp = fopen(path, "wb"); if (!fp) { perror(path); exit(2); } fwrite("FREF", 1, 4, fp); }
  ~RecWriter() { if (fp) fclose(fp); }
  void put(const char *name, const char *dt, const vector<long long> &shape, const void *data, size_t bytes)
  {
    unsigned nl = (unsigned)strlen(name);
    fwrite(&nl, 4, 1, fp); fwrite(name, 1, nl, fp);
    char d[4] = {0, 0, 0, 0}; memcpy(d, dt, strlen(dt) < 4 ? strlen(dt) : 4); fwrite(d, 1, 4, fp);
    unsigned nd = (unsigned)shape.size(); fwrite(&nd, 4, 1, fp);
    for (long long s : shape) fwrite(&s, 8, 1, fp);
    if (bytes) fwrite(data, 1, bytes, fp);
  }
  void f8(const char *n, const vector<long long> &s, const double *p, size_t cnt) { put(n, "f8", s, p, cnt * 8); }
  void i4(const char *n, const vector<long long> &s, const int *p, size_t cnt) { put(n, "i4", s, p, cnt * 4); }
};

static void open_and_read(const string &deck)
{
  InitIGA( );
  fname = deck;
  string aux = deck + ".dat";
  in.open(aux.c_str( ));
  if (!in.is_open( )) { fprintf(stderr, "cannot open %s\n", aux.c_str( )); exit(2); }
  aux = deck + ".pos";
  out.open(aux.c_str( ));
  InpReadData( );
  InpCopyData( );
  in.close( );
  cControl::Init( );
}

static double now_s(void)
{
  return chrono::duration<double>(chrono::steady_clock::now( ).time_since_epoch( )).count( );
}

static int mode_dump(int argc, char **argv)
{
  string deck = argv[2];
  const char *outp = argv[3];
  bool trip = true, solve = true, mass = false, stress = false, geom = false, reac = false, nodal = false;
  const char *ufile = 0;
  double stol = -1.0;
  for (int a = 4; a < argc; a++)
  {
    string s = argv[a];
    if (s == "--no-triplets") trip = false;
    else if (s == "--no-solve") solve = false;
    else if (s == "--mass") mass = true;
    else if (s == "--stress") stress = true;
    else if (s == "--geom") geom = true;
    else if (s == "--reactions") reac = true;
    else if (s == "--nodal") nodal = true;
    else if (s == "--u" && a + 1 < argc) ufile = argv[++a];
    else if (s == "--solver-tol" && a + 1 < argc) stol = atof(argv[++a]);
  }

  // Keep the reference's console feedback (PCG progress) off stdout.
  streambuf *coutbuf = cout.rdbuf( );
  ofstream devnull("/dev/null");
  cout.rdbuf(devnull.rdbuf( ));

  open_and_read(deck);
  int neq = CtrlAccess::NEq( );
  RecWriter w(outp);
  w.i4("neq", {1}, &neq, 1);

  int nnode = cNode::GetNumNode( );
  vector<int> neqmap((size_t)nnode * 3), labels(nnode);
  for (int i = 0; i < nnode; i++)
  {
    cNode *nd = cNode::GetNode(i);
    labels[i] = nd->GetLabel( );
    for (int j = 0; j < 3; j++) neqmap[(size_t)i * 3 + j] = nd->GetDof(j);
  }
  w.i4("node_label", {nnode}, labels.data( ), labels.size( ));
  w.i4("node_eq", {nnode, 3}, neqmap.data( ), neqmap.size( ));

  if (ufile)
  {
    cVector u0(neq);
    FILE *fu = fopen(ufile, "rb");
    if (!fu || fread(u0.Val( ), 8, neq, fu) != (size_t)neq) { fprintf(stderr, "bad --u file\n"); return 2; }
    fclose(fu);
    cControl::AssignDispl(u0);
  }

  int ne = cElement::GetNumElm( );
  int ndof = ne > 0 ? cElement::GetElm(0)->GetNumElmDof( ) : 0;
  for (int e = 0; e < ne; e++)
    if (cElement::GetElm(e)->GetNumElmDof( ) != ndof) { fprintf(stderr, "mixed element sizes are not dumped\n"); return 2; }
  int maxdof = cElement::GetMaxDof( );
  cMatrix Ke(maxdof, maxdof), Me(maxdof, maxdof);
  cVector ge(maxdof);
  vector<int> dofs((size_t)ne * ndof), elab(ne);
  vector<double> KK((size_t)ne * ndof * ndof), GG((size_t)ne * ndof), MM;
  if (mass) MM.resize((size_t)ne * ndof * ndof);
  for (int e = 0; e < ne; e++)
  {
    cElement *elm = cElement::GetElm(e);
    elab[e] = elm->GetLabel( );
    elm->GetElmDofs(&dofs[(size_t)e * ndof]);
    elm->StiffMat(Ke);
    for (int i = 0; i < ndof; i++)
      for (int j = 0; j < ndof; j++) KK[((size_t)e * ndof + i) * ndof + j] = Ke[i][j];
    elm->IntForce(ge);
    for (int i = 0; i < ndof; i++) GG[(size_t)e * ndof + i] = ge[i];
    if (mass)
    {
      elm->MassMat(Me);
      for (int i = 0; i < ndof; i++)
        for (int j = 0; j < ndof; j++) MM[((size_t)e * ndof + i) * ndof + j] = Me[i][j];
    }
  }
  w.i4("elm_label", {ne}, elab.data( ), elab.size( ));
  w.i4("elm_dofs", {ne, ndof}, dofs.data( ), dofs.size( ));
  w.f8("elm_K", {ne, ndof, ndof}, KK.data( ), KK.size( ));
  w.f8("elm_g", {ne, ndof}, GG.data( ), GG.size( ));
  if (mass) w.f8("elm_M", {ne, ndof, ndof}, MM.data( ), MM.size( ));

  cVector f(neq);
  cControl::ExtLoadVector(f);
  w.f8("f", {neq}, f.Val( ), neq);

  if (trip)
  {
    cRecMatrix rec(neq);
    cControl::StiffnessMatrix(&rec);
    long long nt = (long long)rec.V.size( );
    w.i4("K_i", {nt}, rec.I.data( ), rec.I.size( ));
    w.i4("K_j", {nt}, rec.J.data( ), rec.J.size( ));
    w.f8("K_v", {nt}, rec.V.data( ), rec.V.size( ));
  }

  if (solve && !ufile)
  {
    cSysMatrix *K = cSysMatrix::CreateMatrix(CtrlAccess::MatType( ), neq, CtrlAccess::Prof( ));
    double tol = stol > 0 ? stol : CtrlAccess::Tolerance( );
    K->SetParam(CtrlAccess::MaxIt( ), tol);
    cControl::StiffnessMatrix(K);
    cVector u(neq);
    double t0 = now_s( );
    int ok = K->Solve(f, u);
    double t1 = now_s( );
    w.f8("u", {neq}, u.Val( ), neq);
    w.i4("solve_ok", {1}, &ok, 1);
    double ts = t1 - t0;
    w.f8("solve_seconds", {1}, &ts, 1);
    cControl::AssignDispl(u);
    cVector g(neq);
    cControl::IntForceVector(g);
    w.f8("g_of_u", {neq}, g.Val( ), neq);
    delete K;
  }
  if (stress && (ufile || solve))
  {
    const int nip = ne > 0 ? cElement::GetElm(0)->GetNumIntPnt( ) : 0;
    const int nen = ne > 0 ? cElement::GetElm(0)->GetShape( )->GetNumNode( ) : 0;
    vector<double> SE((size_t)ne * nip * 6), SS((size_t)ne * nip * 6), SN((size_t)ne * nen * 6);
    cMatrix Strain(nip, 6), Stress(nip, 6), Nodal(nen, 6);
    for (int e = 0; e < ne; e++)
    {
      cElement *elm = cElement::GetElm(e);
      if (elm->GetNumIntPnt( ) != nip) { fprintf(stderr, "mixed integration orders are not dumped\n"); return 2; }
      elm->IntPntStress(Strain, Stress);
      for (int i = 0; i < nip; i++)
        for (int k = 0; k < 6; k++)
        {
          SE[((size_t)e * nip + i) * 6 + k] = Strain[i][k];
          SS[((size_t)e * nip + i) * 6 + k] = Stress[i][k];
        }
      // extrapolated nodal stresses from the stresses just stored (the
      // printing step's cElmParam::NodalStress)
      if (nodal)
      {
        elm->NodalStress(Nodal);
        for (int a = 0; a < nen; a++)
          for (int k = 0; k < 6; k++) SN[((size_t)e * nen + a) * 6 + k] = Nodal[a][k];
      }
    }
    w.f8("elm_strain", {ne, nip, 6}, SE.data( ), SE.size( ));
    w.f8("elm_stress", {ne, nip, 6}, SS.data( ), SS.size( ));
    if (nodal) w.f8("elm_nodal_stress", {ne, nen, 6}, SN.data( ), SN.size( ));
  }
  if (reac && (ufile || solve))
  {
    // support reactions at the same state (cControl::SuppReactions): element
    // internal forces of the elements touching a support minus the loads
    // touching one, per node label and direction (all nodes, 6 columns)
    const int nnode = cNode::GetNumNode( );
    cMatrix R(nnode, 6);
    cControl::SuppReactions(R);
    vector<double> RR((size_t)nnode * 6);
    for (int i = 0; i < nnode; i++)
      for (int j = 0; j < 6; j++) RR[(size_t)i * 6 + j] = R(i, j);
    w.f8("reactions", {nnode, 6}, RR.data( ), RR.size( ));
  }
  if (geom && (ufile || solve))
  {
    // element geometric stiffness at the solved (or --u) state, the matrix
    // cControl::GeomStiffMatrix assembles for linear buckling
    const int nd = ne > 0 ? cElement::GetElm(0)->GetNumElmDof( ) : 0;
    vector<double> GE((size_t)ne * nd * nd);
    cMatrix Gelm(nd, nd);
    for (int e = 0; e < ne; e++)
    {
      cElement *elm = cElement::GetElm(e);
      elm->GeomStiff(Gelm);
      for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) GE[((size_t)e * nd + i) * nd + j] = Gelm[i][j];
    }
    w.f8("elm_G", {ne, nd, nd}, GE.data( ), GE.size( ));
  }
  cout.rdbuf(coutbuf);
  return 0;
}

static int mode_bench(int argc, char **argv)
{
  string deck = argv[2];
  int iters = argc > 3 ? atoi(argv[3]) : 5;
  int reps = argc > 4 ? atoi(argv[4]) : 1;
  int iters2 = argc > 5 ? atoi(argv[5]) : 0;
  if (reps < 1) reps = 1;
  streambuf *coutbuf = cout.rdbuf( );
  ofstream devnull("/dev/null");
  cout.rdbuf(devnull.rdbuf( ));

  double t0 = now_s( );
  open_and_read(deck);
  double t_read = now_s( ) - t0;
  int neq = CtrlAccess::NEq( );
  int ne = cElement::GetNumElm( );

  cVector f(neq);
  cControl::ExtLoadVector(f);
  cSysMatrix *K = cSysMatrix::CreateMatrix(SYM_SPARSE, neq, CtrlAccess::Prof( ));
  double t1 = now_s( );
  cControl::StiffnessMatrix(K);
  double t_asm = now_s( ) - t1;
  long long nnz_lower = K->GetNumElm( );

  // Element integration alone (no scatter), on the same elements.
  int maxdof = cElement::GetMaxDof( );
  cMatrix Ke(maxdof, maxdof);
  double t2 = now_s( );
  for (int e = 0; e < ne; e++) cElement::GetElm(e)->StiffMat(Ke);
  double t_int = now_s( ) - t2;

  // each rep runs PCGSolver with `iters` iterations and, when a second count
  // is given, once more with `iters2`: the difference separates the cost per
  // iteration from the solver's set-up (its diagonal read through Get)
  cVector u(neq);
  vector<double> t_pcg(reps), t_pcg2(iters2 > 0 ? reps : 0);
  for (int r = 0; r < reps; r++)
  {
    double t3 = now_s( );
    PCGSolver(iters, 1e-300, K, f, u);
    t_pcg[r] = now_s( ) - t3;
    if (iters2 > 0)
    {
      double t4 = now_s( );
      PCGSolver(iters2, 1e-300, K, f, u);
      t_pcg2[r] = now_s( ) - t4;
    }
  }
  cout.rdbuf(coutbuf);
  printf("{\"neq\": %d, \"ne\": %d, \"nnz_lower\": %lld, \"read_s\": %.6f, \"assembly_s\": %.6f, "
         "\"integration_s\": %.6f, \"pcg_iters\": %d, \"pcg_s\": %.6f, \"pcg_rep_s\": [",
         neq, ne, nnz_lower, t_read, t_asm, t_int, iters, t_pcg[0]);
  for (int r = 0; r < reps; r++) printf("%s%.6f", r ? ", " : "", t_pcg[r]);
  printf("], \"pcg_iters2\": %d, \"pcg_rep2_s\": [", iters2);
  for (size_t r = 0; r < t_pcg2.size( ); r++) printf("%s%.6f", r ? ", " : "", t_pcg2[r]);
  printf("]}\n");
  return 0;
}

int main(int argc, char **argv)
{
  ios_base::sync_with_stdio(false);
  if (argc >= 4 && string(argv[1]) == "dump") return mode_dump(argc, argv);
  if (argc >= 3 && string(argv[1]) == "bench") return mode_bench(argc, argv);
  fprintf(stderr, "usage: fastref dump <deck> <out.bin> [opts] | fastref bench <deck> <pcg_iters>\n");
  return 1;
}

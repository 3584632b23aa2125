// internal.h - private types of libfastgpu (not part of the C ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fast_gpu.h"

namespace fastgpu {

// Largest element supported by the integration kernels (hex20) and largest
// Gauss rule (4x4x4).
constexpr int kMaxNodes = 20;
constexpr int kMaxGauss = 64;

// Device-side solver scalars.  All scalars are FP64 even when the vectors
// are FP32; reductions are fixed-order, so a solve is bit-reproducible.
struct PcgState {
  double dot0;    // z.r of the current iterate
  double alpha;
  double beta;
  double lenf;    // |rhs| (the reference's normaliser, PCGSolver)
  double rr;      // r.r after the last update
  double err;     // sqrt(rr) / lenf
  double tol;
  double pw;      // p.w of the last iteration
  double err_true;  // |f - K u| / |f| at the last FP64 residual (mixed path)
  double best_err;  // smallest err_true so far (mixed path stagnation guard)
  int32_t iter;   // iterations completed
  int32_t done;   // 0 running, 1 converged, 2 iteration cap, 3 breakdown, 4 stagnation,
                  // 6 grid-barrier timeout (persistent kernel)
  int32_t maxit;
  int32_t updates;  // FP64 residual replacements (mixed path)
  int32_t null_rhs; // |f| < tol: the solution is u = 0 (PCGSolver returns at once)
  int32_t stall;    // FP64 residual replacements without a 2x improvement
  int32_t final;    // converged on the FP64 residual: later launches do nothing
  int32_t best;     // the last FP64 residual was the smallest so far (mixed path)
  uint32_t arrive_update;   // blocks finished in the fused update kernel (the last one commits)
  uint32_t arrive_dir;      // blocks finished in the fused direction kernel
  int32_t restarts_left;    // mixed path: fresh starts of the recurrence still allowed after a stall
  int32_t fresh;            // the last FP64 residual restarts the recurrence (p = z)
  int32_t restarts;         // fresh starts taken
  int32_t pad_;
};

// 32-bit words of one element's first-touch flags: nn*nn bits, rows padded
// to 16 bytes (bulk-copy size)
inline int first_words(int nn) { return (nn * nn + 127) / 128 * 4; }

struct Bucket {
  int type = 0;            // FAST_ELEM_*
  int nn = 0;              // nodes per element
  int ngp[3] = {0, 0, 0};
  int ng = 0;              // total Gauss points
  int64_t ne = 0;
  std::vector<int32_t> perm;       // colour-sorted position -> original element
  std::vector<int32_t> inv;        // original element -> colour-sorted position
  std::vector<int64_t> color_off;  // [ncolors+1] offsets in colour-sorted order
  std::vector<int32_t> h_conn;     // colour-sorted incidence
  std::vector<int32_t> h_slot;     // colour-sorted slot map (freed after upload)
  bool has_rho = false;
  int tl = 0;                      // 1: total-Lagrangian (St. Venant-Kirchhoff) formulation
  int32_t *d_conn = nullptr;       // [ne][nn] colour-sorted
  double *d_E = nullptr, *d_nu = nullptr, *d_rho = nullptr;
  int32_t *d_slot = nullptr;       // [ne][nn][nn] block index of node pair (a, b)
  double *d_dN = nullptr;          // [ng][nn][3] natural derivatives at the Gauss points
  double *d_N = nullptr;           // [ng][nn] shape functions
  double *d_w = nullptr;           // [ng] Gauss weights
  int64_t ne_regular = 0;          // colour-scheduled elements; the tied ones follow in perm order
  // first-touch flags (when Ctx::first_touch): per colour-sorted element
  // first_words(nn) words, bit a*nn+b set when the element is the first of the
  // stiffness assembly to write the block of its node pair (a, b)
  std::vector<uint32_t> h_first;
  uint32_t *d_first = nullptr;
  // launch shape chosen by fast_gpu_autotune (0: the occupancy-derived default)
  int tune_ctas = 0;               // FP64 element kernels: resident CTAs per SM at most
  int tune_split = 0;              // B-spline FP64 kernels: CTAs sharing one element at most
  int tune_tc_ctas = 0;            // tensor-core element kernels: resident CTAs per SM at most
  int tune_kernel = 0;             // FP64 hex stiffness: 0 CTA per element, 1 warp per element (elem_warp.cu)
  // B-spline solids (FAST_ELEM_BSP_SOLID)
  int pd[3] = {0, 0, 0};           // degree per direction
  int rational = 0;
  int nspan[3] = {0, 0, 0};
  int32_t *d_span = nullptr;       // [ne][4] colour-sorted spans per direction (4th unused)
  double *d_bas = nullptr;         // per direction d at offset bas_off[d]: [nspan][ngp_d][p+1][2] (N, dN/dt)
  int64_t bas_off[3] = {0, 0, 0};
  double *d_wt = nullptr;          // [nnode] control-point weights (rational patches)
  // nodal stress recovery (built on first use): extrapolation matrix and the
  // node -> (element, local node) incidence in element order
  double *d_tr = nullptr;          // [nn][ng]
  int64_t *d_nptr = nullptr;       // [nnode+1]
  int64_t *d_nent = nullptr;       // [ne*nn] entries k*nn + a, ascending k per node
};

// Elements that touch a tied (slave) node.  Their element matrices go to a
// scratch buffer and are scattered as T_e^T K_e T_e onto their expanded node
// list (the non-slave nodes plus the masters of their slave nodes).
struct TiedSet {
  int64_t n = 0;                          // tied elements
  std::vector<int64_t> color_off;         // [ncolors+1] over colour-sorted tied elements
  std::vector<int64_t> h_nptr;            // [n+1] offsets into h_nodes (expanded node lists)
  std::vector<int32_t> h_nodes;
  std::vector<int64_t> h_sptr;            // [n+1] offsets into h_slot (m_e^2 block slots, row-major)
  std::vector<int32_t> h_slot;
  std::vector<int64_t> h_pptr;            // [h_nodes.size()+1] pre-image of each expanded node
  std::vector<int32_t> h_pa;              //   local node of the element
  std::vector<double> h_pt;               //   weight (1 for a non-slave node)
  std::vector<int64_t> h_keoff;           // [n] element matrix offset in the scratch buffer
  std::vector<int64_t> h_eptr;            // [n+1] offsets into h_econn
  std::vector<int32_t> h_econn;           //   each tied element's own nodes, local order
  std::vector<int32_t> h_nn;              // [n] nodes per element
  int64_t ke_total = 0;
  std::vector<std::vector<int32_t>> bucket_pos;  // per bucket: colour-sorted positions, scratch order
  std::vector<int64_t> bucket_keoff;             // per bucket: first scratch offset
  int64_t *d_nptr = nullptr, *d_sptr = nullptr, *d_pptr = nullptr, *d_keoff = nullptr, *d_eptr = nullptr;
  int32_t *d_econn = nullptr;
  int32_t *d_nodes = nullptr, *d_slot = nullptr, *d_pa = nullptr, *d_nn = nullptr;
  double *d_pt = nullptr, *d_ke = nullptr;
  std::vector<int32_t *> d_bucket_pos;
};

// Slave / master maps of the ties, for the load restriction T^T f and the
// displacement prolongation u_s = sum w u_m (gather forms, deterministic).
struct TieMaps {
  int64_t nslave = 0, nmaster = 0;
  int32_t *d_slave = nullptr;   // [nslave]
  int64_t *d_sptr = nullptr;    // [nslave+1]
  int32_t *d_smaster = nullptr; // masters of each slave
  double *d_sw = nullptr;
  int32_t *d_master = nullptr;  // [nmaster] distinct master nodes
  int64_t *d_mptr = nullptr;    // [nmaster+1]
  int32_t *d_mslave = nullptr;  // slaves of each master
  double *d_mw = nullptr;
};

struct PersistPlanHost;  // elem_persist.cu

struct Ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t side_stream = nullptr;  // captures the bodies of conditional graph nodes
  std::string err;
  int sm_count = 148;

  // mesh
  int64_t nnode = 0;
  int32_t neq = 0;
  std::vector<int32_t> h_eq;      // [nnode*3] 1-based, 0 fixed
  std::vector<int32_t> h_dof_of_eq;  // [neq] node-DOF index 3*n+i of equation k+1 (unpadded)
  double *d_X = nullptr;          // [nnode][3]
  uint8_t *d_fix = nullptr;       // [nnode] bit i set: DOF i has no equation
  int32_t *d_dof_of_eq = nullptr; // [neq] padded vector index 4*n+i of equation k+1
  std::vector<Bucket> buckets;
  // face tractions on the device (fast_gpu_set_face_loads)
  int32_t nface = 0, nfn = 0, face_ngp = 0, nfnode = 0;
  int32_t *d_fn = nullptr, *d_floc = nullptr;    // [nface][nfn] nodes, [nface] Local flags
  double *d_fq = nullptr, *d_fe = nullptr;       // [nface][3] tractions, [nface][nfn][3] face forces
  int32_t *d_fnode = nullptr, *d_feq = nullptr;  // [nfnode] loaded nodes, [nfnode][3] their equations
  int32_t *d_fptr = nullptr, *d_fidx = nullptr;  // [nfnode+1] / [nface*nfn]: face-node entries per node
  // tied interfaces
  std::vector<int64_t> h_tslave, h_tptr, h_tmaster;  // copies of fast_gpu_ties
  std::vector<double> h_tweight;
  std::vector<int32_t> h_slave_of;                   // [nnode] tie index of a slave node, -1 otherwise
  TiedSet tied;
  TieMaps tmaps;
  bool has_ties() const { return !h_tslave.empty(); }

  // node-block (3x3) CSR pattern, full (both triangles)
  int64_t nnzb = 0;
  std::vector<int32_t> h_rowptr, h_col, h_diag;
  int32_t *d_rowptr = nullptr, *d_col = nullptr, *d_diag = nullptr;
  // solve layout: each block-row padded to a multiple of 4 blocks, so its
  // structure-of-arrays segments start on 16-byte boundaries (vector loads)
  int64_t nnzb_pad = 0;
  std::vector<int32_t> h_srow, h_scol;
  int32_t *d_srow = nullptr, *d_scol = nullptr;
  int32_t ncolors = 0;
  double pattern_seconds = 0.0;
  int64_t nnz_lower_eq = 0;

  // assembled matrices: [nnzb][3][3] blocks (assembly target, AoS)
  double *d_K = nullptr, *d_M = nullptr;
  // FP32 stiffness from the tensor cores (FAST_ASM_STIFFNESS_TF32), same layout;
  // while K32_current is set it is the stiffness of the context: the FP64 slot
  // is stale and the mixed solve takes its FP64 residuals element by element
  float *d_K32 = nullptr;
  bool K32_current = false;
  // solve copies in row-local SoA layout (FP64 and FP32), rebuilt after each assembly
  double *d_Ks = nullptr, *d_Ms = nullptr;
  float *d_Ks32 = nullptr;
  bool K_ok = false, M_ok = false, Ks_ok = false, Ms_ok = false;
  int32_t *d_status = nullptr;    // device error flags (detJ)
  int32_t *h_status = nullptr;    // pinned

  // nodal displacement state (TL tangent, internal force) and internal force
  double *d_disp = nullptr;       // [nnode][4]
  double *d_gint = nullptr;       // [nnode][4]
  // solver workspace: node vectors padded to 4 entries (x, y, z, 0) per node
  double *d_u = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr, *d_w = nullptr, *d_f = nullptr;
  double *d_p2 = nullptr;         // second search-direction buffer (persistent PCG)
  double *d_dinv = nullptr;       // [nnode][3][4] inverse diagonal (Jacobi) or inverse 3x3 block
  double *d_ubest = nullptr;      // mixed path: FP64 iterate with the smallest true residual
  float *s_x = nullptr, *s_r = nullptr, *s_z = nullptr, *s_p = nullptr, *s_w = nullptr;
  float *s_p2 = nullptr;
  float *s_dinv = nullptr;        // [nnode][3][4]
  int precond_built = -1;         // which preconditioner d_dinv holds
  double *d_partials = nullptr;   // reduction partials [2][kRedBlocks]
  PcgState *d_state = nullptr;
  PcgState *h_state = nullptr;    // pinned
  double *d_eq_tmp = nullptr;     // [neq] staging for host <-> device in equation space
  double *h_eq_tmp = nullptr;     // pinned [neq]

  int64_t launches = 0;          // kernels launched by this context (all entry points)

  // independent problems in one mesh (fast_gpu_set_problems)
  int32_t nprob = 0;
  std::vector<int64_t> h_noff;    // [nprob+1] node offsets
  int64_t *d_noff = nullptr;
  int32_t *d_order = nullptr;     // problems by size, largest first
  int32_t *d_piters = nullptr, *d_pdone = nullptr;
  double *d_perr = nullptr;

  // persistent PCG: systems with at most persist_max_nodes nodes run each
  // chunk of iterations as one cooperative kernel (grid barriers in d_bar)
  int64_t persist_max_nodes = 65536;
  // SpMV lanes per block-row (4, 8, 16 or 32): FP32 takes 4 blocks and FP64 2
  // blocks per lane trip; defaults measured best on a hex20 box (64 blocks per
  // padded row), fast_gpu_autotune measures them on the system at hand
  int lpr32 = 8, lpr64 = 16;
  // Newmark steps and Newton iterations replayed as captured CUDA graphs
  bool graph_steps = true;
  // FP32 SpMV with the matrix streamed through shared memory by bulk copies
  // (spmv_f32_bulk): its row tiles, their largest value / column bytes and grid
  bool spmv32_bulk = false;
  bool spmv32_stream = false;   // FP32 SpMV with cache-streaming matrix loads (8 or 16 lanes)
  bool spmv32_c16 = false;      // FP32 SpMV with 16-bit column offsets (8 or 16 lanes)
  uint16_t *d_scol16 = nullptr; // [nnzb_pad] column offsets from the row's smallest column
  int32_t *d_rowbase = nullptr; // [nnode] that column
  // internal force element by element, then gathered per node (every bucket a
  // hex bucket): element forces [bucket][colour-sorted element][nn][3] at
  // elem_g_off[bucket], and per node the offsets of its elements' entries in
  // bucket, then colour order (the order the colour-by-colour scatter adds
  // them in, so both give the same bits)
  bool force_gather = false;      // available for this mesh
  bool use_force_gather = true;   // FAST_OPT_FORCE_GATHER
  double *d_elem_g = nullptr;
  int64_t *d_gptr = nullptr;      // [nnode + 1]
  int64_t *d_ginc = nullptr;      // [sum of elements x nn]
  std::vector<int64_t> elem_g_off;
  // widest launch shape the element kernels could take since last reset
  // (read by the autotuner to bound its candidates)
  int elem_occ = 0, elem_split_max = 0;
  // the stiffness assembly initialises every block by its first writer (no
  // zero fill; set by the pattern build where that covers every block)
  bool first_touch = false;
  bool zero_fill = false;  // option: zero-fill K all the same
  // the tensor-core stiffness of all buckets in one persistent launch (option)
  bool persist_asm = false;
  PersistPlanHost *persist = nullptr;   // its work list, built on first use
  bool persist_first = false;           // first-touch flags in the work list's arguments
  bool use_first_touch() const { return first_touch && !zero_fill; }
  int32_t *d_tile_row = nullptr;
  int bulk_ntiles = 0, bulk_vbytes = 0, bulk_cbytes = 0, bulk_grid = 0;
  int persist_grid = 0;           // blocks of that kernel (0: not yet sized)
  void *d_bar = nullptr;          // grid barrier words (kBarrierBytes)
  static constexpr size_t kBarrierBytes = 8192;

  // CUDA graphs of one chunk of PCG iterations (captured once, replayed)
  cudaGraphExec_t graph_fp64 = nullptr, graph_mixed = nullptr;
  int graph_fp64_chunk = 0, graph_mixed_chunk = 0;
  int64_t graph_fp64_kernels = 0, graph_mixed_kernels = 0;
  void drop_graphs() {
    if (graph_fp64) cudaGraphExecDestroy(graph_fp64);
    if (graph_mixed) cudaGraphExecDestroy(graph_mixed);
    graph_fp64 = graph_mixed = nullptr;
  }

  // live kernel timing: CUDA events around SpMV launches, assemblies, the
  // learned predictor, internal forces and linear solves (the FAST_KERNEL_*
  // kinds), harvested at each host sync; spans may nest
  static constexpr int kSpanKinds = 8;
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  struct Span { int kind; int64_t id; bool closed; cudaEvent_t a, b; };
  std::vector<Span> spans;
  int64_t span_ids = 0;
  double kt_ms[kSpanKinds] = {};
  int64_t kt_n[kSpanKinds] = {};
  cudaEvent_t take_event();
  int64_t begin_span(int kind);   // span id, -1 when timing is off
  void end_span(int64_t id = -1); // -1: the most recent open span
  void harvest();                 // closed spans only (call after a stream sync)

  bool set_error(const std::string &m) { err = m; return false; }
};

// Resident CTAs per SM of one element-kernel launch: the occupancy `occ`,
// capped by a tuned shape `cap` (0 = none); the widest occupancy seen is kept
// for the autotuner.
inline int elem_per_sm(Ctx &c, int occ, int cap) {
  if (occ < 1) occ = 1;
  if (occ > c.elem_occ) c.elem_occ = occ;
  return (cap > 0 && cap < occ) ? cap : occ;
}

// pattern.cpp
bool build_pattern(Ctx &c, const fast_gpu_mesh &m);

// shape tables (shape_tables.cpp)
bool gauss_rule(int n, double *r, double *w);
void gauss_point_tables(int type, const int ngp[3], std::vector<double> &N, std::vector<double> &dN,
                        std::vector<double> &w);
// stress extrapolation TR [nn][ng] of a hex type and Gauss rule
bool extrapolation_matrix(int type, const int ngp[3], std::vector<double> &TR, const int *pd = nullptr);
int nodes_of(int type);
// B-spline solid kernels exist for these (degree per direction, Gauss order)
bool bsp_supported(const int pd[3], int ngp);
// ... and total-Lagrangian tangents / internal forces (bsp_tl.cu)
bool bsp_tl_supported(const int pd[3], int ngp);
// nodes per element of a bucket description (B-spline solids: product of p+1); 0 = unsupported
int bucket_nodes(const fast_gpu_bucket &bk);
// Per-span univariate basis tables of one patch direction at the Gauss
// points: out[(s * ng + g) * (p + 1) + i] = {N_i, dN_i/dt} of span s.  False
// when the knot vector is not a valid open or clamped vector of this degree.
bool bspline_gauss_tables(int p, int nknots, const double *knots, int ng, int &nspan, std::vector<double> &out);

// kernels (elem_kernels.cu / solve_kernels.cu); all launched on c.stream
cudaError_t launch_zero_matrix(Ctx &c, double *K, bool identity_on_fixed);
// 1 on the diagonal of every fixed DOF (the stiffness slot's convention)
cudaError_t launch_fixed_identity(Ctx &c, double *K);
cudaError_t launch_assemble(Ctx &c, int what, double *target);
// elem_warp.cu: FP64 hex stiffness with one warp per element (one colour)
struct ElemArgs;
bool warp_supported(const Bucket &B);
cudaError_t launch_warp_elements(Ctx &c, const Bucket &B, ElemArgs a, int64_t count);
// the small-strain stiffness of one bucket, every colour (no tied elements)
cudaError_t launch_assemble_bucket(Ctx &c, size_t b, double *target);
// device face loads (face_loads.cu)
void free_face_loads(Ctx &c);
// tied interfaces (ties.cu)
cudaError_t upload_ties(Ctx &c);
void free_ties(Ctx &c);
cudaError_t launch_tied_element_matrices(Ctx &c);   // dense K_e of every tied element into the scratch buffer
cudaError_t launch_tied_assemble(Ctx &c, double *K);
// the tied elements into the FP32 tensor-core stiffness: their FP64 element
// matrices (the scratch buffer) scattered as T_e^T K_e T_e in FP32
cudaError_t launch_tied_assemble32(Ctx &c, float *K32);
// G += K_e u_e of every tied element (node space, u with its slave values,
// from the scratch buffer of the last assembly), every DOF of the element
// (slave DOFs feed the restriction; fixed ones are zeroed by the caller);
// nothing is done while *skip is non-zero
cudaError_t launch_tied_matvec(Ctx &c, const double *u, double *G, const int32_t *skip);
cudaError_t launch_tie_restrict(Ctx &c, double *f);  // f <- T^T f (padded node layout)
cudaError_t launch_tie_zero(Ctx &c, double *v);      // v[slave DOFs] = 0
// v[DOFs without an equation] = 0 (supports and slaves); nothing while *skip
cudaError_t launch_zero_fixed(Ctx &c, double *v, const int32_t *skip);
cudaError_t launch_tie_prolong(Ctx &c, double *u);   // u[slave] = sum w u[master]
cudaError_t launch_element_matrices(Ctx &c, int what, int bucket, int64_t first_sorted, int64_t count,
                                    double *d_out);

// geom.cu: G += sign * geometric stiffness at c.d_disp (small-strain hex
// buckets, colour by colour; fixed rows and columns untouched)
cudaError_t launch_geom_stiffness(Ctx &c, double *G, double sign);

// tl_kernels.cu
cudaError_t launch_tl(Ctx &c, double *K, double *G, bool want_k, bool want_g);
// the same at the nodal displacements U ([nnode][4]); every launch does
// nothing while *skip (a device flag, may be null) is non-zero
cudaError_t launch_tl_at(Ctx &c, double *K, double *G, bool want_k, bool want_g, const double *U, const int32_t *skip);

// elem_tc.cu: stiffness on the tensor cores (TF32 operands split in three, FP32 blocks), small-strain hex buckets
bool tc_supported(const Bucket &B);
// B-spline degrees / rules of the tensor-core kernel (and of the mass kernel)
bool bsp_tc_supported(const int pd[3], int ngp);
cudaError_t launch_assemble_tc(Ctx &c, float *K32);
// one bucket of it, every colour (no zeroing, no tied elements)
cudaError_t launch_assemble_tc_bucket(Ctx &c, size_t b, float *K32);
// elem_persist.cu: the regular elements of every bucket into K32 in one
// cooperative launch, and whether the mesh's buckets allow it
cudaError_t launch_persist_elements(Ctx &c, float *K32);
bool persist_supported(const Ctx &c);
void free_persist_plan(Ctx &c);
cudaError_t launch_element_matrices_tc(Ctx &c, int bucket, int64_t count, double *d_out_and_index);
cudaError_t launch_tl_element(Ctx &c, int what, int bucket, int64_t count, double *d_out_and_index);

constexpr int kRedBlocks = 592;   // fixed reduction grid: 4 x 148 SMs
cudaError_t launch_build_precond(Ctx &c, const double *K, int precond);
// the same from the FP32 blocks of the tensor-core stiffness
cudaError_t launch_build_precond32(Ctx &c, const float *K32, int precond);
// row tiles of the bulk-staged FP32 SpMV (once per pattern)
cudaError_t ensure_bulk_tiles(Ctx &c);
// 16-bit column offsets of the FP32 SpMV (once per pattern; not supported when
// a block-row spans 65,536 nodes or more)
cudaError_t ensure_col16(Ctx &c);
// FP32 blocks -> the FP32 row-local SoA copy
cudaError_t launch_to_soa32(Ctx &c, const float *K32, float *Ks32);
// r = f - K u in FP64 without the assembled matrix: the small-strain internal
// force of every element at u (K u for a linear elastic solid), tie
// restriction / prolongation included; r.r per block into part[spmv grid];
// nothing is done while *skip is non-zero
cudaError_t launch_matfree_residual(Ctx &c, const double *f, const double *u, double *r, double *part,
                                    const int32_t *skip);
// AoS blocks -> row-local SoA copies (either output may be null)
cudaError_t launch_to_soa(Ctx &c, const double *K, double *Ks, float *Ks32);
// PCG on the padded node vectors c.d_f -> c.d_u; state left in c.h_state
cudaError_t pcg_fp64(Ctx &c, bool warm, double tol, int maxit, int chunk, int iter0 = 0);
cudaError_t pcg_mixed(Ctx &c, bool warm, double tol, int maxit, int chunk);
// Records a whole solve of c.d_f -> c.d_u (kernel-per-step form: the
// preconditioner and solve copies must be current) into the graph being
// captured on c.stream: the initialisation, then a WHILE conditional node
// whose body is `chunk` iterations (plus the FP64 residual replacement of the
// mixed path) and a kernel that keeps the loop going while the state is
// running.  The tolerance is read from tol_dev when that is not null.  The
// loop ends at the state's maxit at the latest (the kernels stop there).
cudaError_t record_pcg(Ctx &c, bool mixed, bool warm, double tol, const double *tol_dev, int maxit, int chunk);
constexpr int kDoneBarrierTimeout = 6;  // PcgState::done: a grid-barrier wait ran out
// one CTA per independent problem (node ranges d_noff), FP64 Jacobi/block PCG on c.d_Ks
// from c.d_f into c.d_u; per problem: iterations, |r|/|f| and done (1 conv, 2 cap, 3 breakdown)
// padded row-local SoA copies of K (what = FAST_ASM_STIFFNESS, FP32 too when fp32) or M, rebuilt if stale
cudaError_t solve_layout(Ctx &c, int what, bool fp32);
// the values of K (FAST_ASM_STIFFNESS) or M changed: drop their solve copies and preconditioner
void matrix_changed(Ctx &c, int what);
// solve K u = f on the node-padded vectors c.d_f -> c.d_u (c.d_u is the first iterate when warm);
// returns a FAST_GPU_* status
int solve_nodes(Ctx &c, const fast_gpu_solve_opts *o, bool warm, fast_gpu_solve_report *rep);
cudaError_t launch_pcg_batch(Ctx &c, int nprob, const int32_t *d_order, const int64_t *d_noff, double tol, int maxit,
                             bool warm, int32_t *d_iters, double *d_errs, int32_t *d_done);
cudaError_t launch_residual(Ctx &c, const double *Ks, const double *f, const double *u, double *r,
                            double *rr_out_dev);
cudaError_t launch_spmv(Ctx &c, const double *Ks, const double *x, double *y);
cudaError_t launch_spmv32(Ctx &c, const float *Ks, const float *x, float *y);
cudaError_t launch_eq_to_node(Ctx &c, const double *eqv, double *nodev);
cudaError_t launch_node_to_eq(Ctx &c, const double *nodev, double *eqv);
cudaError_t launch_norm2(Ctx &c, const double *x, int64_t n, double *out_dev);

}  // namespace fastgpu

// fast_gpu.cu - the C ABI of libfastgpu.so (declared in include/fast_gpu.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess) {                                                          \
      c->err = std::string(#call) + ": " + cudaGetErrorString(_e);                    \
      return FAST_GPU_ECUDA;                                                          \
    }                                                                                 \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void **)p, sizeof(T) * count);
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void free_mesh(Ctx &c) {
  c.drop_graphs();
  for (Bucket &B : c.buckets) {
    dfree(B.d_conn); dfree(B.d_E); dfree(B.d_nu); dfree(B.d_rho); dfree(B.d_slot); dfree(B.d_first);
    dfree(B.d_dN); dfree(B.d_N); dfree(B.d_w);
    dfree(B.d_span); dfree(B.d_bas); dfree(B.d_wt);
    dfree(B.d_tr); dfree(B.d_nptr); dfree(B.d_nent);
  }
  free_persist_plan(c);
  c.buckets.clear();
  free_ties(c);
  free_face_loads(c);
  dfree(c.d_X); dfree(c.d_fix); dfree(c.d_dof_of_eq); dfree(c.d_scol16); dfree(c.d_rowbase);
  dfree(c.d_elem_g); dfree(c.d_gptr); dfree(c.d_ginc);
  c.force_gather = false;
  c.elem_g_off.clear();
  c.spmv32_c16 = false;
  dfree(c.d_rowptr); dfree(c.d_col); dfree(c.d_diag); dfree(c.d_srow); dfree(c.d_scol);
  dfree(c.d_tile_row);
  c.bulk_ntiles = 0;
  c.spmv32_bulk = false;
  dfree(c.d_K); dfree(c.d_M); dfree(c.d_Ks); dfree(c.d_Ms); dfree(c.d_Ks32);
  dfree(c.d_u); dfree(c.d_r); dfree(c.d_z); dfree(c.d_p); dfree(c.d_w); dfree(c.d_f); dfree(c.d_dinv);
  dfree(c.d_p2); dfree(c.s_p2);
  dfree(c.d_ubest);
  dfree(c.s_x); dfree(c.s_r); dfree(c.s_z); dfree(c.s_p); dfree(c.s_w); dfree(c.s_dinv);
  dfree(c.d_eq_tmp);
  dfree(c.d_disp); dfree(c.d_gint);
  if (c.h_eq_tmp) cudaFreeHost(c.h_eq_tmp);
  c.h_eq_tmp = nullptr;
  c.K_ok = c.M_ok = c.Ks_ok = c.Ms_ok = false;
  c.precond_built = -1;
  for (void *p : {(void *)c.d_noff, (void *)c.d_order, (void *)c.d_piters, (void *)c.d_pdone, (void *)c.d_perr})
    if (p) cudaFree(p);
  c.d_noff = nullptr; c.d_order = nullptr; c.d_piters = nullptr; c.d_pdone = nullptr; c.d_perr = nullptr;
  c.nprob = 0;
  c.h_noff.clear();
  c.nnode = 0;
  c.neq = 0;
  c.nnzb = 0;
}

int check_ctx(const fast_gpu_ctx *c) { return c ? FAST_GPU_OK : FAST_GPU_EINVAL; }

cudaError_t ensure_soa(Ctx &c, int what, bool fp32);

double *target_of(Ctx &c, int what) {
  if (what == FAST_ASM_STIFFNESS) return c.d_K;
  if (what == FAST_ASM_MASS) return c.d_M;
  return nullptr;
}

void invalidate(Ctx &c, int what) {
  if (what == FAST_ASM_STIFFNESS) { c.Ks_ok = false; c.precond_built = -1; }
  else c.Ms_ok = false;
}

// row-local SoA copies for the solve (FP64, and FP32 when asked)
cudaError_t ensure_soa(Ctx &c, int what, bool fp32) {
  cudaError_t e = cudaSuccess;
  // padded rows: the padding values are zeroed once at allocation and never written
  const size_t nv = (size_t)9 * c.nnzb_pad;
  if (what == FAST_ASM_MASS) {
    if (!c.d_Ms) {
      if ((e = cudaMalloc((void **)&c.d_Ms, sizeof(double) * nv)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(c.d_Ms, 0, sizeof(double) * nv, c.stream)) != cudaSuccess) return e;
    }
    if (!c.Ms_ok) { e = launch_to_soa(c, c.d_M, c.d_Ms, nullptr); c.Ms_ok = (e == cudaSuccess); }
    return e;
  }
  if (c.K32_current) {
    // the tensor-core stiffness: FP32 copy only (there is no FP64 stiffness)
    if (!fp32) return cudaErrorInvalidValue;
    if (!c.d_Ks32) {
      if ((e = cudaMalloc((void **)&c.d_Ks32, sizeof(float) * nv)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(c.d_Ks32, 0, sizeof(float) * nv, c.stream)) != cudaSuccess) return e;
      c.Ks_ok = false;
    }
    if (!c.Ks_ok) {
      e = launch_to_soa32(c, c.d_K32, c.d_Ks32);
      c.Ks_ok = (e == cudaSuccess);
    }
    return e;
  }
  if (!c.d_Ks) {
    if ((e = cudaMalloc((void **)&c.d_Ks, sizeof(double) * nv)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(c.d_Ks, 0, sizeof(double) * nv, c.stream)) != cudaSuccess) return e;
  }
  if (fp32 && !c.d_Ks32) {
    if ((e = cudaMalloc((void **)&c.d_Ks32, sizeof(float) * nv)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(c.d_Ks32, 0, sizeof(float) * nv, c.stream)) != cudaSuccess) return e;
    c.Ks_ok = false;
  }
  if (!c.Ks_ok) {
    // the FP32 copy is always refreshed with the FP64 one once it exists
    e = launch_to_soa(c, c.d_K, c.d_Ks, c.d_Ks32);
    c.Ks_ok = (e == cudaSuccess);
  }
  return e;
}

// (eq i, eq j) 0-based -> flat value index in the block matrix, or -1
int64_t value_index(const Ctx &c, int32_t i, int32_t j) {
  if (i < 0 || j < 0 || i >= c.neq || j >= c.neq) return -1;
  const int32_t di = c.h_dof_of_eq[i], dj = c.h_dof_of_eq[j];
  const int32_t ni = di / 3, pi = di % 3, nj = dj / 3, pj = dj % 3;
  const int32_t *b0 = c.h_col.data() + c.h_rowptr[ni], *b1 = c.h_col.data() + c.h_rowptr[ni + 1];
  const int32_t *p = std::lower_bound(b0, b1, nj);
  if (p == b1 || *p != nj) return -1;
  return (int64_t)(p - c.h_col.data()) * 9 + pi * 3 + pj;
}

// dst += a src over 9 * nnzb block entries (both slots share the pattern)
__global__ void add_mat_kernel(int64_t n, double a, const double *__restrict__ src, double *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = dst[i] + a * src[i];
}

}  // namespace

namespace fastgpu {
cudaError_t solve_layout(Ctx &c, int what, bool fp32) { return ensure_soa(c, what, fp32); }
void matrix_changed(Ctx &c, int what) { invalidate(c, what); }
}  // namespace fastgpu

extern "C" {

int fast_gpu_version(void) { return FAST_GPU_ABI_VERSION; }

int fast_gpu_create(int device, fast_gpu_ctx **out) {
  if (!out) return FAST_GPU_EINVAL;
  *out = nullptr;
  fast_gpu_ctx *c = new (std::nothrow) fast_gpu_ctx();
  if (!c) return FAST_GPU_ENOMEM;
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_status, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_status, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_state, sizeof(PcgState) * 2);
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_state, sizeof(PcgState) * 2);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_partials, sizeof(double) * 16384);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_bar, Ctx::kBarrierBytes);
  if (e == cudaSuccess) e = cudaMemset(c->d_bar, 0, Ctx::kBarrierBytes);
  if (e == cudaSuccess) {
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (!coop) c->persist_max_nodes = 0;
  }
  if (e != cudaSuccess) {
    delete c;
    return FAST_GPU_ECUDA;
  }
  c->stream = c->own_stream;
  *out = c;
  return FAST_GPU_OK;
}

int fast_gpu_set_option(fast_gpu_ctx *c, int32_t option, int64_t value) {
  if (!c) return FAST_GPU_EINVAL;
  if (option == FAST_OPT_PERSISTENT_MAX_NODES) {
    if (value < 0) return FAST_GPU_EINVAL;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
    c->persist_max_nodes = coop ? value : 0;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_SPMV_LANES_FP32 || option == FAST_OPT_SPMV_LANES_FP64) {
    if (value != 4 && value != 8 && value != 16 && value != 32) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    c->drop_graphs();  // captured iterations hold the old launch shape
    (option == FAST_OPT_SPMV_LANES_FP32 ? c->lpr32 : c->lpr64) = (int)value;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_SPMV_BULK_FP32) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    if (value) CK(ensure_bulk_tiles(*c));
    c->drop_graphs();
    c->spmv32_bulk = value != 0;
    if (value) c->spmv32_stream = c->spmv32_c16 = false;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_GRAPH_STEPS) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    c->graph_steps = value != 0;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_SPMV_STREAM_FP32) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    c->drop_graphs();
    c->spmv32_stream = value != 0;
    if (value) c->spmv32_bulk = c->spmv32_c16 = false;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_SPMV_COL16_FP32) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    if (value) {
      if (!c->d_K) return FAST_GPU_ESTATE;
      const cudaError_t e = ensure_col16(*c);
      if (e == cudaErrorNotSupported) { c->err = "set_option: a block-row spans 65,536 nodes or more"; return FAST_GPU_ENOTSUP; }
      CK(e);
    }
    c->drop_graphs();
    c->spmv32_c16 = value != 0;
    if (value) c->spmv32_bulk = c->spmv32_stream = false;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_FORCE_GATHER) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    c->drop_graphs();
    c->use_force_gather = value != 0;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_PERSISTENT_ASSEMBLY) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    c->persist_asm = value != 0;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_ZERO_FILL) {
    if (value != 0 && value != 1) return FAST_GPU_EINVAL;
    c->zero_fill = value != 0;
    return FAST_GPU_OK;
  }
  if (option == FAST_OPT_ELEM_SHAPE) {
    const int64_t b = (value >> 24) & 0xFF, kern = value >> 32;
    if (value < 0 || b >= (int64_t)c->buckets.size() || kern < 0 || kern > 1) return FAST_GPU_EINVAL;
    if (kern == 1 && !warp_supported(c->buckets[(size_t)b])) return FAST_GPU_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    c->drop_graphs();
    Bucket &B = c->buckets[(size_t)b];
    B.tune_ctas = (int)(value & 0xFF);
    B.tune_split = (int)((value >> 8) & 0xFF);
    B.tune_tc_ctas = (int)((value >> 16) & 0xFF);
    B.tune_kernel = (int)kern;
    return FAST_GPU_OK;
  }
  return FAST_GPU_EINVAL;
}

int fast_gpu_destroy(fast_gpu_ctx *c) {
  if (!c) return FAST_GPU_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_mesh(*c);
  dfree(c->d_status);
  if (c->h_status) cudaFreeHost(c->h_status);
  dfree(c->d_state);
  if (c->h_state) cudaFreeHost(c->h_state);
  dfree(c->d_partials);
  if (c->d_bar) cudaFree(c->d_bar);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  if (c->side_stream) cudaStreamDestroy(c->side_stream);
  delete c;
  return FAST_GPU_OK;
}

const char *fast_gpu_last_error(const fast_gpu_ctx *c) { return c ? c->err.c_str() : "null context"; }

int fast_gpu_set_stream(fast_gpu_ctx *c, void *s) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  c->stream = s ? (cudaStream_t)s : c->own_stream;
  return FAST_GPU_OK;
}

int fast_gpu_synchronize(fast_gpu_ctx *c) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  CK(cudaStreamSynchronize(c->stream));
  return FAST_GPU_OK;
}

int fast_gpu_upload_mesh(fast_gpu_ctx *c, const fast_gpu_mesh *m) {
  if (check_ctx(c) || !m || m->num_nodes <= 0 || !m->coords || !m->node_eq || m->num_buckets <= 0 || !m->buckets) {
    if (c) c->err = "upload_mesh: invalid mesh description";
    return FAST_GPU_EINVAL;
  }
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  free_mesh(*c);
  const int64_t nnode = m->num_nodes;
  c->nnode = nnode;
  c->neq = m->num_eq;
  c->h_eq.assign(m->node_eq, m->node_eq + 3 * nnode);
  c->h_dof_of_eq.assign(std::max(0, m->num_eq), -1);
  std::vector<uint8_t> fix(nnode, 0);
  for (int64_t n = 0; n < nnode; n++)
    for (int i = 0; i < 3; i++) {
      const int32_t q = c->h_eq[3 * n + i];
      if (q <= 0) {
        fix[n] |= (uint8_t)(1 << i);
      } else {
        if (q > m->num_eq || c->h_dof_of_eq[q - 1] != -1) {
          c->err = "upload_mesh: node_eq is not a numbering of 1..num_eq";
          return FAST_GPU_EINVAL;
        }
        c->h_dof_of_eq[q - 1] = (int32_t)(3 * n + i);
      }
    }
  for (int32_t k = 0; k < m->num_eq; k++)
    if (c->h_dof_of_eq[k] < 0) {
      c->err = "upload_mesh: equation without a DOF";
      return FAST_GPU_EINVAL;
    }
  c->buckets.resize(m->num_buckets);
  for (int b = 0; b < m->num_buckets; b++) {
    const fast_gpu_bucket &bk = m->buckets[b];
    Bucket &B = c->buckets[b];
    B.type = bk.elem_type;
    B.nn = bucket_nodes(bk);
    if (!B.nn) {
      c->err = bk.elem_type == FAST_ELEM_BSP_SOLID
                   ? "upload_mesh: B-spline solid bucket needs a patch of degree 2 to 5 in every direction"
                   : "upload_mesh: unsupported element type";
      return FAST_GPU_ENOTSUP;
    }
    for (int k = 0; k < 3; k++) B.ngp[k] = bk.ngp[k];
    B.ng = B.ngp[0] * B.ngp[1] * B.ngp[2];
    if (B.type == FAST_ELEM_BSP_SOLID)
      for (int d = 0; d < 3; d++) B.pd[d] = bk.patch->degree[d];
    const bool ok_rule = (B.ngp[0] == B.ngp[1] && B.ngp[1] == B.ngp[2]) &&
                         ((B.type == FAST_ELEM_HEX8 && (B.ngp[0] == 1 || B.ngp[0] == 2 || B.ngp[0] == 3)) ||
                          (B.type == FAST_ELEM_HEX20 && (B.ngp[0] >= 2 && B.ngp[0] <= 4)) ||
                          (B.type == FAST_ELEM_BSP_SOLID && bsp_supported(B.pd, B.ngp[0]) &&
                           (bk.formulation != FAST_FORM_TOTAL_LAGRANGIAN || bsp_tl_supported(B.pd, B.ngp[0]))));
    if (!ok_rule) { c->err = "upload_mesh: unsupported Gauss rule for this element type"; return FAST_GPU_ENOTSUP; }
    B.ne = bk.num_elems;
    if (B.ne <= 0 || !bk.conn || !bk.E || !bk.nu) { c->err = "upload_mesh: empty bucket"; return FAST_GPU_EINVAL; }
    B.has_rho = bk.rho != nullptr;
    if (bk.formulation != FAST_FORM_SMALL_STRAIN && bk.formulation != FAST_FORM_TOTAL_LAGRANGIAN) {
      c->err = "upload_mesh: unknown element formulation";
      return FAST_GPU_ENOTSUP;
    }
    B.tl = bk.formulation == FAST_FORM_TOTAL_LAGRANGIAN;
    if (B.type == FAST_ELEM_BSP_SOLID) {
      const fast_gpu_patch &P = *bk.patch;
      if (B.has_rho && !bsp_tc_supported(B.pd, B.ngp[0])) {
        c->err = "upload_mesh: B-spline solids take a density (mass matrix) for degrees (2,2,2), (3,3,3), (3,3,2)";
        return FAST_GPU_ENOTSUP;
      }
      if (!P.span) { c->err = "upload_mesh: B-spline solid bucket without element spans"; return FAST_GPU_EINVAL; }
      for (int d = 0; d < 3; d++) {
        std::vector<double> tab;
        if (!bspline_gauss_tables(B.pd[d], P.num_knots[d], P.knots[d], B.ngp[d], B.nspan[d], tab)) {
          c->err = "upload_mesh: invalid knot vector in patch direction " + std::to_string(d);
          return FAST_GPU_EINVAL;
        }
      }
      for (int64_t e = 0; e < B.ne; e++)
        for (int d = 0; d < 3; d++)
          if (P.span[3 * e + d] < 0 || P.span[3 * e + d] >= B.nspan[d]) {
            c->err = "upload_mesh: element " + std::to_string(e) + " names a knot span outside its patch";
            return FAST_GPU_EINVAL;
          }
      B.rational = P.rational ? 1 : 0;
    }
  }
  if (m->ties && m->ties->num_slaves > 0)
    for (const Bucket &B : c->buckets)
      if (B.tl || B.has_rho) {
        c->err = "upload_mesh: tied interfaces support small-strain stiffness buckets only";
        return FAST_GPU_ENOTSUP;
      }
  if (!build_pattern(*c, *m)) return FAST_GPU_EINVAL;
  // slave DOFs leave the system: flagged like fixed ones (identity diagonal)
  for (int64_t n = 0; n < nnode; n++)
    if (c->h_slave_of[n] >= 0) fix[n] = 7;

  CK(dalloc(&c->d_X, 3 * nnode));
  CK(cudaMemcpy(c->d_X, m->coords, sizeof(double) * 3 * nnode, cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_fix, nnode));
  CK(cudaMemcpy(c->d_fix, fix.data(), nnode, cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_dof_of_eq, c->neq));
  {
    std::vector<int32_t> d4(c->neq);
    for (int32_t k = 0; k < c->neq; k++) d4[k] = 4 * (c->h_dof_of_eq[k] / 3) + c->h_dof_of_eq[k] % 3;
    if (c->neq) CK(cudaMemcpy(c->d_dof_of_eq, d4.data(), sizeof(int32_t) * c->neq, cudaMemcpyHostToDevice));
  }
  CK(dalloc(&c->d_rowptr, nnode + 1));
  CK(cudaMemcpy(c->d_rowptr, c->h_rowptr.data(), sizeof(int32_t) * (nnode + 1), cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_col, c->nnzb));
  CK(cudaMemcpy(c->d_col, c->h_col.data(), sizeof(int32_t) * c->nnzb, cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_diag, nnode));
  CK(cudaMemcpy(c->d_diag, c->h_diag.data(), sizeof(int32_t) * nnode, cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_srow, nnode + 1));
  CK(cudaMemcpy(c->d_srow, c->h_srow.data(), sizeof(int32_t) * (nnode + 1), cudaMemcpyHostToDevice));
  CK(dalloc(&c->d_scol, c->nnzb_pad));
  CK(cudaMemcpy(c->d_scol, c->h_scol.data(), sizeof(int32_t) * c->nnzb_pad, cudaMemcpyHostToDevice));
  for (int b = 0; b < m->num_buckets; b++) {
    const fast_gpu_bucket &bk = m->buckets[b];
    Bucket &B = c->buckets[b];
    const int64_t ne = B.ne;
    std::vector<double> E(ne), nu(ne), rho;
    for (int64_t s = 0; s < ne; s++) { E[s] = bk.E[B.perm[s]]; nu[s] = bk.nu[B.perm[s]]; }
    CK(dalloc(&B.d_conn, ne * B.nn));
    CK(cudaMemcpy(B.d_conn, B.h_conn.data(), sizeof(int32_t) * ne * B.nn, cudaMemcpyHostToDevice));
    CK(dalloc(&B.d_slot, ne * B.nn * B.nn));
    CK(cudaMemcpy(B.d_slot, B.h_slot.data(), sizeof(int32_t) * ne * B.nn * B.nn, cudaMemcpyHostToDevice));
    std::vector<int32_t>().swap(B.h_slot);
    if (!B.h_first.empty()) {
      CK(dalloc(&B.d_first, B.h_first.size()));
      CK(cudaMemcpy(B.d_first, B.h_first.data(), sizeof(uint32_t) * B.h_first.size(), cudaMemcpyHostToDevice));
      std::vector<uint32_t>().swap(B.h_first);
    }
    CK(dalloc(&B.d_E, ne));
    CK(cudaMemcpy(B.d_E, E.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
    CK(dalloc(&B.d_nu, ne));
    CK(cudaMemcpy(B.d_nu, nu.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
    if (B.has_rho) {
      rho.resize(ne);
      for (int64_t s = 0; s < ne; s++) rho[s] = bk.rho[B.perm[s]];
      CK(dalloc(&B.d_rho, ne));
      CK(cudaMemcpy(B.d_rho, rho.data(), sizeof(double) * ne, cudaMemcpyHostToDevice));
    }
    std::vector<double> N, dN, w;
    if (B.type == FAST_ELEM_BSP_SOLID) {
      const fast_gpu_patch &P = *bk.patch;
      std::vector<double> all;
      for (int d = 0; d < 3; d++) {
        std::vector<double> tab;
        int ns = 0;
        bspline_gauss_tables(B.pd[d], P.num_knots[d], P.knots[d], B.ngp[d], ns, tab);
        B.bas_off[d] = (int64_t)all.size();
        all.insert(all.end(), tab.begin(), tab.end());
      }
      CK(dalloc(&B.d_bas, all.size()));
      CK(cudaMemcpy(B.d_bas, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice));
      std::vector<int32_t> sp(4 * ne, 0);
      for (int64_t s = 0; s < ne; s++)
        for (int d = 0; d < 3; d++) sp[4 * s + d] = P.span[3 * (int64_t)B.perm[s] + d];
      CK(dalloc(&B.d_span, 4 * ne));
      CK(cudaMemcpy(B.d_span, sp.data(), sizeof(int32_t) * sp.size(), cudaMemcpyHostToDevice));
      if (B.rational && P.weights) {
        CK(dalloc(&B.d_wt, nnode));
        CK(cudaMemcpy(B.d_wt, P.weights, sizeof(double) * nnode, cudaMemcpyHostToDevice));
      }
      // Gauss weights only: the shape functions come from the span tables
      double r[6], wr[6], ws[6], wt[6];
      gauss_rule(B.ngp[0], r, wr);
      gauss_rule(B.ngp[1], r, ws);
      gauss_rule(B.ngp[2], r, wt);
      for (int i = 0; i < B.ngp[2]; i++)
        for (int j = 0; j < B.ngp[1]; j++)
          for (int l = 0; l < B.ngp[0]; l++) w.push_back(wr[l] * ws[j] * wt[i]);
      CK(dalloc(&B.d_w, w.size()));
      CK(cudaMemcpy(B.d_w, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice));
      continue;
    }
    gauss_point_tables(B.type, B.ngp, N, dN, w);
    CK(dalloc(&B.d_N, N.size()));
    CK(cudaMemcpy(B.d_N, N.data(), sizeof(double) * N.size(), cudaMemcpyHostToDevice));
    CK(dalloc(&B.d_dN, dN.size()));
    CK(cudaMemcpy(B.d_dN, dN.data(), sizeof(double) * dN.size(), cudaMemcpyHostToDevice));
    CK(dalloc(&B.d_w, w.size()));
    CK(cudaMemcpy(B.d_w, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice));
  }
  CK(upload_ties(*c));
  {
    // the per-node gather of the element-wise internal force (hex buckets
    // only): each node's element entries in bucket, then colour-sorted order
    bool all_hex = !c->buckets.empty();
    for (const Bucket &B : c->buckets)
      all_hex = all_hex && ((B.type == FAST_ELEM_HEX8 && (B.ng == 1 || B.ng == 8 || B.ng == 27)) ||
                            (B.type == FAST_ELEM_HEX20 && (B.ng == 8 || B.ng == 27 || B.ng == 64)));
    if (all_hex) {
      std::vector<int64_t> ptr(nnode + 1, 0);
      c->elem_g_off.assign(c->buckets.size(), 0);
      int64_t off = 0;
      for (size_t b = 0; b < c->buckets.size(); b++) {
        const Bucket &B = c->buckets[b];
        const int64_t nreg = B.color_off.empty() ? 0 : B.color_off.back();
        c->elem_g_off[b] = off;
        for (int64_t e = 0; e < nreg * B.nn; e++) ptr[B.h_conn[e] + 1]++;
        off += nreg * B.nn * 3;
      }
      for (int64_t n = 0; n < nnode; n++) ptr[n + 1] += ptr[n];
      std::vector<int64_t> inc(ptr[nnode]), pos(ptr.begin(), ptr.end() - 1);
      for (size_t b = 0; b < c->buckets.size(); b++) {
        const Bucket &B = c->buckets[b];
        const int64_t nreg = B.color_off.empty() ? 0 : B.color_off.back();
        for (int64_t e = 0; e < nreg * B.nn; e++) inc[pos[B.h_conn[e]]++] = c->elem_g_off[b] + 3 * e;
      }
      CK(dalloc(&c->d_elem_g, off));
      CK(dalloc(&c->d_gptr, nnode + 1));
      CK(cudaMemcpy(c->d_gptr, ptr.data(), sizeof(int64_t) * (nnode + 1), cudaMemcpyHostToDevice));
      CK(dalloc(&c->d_ginc, inc.size()));
      if (!inc.empty()) CK(cudaMemcpy(c->d_ginc, inc.data(), sizeof(int64_t) * inc.size(), cudaMemcpyHostToDevice));
      c->force_gather = true;
    }
  }
  const int64_t n4 = 4 * nnode;
  CK(dalloc(&c->d_K, 9 * c->nnzb));
  CK(dalloc(&c->d_u, n4)); CK(dalloc(&c->d_r, n4)); CK(dalloc(&c->d_z, n4)); CK(dalloc(&c->d_p, n4));
  CK(dalloc(&c->d_p2, n4)); CK(dalloc(&c->s_p2, n4));
  CK(dalloc(&c->d_w, n4)); CK(dalloc(&c->d_f, n4)); CK(dalloc(&c->d_dinv, 12 * nnode));
  CK(dalloc(&c->d_ubest, n4));
  CK(dalloc(&c->s_x, n4)); CK(dalloc(&c->s_r, n4)); CK(dalloc(&c->s_z, n4)); CK(dalloc(&c->s_p, n4));
  CK(dalloc(&c->s_w, n4)); CK(dalloc(&c->s_dinv, 12 * nnode));
  CK(cudaMemset(c->d_p, 0, sizeof(double) * n4));
  CK(cudaMemset(c->s_p, 0, sizeof(float) * n4));
  CK(dalloc(&c->d_disp, n4));
  CK(dalloc(&c->d_gint, n4));
  CK(cudaMemset(c->d_disp, 0, sizeof(double) * n4));
  CK(dalloc(&c->d_eq_tmp, std::max<int64_t>(2 * (int64_t)c->neq, 1)));
  CK(cudaMallocHost((void **)&c->h_eq_tmp, sizeof(double) * std::max<int64_t>(2 * (int64_t)c->neq, 1)));
  return FAST_GPU_OK;
}

int fast_gpu_pattern_info(fast_gpu_ctx *c, int64_t *nnzb, int64_t *nnz_lower, int32_t *ncol, double *secs) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  if (nnzb) *nnzb = c->nnzb;
  if (nnz_lower) *nnz_lower = c->nnz_lower_eq;
  if (ncol) *ncol = c->ncolors;
  if (secs) *secs = c->pattern_seconds;
  return FAST_GPU_OK;
}

int fast_gpu_update_coords(fast_gpu_ctx *c, const double *coords) {
  if (check_ctx(c) || !coords || !c->d_X) return FAST_GPU_EINVAL;
  CK(cudaMemcpyAsync(c->d_X, coords, sizeof(double) * 3 * c->nnode, cudaMemcpyHostToDevice, c->stream));
  c->K_ok = c->M_ok = false;
  invalidate(*c, FAST_ASM_STIFFNESS);
  invalidate(*c, FAST_ASM_MASS);
  return FAST_GPU_OK;
}

int fast_gpu_update_material(fast_gpu_ctx *c, int32_t b, const double *E, const double *nu) {
  if (check_ctx(c) || b < 0 || b >= (int)c->buckets.size()) return FAST_GPU_EINVAL;
  Bucket &B = c->buckets[b];
  if (!c->h_eq_tmp || B.ne > 2 * (int64_t)std::max(c->neq, 1)) {
    // permute through a temporary host buffer
    std::vector<double> t(B.ne);
    if (E) {
      for (int64_t s = 0; s < B.ne; s++) t[s] = E[B.perm[s]];
      CK(cudaMemcpyAsync(B.d_E, t.data(), sizeof(double) * B.ne, cudaMemcpyHostToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    if (nu) {
      for (int64_t s = 0; s < B.ne; s++) t[s] = nu[B.perm[s]];
      CK(cudaMemcpyAsync(B.d_nu, t.data(), sizeof(double) * B.ne, cudaMemcpyHostToDevice, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  } else {
    double *h = c->h_eq_tmp;
    if (E) {
      CK(cudaStreamSynchronize(c->stream));
      for (int64_t s = 0; s < B.ne; s++) h[s] = E[B.perm[s]];
      CK(cudaMemcpyAsync(B.d_E, h, sizeof(double) * B.ne, cudaMemcpyHostToDevice, c->stream));
    }
    if (nu) {
      CK(cudaStreamSynchronize(c->stream));
      for (int64_t s = 0; s < B.ne; s++) h[s] = nu[B.perm[s]];
      CK(cudaMemcpyAsync(B.d_nu, h, sizeof(double) * B.ne, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  c->K_ok = c->M_ok = false;
  invalidate(*c, FAST_ASM_STIFFNESS);
  invalidate(*c, FAST_ASM_MASS);
  return FAST_GPU_OK;
}

int fast_gpu_set_displacement_device(fast_gpu_ctx *c, const double *d_u) {
  if (check_ctx(c) || !d_u || !c->d_disp) return FAST_GPU_EINVAL;
  CK(launch_eq_to_node(*c, d_u, c->d_disp));
  return FAST_GPU_OK;
}

int fast_gpu_set_displacement(fast_gpu_ctx *c, const double *u) {
  if (check_ctx(c) || !u || !c->d_disp) return FAST_GPU_EINVAL;
  const size_t nb = sizeof(double) * c->neq;
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(c->h_eq_tmp, u, nb);
  CK(cudaMemcpyAsync(c->d_eq_tmp, c->h_eq_tmp, nb, cudaMemcpyHostToDevice, c->stream));
  CK(launch_eq_to_node(*c, c->d_eq_tmp, c->d_disp));
  return FAST_GPU_OK;
}

int fast_gpu_internal_force_device(fast_gpu_ctx *c, double *d_g) {
  if (c && c->has_ties()) { c->err = "internal_force: not available with tied interfaces"; return FAST_GPU_ENOTSUP; }
  if (check_ctx(c) || !d_g || !c->d_gint) return FAST_GPU_EINVAL;
  const int64_t sp = c->begin_span(FAST_KERNEL_INTERNAL_FORCE);
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  CK(cudaMemsetAsync(c->d_gint, 0, sizeof(double) * 4 * c->nnode, c->stream));
  CK(launch_tl(*c, nullptr, c->d_gint, false, true));
  CK(launch_node_to_eq(*c, c->d_gint, d_g));
  c->end_span(sp);
  return FAST_GPU_OK;
}

int fast_gpu_internal_force(fast_gpu_ctx *c, double *g) {
  if (check_ctx(c) || !g) return FAST_GPU_EINVAL;
  const int rc = fast_gpu_internal_force_device(c, c->d_eq_tmp);
  if (rc != FAST_GPU_OK) return rc;
  const size_t nb = sizeof(double) * c->neq;
  CK(cudaMemcpyAsync(c->h_eq_tmp, c->d_eq_tmp, nb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(g, c->h_eq_tmp, nb);
  if (c->h_status[0] & 1) {
    c->err = "internal_force: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  return FAST_GPU_OK;
}

int fast_gpu_zero(fast_gpu_ctx *c, int32_t what) {
  if (check_ctx(c) || !c->d_K) return FAST_GPU_ESTATE;
  if (what == FAST_ASM_MASS && !c->d_M) CK(dalloc(&c->d_M, 9 * c->nnzb));
  double *T = target_of(*c, what);
  if (!T) return FAST_GPU_EINVAL;
  CK(launch_zero_matrix(*c, T, what == FAST_ASM_STIFFNESS));
  if (what == FAST_ASM_STIFFNESS) { c->K_ok = true; c->K32_current = false; } else c->M_ok = true;
  invalidate(*c, what);
  return FAST_GPU_OK;
}

namespace {
// FAST_ASM_STIFFNESS_TF32: the stiffness on the tensor cores, FP32 blocks
int assemble_tf32(fast_gpu_ctx *c) {
  for (const Bucket &B : c->buckets)
    if (!tc_supported(B)) {
      c->err = "assemble: the tensor-core stiffness takes small-strain hex8 / hex20 and B-spline (2,2,2), "
               "(3,3,3), (3,3,2) buckets only";
      return FAST_GPU_ENOTSUP;
    }
  if (!c->d_K32) CK(cudaMalloc((void **)&c->d_K32, sizeof(float) * 9 * (size_t)c->nnzb));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  c->begin_span(FAST_KERNEL_ASSEMBLE_TF32);
  CK(launch_assemble_tc(*c, c->d_K32));
  c->end_span();
  CK(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->harvest();
  c->K32_current = true;
  c->K_ok = false;          // the FP64 stiffness slot no longer holds the current stiffness
  invalidate(*c, FAST_ASM_STIFFNESS);
  if (c->h_status[0] & 4) { c->err = "assemble: a tensor-core kernel's wait timed out"; return FAST_GPU_ECUDA; }
  if (c->h_status[0] & 1) {
    c->err = "assemble: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  return FAST_GPU_OK;
}
}  // namespace

int fast_gpu_assemble(fast_gpu_ctx *c, int32_t what) {
  if (check_ctx(c) || !c->d_K) { if (c) c->err = "assemble: no mesh"; return FAST_GPU_ESTATE; }
  if (what == FAST_ASM_STIFFNESS_TF32) return assemble_tf32(c);
  if (what != FAST_ASM_STIFFNESS && what != FAST_ASM_MASS) return FAST_GPU_EINVAL;
  if (what == FAST_ASM_STIFFNESS) c->K32_current = false;
  if (what == FAST_ASM_MASS && !c->d_M) CK(dalloc(&c->d_M, 9 * c->nnzb));
  double *T = target_of(*c, what);
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  if (what == FAST_ASM_STIFFNESS) c->begin_span(2);
  // (with first-touch flags every block is stored by its first writer)
  if (!(what == FAST_ASM_STIFFNESS && c->use_first_touch())) CK(launch_zero_matrix(*c, T, what == FAST_ASM_STIFFNESS));
  CK(launch_assemble(*c, what, T));
  if (what == FAST_ASM_STIFFNESS) CK(launch_tl(*c, T, nullptr, true, false));
  if (what == FAST_ASM_STIFFNESS) c->end_span();
  CK(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->harvest();
  if (what == FAST_ASM_STIFFNESS) c->K_ok = true; else c->M_ok = true;
  invalidate(*c, what);
  if (c->h_status[0] & 1) {
    c->err = "assemble: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  return FAST_GPU_OK;
}

int fast_gpu_add(fast_gpu_ctx *c, int32_t what, int32_t i, int32_t j, double v) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  if (what == FAST_ASM_STIFFNESS && c->K32_current) {
    c->err = "add: the current stiffness is the tensor-core FP32 one; assemble FAST_ASM_STIFFNESS to edit entries";
    return FAST_GPU_ESTATE;
  }
  double *T = target_of(*c, what);
  if (!T) return FAST_GPU_ESTATE;
  const int64_t k1 = value_index(*c, i, j);
  if (k1 < 0) { c->err = "add: (i, j) outside the pattern"; return FAST_GPU_ENOTFOUND; }
  const int64_t k2 = value_index(*c, j, i);
  double a = 0, b = 0;
  CK(cudaMemcpyAsync(&a, T + k1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  a += v;
  CK(cudaMemcpyAsync(T + k1, &a, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (k2 != k1) {
    CK(cudaMemcpyAsync(&b, T + k2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    b += v;
    CK(cudaMemcpyAsync(T + k2, &b, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  invalidate(*c, what);
  return FAST_GPU_OK;
}

int fast_gpu_add_mat(fast_gpu_ctx *c, int32_t dst, double a, int32_t src) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  if (dst != FAST_ASM_STIFFNESS || src != FAST_ASM_MASS) {
    c->err = "add_mat: only K += a M (dst FAST_ASM_STIFFNESS, src FAST_ASM_MASS)";
    return FAST_GPU_EINVAL;
  }
  if (!c->d_K || !c->d_M || !c->K_ok || !c->M_ok) { c->err = "add_mat: K and M must be assembled"; return FAST_GPU_ESTATE; }
  const int64_t n = 9 * c->nnzb;
  add_mat_kernel<<<4 * c->sm_count, 256, 0, c->stream>>>(n, a, c->d_M, c->d_K);
  c->launches++;
  CK(cudaGetLastError());
  invalidate(*c, FAST_ASM_STIFFNESS);
  return FAST_GPU_OK;
}

int fast_gpu_get(fast_gpu_ctx *c, int32_t what, int32_t i, int32_t j, double *v) {
  if (check_ctx(c) || !v) return FAST_GPU_EINVAL;
  double *T = target_of(*c, what);
  if (!T) return FAST_GPU_ESTATE;
  const int64_t k = value_index(*c, i, j);
  if (k < 0) { *v = 0.0; return FAST_GPU_OK; }
  CK(cudaMemcpyAsync(v, T + k, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return FAST_GPU_OK;
}

int fast_gpu_mult_vect(fast_gpu_ctx *c, int32_t what, const double *x, double *y) {
  if (check_ctx(c) || !x || !y) return FAST_GPU_EINVAL;
  double *T = target_of(*c, what);
  if (!T || (what == FAST_ASM_STIFFNESS && !c->K_ok) || (what == FAST_ASM_MASS && !c->M_ok)) return FAST_GPU_ESTATE;
  const size_t nb = sizeof(double) * c->neq;
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(c->h_eq_tmp, x, nb);
  CK(cudaMemcpyAsync(c->d_eq_tmp, c->h_eq_tmp, nb, cudaMemcpyHostToDevice, c->stream));
  CK(ensure_soa(*c, what, false));
  CK(launch_eq_to_node(*c, c->d_eq_tmp, c->d_z));
  CK(launch_spmv(*c, what == FAST_ASM_MASS ? c->d_Ms : c->d_Ks, c->d_z, c->d_w));
  CK(launch_node_to_eq(*c, c->d_w, c->d_eq_tmp));
  CK(cudaMemcpyAsync(c->h_eq_tmp, c->d_eq_tmp, nb, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(y, c->h_eq_tmp, nb);
  return FAST_GPU_OK;
}

namespace {

int solve_node_space(fast_gpu_ctx *c, const fast_gpu_solve_opts *o, bool warm, fast_gpu_solve_report *rep) {
  // c->d_f holds the padded load, c->d_u the initial / returned solution
  fast_gpu_solve_opts opts{};
  if (o) opts = *o;
  const int maxit = opts.maxit > 0 ? opts.maxit : std::max(20 * c->neq, 100);
  const double tol = opts.tol > 0 ? opts.tol : 1e-5;
  const int precond = opts.precond;
  if (precond != FAST_PRECOND_JACOBI && precond != FAST_PRECOND_BLOCK_JACOBI) return FAST_GPU_EINVAL;
  const bool mixed = opts.precision == FAST_PREC_MIXED;
  if (!mixed && opts.precision != FAST_PREC_FP64) return FAST_GPU_EINVAL;
  const bool k32 = c->K32_current;
  if (k32 && !mixed) {
    c->err = "solve: the tensor-core stiffness serves the mixed-precision solve; assemble FAST_ASM_STIFFNESS "
             "for an FP64 solve";
    return FAST_GPU_ESTATE;
  }
  if (c->precond_built != precond)
    CK(k32 ? launch_build_precond32(*c, c->d_K32, precond) : launch_build_precond(*c, c->d_K, precond));
  CK(ensure_soa(*c, FAST_ASM_STIFFNESS, mixed));
  const int chunk = opts.check_every > 0 ? opts.check_every : (mixed ? 50 : 32);
  fast_gpu_solve_report R{};
  if (mixed) {
    CK(pcg_mixed(*c, warm, tol, maxit, chunk));
    R.outer = c->h_state->updates;
    int done = c->h_state->done, it = c->h_state->iter;
    if ((done == 3 || done == 4) && it < maxit && k32) {
      // The tensor-core FP32 stiffness (entries to about 1e-6 of the largest
      // on degree-3 B-splines) could not take this system to the tolerance
      // against its element-by-element FP64 residual, restarts included:
      // assemble the FP64 stiffness and go on with the mixed iteration on it
      // from the best FP64 iterate seen (its FP32 copy is the rounded FP64 K).
      R.escalated = 2;
      CK(cudaMemcpyAsync(c->d_u, c->d_ubest, sizeof(double) * 4 * c->nnode, cudaMemcpyDeviceToDevice, c->stream));
      if (!c->use_first_touch()) CK(launch_zero_matrix(*c, c->d_K, true));
      CK(launch_assemble(*c, FAST_ASM_STIFFNESS, c->d_K));
      c->K_ok = true;
      c->K32_current = false;
      invalidate(*c, FAST_ASM_STIFFNESS);
      CK(launch_build_precond(*c, c->d_K, precond));
      c->precond_built = precond;
      CK(ensure_soa(*c, FAST_ASM_STIFFNESS, true));
      CK(pcg_mixed(*c, true, tol, maxit - it, chunk));
      R.outer += c->h_state->updates;
      c->h_state->iter += it;
      done = c->h_state->done;
      it = c->h_state->iter;
    }
    if ((done == 3 || done == 4) && it < maxit && !c->K32_current) {
      // FP32 iterates stopped making progress (ill-conditioned system): go on
      // with the FP64 iteration from the best FP64 iterate seen
      R.escalated |= 1;
      CK(cudaMemcpyAsync(c->d_u, c->d_ubest, sizeof(double) * 4 * c->nnode, cudaMemcpyDeviceToDevice, c->stream));
      CK(pcg_fp64(*c, true, tol, maxit, chunk, it));
    }
  } else {
    CK(pcg_fp64(*c, warm, tol, maxit, chunk));
    R.outer = 1;
  }
  c->harvest();
  const PcgState &st = *c->h_state;
  R.iterations = st.iter;
  R.rel_residual = (mixed && !(R.escalated & 1)) ? st.err_true : st.err;
  R.converged = (st.done == 1);
  // true FP64 residual |f - K u| / |f| (element by element on the tensor-core stiffness)
  {
    double *d_rr = c->d_partials + 12290;
    double *d_ff = c->d_partials + 12291;
    CK(launch_residual(*c, c->K32_current ? nullptr : c->d_Ks, c->d_f, c->d_u, c->d_r, d_rr));  // null: element by element
    CK(launch_norm2(*c, c->d_f, 4 * c->nnode, d_ff));
    double h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, d_rr, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    R.true_rel_residual = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
  }
  if (rep) *rep = R;
  if (st.done == kDoneBarrierTimeout) {
    c->err = "solve: a grid-barrier wait of the persistent PCG kernel timed out";
    return FAST_GPU_ECUDA;
  }
  if (st.done == 3) {
    c->err = "solve: breakdown (non-positive or non-finite p.Kp or residual)";
    return FAST_GPU_ENONCONV;
  }
  if (st.done == 4) {
    c->err = "solve: FP64 residual stagnated above the tolerance (attainable accuracy reached)";
    return FAST_GPU_ENONCONV;
  }
  if (!R.converged) {
    c->err = "solve: no convergence within the iteration cap";
    return FAST_GPU_ENONCONV;
  }
  return FAST_GPU_OK;
}

}  // namespace

extern "C++" {
namespace fastgpu {
int solve_nodes(Ctx &c, const fast_gpu_solve_opts *o, bool warm, fast_gpu_solve_report *rep) {
  return solve_node_space(static_cast<fast_gpu_ctx *>(&c), o, warm, rep);
}
}  // namespace fastgpu
}

int fast_gpu_solve_device(fast_gpu_ctx *c, const double *d_f, double *d_u, const fast_gpu_solve_opts *o,
                          fast_gpu_solve_report *rep) {
  if (check_ctx(c) || !d_f || !d_u) return FAST_GPU_EINVAL;
  if (!c->K_ok && !c->K32_current) { c->err = "solve: matrix not assembled"; return FAST_GPU_ESTATE; }
  const bool warm = o && o->warm_start;
  const int64_t sp = c->begin_span(FAST_KERNEL_LINEAR_SOLVE);
  CK(launch_eq_to_node(*c, d_f, c->d_f));
  CK(launch_tie_restrict(*c, c->d_f));
  if (warm) {
    CK(launch_eq_to_node(*c, d_u, c->d_u));
    CK(launch_tie_zero(*c, c->d_u));
  }
  const int rc = solve_node_space(c, o, warm, rep);
  if (rc == FAST_GPU_OK || rc == FAST_GPU_ENONCONV) {
    CK(launch_tie_prolong(*c, c->d_u));
    CK(launch_node_to_eq(*c, c->d_u, d_u));
  }
  c->end_span(sp);
  return rc;
}

int fast_gpu_solve(fast_gpu_ctx *c, const double *f, double *u, const fast_gpu_solve_opts *o,
                   fast_gpu_solve_report *rep) {
  if (check_ctx(c) || !f || !u) return FAST_GPU_EINVAL;
  if (!c->K_ok && !c->K32_current) { c->err = "solve: matrix not assembled"; return FAST_GPU_ESTATE; }
  const size_t nb = sizeof(double) * c->neq;
  double *d_feq = c->d_eq_tmp, *d_ueq = c->d_eq_tmp + c->neq;
  CK(cudaStreamSynchronize(c->stream));
  std::memcpy(c->h_eq_tmp, f, nb);
  if (o && o->warm_start) std::memcpy(c->h_eq_tmp + c->neq, u, nb);
  CK(cudaMemcpyAsync(d_feq, c->h_eq_tmp, (o && o->warm_start) ? 2 * nb : nb, cudaMemcpyHostToDevice, c->stream));
  const int rc = fast_gpu_solve_device(c, d_feq, d_ueq, o, rep);
  if (rc == FAST_GPU_OK || rc == FAST_GPU_ENONCONV) {
    CK(cudaMemcpyAsync(c->h_eq_tmp, d_ueq, nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(u, c->h_eq_tmp, nb);
  }
  return rc;
}

int fast_gpu_get_lower_csr(fast_gpu_ctx *c, int32_t what, int64_t *nnz, int64_t *rowptr, int32_t *col, double *val) {
  if (check_ctx(c) || !nnz) return FAST_GPU_EINVAL;
  const bool k32 = what == FAST_ASM_STIFFNESS_TF32;
  if (k32 && !c->K32_current) { c->err = "get_lower_csr: no tensor-core stiffness assembled"; return FAST_GPU_ESTATE; }
  double *T = k32 ? nullptr : target_of(*c, what);
  if (!T && !k32) return FAST_GPU_ESTATE;
  // count per equation row
  const int32_t neq = c->neq;
  std::vector<int64_t> cnt(neq + 1, 0);
  for (int32_t i = 0; i < neq; i++) {
    const int32_t d = c->h_dof_of_eq[i], n = d / 3;
    for (int32_t k = c->h_rowptr[n]; k < c->h_rowptr[n + 1]; k++)
      for (int q = 0; q < 3; q++) {
        const int32_t ej = c->h_eq[3 * (int64_t)c->h_col[k] + q];
        if (ej && ej - 1 <= i) cnt[i + 1]++;
      }
  }
  for (int32_t i = 0; i < neq; i++) cnt[i + 1] += cnt[i];
  *nnz = cnt[neq];
  if (!col || !val || !rowptr) return FAST_GPU_OK;
  std::vector<double> hv((size_t)9 * c->nnzb);
  if (k32) {
    std::vector<float> hf(hv.size());
    CK(cudaMemcpyAsync(hf.data(), c->d_K32, sizeof(float) * hf.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < hv.size(); k++) hv[k] = (double)hf[k];
  } else {
    CK(cudaMemcpyAsync(hv.data(), T, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  std::memcpy(rowptr, cnt.data(), sizeof(int64_t) * (neq + 1));
  std::vector<std::pair<int32_t, double>> row;
  for (int32_t i = 0; i < neq; i++) {
    const int32_t d = c->h_dof_of_eq[i], n = d / 3, p = d % 3;
    row.clear();
    for (int32_t k = c->h_rowptr[n]; k < c->h_rowptr[n + 1]; k++)
      for (int q = 0; q < 3; q++) {
        const int32_t ej = c->h_eq[3 * (int64_t)c->h_col[k] + q];
        if (ej && ej - 1 <= i) row.emplace_back(ej - 1, hv[(size_t)k * 9 + p * 3 + q]);
      }
    std::sort(row.begin(), row.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    int64_t o = cnt[i];
    for (auto &pr : row) { col[o] = pr.first; val[o] = pr.second; o++; }
  }
  return FAST_GPU_OK;
}

int fast_gpu_element_matrices(fast_gpu_ctx *c, int32_t what, int32_t b, int64_t first, int64_t count, double *Ke) {
  if (check_ctx(c) || !Ke || b < 0 || b >= (int)c->buckets.size()) return FAST_GPU_EINVAL;
  const Bucket &B = c->buckets[b];
  if (first < 0 || count <= 0 || first + count > B.ne) return FAST_GPU_EINVAL;
  if (what == FAST_ASM_MASS && !B.has_rho) { c->err = "element_matrices: bucket has no density"; return FAST_GPU_ESTATE; }
  if (what != FAST_ASM_STIFFNESS && what != FAST_ASM_MASS && what != FAST_ASM_INTERNAL_FORCE &&
      what != FAST_ASM_STIFFNESS_TF32)
    return FAST_GPU_EINVAL;
  if (what == FAST_ASM_STIFFNESS_TF32 && !tc_supported(B)) {
    c->err = "element_matrices: the tensor-core stiffness takes small-strain hex8 / hex20 and B-spline (2,2,2), "
             "(3,3,3), (3,3,2) buckets only";
    return FAST_GPU_ENOTSUP;
  }
  if (B.type == FAST_ELEM_BSP_SOLID && ((what == FAST_ASM_MASS && !bsp_tc_supported(B.pd, B.ngp[0])) ||
                                        (what == FAST_ASM_INTERNAL_FORCE && !bsp_tl_supported(B.pd, B.ngp[0])))) {
    c->err = "element_matrices: B-spline solids provide the mass matrix for degrees up to 3 and the internal "
             "force for the tangent kernels' degrees";
    return FAST_GPU_ENOTSUP;
  }
  const int nd = 3 * B.nn;
  const size_t mat_bytes = sizeof(double) * (size_t)count * (what == FAST_ASM_INTERNAL_FORCE ? nd : nd * nd);
  double *buf = nullptr;
  CK(cudaMalloc((void **)&buf, mat_bytes + sizeof(int32_t) * count + 16));
  std::vector<int32_t> idx(count);
  for (int64_t k = 0; k < count; k++) idx[k] = B.inv[first + k];
  cudaError_t e = cudaMemcpyAsync((char *)buf + mat_bytes, idx.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, mat_bytes, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream);
  if (e == cudaSuccess) {
    if (what == FAST_ASM_INTERNAL_FORCE) e = launch_tl_element(*c, 1, b, count, buf);
    else if (what == FAST_ASM_STIFFNESS_TF32) e = launch_element_matrices_tc(*c, b, count, buf);
    else if (what == FAST_ASM_STIFFNESS && B.tl) e = launch_tl_element(*c, 0, b, count, buf);
    else e = launch_element_matrices(*c, what, b, 0, count, buf);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(Ke, buf, mat_bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(buf);
  if (e != cudaSuccess) { c->err = std::string("element_matrices: ") + cudaGetErrorString(e); return FAST_GPU_ECUDA; }
  return FAST_GPU_OK;
}

int fast_gpu_inspect_pattern(const fast_gpu_mesh *m, int64_t *nnzb, int64_t *nnz_lower, int32_t *ncol,
                             int32_t *rowptr, int32_t *col, int32_t *color) {
  if (!m || m->num_nodes <= 0 || !m->node_eq || m->num_buckets <= 0 || !m->buckets) return FAST_GPU_EINVAL;
  Ctx c;
  c.nnode = m->num_nodes;
  c.h_eq.assign(m->node_eq, m->node_eq + 3 * m->num_nodes);
  c.buckets.resize(m->num_buckets);
  for (int b = 0; b < m->num_buckets; b++) {
    c.buckets[b].type = m->buckets[b].elem_type;
    c.buckets[b].nn = bucket_nodes(m->buckets[b]);
    c.buckets[b].ne = m->buckets[b].num_elems;
    if (!c.buckets[b].nn || !m->buckets[b].conn) return FAST_GPU_ENOTSUP;
  }
  if (!build_pattern(c, *m)) return FAST_GPU_EINVAL;
  if (nnzb) *nnzb = c.nnzb;
  if (nnz_lower) *nnz_lower = c.nnz_lower_eq;
  if (ncol) *ncol = c.ncolors;
  if (rowptr) std::memcpy(rowptr, c.h_rowptr.data(), sizeof(int32_t) * (m->num_nodes + 1));
  if (col) std::memcpy(col, c.h_col.data(), sizeof(int32_t) * c.nnzb);
  if (color) {
    const Bucket &B = c.buckets[0];
    for (size_t k = 0; k + 1 < B.color_off.size(); k++)
      for (int64_t s = B.color_off[k]; s < B.color_off[k + 1]; s++) color[B.perm[s]] = (int32_t)k;
    for (int64_t s = B.ne_regular; s < B.ne; s++) color[B.perm[s]] = -1;  // tied: scattered separately
  }
  // the slot map must cover every node pair of the colour-scheduled elements
  for (const Bucket &B : c.buckets)
    for (int64_t k = 0; k < B.ne_regular * B.nn * B.nn; k++)
      if (B.h_slot[k] < 0) return FAST_GPU_EINVAL;
  return FAST_GPU_OK;
}

int fast_gpu_launch_count(fast_gpu_ctx *c, int64_t *n) {
  if (check_ctx(c) || !n) return FAST_GPU_EINVAL;
  *n = c->launches;
  return FAST_GPU_OK;
}

int fast_gpu_kernel_timing(fast_gpu_ctx *c, int32_t enable) {
  if (check_ctx(c)) return FAST_GPU_EINVAL;
  CK(cudaStreamSynchronize(c->stream));
  c->harvest();
  c->timing = enable != 0;
  for (int k = 0; k < Ctx::kSpanKinds; k++) { c->kt_ms[k] = 0; c->kt_n[k] = 0; }
  return FAST_GPU_OK;
}

int fast_gpu_kernel_stats(fast_gpu_ctx *c, int32_t which, int64_t *launches, double *total_ms, double *bytes) {
  if (check_ctx(c) || which < 0 || which >= Ctx::kSpanKinds) return FAST_GPU_EINVAL;
  CK(cudaStreamSynchronize(c->stream));
  c->harvest();
  if (launches) *launches = c->kt_n[which];
  if (total_ms) *total_ms = c->kt_ms[which];
  if (bytes) {
    const double n4 = 4.0 * c->nnode;
    double algo = 0.0;
    // SpMV: block values + column indices + row pointers + x read once + y written once
    // (the padding blocks of the solve layout are not counted: they are overhead)
    if (which == FAST_KERNEL_SPMV_FP64) algo = (double)c->nnzb * (9 * 8 + 4) + 4.0 * (c->nnode + 1) + 2.0 * 8 * n4;
    // (16-bit column offsets: 2 bytes per block plus a 4-byte base per row)
    if (which == FAST_KERNEL_SPMV_FP32)
      algo = c->spmv32_c16 ? (double)c->nnzb * (9 * 4 + 2) + 4.0 * (c->nnode + 1) + 4.0 * c->nnode + 2.0 * 4 * n4
                           : (double)c->nnzb * (9 * 4 + 4) + 4.0 * (c->nnode + 1) + 2.0 * 4 * n4;
    if (which == FAST_KERNEL_ASSEMBLE || which == FAST_KERNEL_ASSEMBLE_TF32) {
      // scatter model per element: incidence + coordinates + fixity + E, nu + slot map + 3x3 block
      // read-modify-write (72-byte FP64 or 36-byte FP32 blocks), plus the zero fill of the block
      // values; with first-touch stores the zero fill is gone, each block's first write reads
      // nothing, and the flag words are read instead
      const double blk = which == FAST_KERNEL_ASSEMBLE ? 72.0 : 36.0;
      const bool ft = c->use_first_touch();
      for (const Bucket &B : c->buckets) {
        const double nn = B.nn;
        algo += (double)B.ne * (nn * (4 + 24 + 1) + 16 + nn * nn * (4 + 2 * blk));
        if (ft) algo += (double)B.ne * 4.0 * first_words(B.nn);
      }
      algo += ft ? -blk * c->nnzb : blk * c->nnzb;
    }
    *bytes = algo;
  }
  return FAST_GPU_OK;
}

}  // extern "C"

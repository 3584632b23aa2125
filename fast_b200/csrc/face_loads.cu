// face_loads.cu - uniform face tractions integrated on the device
// (fast_gpu_set_face_loads, fast_gpu_face_load_device).
//
// The same integral as the host integrator in loads.cpp, which restates
// cElemLoad::ExtForce (load/load.cpp:618-706) for %LOAD.CASE.AREA.UNIFORM:
// f_e = sum over the face's Gauss points of N^T q |dx/dr x dx/ds| w, on the
// Q4 / Q8 surface shape (shp/shpplane.cpp:353-488), with Local = 1 rotating q
// from the face frame (u = dx/dr, w = u x dx/ds, v = w x u; cShapeSurf::
// LocalSys, shp/shpsurf.cpp:121-160).  It reads the context's current
// coordinates.
//
// One thread integrates one face into fe[face][node][3]; then one thread per
// loaded node sums the entries of the faces that share it, in face order, and
// writes the node's equations: no atomics, the same f on every call.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

__constant__ double cGaussR[6][6] = {
    {0.000000000000000},
    {-0.577350269189626, 0.577350269189626},
    {-0.774596669241483, 0.000000000000000, 0.774596669241483},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
    {-0.906179845938664, -0.538469310105683, 0.000000000000000, 0.538469310105683, 0.906179845938664},
    {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466264,
     0.932469514203152}};
__constant__ double cGaussW[6][6] = {
    {2.000000000000000},
    {1.000000000000000, 1.000000000000000},
    {0.555555555555556, 0.888888888888889, 0.555555555555556},
    {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454},
    {0.236926885056189, 0.478628670499367, 0.568888888888889, 0.478628670499367, 0.236926885056189},
    {0.171324492379170, 0.360761573048139, 0.467913934572691, 0.467913934572691, 0.360761573048139,
     0.171324492379170}};

// surface shape functions and their (r, s) derivatives: Q4 (corners) or Q8
// (corners 0, 2, 4, 6 and mid-sides 1, 3, 5, 7)
template <int NF>
__device__ __forceinline__ void face_shape(double r, double s, double *N, double *dN) {
  if (NF == 4) {
    const double rn[4] = {-1, 1, 1, -1}, sn[4] = {-1, -1, 1, 1};
#pragma unroll
    for (int a = 0; a < 4; a++) {
      N[a] = 0.25 * (1 + rn[a] * r) * (1 + sn[a] * s);
      dN[2 * a] = 0.25 * rn[a] * (1 + sn[a] * s);
      dN[2 * a + 1] = 0.25 * sn[a] * (1 + rn[a] * r);
    }
  } else {
    const double rn[8] = {-1, 0, 1, 1, 1, 0, -1, -1}, sn[8] = {-1, -1, -1, 0, 1, 1, 1, 0};
#pragma unroll
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
}

template <int NF>
__global__ void face_forces(int32_t nface, int ngp, const int32_t *__restrict__ fn, const double *__restrict__ fq,
                            const int32_t *__restrict__ floc, const double *__restrict__ X, double *__restrict__ fe) {
  const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nface) return;
  double x[3 * NF], f[3 * NF];
#pragma unroll
  for (int a = 0; a < NF; a++) {
    const int64_t n = fn[(int64_t)k * NF + a];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      x[3 * a + d] = X[3 * n + d];
      f[3 * a + d] = 0.0;
    }
  }
  const double q0 = fq[3 * k], q1 = fq[3 * k + 1], q2 = fq[3 * k + 2];
  const bool loc = floc[k] != 0;
  for (int i = 0; i < ngp; i++)
    for (int j = 0; j < ngp; j++) {
      const double r = cGaussR[ngp - 1][j], s = cGaussR[ngp - 1][i];
      const double wgt = cGaussW[ngp - 1][j] * cGaussW[ngp - 1][i];
      double N[NF], dN[2 * NF];
      face_shape<NF>(r, s, N, dN);
      double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
#pragma unroll
      for (int a = 0; a < NF; a++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          tr[d] += dN[2 * a] * x[3 * a + d];
          ts[d] += dN[2 * a + 1] * x[3 * a + d];
        }
      const double nv0 = tr[1] * ts[2] - tr[2] * ts[1], nv1 = tr[2] * ts[0] - tr[0] * ts[2],
                   nv2 = tr[0] * ts[1] - tr[1] * ts[0];
      const double detJ = sqrt(nv0 * nv0 + nv1 * nv1 + nv2 * nv2);
      double val[3] = {q0, q1, q2};
      if (loc) {
        const double lu = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
        const double lv = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
        const double u[3] = {tr[0] / lu, tr[1] / lu, tr[2] / lu}, v[3] = {ts[0] / lv, ts[1] / lv, ts[2] / lv};
        const double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        const double v2[3] = {w[1] * u[2] - w[2] * u[1], w[2] * u[0] - w[0] * u[2], w[0] * u[1] - w[1] * u[0]};
#pragma unroll
        for (int d = 0; d < 3; d++) val[d] = u[d] * q0 + v2[d] * q1 + w[d] * q2;
      }
      const double coeff = wgt * detJ;
#pragma unroll
      for (int a = 0; a < NF; a++)
#pragma unroll
        for (int d = 0; d < 3; d++) f[3 * a + d] += N[a] * (coeff * val[d]);
    }
#pragma unroll
  for (int t = 0; t < 3 * NF; t++) fe[(int64_t)k * 3 * NF + t] = f[t];
}

// f[eq] = scale * sum of the node's face entries, in face order
__global__ void face_gather(int32_t nfnode, const int32_t *__restrict__ feq, const int32_t *__restrict__ fptr,
                            const int32_t *__restrict__ fidx, const double *__restrict__ fe, double scale,
                            double *__restrict__ f) {
  const int32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nfnode) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int32_t p = fptr[j]; p < fptr[j + 1]; p++) {
    const double *v = fe + 3 * (int64_t)fidx[p];
    a0 += v[0];
    a1 += v[1];
    a2 += v[2];
  }
  const double a[3] = {a0, a1, a2};
  for (int d = 0; d < 3; d++) {
    const int32_t e = feq[3 * j + d];
    if (e > 0) f[e - 1] = scale * a[d];
  }
}

template <class T>
cudaError_t up(T **d, const std::vector<T> &h) {
  *d = nullptr;
  cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(1, h.size()));
  if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

namespace fastgpu {
void free_face_loads(Ctx &c) {
  for (void *p : {(void *)c.d_fn, (void *)c.d_floc, (void *)c.d_fq, (void *)c.d_fe, (void *)c.d_fnode,
                  (void *)c.d_feq, (void *)c.d_fptr, (void *)c.d_fidx})
    if (p) cudaFree(p);
  c.d_fn = c.d_floc = c.d_fnode = c.d_feq = c.d_fptr = c.d_fidx = nullptr;
  c.d_fq = c.d_fe = nullptr;
  c.nface = c.nfn = c.face_ngp = c.nfnode = 0;
}
}  // namespace fastgpu

#define FCK(call)                                                                  \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      c->err = std::string("face loads: ") + #call + ": " + cudaGetErrorString(_e); \
      return FAST_GPU_ECUDA;                                                       \
    }                                                                              \
  } while (0)

extern "C" int fast_gpu_set_face_loads(fast_gpu_ctx *c, int32_t num_faces, int32_t nodes_per_face,
                                       const int32_t *face_nodes, const double *q, const int32_t *local,
                                       int32_t ngp1d) {
  if (!c || num_faces < 0 || (num_faces > 0 && (!face_nodes || !q))) return FAST_GPU_EINVAL;
  if (c->nnode <= 0) { c->err = "set_face_loads: no mesh"; return FAST_GPU_ESTATE; }
  if (nodes_per_face != 4 && nodes_per_face != 8) return FAST_GPU_ENOTSUP;
  if (ngp1d < 1 || ngp1d > 6) return FAST_GPU_EINVAL;
  const int nf = nodes_per_face;
  for (int64_t t = 0; t < (int64_t)num_faces * nf; t++)
    if (face_nodes[t] < 0 || face_nodes[t] >= c->nnode) {
      c->err = "set_face_loads: face node out of range";
      return FAST_GPU_EINVAL;
    }

  FCK(cudaStreamSynchronize(c->stream));
  free_face_loads(*c);
  // loaded nodes and, per node, its (face, local node) entries in face order
  std::vector<int32_t> cnt(c->nnode + 1, 0);
  for (int64_t t = 0; t < (int64_t)num_faces * nf; t++) cnt[face_nodes[t] + 1]++;
  std::vector<int32_t> node_of, pos(c->nnode, -1), ptr(1, 0);
  for (int64_t n = 0; n < c->nnode; n++)
    if (cnt[n + 1]) { pos[n] = (int32_t)node_of.size(); node_of.push_back((int32_t)n); ptr.push_back(cnt[n + 1]); }
  for (size_t j = 0; j + 1 < ptr.size(); j++) ptr[j + 1] += ptr[j];
  std::vector<int32_t> idx((size_t)num_faces * nf), fill(ptr.begin(), ptr.end() - 1), eqs(3 * node_of.size());
  for (int64_t t = 0; t < (int64_t)num_faces * nf; t++) idx[fill[pos[face_nodes[t]]]++] = (int32_t)t;
  for (size_t j = 0; j < node_of.size(); j++)
    for (int d = 0; d < 3; d++) eqs[3 * j + d] = c->h_eq[3 * (size_t)node_of[j] + d];
  std::vector<int32_t> fn(face_nodes, face_nodes + (int64_t)num_faces * nf), loc(num_faces, 0);
  if (local)
    for (int32_t k = 0; k < num_faces; k++) loc[k] = local[k];
  std::vector<double> fq(q, q + 3 * (int64_t)num_faces);
  FCK(up(&c->d_fn, fn));
  FCK(up(&c->d_floc, loc));
  FCK(up(&c->d_fq, fq));
  FCK(up(&c->d_fnode, node_of));
  FCK(up(&c->d_feq, eqs));
  FCK(up(&c->d_fptr, ptr));
  FCK(up(&c->d_fidx, idx));
  FCK(cudaMalloc((void **)&c->d_fe, sizeof(double) * 3 * std::max<int64_t>(1, (int64_t)num_faces * nf)));
  c->nface = num_faces;
  c->nfn = nf;
  c->face_ngp = ngp1d;
  c->nfnode = (int32_t)node_of.size();
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_face_load_device(fast_gpu_ctx *c, double scale, double *d_f) {
  if (!c || !d_f) return FAST_GPU_EINVAL;
  if (c->neq <= 0) { c->err = "face_load_device: no mesh"; return FAST_GPU_ESTATE; }
  FCK(cudaMemsetAsync(d_f, 0, sizeof(double) * c->neq, c->stream));
  if (c->nface == 0) return FAST_GPU_OK;
  const unsigned gf = (unsigned)((c->nface + 127) / 128);
  if (c->nfn == 4)
    face_forces<4><<<gf, 128, 0, c->stream>>>(c->nface, c->face_ngp, c->d_fn, c->d_fq, c->d_floc, c->d_X, c->d_fe);
  else
    face_forces<8><<<gf, 128, 0, c->stream>>>(c->nface, c->face_ngp, c->d_fn, c->d_fq, c->d_floc, c->d_X, c->d_fe);
  face_gather<<<(unsigned)((c->nfnode + 255) / 256), 256, 0, c->stream>>>(c->nfnode, c->d_feq, c->d_fptr, c->d_fidx,
                                                                          c->d_fe, scale, d_f);
  c->launches += 2;
  FCK(cudaGetLastError());
  return FAST_GPU_OK;
}

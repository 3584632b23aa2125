// reactions.cpp - support reactions at the current displacements
// (fast_gpu_support_reactions): cControl::SuppReactions (ctrl/ctrl.cpp:844-882).
//
//   R = sum over elements with a supported node of the element's internal
//       force, added to all its nodes (cElement::AddReactions,
//       elc/element.cpp:3106-3126), in element order;
//     - sum over face loads with a supported node of their nodal forces
//       (cElemLoad::HasSupp / AddReactions, load/load.cpp:726-760), and over
//       nodal loads on supported nodes (cNodalLoad::AddReactions, :586-600).
//
// The element forces come from the device (the internal-force kernels in
// element-output mode), the face loads from the host integrator with every
// DOF given an equation, so the forces on restrained DOFs are kept.
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

extern "C" int fast_gpu_support_reactions(fast_gpu_ctx *c, const uint8_t *supported, int32_t num_faces,
                                          int32_t nodes_per_face, const int32_t *face_nodes, const double *q,
                                          const int32_t *local, int32_t ngp1d, const double *nodal_f,
                                          double load_factor, double *R) {
  if (!c || !R || num_faces < 0 || (num_faces > 0 && (!face_nodes || !q))) return FAST_GPU_EINVAL;
  if (!c->d_X || c->nnode <= 0) { c->err = "support_reactions: no mesh"; return FAST_GPU_ESTATE; }
  if (c->has_ties()) { c->err = "tied interfaces support linear static solves only"; return FAST_GPU_ENOTSUP; }
  const int64_t nnode = c->nnode;
  // supported nodes: given, or every node with a DOF without an equation
  std::vector<uint8_t> sup(nnode, 0);
  for (int64_t n = 0; n < nnode; n++)
    sup[n] = supported ? (supported[n] != 0)
                       : (c->h_eq[3 * n] == 0 || c->h_eq[3 * n + 1] == 0 || c->h_eq[3 * n + 2] == 0);
  std::memset(R, 0, sizeof(double) * 3 * nnode);
  for (int b = 0; b < (int)c->buckets.size(); b++) {
    const Bucket &B = c->buckets[b];
    const int nn = B.nn;
    std::vector<int64_t> touch;  // caller-order elements with a supported node
    for (int64_t k = 0; k < B.ne; k++) {
      const int32_t *en = &B.h_conn[(size_t)B.inv[k] * nn];
      for (int a = 0; a < nn; a++)
        if (sup[en[a]]) { touch.push_back(k); break; }
    }
    if (touch.empty()) continue;
    // element forces of [first, last] in one call, in caller order
    const int64_t first = touch.front(), count = touch.back() - first + 1;
    std::vector<double> g((size_t)count * 3 * nn);
    const int rc = fast_gpu_element_matrices(c, FAST_ASM_INTERNAL_FORCE, b, first, count, g.data());
    if (rc != FAST_GPU_OK) return rc;
    for (int64_t k : touch) {
      const int32_t *en = &B.h_conn[(size_t)B.inv[k] * nn];
      const double *ge = &g[(size_t)(k - first) * 3 * nn];
      for (int a = 0; a < nn; a++)
        for (int i = 0; i < 3; i++) R[3 * (int64_t)en[a] + i] += ge[3 * a + i];
    }
  }
  if (num_faces > 0) {
    std::vector<int32_t> fsub, lsub;
    std::vector<double> qsub;
    int32_t nsub = 0;
    for (int32_t f = 0; f < num_faces; f++) {
      bool hit = false;
      for (int k = 0; k < nodes_per_face; k++) hit |= face_nodes[(size_t)f * nodes_per_face + k] >= 0 &&
                                                      face_nodes[(size_t)f * nodes_per_face + k] < nnode &&
                                                      sup[face_nodes[(size_t)f * nodes_per_face + k]];
      if (!hit) continue;
      fsub.insert(fsub.end(), face_nodes + (size_t)f * nodes_per_face, face_nodes + (size_t)(f + 1) * nodes_per_face);
      qsub.insert(qsub.end(), q + 3 * (size_t)f, q + 3 * (size_t)(f + 1));
      lsub.push_back(local ? local[f] : 0);
      nsub++;
    }
    if (nsub > 0) {
      std::vector<double> X((size_t)3 * nnode), ff((size_t)3 * nnode, 0.0);
      cudaError_t e = cudaMemcpy(X.data(), c->d_X, sizeof(double) * X.size(), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { c->err = std::string("support_reactions: ") + cudaGetErrorString(e); return FAST_GPU_ECUDA; }
      std::vector<int32_t> eq_all((size_t)3 * nnode);
      for (size_t i = 0; i < eq_all.size(); i++) eq_all[i] = (int32_t)i + 1;
      const int rc = fast_gpu_face_load_vector(nnode, X.data(), eq_all.data(), (int32_t)(3 * nnode), nsub,
                                               nodes_per_face, fsub.data(), qsub.data(), lsub.data(), ngp1d, ff.data());
      if (rc != FAST_GPU_OK) return rc;
      for (size_t i = 0; i < ff.size(); i++) R[i] -= load_factor * ff[i];
    }
  }
  if (nodal_f)
    for (int64_t n = 0; n < nnode; n++)
      if (sup[n])
        for (int i = 0; i < 3; i++) R[3 * n + i] -= load_factor * nodal_f[3 * n + i];
  return FAST_GPU_OK;
}

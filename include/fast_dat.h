/* fast_dat.h - C ABI of the deck reader in libfastgpu.so: the solid subset
 * of FAST's .dat input read on all host cores, straight into the arrays the
 * device mesh (fast_gpu_mesh / fast_gpu_bucket) takes.
 *
 * It replaces, for hex8 / hex20 solid decks, the reference's sequential
 * keyword loop InpReadData (main/input.cpp:355-401) with Utl::NextLabel
 * (main/utl.cpp:125-133) and the block readers that the hot path needs:
 *   %NODE, %NODE.COORD          cNode::ReadNumNode / ReadCoord (node/node.cpp:61-102)
 *   %NODE.SOLVER.ORDER          cNode::ReadSolverOrder (node/node.cpp:248-284)
 *   %NODE.SUPPORT               cNode::ReadSupp (node/node.cpp:289-330)
 *   %MATERIAL.ISOTROPIC         cMaterial::ReadElastIso (mat/material.cpp:95-119)
 *   %MATERIAL.DENSITY           cMaterial::ReadDensity (mat/material.cpp:721-745)
 *   %SECTION.HOMOGENEOUS.ISOTROPIC.3D  cSection::ReadHomIso3D (sec/section.cpp:96-119)
 *   %INTEGRATION.ORDER          cElement::ReadIntOrd (elc/element.cpp:194-228)
 *   %ELEMENT, %ELEMENT.BRICK8/BRICK8TL/BRICK20/BRICK20TL
 *                               cElement::ReadNumElm / ReadBrick* (elc/element.cpp:301-316,
 *                               1985-2090) with cElmParam::Read (elc/elmparam.cpp:221-247)
 *   %PATCH, %CONTROL.POINT.WEIGHT, %ELEMENT.BSPLINE.SOLID(TL)
 *                               one 'bspsol' patch with 'General' knot vectors (cBspPat::Read
 *                               geom/patch.cpp:1459-1484, cShapeBsp::ReadIGA shp/shpbsp.cpp:57-116)
 *   %LOAD.CASE.NODAL.FORCE      cLoad::ReadNodalLoads (load/load.cpp:53-87)
 *   %LOAD.CASE.AREA.UNIFORM     cLoad::ReadFaceUnifLoads + cFaceUnifLoad::Read
 *                               (load/load.cpp:229-248, 1440-1478)
 *   %HEADER.ANALYSIS.*          the cControl / cCtrlNewmark / cCtrlArcLength readers
 *                               named in main/input.cpp:196-215
 * with the reference's meaning of each record: the i-th %NODE.COORD record is
 * node i+1 (its own label is not used), sections, materials and elements are
 * addressed by label, integration orders by position, support and load
 * records by node label.  Labels outside their ranges, unreadable numbers and
 * elements not defined exactly once are errors (the reference stops there).
 * Other blocks are skipped, as the reference skips labels it does not know.
 *
 * Status codes are fast_gpu.h's (FAST_GPU_OK, FAST_GPU_EINVAL for a deck
 * error, FAST_GPU_ENOTSUP for decks outside this subset: more than one
 * element type or integration order, ties, other patch kinds, area loads on
 * B-spline solids). */
#ifndef FAST_DAT_H
#define FAST_DAT_H

#include <stdint.h>

#include "fast_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fast_dat fast_dat;

typedef struct {
  int64_t num_nodes;
  int64_t num_elems;
  int64_t num_faces;          /* %LOAD.CASE.AREA.UNIFORM records                     */
  int32_t nodes_per_face;     /* 4 (Q4 faces of hex8) or 8 (Q8 faces of hex20)       */
  int32_t elem_type;          /* FAST_ELEM_HEX8, FAST_ELEM_HEX20 or FAST_ELEM_BSP_SOLID  */
  int32_t nodes_per_elem;     /* 8, 20 or the patch's (p+1)(q+1)(r+1)                */
  int32_t formulation;        /* FAST_FORM_SMALL_STRAIN or FAST_FORM_TOTAL_LAGRANGIAN */
  int32_t ngp[3];             /* Gauss points per direction (the deck's one order)   */
  int32_t has_density;        /* %MATERIAL.DENSITY present                           */
  int32_t has_solver_order;   /* %NODE.SOLVER.ORDER present                          */
  int32_t has_nodal_forces;   /* %LOAD.CASE.NODAL.FORCE present                      */
  int32_t max_iter;           /* MAXIMUM.ITERATIONS (0 when absent)                  */
  int32_t max_steps;          /* MAXIMUM.STEPS (1)                                   */
  int32_t target_iter;        /* TARGET.ITERATIONS (-1 when absent)                  */
  int32_t print_step;         /* PRINT.STEPS (1)                                     */
  int32_t has_arc_length;     /* ARC-LENGTH present                                  */
  double  tol;                /* TOLERANCE (1e-5)                                    */
  double  step_factor;        /* STEP.FACTOR (1)                                     */
  double  arc_load_coeff;     /* ARC-LENGTH load coefficient                         */
  double  time_step;          /* TIME.STEP (0)                                       */
  double  newmark[2];         /* NEWMARK.PARAMETERS gamma, beta (0.5, 0.25)          */
  char    algorithm[32];      /* ALGORITHM, without quotes ("" when absent)          */
  char    matrix_type[32];    /* MATRIX.TYPE, without quotes                         */
  char    title[128];         /* first line after %HEADER                            */
  /* B-spline solid decks (elem_type FAST_ELEM_BSP_SOLID) */
  int32_t patch_degree[3];
  int32_t patch_num_knots[3]; /* knot vector lengths, multiplicities expanded         */
  int32_t patch_rational;
  int32_t has_weights;        /* %CONTROL.POINT.WEIGHT present                       */
  int64_t patch_num_cps;      /* control points of the patch                         */
} fast_dat_info;

/* Reads the deck at path with up to `threads` host threads (0: all cores).
 * On success *out holds the deck (release it with fast_dat_free).  On a deck
 * error *out still holds a handle whose fast_dat_error() says what and
 * where (file line); release it too.  *out is NULL only when memory ran out
 * or out itself is NULL. */
int fast_dat_read(const char *path, int32_t threads, fast_dat **out);
const char *fast_dat_error(const fast_dat *dat);
void fast_dat_free(fast_dat *dat);

int fast_dat_get_info(const fast_dat *dat, fast_dat_info *info);
/* coords [num_nodes][3]; fixed [num_nodes][3] (1 = restrained), solver_rank
 * [num_nodes] (the 1-based %NODE.SOLVER.ORDER entry of each node), nodal_f
 * [num_nodes][3] (summed nodal forces); any output may be NULL. */
int fast_dat_get_nodes(const fast_dat *dat, double *coords, uint8_t *fixed, int64_t *solver_rank, double *nodal_f);
/* conn [num_elems][nodes_per_elem] 0-based node indices in FAST's local
 * order, element i = label i+1; E, nu, rho [num_elems]; any may be NULL. */
int fast_dat_get_elements(const fast_dat *dat, int32_t *conn, double *E, double *nu, double *rho);
/* elem [num_faces] 0-based element, corners [num_faces][3] 0-based nodes as
 * written, face_nodes [num_faces][nodes_per_face] the loaded face in its
 * face-shape order (the first face of the element's cShapeBrick8/20::GetFace
 * table, shp/shpsolid.cpp:264-276, 459-471, whose corners hold the three),
 * local [num_faces], q [num_faces][3]: face_nodes, q and local are the
 * arguments fast_gpu_set_face_loads and fast_gpu_face_load_vector take; any
 * output may be NULL. */
int fast_dat_get_faces(const fast_dat *dat, int32_t *elem, int32_t *corners, int32_t *face_nodes, int32_t *local,
                       double *q);
/* B-spline solid decks: knots (the three expanded vectors one after the
 * other), span [num_elems][3] 0-based non-zero knot spans, weights
 * [num_nodes] (1 where none is given), cps [patch_num_cps] the node of each
 * patch control point (r fastest); any may be NULL. */
int fast_dat_get_patch(const fast_dat *dat, double *knots, int32_t *span, double *weights, int32_t *cps);
/* A bucket whose arrays point into the deck (valid until fast_dat_free):
 * uploads without copies through fast_gpu_mesh.buckets. */
int fast_dat_bucket(const fast_dat *dat, fast_gpu_bucket *bucket);

#ifdef __cplusplus
}
#endif

#endif /* FAST_DAT_H */

/* fast_pos.h - C ABI of the result writer in libfastgpu.so: FAST's .pos
 * output for solid decks, formatted on all host cores.
 *
 * It writes what the reference's main program and controller write
 * (main/main.cpp:108-121, cControl::PrintResult ctrl/ctrl.cpp:1117-1304,
 * cControl::End :597-622), byte for byte for the blocks below:
 *   "%HEADER", the generator line, the deck's own text from its second line
 *   up to "%END" (InpCopyData, main/input.cpp:405-420);
 *   at the first step "%RESULT" and "%RESULT.CASE" with the blank step-list
 *   area (13 spaces per line, floor(1.1 * max_steps) + 1 lines);
 *   per step: %RESULT.CASE.STEP, .FACTOR, .NODAL.DISPLACEMENT (six values,
 *   the rotations 0 for solids), .NODAL.REACTIONS when given, .ELEMENT.GAUSS.SCALAR(.DATA)
 *   (cControl::PrintIntPntStress :2189-2260), .ELEMENT.NODAL.SCALAR(.DATA)
 *   (PrintNodalStress :2264-2320) and, when asked for, .NODAL.SCALAR(.DATA)
 *   (PrintAvrNodalStress :2397-2470), and for Newmark the .VELOCITY and
 *   .ACCELERATION blocks;
 *   the vibration or buckling modes of an eigen analysis;
 *   at the end "%END" and the step list written over the blank area (after
 *   it when no step was printed, as for a modal analysis).
 * Numbers are printed as iostream prints them with scientific, showpos and
 * setprecision(precision): a sign, one digit, the point, `precision` digits,
 * the exponent with at least two digits.  Node i is label i+1, element k
 * label k+1, stresses in Voigt order xx yy zz xy xz yz.  The IGA and
 * micro-model blocks are not written.  Status codes are fast_gpu.h's (FAST_GPU_EINVAL for bad
 * arguments or an I/O error). */
#ifndef FAST_POS_H
#define FAST_POS_H

#include <stdint.h>

#include "fast_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fast_pos fast_pos;

typedef struct {
  const char *header_line;  /* the file's second line, without newline (NULL: the library's own) */
  int32_t precision;        /* %HEADER.OUTPUT.PRECISION (the reference's default is 5) */
  int32_t max_steps;        /* MAXIMUM.STEPS: sizes the step-list area                 */
  int32_t print_average;    /* %HEADER.PRINT.AVERAGE.NODAL.STRESS: write .NODAL.SCALAR  */
  int32_t threads;          /* formatting threads, 0: all cores                         */
} fast_pos_opts;

/* Creates pos_path and writes the header and the echo of the deck at
 * dat_path.  *out is set whenever it is not NULL and memory allowed; on an
 * error fast_pos_error() says why; release it with fast_pos_free. */
int fast_pos_open(const char *pos_path, const char *dat_path, const fast_pos_opts *opts, fast_pos **out);
/* One printed step.  displ [num_nodes][3]; gauss_stress [num_elems][points][6]
 * and elem_nodal [num_elems][nodes_per_elem][6] may be NULL (block not
 * written); nodal_avg [num_nodes][6] is required when print_average. */
int fast_pos_step(fast_pos *pos, double factor, int64_t num_nodes, const double *displ, int64_t num_elems,
                  int32_t points, const double *gauss_stress, int32_t nodes_per_elem, const double *elem_nodal,
                  const double *nodal_avg);
/* Support reactions for the next fast_pos_step, printed after its
 * displacements (%RESULT.CASE.STEP.NODAL.REACTIONS, ctrl/ctrl.cpp:1222-1257,
 * when %HEADER.PRINT.SUPPORT.REACTIONS is set): nodes [count] the 0-based
 * supported nodes in ascending order, R [count][3] (e.g. the supported rows
 * of fast_gpu_support_reactions); five digits as the reference prints them. */
int fast_pos_reactions(fast_pos *pos, int64_t count, const int64_t *nodes, const double *R);
/* Nodal velocities and accelerations of a printed Newmark step, after its
 * fast_pos_step (cCtrlNewmark::PrintVelAcc, ctrl/ctrlnewmark.cpp:282-330):
 * v, a [num_nodes][3], rotations printed 0. */
int fast_pos_velacc(fast_pos *pos, int64_t num_nodes, const double *v, const double *a);
/* Eigen-analysis output (cCtrlModal::PrintMode ctrl/ctrlmodal.cpp:129-156,
 * cCtrlLinStab::PrintMode ctrl/ctrllinstab.cpp:156-185): the .MODES header,
 * then per mode its value (natural frequency, or buckling factor) and its
 * eigenvector block.  modes [num_modes][num_nodes][3] (rotations printed 0). */
#define FAST_POS_VIBRATION 0
#define FAST_POS_BUCKLING  1
int fast_pos_modes(fast_pos *pos, int32_t kind, int32_t num_modes, const double *values, int64_t num_nodes,
                   const double *modes);
/* "%END" and the step list; the file is complete after this. */
int fast_pos_finish(fast_pos *pos);
const char *fast_pos_error(const fast_pos *pos);
void fast_pos_free(fast_pos *pos);   /* closes the file if still open */

#ifdef __cplusplus
}
#endif

#endif /* FAST_POS_H */

/*
 * pcfd_oracle.h -- CPU restatement (FP64, OpenMP) of the ParaCFD composite pressure operator,
 * its multigrid preconditioner and Krylov solvers, and the projection divergence/correction.
 * TEST INFRASTRUCTURE: used by tests/ as a checker and by bench.py's CPU-baseline leg only.
 *
 * Follows (reference paths): CompositeAmrPressureSystem::apply_cpu / diagonal_cpu
 * (src/core/fluid/amr_pressure.cpp:498-543), DeviceCompositeAmrPressureSolver setup, V-cycle,
 * PCG and GCRO (src/core/fluid/amr_pressure.cu:857-1154, 1267-1698), composite_amr_divergence_cpu
 * / _projection_rhs_cpu / _correct_fluxes_cpu (amr_pressure.cpp:479-496).  The reference has no
 * CPU pressure solver; this file is the CPU one.
 */
#ifndef PCFD_ORACLE_H
#define PCFD_ORACLE_H
#include "../include/paracfd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct po_system po_system;

po_system* po_create(const pcfd_topology* topology);
void po_destroy(po_system* s);
int po_threads(void);
void po_apply(po_system* s, const double* p, double* out, int orthogonal);
void po_diagonal(po_system* s, double* diagonal);
void po_precondition(po_system* s, const double* r, double* z);
/* From now on po_precondition / po_solve use the composite cycle of paracfd_b200 (its
 * PCFD_MG_CYCLE_COMPOSITE in FP64): `steps` smoothing steps per stage (0: 6), Chebyshev stage
 * smoothing on [2 / stage_ratio, 2] (< 2: damped Jacobi), fine Chebyshev-Richardson steps on
 * [2 / fine_ratio, 2] (< 2: w = 2/3), an explicit inverse on a coarsest stage of <= 512 cells. */
void po_set_composite(po_system* s, int steps, int stage_ratio, int fine_ratio);
/* returns converged; out[0] relative residual, out[1] iterations, out[2] preconditioner applications */
int po_solve(po_system* s, double* x, const double* b, double tolerance, int max_iterations, int warm_start,
             double* out3);
/* faces in the compact per-brick layout of paracfd_b200.h; special velocities FP32 (cf then eb) */
void po_divergence(po_system* s, const float* u, const float* v, const float* w, const float* special,
                   double* integrated, double* divergence);
void po_correct(po_system* s, const double* pressure, double rho, double dt, float* u, float* v, float* w,
                float* special);

#ifdef __cplusplus
}
#endif
#endif

/*
 * pdlpgpu_components.h -- the engine's building blocks, one call each, for
 * parity testing against the reference's components and for diagnostics.
 * Host arrays in the caller's (original) order; each call uploads, runs the
 * device kernels of that component once, and downloads.
 *
 * Each entry point replaces one reference routine:
 */
#ifndef PDLPGPU_COMPONENTS_H
#define PDLPGPU_COMPONENTS_H

#include "pdlpgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SparseMatrix::multiply / transposeMultiply
 * (pdlp_engine/src/sparse_matrix.cpp:343-419): out = A x, or A^T y when
 * `transpose` is 1. `precision` 0 computes in FP64, 1 in FP32 (inputs and
 * outputs are converted). Returns 0 on success. */
int32_t pdlpgpu_spmv(const pdlpgpu_lp* lp, int32_t transpose, int32_t precision,
                     const double* in, double* out);

/* RuizScaler::equilibrate (pdlp_engine/src/scaling.cpp:55-136): the row and
 * column scale vectors and the scaled coefficients in canonical CSR order
 * (any output may be NULL). Returns 0 on success. */
int32_t pdlpgpu_ruiz(const pdlpgpu_lp* lp, int32_t iterations, double* row_scale,
                     double* col_scale, double* scaled_values);

/* Preconditioner::compute (pdlp_engine/src/preconditioner.cpp:31-80) on the
 * given matrix. Returns 0 on success. */
int32_t pdlpgpu_precondition(const pdlpgpu_lp* lp, double* tau, double* tau_inverse,
                             double* sigma, double* sigma_inverse);

/* CpuPdhgKernel::trial (pdlp_engine/src/pdhg_kernel.cpp:189-277) on an
 * explicit state of the given (working) LP: x', y', A x' and the reductions
 * {sum dx^2/tau, sum dy^2/sigma, dy'A dx}. `precision` as for pdlpgpu_spmv.
 * Returns 0 on success. */
int32_t pdlpgpu_trial(const pdlpgpu_lp* lp, int32_t precision, const double* tau,
                      const double* tau_inverse, const double* sigma,
                      const double* sigma_inverse, const double* x, const double* y,
                      const double* ax, double step, double weight, double* x_out,
                      double* y_out, double* ax_out, double* reductions);

/* TerminationChecker::evaluate (pdlp_engine/src/termination.cpp:211-325) of
 * (x, y), and InfeasibilityDetector::testDualRay / testPrimalRay
 * (pdlp_engine/src/infeasibility.cpp:51-192) of the directions y - ry and
 * x - rx. metrics[8] = {primal objective, dual objective, primal residual,
 * dual residual, relative gap, kkt, finite, dual valid}; verdicts[6] =
 * {dual proves, dual value, dual relative violation, primal proves, primal
 * value, primal relative violation}. Returns 0 on success. */
int32_t pdlpgpu_evaluate(const pdlpgpu_lp* lp, double infeasibility_tolerance,
                         const double* x, const double* y, const double* rx,
                         const double* ry, double* metrics, double* verdicts);

/* Layout statistics without a device (host only): slices, slots and real
 * entries of both sides, for the tuning in `ext` (NULL = autotune).
 * stats[8] = {a slices, a slots, a entries, at slices, at slots, at entries,
 * lane elements, vector width}. Returns 0, or -1 for an invalid matrix. */
int32_t pdlpgpu_layout_stats(const pdlpgpu_lp* lp, const pdlpgpu_ext_options* ext,
                             int64_t* stats);

/* The layout's own product on the host (no device): walks the SELL-G slices
 * exactly as the kernels do, to show the layout encodes A. out = A x. */
int32_t pdlpgpu_layout_multiply(const pdlpgpu_lp* lp, const pdlpgpu_ext_options* ext,
                                const double* x, double* out);

#ifdef __cplusplus
}
#endif

#endif

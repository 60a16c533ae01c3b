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

/* No counterpart in the reference. The fused trial of pdlpgpu_trial for
 * callers that cannot let the library allocate device memory: a process that
 * owns all device memory through its own pool and budget, or a loop that must
 * not take the device-wide synchronisation of cudaMalloc. Every pointer is
 * device memory the caller owns: A and A^T as CSR (int64 starts, int32
 * indices, FP64 values), the vectors of pdlpgpu_trial, the outputs, and
 * `reductions` (3 doubles: sum dx^2/tau, sum dy^2/sigma, dy'A dx). `stream`
 * is a cudaStream_t (NULL = default stream); the call only enqueues work.
 * Scratch is a fixed 192 KiB static device array inside the library, so rows
 * and columns are limited to 8,388,608 each (larger sizes are rejected with an
 * error), and a NULL pointer that a launch would read or write is rejected
 * before anything is enqueued. The first call in each CUDA context (the
 * device's primary context, again after cudaDeviceReset, or a caller's own
 * driver context) looks up that array's address in that context, so make the
 * first call in each context before any stream capture. All calls share
 * the array: calls that overlap on the GPU race; each call writes every slot
 * it later reads, so nothing needs clearing between calls. Returns 0, or -1
 * with pdlpgpu_last_error() set. */
int32_t pdlpgpu_trial_noalloc(int32_t rows, int32_t cols, const int64_t* a_row_start,
                              const int32_t* a_col_index, const double* a_values,
                              const int64_t* at_row_start, const int32_t* at_col_index,
                              const double* at_values, const double* objective,
                              const double* var_lower, const double* var_upper,
                              const double* tau, const double* tau_inverse,
                              const double* row_lower, const double* row_upper,
                              const double* sigma, const double* sigma_inverse,
                              const double* x, const double* y, const double* ax, double step,
                              double weight, double* x_out, double* y_out, double* ax_out,
                              double* reductions, void* stream);

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

/* No counterpart in the reference (pdlp_engine/README.md:226-233 names it as
 * the restart metric still missing there): the normalised duality gap
 * rho(r; z) of z = (x, y) for L(x, y) = c'x + y'Ax - h*(y) (h* the support
 * function of the row bounds) over the box of x and the dual domain, in the
 * ball ||(dx, dy)||_w^2 = w ||dx||^2 + ||dy||^2 / w <= r^2 whose radius r is
 * the distance from z to (x_ref, y_ref). g = c + A'y [n] and a = A x [m] are
 * given; bounds may be infinite. out[2] = {gap, radius}; the gap is +inf
 * when the radius is zero. The device routine is the one the check stage
 * uses for PDLPGPU_RESTART_NORMALIZED_GAP. Returns 0 on success. */
int32_t pdlpgpu_normalized_gap(int32_t n, int32_t m, double weight, const double* x,
                               const double* g, const double* x_lower, const double* x_upper,
                               const double* x_ref, const double* y, const double* a,
                               const double* r_lower, const double* r_upper, const double* y_ref,
                               double* out);

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

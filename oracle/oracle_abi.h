/*
 * oracle_abi.h -- the C interface shared by the two CPU oracles of this
 * repository. TEST INFRASTRUCTURE ONLY: nothing in the product links it.
 *
 *   oracle/_ref/libpdlp_ref*.so  the reference pdlp_engine compiled from its own
 *                                sources, wrapped by ref_shim.cpp
 *   oracle/_port/libpdlp_port.so the plain-C restatement in pdlp_port.c
 *
 * Both export exactly these symbols, so a test can run the same case through
 * either one and compare.  Every routine works on the serial path of the
 * reference (threadCount = 1), which is the deterministic one.
 */
#ifndef PDLP_ORACLE_ABI_H
#define PDLP_ORACLE_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A linear program in the reference's CompiledLp form
 * (pdlp_engine/include/pdlp/compiled_lp.h:13-28):
 *   minimize c'x + offset  s.t.  rowLower <= A x <= rowUpper,
 *                                varLower <= x <= varUpper.
 * A is canonical CSR: rows sorted by column, no duplicates, no zeros --
 * what SparseMatrix::fromTriplets produces. Infinite bounds are IEEE inf. */
typedef struct orc_lp {
    int32_t rows;
    int32_t cols;
    int64_t nnz;
    const int64_t* row_start;
    const int32_t* col_index;
    const double* values;
    const double* objective;
    double objective_offset;
    const double* row_lower;
    const double* row_upper;
    const double* var_lower;
    const double* var_upper;
} orc_lp;

/* PdlpOptions field for field (pdlp_engine/include/pdlp/pdlp_options.h:7-75).
 * Booleans are int32 0/1. */
typedef struct orc_options {
    int64_t iteration_limit;
    double time_limit_seconds;
    double primal_tolerance;
    double dual_tolerance;
    double gap_tolerance;
    int32_t termination_check_frequency;
    int32_t power_iteration_count;
    int32_t thread_count;
    int64_t parallel_nonzero_threshold;
    double initial_step_safety;
    double minimum_step_scale;
    double maximum_primal_weight;
    double minimum_primal_weight;
    int32_t use_ruiz_scaling;
    int32_t ruiz_iterations;
    int32_t detect_infeasibility;
    double infeasibility_tolerance;
    int32_t use_diagonal_preconditioning;
    int32_t use_adaptive_linesearch;
    int32_t maximum_step_trials;
    int32_t use_averaging;
    int32_t use_restarts;
    int32_t use_feasibility_polishing;
    int32_t minimum_restart_iterations;
    int32_t maximum_restart_iterations;
    double restart_sufficient_decay;
    double restart_necessary_decay;
    double restart_artificial_fraction;
    double initial_primal_weight;
    double primal_weight_smoothing;
    int32_t polishing_iterations;
} orc_options;

/* PdlpResult's scalars (pdlp_engine/include/pdlp/pdlp_result.h:26-62). */
typedef struct orc_result {
    int32_t status;          /* PdlpStatus order: 0 optimal .. 6 invalid_problem */
    int32_t has_dual_ray;
    int32_t has_primal_ray;
    int32_t restart_count;
    int64_t iterations;
    int64_t step_trials;
    double primal_objective;
    double dual_objective;
    double primal_residual;
    double dual_residual;
    double relative_gap;
    double solve_time_seconds;
    double final_step_size;
    double static_step_bound;
    double final_primal_weight;
    int32_t primal_size;     /* 0 when the result carries no point */
    int32_t dual_size;
    char message[160];
} orc_result;

void orc_default_options(orc_options* options);

/* PdlpSolver::solve. primal/dual/dual_ray/primal_ray are caller buffers of
 * length cols/rows/rows/cols; each may be NULL. Returns the status. */
int orc_solve(const orc_lp* lp, const orc_options* options, double* primal,
              double* dual, double* dual_ray, double* primal_ray, orc_result* out);

/* SparseMatrix::fromTriplets. Output arrays are sized for `count` entries;
 * *nnz_out receives the merged count. Returns 0, or -1 for invalid input. */
int orc_from_triplets(int32_t rows, int32_t cols, int64_t count,
                      const int32_t* row, const int32_t* col, const double* value,
                      int64_t* row_start, int32_t* col_index, double* values,
                      int64_t* col_start, int32_t* row_index, double* csc_values,
                      int64_t* nnz_out);

/* SparseMatrix::multiply / transposeMultiply (serial). */
void orc_multiply(const orc_lp* lp, const double* x, double* ax);
void orc_transpose_multiply(const orc_lp* lp, const double* y, double* aty);

/* RuizScaler::equilibrate: scale vectors, the scaled CSR values, and the
 * scaled objective and bounds. Any output may be NULL. */
void orc_ruiz(const orc_lp* lp, int32_t iterations, double* row_scale,
              double* col_scale, double* scaled_values, double* scaled_objective,
              double* scaled_row_lower, double* scaled_row_upper,
              double* scaled_var_lower, double* scaled_var_upper);
double orc_condition_spread(const orc_lp* lp);

/* Preconditioner::compute and estimateSpectralNorm. */
void orc_precondition(const orc_lp* lp, int32_t enabled, double* tau,
                      double* tau_inverse, double* sigma, double* sigma_inverse);
double orc_spectral_norm(const orc_lp* lp, int32_t iterations, int32_t* converged);

/* CpuPdhgKernel::trial on an explicit state (serial). reductions[0..2] =
 * primal movement, dual movement, interaction; returns finite flag. */
int orc_trial(const orc_lp* working, const double* tau, const double* tau_inverse,
              const double* sigma, const double* sigma_inverse, const double* x,
              const double* y, const double* ax, double step, double weight,
              double* x_out, double* y_out, double* ax_out, double* reductions);

/* TerminationChecker::evaluate. metrics = {primalObjective, dualObjective,
 * primalResidual, dualResidual, relativeGap, kktScore, finite, dualValid}. */
void orc_evaluate(const orc_lp* lp, const double* x, const double* y, double* metrics);

/* InfeasibilityDetector::testDualRay / testPrimalRay.
 * verdict = {proves, certificateValue, relativeViolation}. */
void orc_test_dual_ray(const orc_lp* lp, double tolerance, const double* direction,
                       double* verdict);
void orc_test_primal_ray(const orc_lp* lp, double tolerance, const double* direction,
                         double* verdict);

#ifdef __cplusplus
}
#endif

#endif

/*
 * pdlpgpu.h -- C ABI of the B200-native PDLP engine.
 *
 * A drop-in for the PDLP dispatch target of Aryan-Kumar06/optimisation_solver:
 *
 *   pdlp::PdlpResult pdlp::PdlpSolver::solve(const CompiledLp&, const PdlpOptions&) const
 *   (pdlp_engine/include/pdlp/pdlp_solver.h:9-15, called by solver::runPdlp at
 *    src/solver/orchestrator.cpp:337)
 *
 * Plain pointers and sizes only; no C++ or CUDA types cross this boundary.
 * The header-only C++ facade in pdlpgpu.hpp restores the reference signature.
 *
 * Conventions kept from the reference:
 *   - the LP is  min c'x + offset  s.t.  row_lower <= A x <= row_upper,
 *     var_lower <= x <= var_upper, IEEE +-inf for absent bounds
 *     (pdlp_engine/include/pdlp/compiled_lp.h:13-28);
 *   - row duals carry the PDLP sign: stationarity is c + A'y
 *     (include/adapter/pdlp_adapter.h:18-28);
 *   - solve never throws / aborts: invalid input or options give status
 *     INVALID_PROBLEM with a message (pdlp_engine/src/pdlp_solver.cpp:121-134),
 *     CUDA errors give NUMERICAL_FAILURE with the CUDA error string.
 */
#ifndef PDLPGPU_H
#define PDLPGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDLPGPU_ABI_VERSION 1

/* PdlpStatus, same order and spellings (pdlp_engine/include/pdlp/pdlp_result.h:10-24,
 * pdlp_engine/src/pdlp_solver.cpp:103-114). */
enum {
    PDLPGPU_OPTIMAL = 0,
    PDLPGPU_INFEASIBLE = 1,
    PDLPGPU_UNBOUNDED = 2,
    PDLPGPU_ITERATION_LIMIT = 3,
    PDLPGPU_TIME_LIMIT = 4,
    PDLPGPU_NUMERICAL_FAILURE = 5,
    PDLPGPU_INVALID_PROBLEM = 6
};

/* Replaces pdlp::CompiledLp (pdlp_engine/include/pdlp/compiled_lp.h:17-63).
 * The matrix is CSR with int64 row starts, int32 column indices and float64
 * values, as SparseMatrix stores it (pdlp_engine/include/pdlp/sparse_matrix.h:128-130).
 * Non-canonical input (unsorted rows, duplicate entries, explicit zeros) is
 * canonicalised as SparseMatrix::fromTriplets does. All arrays are borrowed. */
typedef struct pdlpgpu_lp {
    int32_t num_rows;
    int32_t num_cols;
    const int64_t* row_start;      /* [num_rows + 1] */
    const int32_t* col_index;      /* [row_start[num_rows]] */
    const double* values;          /* [row_start[num_rows]] */
    const double* objective;       /* [num_cols] */
    double objective_offset;
    const double* row_lower;       /* [num_rows] */
    const double* row_upper;       /* [num_rows] */
    const double* var_lower;       /* [num_cols] */
    const double* var_upper;       /* [num_cols] */
} pdlpgpu_lp;

/* Replaces pdlp::PdlpOptions field for field, same defaults
 * (pdlp_engine/include/pdlp/pdlp_options.h:7-75). Booleans are int32 0/1.
 * thread_count and parallel_nonzero_threshold are accepted and ignored: the
 * device engine has no host worker pool. */
typedef struct pdlpgpu_options {
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
} pdlpgpu_options;

/* Precision of the PDHG iterations. */
enum {
    PDLPGPU_PRECISION_FP64 = 0,   /* FP64 everywhere: the reference's arithmetic */
    PDLPGPU_PRECISION_MIXED = 1   /* FP32 A and iterates; FP64 checks, objective, final FP64 stage */
};

/* Device layout of a session's trial kernels. */
enum {
    PDLPGPU_LAYOUT_AUTO = 0,         /* interleaved for sessions of 16 or more instances */
    PDLPGPU_LAYOUT_SELL = 1,         /* one SELL-G matrix walk per instance */
    PDLPGPU_LAYOUT_INTERLEAVED = 2   /* vectors [line][instance]; a warp serves 32 instances */
};

/* Score of the restart test (RestartController::choose, restart_controller.cpp:8-63,
 * keeps its thresholds and decisions; only the compared score changes). */
enum {
    PDLPGPU_RESTART_KKT = 0,         /* the reference's: the relative KKT error of each candidate */
    PDLPGPU_RESTART_NORMALIZED_GAP = 1 /* the normalised duality gap of each candidate at the radius
                                        * of its distance to the last restart point (weighted by
                                        * the primal weight, in the scaled space of the iterations);
                                        * pdlp_engine/README.md:226-233 names it as the missing metric */
};

/* Extensions with no counterpart in PdlpOptions. Zero means "default". */
typedef struct pdlpgpu_ext_options {
    int32_t precision;             /* PDLPGPU_PRECISION_* */
    int32_t device;                /* CUDA device ordinal */
    int32_t lane_elements;         /* SpMV tuning: target nonzeros per lane (0 = autotune) */
    int32_t vector_width;          /* SpMV tuning: 1, 2 or 4 elements per lane load (0 = autotune) */
    int32_t chunk_slack;           /* extra trial slots per captured check interval (0 = 4) */
    int32_t fp32_stall_checks;     /* mixed: checks without progress before the FP64 stage (0 = 8) */
    int32_t fp32_switch_factor;    /* mixed: stalls count once the best KKT <= min(factor * tol, 1e-5) (0 = 1000) */
    int32_t disable_graphs;        /* 1: launch kernels directly instead of CUDA graphs */
    int32_t cta_slots;             /* SpMV tuning: matrix slots per CTA (0 = autotune) */
    int32_t layout;                /* sessions: PDLPGPU_LAYOUT_* */
    int32_t lane_instances;        /* interleaved layout: instances per lane, 1, 2 or 4 (0 = auto) */
    int32_t two_kernel_trials;     /* 1: never fuse a check interval's trials into one cluster launch */
    int32_t restart_metric;        /* PDLPGPU_RESTART_*: the score the restart test compares */
    int32_t reserved[3];
} pdlpgpu_ext_options;

/* Optional warm start (this engine's extension; the reference starts from the
 * box projection of 0 and y = 0, pdlp_engine/src/pdlp_solver.cpp:168-176).
 * Original coordinates, PDLP dual sign. Any pointer may be NULL. The starting
 * point is the better, by KKT score, of the warm point and the cold point. */
typedef struct pdlpgpu_warmstart {
    const double* primal;          /* [num_cols] */
    const double* row_dual;        /* [num_rows] */
    double primal_weight;          /* <= 0: use options.initial_primal_weight */
} pdlpgpu_warmstart;

/* Replaces pdlp::PdlpResult (pdlp_engine/include/pdlp/pdlp_result.h:26-62).
 * Arrays are owned by the result and released by pdlpgpu_result_free. */
typedef struct pdlpgpu_result {
    int32_t status;
    char status_message[160];
    int32_t num_rows;
    int32_t num_cols;
    double* primal;                /* [num_cols] or NULL when no point exists */
    double* row_dual;              /* [num_rows] or NULL */
    double* dual_ray;              /* [num_rows] when status == INFEASIBLE, else NULL */
    double* primal_ray;            /* [num_cols] when status == UNBOUNDED, else NULL */
    double primal_objective;
    double dual_objective;
    double primal_residual;
    double dual_residual;
    double relative_gap;
    int64_t iterations;
    int64_t step_trials;
    int32_t restart_count;
    double solve_time_seconds;
    double final_step_size;
    double static_step_bound;
    double final_primal_weight;
    /* extensions */
    int32_t precision_used;        /* 0 fp64, 1 fp32 only, 2 fp32 then fp64 */
    int64_t fp64_iterations;       /* iterations run in the FP64 stage of a mixed solve */
    double device_seconds;         /* CUDA-event time of the iteration loop */
} pdlpgpu_result;

/* --- entry points --------------------------------------------------------- */

/* Fill with the reference defaults (pdlp_options.h:7-75) / zero extensions. */
void pdlpgpu_default_options(pdlpgpu_options* options);
void pdlpgpu_default_ext_options(pdlpgpu_ext_options* ext);

/* PdlpSolver::solve. `warm` and `ext` may be NULL. *result is allocated by the
 * engine. Returns the status. */
int32_t pdlpgpu_solve(const pdlpgpu_lp* lp, const pdlpgpu_options* options,
                      const pdlpgpu_warmstart* warm, pdlpgpu_result** result);
int32_t pdlpgpu_solve_ex(const pdlpgpu_lp* lp, const pdlpgpu_options* options,
                         const pdlpgpu_ext_options* ext, const pdlpgpu_warmstart* warm,
                         pdlpgpu_result** result);

/* Many independent LPs of any sizes in one batched device solve (no
 * counterpart in the reference, which solves one LP per call). results[i]
 * receives instance i. `warm` may be NULL or hold NULL entries. Returns the
 * number of instances that ended OPTIMAL, or -1 on a setup failure. */
int32_t pdlpgpu_solve_batch(const pdlpgpu_lp* const* lps, int32_t count,
                            const pdlpgpu_options* options, const pdlpgpu_ext_options* ext,
                            const pdlpgpu_warmstart* const* warm, pdlpgpu_result** results);

/* Times the two PDHG trial kernels of a batch of LPs (as pdlpgpu_solve_batch
 * lays them out) with CUDA events, `reps` launches each, every instance
 * active, after the setup; no solve. out[6] = {primal ms per launch, dual ms
 * per launch, primal algorithmic bytes per launch, dual algorithmic bytes per
 * launch, padded slots of the A^T side, padded slots of the A side}. No
 * counterpart in the reference. Returns 0, or -1 with pdlpgpu_last_error(). */
int32_t pdlpgpu_batch_time_kernels(const pdlpgpu_lp* const* lps, int32_t count,
                                   const pdlpgpu_options* options, const pdlpgpu_ext_options* ext,
                                   int32_t reps, double* out);

void pdlpgpu_result_free(pdlpgpu_result* result);

/* toString(PdlpStatus) (pdlp_engine/src/pdlp_solver.cpp:103-114). */
const char* pdlpgpu_status_string(int32_t status);

/* Last error text of the calling thread (setup failures). */
const char* pdlpgpu_last_error(void);

/* Number of CUDA devices visible (0 on a host without a GPU). */
int32_t pdlpgpu_device_count(void);

#ifdef __cplusplus
}
#endif

#endif /* PDLPGPU_H */

/*
 * pdlpgpu_presolve.h -- the reference's presolve, fast and exact.
 *
 * pdlpgpu_presolve replaces presolve::Presolver::run
 * (include/presolve/presolver.h:11, src/presolve/presolver.cpp:1045-1155), the
 * single presolve pass that solver::solve runs on every model before the
 * engines (src/solver/orchestrator.cpp:596-597). It returns the reference's
 * PresolveResult (include/presolve/presolve_result.h:10-25) field for field:
 * the reduced model, the infeasible and converged flags, the size counts, the
 * transformation log (include/presolve/transformation.h:23-44) with the local
 * index each step saw, and the postsolve metadata (fixed-variable and
 * removed-constraint records, both index maps, both objective offsets). Every
 * number is the one the reference computes: the same passes in the same order
 * (zero coefficients, the infeasibility test, empty rows, fixed variables,
 * singleton rows, bound tightening, redundant rows, duplicate and parallel
 * rows; at most 50 passes), the same arithmetic in the same order, the same
 * early exits with the model as the reference leaves it.
 *
 * What changes is the cost. The reference erases variables and rows from
 * vectors and renumbers every term on each removal, scans every row for each
 * fixed variable, and compares every pair of rows for parallelism (O(m^2)
 * coefficient maps per pass, presolver.cpp:906-907), so a model with 10^5
 * rows does not get through it. Here rows and variables keep stable ids with
 * alive flags, a fixed variable visits only the rows that hold it (column
 * lists), rows are grouped by their exact support before the pairwise
 * parallel test, and the local indices the log records are recovered with
 * prefix counts. One pass costs O(nnz log nnz) plus bound tightening, where
 * the reference sums, for each term of a row, the activity of the row's
 * other terms in row order (O(L^2) for a row of L terms): here each sum is
 * bracketed by a proven rounding-error bound and formed (from an exact
 * running prefix) only where the bracket does not already show that the term
 * moves no bound, so a row costs O(L) per pass plus O(L) per term that
 * tightens. Rows whose inputs did not change since a sweep that moved nothing
 * are passed over.
 *
 * Input: a model::Model (include/model/model.h) as arrays. Terms must name
 * existing variables and carry finite values -- what model::Model::validate
 * (src/model/model.cpp:9-146) checks and solver::solve requires before it
 * presolves (orchestrator.cpp:584); other models are refused with -1. Names
 * do not enter: the log's entity names and the records' names follow from the
 * original indices, and include/pdlpgpu_presolve.hpp fills them in.
 *
 * Host code only: no CUDA call, usable on a host without a GPU. The
 * read-only steps (the infeasibility test, the rows' activities) of models
 * above 4096 rows run on up to 16 host threads; PDLPGPU_PRESOLVE_THREADS=k
 * caps them at k (1: the calling thread only). The result does not depend on
 * it. PDLPGPU_PRESOLVE_TRACE=1 prints each pass's step times on stderr.
 */
#ifndef PDLPGPU_PRESOLVE_H
#define PDLPGPU_PRESOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* presolve::TransformationType, same order. */
enum {
    PDLPGPU_TR_REMOVE_VARIABLE = 0,
    PDLPGPU_TR_REMOVE_CONSTRAINT = 1,
    PDLPGPU_TR_FIX_VARIABLE = 2,
    PDLPGPU_TR_SUBSTITUTE_VARIABLE = 3,
    PDLPGPU_TR_TIGHTEN_LOWER = 4,
    PDLPGPU_TR_TIGHTEN_UPPER = 5
};

/* The reason strings of the log and of the removed-constraint records, as
 * codes; pdlpgpu_presolve_reason_string gives the reference's text. */
enum {
    PDLPGPU_PR_FIXED_BY_BOUNDS = 0,        /* fixVariable */
    PDLPGPU_PR_SINGLETON_LOWER = 1,        /* processSingletonRow */
    PDLPGPU_PR_SINGLETON_UPPER = 2,
    PDLPGPU_PR_SINGLETON_ROW = 3,
    PDLPGPU_PR_TIGHTENED_LOWER = 4,        /* tightenBounds */
    PDLPGPU_PR_TIGHTENED_UPPER = 5,
    PDLPGPU_PR_REDUNDANT = 6,              /* removeRedundantConstraints */
    PDLPGPU_PR_DUPLICATE = 7,              /* removeDuplicateAndParallelRows */
    PDLPGPU_PR_EMPTY_ROW = 8,              /* run, empty rows */
    PDLPGPU_PR_EMPTY_ROW_INFEASIBLE = 9
};

/* A model::Model as arrays (borrowed for the call). var_type holds
 * model::VariableType (0 continuous, 1 integer, 2 binary); rows are CSR with
 * their terms in the constraint's own order (duplicates and zeros allowed);
 * the objective's linear and quadratic terms are lists in their own order. */
typedef struct pdlpgpu_presolve_model {
    int64_t num_variables;
    int64_t num_constraints;
    const double* var_lower;
    const double* var_upper;
    const int8_t* var_type;
    const double* row_lower;
    const double* row_upper;
    const int64_t* row_start;    /* num_constraints + 1 */
    const int32_t* row_index;
    const double* row_value;
    double objective_offset;
    int64_t num_objective_terms;
    const int32_t* objective_index;
    const double* objective_value;
    int64_t num_quadratic_terms;
    const int32_t* quadratic_index1;
    const int32_t* quadratic_index2;
    const double* quadratic_value;
} pdlpgpu_presolve_model;

/* PresolveResult as arrays owned by the result (release with
 * pdlpgpu_presolve_free). Indices of variables and rows in the reduced model
 * are local (0 .. presolved_* - 1); "origin" arrays give the original index of
 * each; -1 stands for presolve::INVALID_ORIGINAL_INDEX in the log. */
typedef struct pdlpgpu_presolve_result {
    int32_t infeasible;
    int32_t converged;
    /* 0 when the first infeasibility test refused the input: the reference
     * then returns before it fills the index maps (they stay empty) and the
     * reduced model is the input unchanged. */
    int32_t has_maps;
    int64_t original_variables;
    int64_t original_constraints;
    int64_t presolved_variables;
    int64_t presolved_constraints;
    double initial_objective_offset;
    double presolved_objective_offset;

    /* reduced model */
    const int64_t* variable_origin;      /* presolved_variables */
    const double* var_lower;
    const double* var_upper;
    const int64_t* constraint_origin;    /* presolved_constraints */
    const double* row_lower;
    const double* row_upper;
    const int64_t* row_start;            /* presolved_constraints + 1 */
    const int32_t* row_index;
    const double* row_value;
    int64_t num_objective_terms;
    const int32_t* objective_index;
    const double* objective_value;
    int64_t num_quadratic_terms;
    const int32_t* quadratic_index1;
    const int32_t* quadratic_index2;
    const double* quadratic_value;

    /* transformation log, in order */
    int64_t num_transformations;
    const int32_t* tr_type;
    const int32_t* tr_reason;
    const int64_t* tr_index;
    const int64_t* tr_variable;          /* original index or -1 */
    const int64_t* tr_constraint;        /* original index or -1 */
    const double* tr_old_value;
    const double* tr_new_value;
    const double* tr_offset_change;

    /* FixedVariableRecord, in order; cross contributions as CSR
     * (fixed_cross_start[num_fixed + 1]) by increasing original index */
    int64_t num_fixed;
    const int64_t* fixed_origin;
    const double* fixed_value;
    const double* fixed_linear;
    const double* fixed_quadratic_diagonal;
    const int64_t* fixed_cross_start;
    const int64_t* fixed_cross_variable;
    const double* fixed_cross_value;

    /* RemovedConstraintRecord, in order */
    int64_t num_removed;
    const int64_t* removed_origin;
    const double* removed_lower;
    const double* removed_upper;
    const int32_t* removed_reason;
    const int8_t* removed_singleton;
    const int64_t* removed_singleton_variable;
    const double* removed_singleton_coefficient;
    const int8_t* removed_duplicate;
    const int64_t* removed_duplicate_of;
    const double* removed_scale;
} pdlpgpu_presolve_result;

/* Runs the presolve. Returns 0 and a result, or -1 (nothing allocated) with
 * pdlpgpu_last_error() saying which input is refused: a NULL array with a
 * positive count, a negative count, row_start not non-decreasing from 0, a
 * term naming no variable, a non-finite coefficient, a variable type other
 * than 0, 1, 2. */
int32_t pdlpgpu_presolve(const pdlpgpu_presolve_model* model, pdlpgpu_presolve_result** result);
void pdlpgpu_presolve_free(pdlpgpu_presolve_result* result);

/* The reference's reason text for a PDLPGPU_PR_* code; "" for another. */
const char* pdlpgpu_presolve_reason_string(int32_t reason);

#ifdef __cplusplus
}
#endif

#endif /* PDLPGPU_PRESOLVE_H */

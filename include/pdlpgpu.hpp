// pdlpgpu.hpp -- header-only C++ facade with the reference's exact signature:
//
//   pdlp::PdlpResult pdlpgpu::PdlpSolver::solve(const pdlp::CompiledLp&,
//                                               const pdlp::PdlpOptions&) const;
//
// It replaces pdlp::PdlpSolver (pdlp_engine/include/pdlp/pdlp_solver.h:9-15)
// at its production call site, solver::runPdlp
// (src/solver/orchestrator.cpp:337), by changing only the namespace. Include it
// where the reference's pdlp headers are on the include path and link
// libpdlpgpu.so. The reference's types are converted field for field; nothing
// of this engine's own types leaks into the caller.
#pragma once

#include "pdlp/compiled_lp.h"
#include "pdlp/pdlp_options.h"
#include "pdlp/pdlp_result.h"
#include "pdlpgpu.h"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace pdlpgpu {

class PdlpSolver {
public:
    // Precision and device are this engine's extensions; the defaults give
    // the reference's FP64 arithmetic on device 0.
    explicit PdlpSolver(int32_t precision = PDLPGPU_PRECISION_FP64, int32_t device = 0)
        : precision_(precision), device_(device) {}

    pdlp::PdlpResult solve(const pdlp::CompiledLp& problem,
                           const pdlp::PdlpOptions& options = {}) const {
        // The C ABI carries the vectors as bare pointers, so the checks that
        // need their lengths run here, in CompiledLp::validate's order
        // (pdlp_engine/include/pdlp/compiled_lp.h:32-45); the engine checks
        // the rest.
        auto reject = [](const char* message) {
            pdlp::PdlpResult out;   // defaults are the invalid-problem result
            out.status = pdlp::PdlpStatus::InvalidProblem;
            out.statusMessage = message;
            return out;
        };
        const std::size_t n = static_cast<std::size_t>(problem.numColumns());
        const std::size_t m = static_cast<std::size_t>(problem.numRows());
        if (!problem.matrix.validate()) return reject("CompiledLp contains an invalid sparse matrix");
        if (problem.objective.size() != n || problem.variableLower.size() != n ||
            problem.variableUpper.size() != n)
            return reject("CompiledLp column vector dimensions do not match A");
        if (problem.rowLower.size() != m || problem.rowUpper.size() != m)
            return reject("CompiledLp row vector dimensions do not match A");
        const pdlp::SparseMatrix& a = problem.matrix;
        pdlpgpu_lp lp;
        lp.num_rows = problem.numRows();
        lp.num_cols = problem.numColumns();
        lp.row_start = a.csrRowStart().data();
        lp.col_index = a.csrColumnIndex().data();
        lp.values = a.csrValues().data();
        lp.objective = problem.objective.data();
        lp.objective_offset = problem.objectiveOffset;
        lp.row_lower = problem.rowLower.data();
        lp.row_upper = problem.rowUpper.data();
        lp.var_lower = problem.variableLower.data();
        lp.var_upper = problem.variableUpper.data();

        pdlpgpu_options o;
        o.iteration_limit = options.iterationLimit;
        o.time_limit_seconds = options.timeLimitSeconds;
        o.primal_tolerance = options.primalTolerance;
        o.dual_tolerance = options.dualTolerance;
        o.gap_tolerance = options.gapTolerance;
        o.termination_check_frequency = options.terminationCheckFrequency;
        o.power_iteration_count = options.powerIterationCount;
        o.thread_count = options.threadCount;
        o.parallel_nonzero_threshold = options.parallelNonzeroThreshold;
        o.initial_step_safety = options.initialStepSafety;
        o.minimum_step_scale = options.minimumStepScale;
        o.maximum_primal_weight = options.maximumPrimalWeight;
        o.minimum_primal_weight = options.minimumPrimalWeight;
        o.use_ruiz_scaling = options.useRuizScaling;
        o.ruiz_iterations = options.ruizIterations;
        o.detect_infeasibility = options.detectInfeasibility;
        o.infeasibility_tolerance = options.infeasibilityTolerance;
        o.use_diagonal_preconditioning = options.useDiagonalPreconditioning;
        o.use_adaptive_linesearch = options.useAdaptiveLinesearch;
        o.maximum_step_trials = options.maximumStepTrials;
        o.use_averaging = options.useAveraging;
        o.use_restarts = options.useRestarts;
        o.use_feasibility_polishing = options.useFeasibilityPolishing;
        o.minimum_restart_iterations = options.minimumRestartIterations;
        o.maximum_restart_iterations = options.maximumRestartIterations;
        o.restart_sufficient_decay = options.restartSufficientDecay;
        o.restart_necessary_decay = options.restartNecessaryDecay;
        o.restart_artificial_fraction = options.restartArtificialFraction;
        o.initial_primal_weight = options.initialPrimalWeight;
        o.primal_weight_smoothing = options.primalWeightSmoothing;
        o.polishing_iterations = options.polishingIterations;

        pdlpgpu_ext_options ext;
        pdlpgpu_default_ext_options(&ext);
        ext.precision = precision_;
        ext.device = device_;

        pdlpgpu_result* r = nullptr;
        pdlpgpu_solve_ex(&lp, &o, &ext, nullptr, &r);
        pdlp::PdlpResult out;
        out.status = static_cast<pdlp::PdlpStatus>(r->status);
        out.statusMessage = r->status_message;
        if (r->primal) out.primal.assign(r->primal, r->primal + r->num_cols);
        if (r->row_dual) out.rowDual.assign(r->row_dual, r->row_dual + r->num_rows);
        if (r->dual_ray) out.dualRay.assign(r->dual_ray, r->dual_ray + r->num_rows);
        if (r->primal_ray) out.primalRay.assign(r->primal_ray, r->primal_ray + r->num_cols);
        out.primalObjective = r->primal_objective;
        out.dualObjective = r->dual_objective;
        out.primalResidual = r->primal_residual;
        out.dualResidual = r->dual_residual;
        out.relativeGap = r->relative_gap;
        out.iterations = r->iterations;
        out.stepTrials = r->step_trials;
        out.restartCount = r->restart_count;
        out.solveTimeSeconds = r->solve_time_seconds;
        out.finalStepSize = r->final_step_size;
        out.staticStepBound = r->static_step_bound;
        out.finalPrimalWeight = r->final_primal_weight;
        pdlpgpu_result_free(r);
        return out;
    }

private:
    int32_t precision_;
    int32_t device_;
};

}  // namespace pdlpgpu

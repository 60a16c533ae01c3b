// ref_shim.cpp -- exposes the reference pdlp_engine (compiled from its own,
// unmodified sources by oracle/Makefile) through the C interface in
// oracle_abi.h. TEST INFRASTRUCTURE ONLY: the parity tests and the CPU
// baseline of bench.py load the resulting oracle/_ref/libpdlp_ref*.so; the
// product never does.
//
// Each function converts the plain arrays into the reference's own types and
// calls the reference's own entry point, so the numbers it returns are the
// reference's numbers.
#include "oracle_abi.h"

#include "pdlp/infeasibility.h"
#include "pdlp/pdhg_kernel.h"
#include "pdlp/pdlp_solver.h"
#include "pdlp/preconditioner.h"
#include "pdlp/scaling.h"
#include "pdlp/termination.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

namespace {

std::vector<double> copyOf(const double* data, int64_t count) {
    return std::vector<double>(data, data + count);
}

// CompiledLp from canonical CSR, through SparseMatrix::fromTriplets exactly as
// the reference's adapter builds it (src/adapter/pdlp_adapter.cpp:124-167).
pdlp::CompiledLp toCompiled(const orc_lp* lp) {
    std::vector<pdlp::MatrixTriplet> triplets;
    triplets.reserve(static_cast<std::size_t>(lp->nnz));
    for (int32_t i = 0; i < lp->rows; ++i) {
        for (int64_t k = lp->row_start[i]; k < lp->row_start[i + 1]; ++k) {
            triplets.push_back({i, lp->col_index[k], lp->values[k]});
        }
    }
    pdlp::CompiledLp problem;
    problem.matrix = pdlp::SparseMatrix::fromTriplets(lp->rows, lp->cols, std::move(triplets));
    problem.objective = copyOf(lp->objective, lp->cols);
    problem.objectiveOffset = lp->objective_offset;
    problem.rowLower = copyOf(lp->row_lower, lp->rows);
    problem.rowUpper = copyOf(lp->row_upper, lp->rows);
    problem.variableLower = copyOf(lp->var_lower, lp->cols);
    problem.variableUpper = copyOf(lp->var_upper, lp->cols);
    return problem;
}

pdlp::PdlpOptions toOptions(const orc_options* o) {
    pdlp::PdlpOptions p;
    p.iterationLimit = o->iteration_limit;
    p.timeLimitSeconds = o->time_limit_seconds;
    p.primalTolerance = o->primal_tolerance;
    p.dualTolerance = o->dual_tolerance;
    p.gapTolerance = o->gap_tolerance;
    p.terminationCheckFrequency = o->termination_check_frequency;
    p.powerIterationCount = o->power_iteration_count;
    p.threadCount = o->thread_count;
    p.parallelNonzeroThreshold = o->parallel_nonzero_threshold;
    p.initialStepSafety = o->initial_step_safety;
    p.minimumStepScale = o->minimum_step_scale;
    p.maximumPrimalWeight = o->maximum_primal_weight;
    p.minimumPrimalWeight = o->minimum_primal_weight;
    p.useRuizScaling = o->use_ruiz_scaling != 0;
    p.ruizIterations = o->ruiz_iterations;
    p.detectInfeasibility = o->detect_infeasibility != 0;
    p.infeasibilityTolerance = o->infeasibility_tolerance;
    p.useDiagonalPreconditioning = o->use_diagonal_preconditioning != 0;
    p.useAdaptiveLinesearch = o->use_adaptive_linesearch != 0;
    p.maximumStepTrials = o->maximum_step_trials;
    p.useAveraging = o->use_averaging != 0;
    p.useRestarts = o->use_restarts != 0;
    p.useFeasibilityPolishing = o->use_feasibility_polishing != 0;
    p.minimumRestartIterations = o->minimum_restart_iterations;
    p.maximumRestartIterations = o->maximum_restart_iterations;
    p.restartSufficientDecay = o->restart_sufficient_decay;
    p.restartNecessaryDecay = o->restart_necessary_decay;
    p.restartArtificialFraction = o->restart_artificial_fraction;
    p.initialPrimalWeight = o->initial_primal_weight;
    p.primalWeightSmoothing = o->primal_weight_smoothing;
    p.polishingIterations = o->polishing_iterations;
    return p;
}

void putVector(const std::vector<double>& v, double* out) {
    if (out != nullptr && !v.empty()) {
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    }
}

}  // namespace

extern "C" {

void orc_default_options(orc_options* o) {
    const pdlp::PdlpOptions p;
    o->iteration_limit = p.iterationLimit;
    o->time_limit_seconds = p.timeLimitSeconds;
    o->primal_tolerance = p.primalTolerance;
    o->dual_tolerance = p.dualTolerance;
    o->gap_tolerance = p.gapTolerance;
    o->termination_check_frequency = p.terminationCheckFrequency;
    o->power_iteration_count = p.powerIterationCount;
    o->thread_count = p.threadCount;
    o->parallel_nonzero_threshold = p.parallelNonzeroThreshold;
    o->initial_step_safety = p.initialStepSafety;
    o->minimum_step_scale = p.minimumStepScale;
    o->maximum_primal_weight = p.maximumPrimalWeight;
    o->minimum_primal_weight = p.minimumPrimalWeight;
    o->use_ruiz_scaling = p.useRuizScaling;
    o->ruiz_iterations = p.ruizIterations;
    o->detect_infeasibility = p.detectInfeasibility;
    o->infeasibility_tolerance = p.infeasibilityTolerance;
    o->use_diagonal_preconditioning = p.useDiagonalPreconditioning;
    o->use_adaptive_linesearch = p.useAdaptiveLinesearch;
    o->maximum_step_trials = p.maximumStepTrials;
    o->use_averaging = p.useAveraging;
    o->use_restarts = p.useRestarts;
    o->use_feasibility_polishing = p.useFeasibilityPolishing;
    o->minimum_restart_iterations = p.minimumRestartIterations;
    o->maximum_restart_iterations = p.maximumRestartIterations;
    o->restart_sufficient_decay = p.restartSufficientDecay;
    o->restart_necessary_decay = p.restartNecessaryDecay;
    o->restart_artificial_fraction = p.restartArtificialFraction;
    o->initial_primal_weight = p.initialPrimalWeight;
    o->primal_weight_smoothing = p.primalWeightSmoothing;
    o->polishing_iterations = p.polishingIterations;
}

int orc_solve(const orc_lp* lp, const orc_options* options, double* primal,
              double* dual, double* dual_ray, double* primal_ray, orc_result* out) {
    std::memset(out, 0, sizeof(*out));
    pdlp::CompiledLp problem;
    try {
        problem = toCompiled(lp);
    } catch (const std::exception& error) {
        out->status = static_cast<int32_t>(pdlp::PdlpStatus::InvalidProblem);
        std::snprintf(out->message, sizeof(out->message), "%s", error.what());
        return out->status;
    }
    const pdlp::PdlpResult r = pdlp::PdlpSolver{}.solve(problem, toOptions(options));
    out->status = static_cast<int32_t>(r.status);
    out->has_dual_ray = r.dualRay.empty() ? 0 : 1;
    out->has_primal_ray = r.primalRay.empty() ? 0 : 1;
    out->restart_count = r.restartCount;
    out->iterations = r.iterations;
    out->step_trials = r.stepTrials;
    out->primal_objective = r.primalObjective;
    out->dual_objective = r.dualObjective;
    out->primal_residual = r.primalResidual;
    out->dual_residual = r.dualResidual;
    out->relative_gap = r.relativeGap;
    out->solve_time_seconds = r.solveTimeSeconds;
    out->final_step_size = r.finalStepSize;
    out->static_step_bound = r.staticStepBound;
    out->final_primal_weight = r.finalPrimalWeight;
    out->primal_size = static_cast<int32_t>(r.primal.size());
    out->dual_size = static_cast<int32_t>(r.rowDual.size());
    std::snprintf(out->message, sizeof(out->message), "%s", r.statusMessage.c_str());
    putVector(r.primal, primal);
    putVector(r.rowDual, dual);
    putVector(r.dualRay, dual_ray);
    putVector(r.primalRay, primal_ray);
    return out->status;
}

int orc_from_triplets(int32_t rows, int32_t cols, int64_t count, const int32_t* row,
                      const int32_t* col, const double* value, int64_t* row_start,
                      int32_t* col_index, double* values, int64_t* col_start,
                      int32_t* row_index, double* csc_values, int64_t* nnz_out) {
    std::vector<pdlp::MatrixTriplet> triplets(static_cast<std::size_t>(count));
    for (int64_t k = 0; k < count; ++k) {
        triplets[static_cast<std::size_t>(k)] = {row[k], col[k], value[k]};
    }
    pdlp::SparseMatrix m;
    try {
        m = pdlp::SparseMatrix::fromTriplets(rows, cols, std::move(triplets));
    } catch (const std::exception&) {
        return -1;
    }
    std::copy(m.csrRowStart().begin(), m.csrRowStart().end(), row_start);
    std::copy(m.csrColumnIndex().begin(), m.csrColumnIndex().end(), col_index);
    std::copy(m.csrValues().begin(), m.csrValues().end(), values);
    std::copy(m.cscColumnStart().begin(), m.cscColumnStart().end(), col_start);
    std::copy(m.cscRowIndex().begin(), m.cscRowIndex().end(), row_index);
    std::copy(m.cscValues().begin(), m.cscValues().end(), csc_values);
    *nnz_out = static_cast<int64_t>(m.nonzeros());
    return 0;
}

void orc_multiply(const orc_lp* lp, const double* x, double* ax) {
    const pdlp::CompiledLp p = toCompiled(lp);
    std::vector<double> result;
    p.matrix.multiply(copyOf(x, lp->cols), result);
    putVector(result, ax);
}

void orc_transpose_multiply(const orc_lp* lp, const double* y, double* aty) {
    const pdlp::CompiledLp p = toCompiled(lp);
    std::vector<double> result;
    p.matrix.transposeMultiply(copyOf(y, lp->rows), result);
    putVector(result, aty);
}

void orc_ruiz(const orc_lp* lp, int32_t iterations, double* row_scale, double* col_scale,
              double* scaled_values, double* scaled_objective, double* scaled_row_lower,
              double* scaled_row_upper, double* scaled_var_lower, double* scaled_var_upper) {
    const pdlp::CompiledLp p = toCompiled(lp);
    const pdlp::ProblemScaling s = pdlp::RuizScaler::equilibrate(p, iterations);
    putVector(s.rowScale, row_scale);
    putVector(s.columnScale, col_scale);
    putVector(s.problem.matrix.csrValues(), scaled_values);
    putVector(s.problem.objective, scaled_objective);
    putVector(s.problem.rowLower, scaled_row_lower);
    putVector(s.problem.rowUpper, scaled_row_upper);
    putVector(s.problem.variableLower, scaled_var_lower);
    putVector(s.problem.variableUpper, scaled_var_upper);
}

double orc_condition_spread(const orc_lp* lp) {
    return pdlp::RuizScaler::conditionSpread(toCompiled(lp).matrix);
}

void orc_precondition(const orc_lp* lp, int32_t enabled, double* tau, double* tau_inverse,
                      double* sigma, double* sigma_inverse) {
    const pdlp::DiagonalPreconditioner d =
        pdlp::Preconditioner::compute(toCompiled(lp), enabled != 0);
    putVector(d.primalScale, tau);
    putVector(d.primalScaleInverse, tau_inverse);
    putVector(d.dualScale, sigma);
    putVector(d.dualScaleInverse, sigma_inverse);
}

double orc_spectral_norm(const orc_lp* lp, int32_t iterations, int32_t* converged) {
    bool flag = false;
    const double norm =
        pdlp::Preconditioner::estimateSpectralNorm(toCompiled(lp).matrix, iterations, &flag);
    if (converged != nullptr) {
        *converged = flag ? 1 : 0;
    }
    return norm;
}

int orc_trial(const orc_lp* working, const double* tau, const double* tau_inverse,
              const double* sigma, const double* sigma_inverse, const double* x,
              const double* y, const double* ax, double step, double weight, double* x_out,
              double* y_out, double* ax_out, double* reductions) {
    const pdlp::CompiledLp p = toCompiled(working);
    pdlp::DiagonalPreconditioner d;
    d.primalScale = copyOf(tau, working->cols);
    d.primalScaleInverse = copyOf(tau_inverse, working->cols);
    d.dualScale = copyOf(sigma, working->rows);
    d.dualScaleInverse = copyOf(sigma_inverse, working->rows);
    pdlp::PdlpState state;
    state.primal = copyOf(x, working->cols);
    state.dual = copyOf(y, working->rows);
    state.rowActivity = copyOf(ax, working->rows);
    pdlp::StepParameters steps;
    steps.globalStep = step;
    steps.primalWeight = weight;
    pdlp::CpuPdhgKernel kernel(p);
    const pdlp::KernelTrialResult r = kernel.trial(state, d, steps);
    kernel.commit(state);
    putVector(state.primal, x_out);
    putVector(state.dual, y_out);
    putVector(state.rowActivity, ax_out);
    reductions[0] = r.primalMovementWeighted;
    reductions[1] = r.dualMovementWeighted;
    reductions[2] = r.interaction;
    return r.finite ? 1 : 0;
}

void orc_evaluate(const orc_lp* lp, const double* x, const double* y, double* metrics) {
    const pdlp::CompiledLp p = toCompiled(lp);
    pdlp::TerminationChecker checker(pdlp::PdlpOptions{}, p);
    const pdlp::CandidateMetrics m =
        checker.evaluate(copyOf(x, lp->cols), copyOf(y, lp->rows));
    metrics[0] = m.primalObjective;
    metrics[1] = m.dualObjective;
    metrics[2] = m.primalResidual;
    metrics[3] = m.dualResidual;
    metrics[4] = m.relativeGap;
    metrics[5] = m.kktScore;
    metrics[6] = m.finite ? 1.0 : 0.0;
    metrics[7] = m.dualObjectiveValid ? 1.0 : 0.0;
}

void orc_test_dual_ray(const orc_lp* lp, double tolerance, const double* direction,
                       double* verdict) {
    const pdlp::CompiledLp p = toCompiled(lp);
    pdlp::PdlpOptions options;
    options.infeasibilityTolerance = tolerance;
    pdlp::InfeasibilityDetector detector(p, options);
    const pdlp::InfeasibilityVerdict v = detector.testDualRay(copyOf(direction, lp->rows));
    verdict[0] = v.provesPrimalInfeasible ? 1.0 : 0.0;
    verdict[1] = v.certificateValue;
    verdict[2] = v.relativeViolation;
}

void orc_test_primal_ray(const orc_lp* lp, double tolerance, const double* direction,
                         double* verdict) {
    const pdlp::CompiledLp p = toCompiled(lp);
    pdlp::PdlpOptions options;
    options.infeasibilityTolerance = tolerance;
    pdlp::InfeasibilityDetector detector(p, options);
    const pdlp::InfeasibilityVerdict v = detector.testPrimalRay(copyOf(direction, lp->cols));
    verdict[0] = v.provesUnbounded ? 1.0 : 0.0;
    verdict[1] = v.certificateValue;
    verdict[2] = v.relativeViolation;
}

}  // extern "C"

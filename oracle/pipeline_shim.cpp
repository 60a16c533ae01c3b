// pipeline_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C interface over the reference's own pipeline for the Python tests: the
// MPS reader (src/mps/mps_reader.cpp), the PDLP adapter
// (src/adapter/pdlp_adapter.cpp:21-189) and solver::solve
// (src/solver/orchestrator.cpp). oracle/Makefile links it twice from the
// reference's sources where they lie: with the reference's
// pdlp_engine/src/pdlp_solver.cpp (libpipeline_ref.so), and with the GPU
// engine's pdlp::PdlpSolver::solve (include/pdlpgpu_override.hpp) linked in
// its place (libpipeline_gpu.so), so that solver::runPdlp reaches the GPU
// with no reference line changed. Only the pl_* functions are exported.
#include "adapter/pdlp_adapter.h"
#include "model/model.h"
#include "mps/mps_reader.h"
#include "pdlp/compiled_lp.h"
#include "solver/orchestrator.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#define PL_API extern "C" __attribute__((visibility("default")))

namespace {

void put(char* dst, int len, const std::string& s) {
    if (dst == nullptr || len <= 0) return;
    const std::size_t k = std::min<std::size_t>(s.size(), static_cast<std::size_t>(len - 1));
    std::memcpy(dst, s.data(), k);
    dst[k] = '\0';
}

}  // namespace

struct pl_model {
    model::Model model;
    std::vector<std::string> warnings;   // the reader's, when read from a file
    pdlp::CompiledLp compiled;
    adapter::PdlpTranslation translation;
};

struct pl_solve_out {
    int32_t status;            // solver::SolveStatus
    int32_t executed_engine;   // solver::Engine
    int32_t has_primal;
    int32_t has_duals;
    double objective;
    double max_dual_residual;
    int64_t iterations;
    int64_t reduced_variables;
    int64_t reduced_constraints;
    char status_name[32];
    char message[256];
};

// Reads an MPS file with the reference MpsReader. Returns 0, or -1 with the
// reader's message.
PL_API int pl_read_mps(const char* path, pl_model** out, char* message, int message_len) {
    try {
        mps::MpsReader reader;
        auto* h = new pl_model;
        try {
            h->model = reader.read(path);
        } catch (...) {
            delete h;
            throw;
        }
        h->warnings = reader.warnings();
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        put(message, message_len, e.what());
        return -1;
    }
}

PL_API void pl_model_free(pl_model* h) { delete h; }

PL_API void pl_model_dims(const pl_model* h, int64_t* variables, int64_t* constraints) {
    *variables = static_cast<int64_t>(h->model.variables.size());
    *constraints = static_cast<int64_t>(h->model.constraints.size());
}

// adapter::toCompiledLp of the model read. Returns 0 with the dimensions, or
// -1 with the adapter's error.
PL_API int pl_compile(pl_model* h, int32_t* rows, int32_t* cols, int64_t* nnz, char* message,
                      int message_len) {
    adapter::AdapterOptions options;
    h->translation = adapter::toCompiledLp(h->model, h->compiled, options);
    if (!h->translation.ok) {
        put(message, message_len, h->translation.error);
        return -1;
    }
    *rows = h->compiled.numRows();
    *cols = h->compiled.numColumns();
    *nnz = static_cast<int64_t>(h->compiled.matrix.csrValues().size());
    return 0;
}

PL_API void pl_compiled_copy(const pl_model* h, int64_t* row_start, int32_t* col_index,
                             double* values, double* objective, double* objective_offset,
                             double* row_lower, double* row_upper, double* var_lower,
                             double* var_upper) {
    const pdlp::CompiledLp& c = h->compiled;
    const auto& a = c.matrix;
    std::copy(a.csrRowStart().begin(), a.csrRowStart().end(), row_start);
    std::copy(a.csrColumnIndex().begin(), a.csrColumnIndex().end(), col_index);
    std::copy(a.csrValues().begin(), a.csrValues().end(), values);
    std::copy(c.objective.begin(), c.objective.end(), objective);
    *objective_offset = c.objectiveOffset;
    std::copy(c.rowLower.begin(), c.rowLower.end(), row_lower);
    std::copy(c.rowUpper.begin(), c.rowUpper.end(), row_upper);
    std::copy(c.variableLower.begin(), c.variableLower.end(), var_lower);
    std::copy(c.variableUpper.begin(), c.variableUpper.end(), var_upper);
}

// solver::solve of the model read (presolve, dispatch, engine, postsolve).
// force_engine < 0 leaves dispatch to the reference. Vectors are written when
// the result has them: x and reduced_costs [variables], duals [constraints].
PL_API int pl_solve(const pl_model* h, int32_t force_engine, double tolerance,
                    double time_limit_seconds, int32_t threads, pl_solve_out* out, double* x,
                    double* duals, double* reduced_costs) {
    try {
        solver::SolverOptions options;
        if (force_engine >= 0) options.forceEngine = static_cast<solver::Engine>(force_engine);
        options.tolerance = tolerance;
        options.timeLimitSeconds = time_limit_seconds;
        options.threadCount = threads;
        const solver::SolveResult r = solver::solve(h->model, options);
        out->status = static_cast<int32_t>(r.status);
        out->executed_engine = static_cast<int32_t>(r.executedEngine);
        out->has_primal = r.hasPrimal ? 1 : 0;
        out->has_duals = r.hasDuals ? 1 : 0;
        out->objective = r.objectiveValue;
        out->max_dual_residual = r.maxDualResidual;
        out->iterations = r.iterations;
        out->reduced_variables = static_cast<int64_t>(r.reducedVariableCount);
        out->reduced_constraints = static_cast<int64_t>(r.reducedConstraintCount);
        put(out->status_name, sizeof(out->status_name), solver::toString(r.status));
        put(out->message, sizeof(out->message), r.message);
        if (r.hasPrimal && x != nullptr)
            std::copy(r.variableValues.begin(), r.variableValues.end(), x);
        if (r.hasDuals && duals != nullptr)
            std::copy(r.constraintDuals.begin(), r.constraintDuals.end(), duals);
        if (r.hasDuals && reduced_costs != nullptr)
            std::copy(r.reducedCosts.begin(), r.reducedCosts.end(), reduced_costs);
        return 0;
    } catch (const std::exception& e) {
        put(out->message, sizeof(out->message), e.what());
        return -1;
    }
}

// The Model IR as flat arrays, so a model read here can travel as a fixture
// and be rebuilt where the MPS file is absent. Term lists are kept in their
// stored order (duplicates included). Quadratic terms are not carried.
PL_API void pl_model_sizes(const pl_model* h, int64_t* objective_terms, int64_t* row_terms,
                           int64_t* quadratic_terms) {
    const model::Model& m = h->model;
    *objective_terms = static_cast<int64_t>(m.objective.linearTerms.size());
    int64_t k = 0;
    for (const auto& c : m.constraints) k += static_cast<int64_t>(c.linearTerms.size());
    *row_terms = k;
    *quadratic_terms = static_cast<int64_t>(m.objective.quadraticTerms.size());
}

PL_API void pl_model_export(const pl_model* h, int32_t* sense, double* offset,
                            int32_t* objective_index, double* objective_value,
                            int32_t* var_type, double* var_lower, double* var_upper,
                            double* row_lower, double* row_upper, int64_t* row_start,
                            int32_t* row_index, double* row_value) {
    const model::Model& m = h->model;
    *sense = m.objective.sense == model::ObjectiveSense::Maximize ? 1 : 0;
    *offset = m.objective.offset;
    for (std::size_t k = 0; k < m.objective.linearTerms.size(); ++k) {
        objective_index[k] = m.objective.linearTerms[k].variableIndex;
        objective_value[k] = m.objective.linearTerms[k].value;
    }
    for (std::size_t j = 0; j < m.variables.size(); ++j) {
        var_type[j] = static_cast<int32_t>(m.variables[j].type);
        var_lower[j] = m.variables[j].lowerBound;
        var_upper[j] = m.variables[j].upperBound;
    }
    int64_t k = 0;
    row_start[0] = 0;
    for (std::size_t i = 0; i < m.constraints.size(); ++i) {
        const auto& c = m.constraints[i];
        row_lower[i] = c.lowerBound;
        row_upper[i] = c.upperBound;
        for (const auto& t : c.linearTerms) {
            row_index[k] = t.variableIndex;
            row_value[k] = t.value;
            ++k;
        }
        row_start[i + 1] = k;
    }
}

PL_API pl_model* pl_model_import(int64_t variables, int64_t constraints, int32_t sense,
                                 double offset, int64_t objective_terms,
                                 const int32_t* objective_index, const double* objective_value,
                                 const int32_t* var_type, const double* var_lower,
                                 const double* var_upper, const double* row_lower,
                                 const double* row_upper, const int64_t* row_start,
                                 const int32_t* row_index, const double* row_value) {
    auto* h = new pl_model;
    model::Model& m = h->model;
    m.objective.sense = sense ? model::ObjectiveSense::Maximize : model::ObjectiveSense::Minimize;
    m.objective.offset = offset;
    for (int64_t k = 0; k < objective_terms; ++k)
        m.objective.linearTerms.push_back({objective_index[k], objective_value[k]});
    m.variables.resize(static_cast<std::size_t>(variables));
    for (int64_t j = 0; j < variables; ++j) {
        auto& v = m.variables[static_cast<std::size_t>(j)];
        v.name = "x" + std::to_string(j);
        v.type = static_cast<model::VariableType>(var_type[j]);
        v.lowerBound = var_lower[j];
        v.upperBound = var_upper[j];
    }
    m.constraints.resize(static_cast<std::size_t>(constraints));
    for (int64_t i = 0; i < constraints; ++i) {
        auto& c = m.constraints[static_cast<std::size_t>(i)];
        c.name = "r" + std::to_string(i);
        c.lowerBound = row_lower[i];
        c.upperBound = row_upper[i];
        for (int64_t k = row_start[i]; k < row_start[i + 1]; ++k)
            c.linearTerms.push_back({row_index[k], row_value[k]});
    }
    return h;
}

// Names and warnings: kind 0 the model name, 1 variable `index`, 2 row
// `index`, 3 warning `index`; NULL out of range.
PL_API const char* pl_name(const pl_model* h, int32_t kind, int64_t index) {
    const model::Model& m = h->model;
    if (kind == 0) return m.name.c_str();
    if (index < 0) return nullptr;
    const std::size_t k = static_cast<std::size_t>(index);
    if (kind == 1) return k < m.variables.size() ? m.variables[k].name.c_str() : nullptr;
    if (kind == 2) return k < m.constraints.size() ? m.constraints[k].name.c_str() : nullptr;
    if (kind == 3) return k < h->warnings.size() ? h->warnings[k].c_str() : nullptr;
    return nullptr;
}

PL_API int64_t pl_warning_count(const pl_model* h) { return static_cast<int64_t>(h->warnings.size()); }

// Quadratic objective terms in stored order.
PL_API void pl_model_quadratic(const pl_model* h, int32_t* i, int32_t* j, double* value) {
    const auto& q = h->model.objective.quadraticTerms;
    for (std::size_t k = 0; k < q.size(); ++k) {
        i[k] = q[k].variableIndex1;
        j[k] = q[k].variableIndex2;
        value[k] = q[k].value;
    }
}

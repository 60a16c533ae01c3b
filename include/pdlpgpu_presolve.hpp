// pdlpgpu_presolve.hpp -- the fast presolve with the reference's types.
//
// pdlpgpu::presolve_model(const model::Model&) returns the
// presolve::PresolveResult that presolve::Presolver::run
// (include/presolve/presolver.h:11) returns for the same model, names and
// reason strings included, computed by pdlpgpu_presolve (pdlpgpu_presolve.h).
// Header only; compile against the reference's include/ tree and link
// libpdlpgpu.so. A model whose terms name no variable or carry non-finite
// values (what model::Model::validate refuses) throws std::invalid_argument
// with the library's message; solver::solve validates before it presolves
// (src/solver/orchestrator.cpp:584), so its models never do.
#pragma once

#include "model/model.h"
#include "pdlpgpu.h"
#include "pdlpgpu_presolve.h"
#include "presolve/presolve_result.h"
#include "presolve/transformation.h"

#include <cstdint>
#include <stdexcept>
#include <vector>

namespace pdlpgpu {

inline presolve::PresolveResult presolve_model(const model::Model& input) {
    const std::size_t n = input.variables.size(), m = input.constraints.size();
    std::vector<double> vlo(n), vhi(n), rlo(m), rhi(m), rv, ov, qv;
    std::vector<int8_t> vt(n);
    std::vector<int64_t> rs(m + 1, 0);
    std::vector<int32_t> ri, oi, qi, qj;
    for (std::size_t v = 0; v < n; ++v) {
        vlo[v] = input.variables[v].lowerBound;
        vhi[v] = input.variables[v].upperBound;
        vt[v] = static_cast<int8_t>(input.variables[v].type);
    }
    for (std::size_t r = 0; r < m; ++r) {
        const model::Constraint& c = input.constraints[r];
        rlo[r] = c.lowerBound;
        rhi[r] = c.upperBound;
        for (const model::LinearTerm& t : c.linearTerms) {
            ri.push_back(t.variableIndex);
            rv.push_back(t.value);
        }
        rs[r + 1] = static_cast<int64_t>(ri.size());
    }
    for (const model::LinearTerm& t : input.objective.linearTerms) {
        oi.push_back(t.variableIndex);
        ov.push_back(t.value);
    }
    for (const model::QuadraticTerm& t : input.objective.quadraticTerms) {
        qi.push_back(t.variableIndex1);
        qj.push_back(t.variableIndex2);
        qv.push_back(t.value);
    }
    pdlpgpu_presolve_model in{};
    in.num_variables = static_cast<int64_t>(n);
    in.num_constraints = static_cast<int64_t>(m);
    in.var_lower = vlo.data();
    in.var_upper = vhi.data();
    in.var_type = vt.data();
    in.row_lower = rlo.data();
    in.row_upper = rhi.data();
    in.row_start = rs.data();
    in.row_index = ri.data();
    in.row_value = rv.data();
    in.objective_offset = input.objective.offset;
    in.num_objective_terms = static_cast<int64_t>(oi.size());
    in.objective_index = oi.data();
    in.objective_value = ov.data();
    in.num_quadratic_terms = static_cast<int64_t>(qi.size());
    in.quadratic_index1 = qi.data();
    in.quadratic_index2 = qj.data();
    in.quadratic_value = qv.data();

    pdlpgpu_presolve_result* r = nullptr;
    if (pdlpgpu_presolve(&in, &r) != 0) throw std::invalid_argument(pdlpgpu_last_error());

    presolve::PresolveResult out;
    out.infeasible = r->infeasible != 0;
    out.converged = r->converged != 0;
    out.originalVariables = static_cast<std::size_t>(r->original_variables);
    out.originalConstraints = static_cast<std::size_t>(r->original_constraints);
    out.presolvedVariables = static_cast<std::size_t>(r->presolved_variables);
    out.presolvedConstraints = static_cast<std::size_t>(r->presolved_constraints);

    model::Model& red = out.model;
    red.name = input.name;
    red.objective.sense = input.objective.sense;
    red.objective.offset = r->presolved_objective_offset;
    for (int64_t k = 0; k < r->num_objective_terms; ++k)
        red.objective.linearTerms.push_back({r->objective_index[k], r->objective_value[k]});
    for (int64_t k = 0; k < r->num_quadratic_terms; ++k)
        red.objective.quadraticTerms.push_back(
            {r->quadratic_index1[k], r->quadratic_index2[k], r->quadratic_value[k]});
    red.variables.reserve(static_cast<std::size_t>(r->presolved_variables));
    for (int64_t k = 0; k < r->presolved_variables; ++k) {
        model::Variable v = input.variables[static_cast<std::size_t>(r->variable_origin[k])];
        v.lowerBound = r->var_lower[k];
        v.upperBound = r->var_upper[k];
        red.variables.push_back(std::move(v));
    }
    red.constraints.reserve(static_cast<std::size_t>(r->presolved_constraints));
    for (int64_t k = 0; k < r->presolved_constraints; ++k) {
        model::Constraint c;
        c.name = input.constraints[static_cast<std::size_t>(r->constraint_origin[k])].name;
        c.lowerBound = r->row_lower[k];
        c.upperBound = r->row_upper[k];
        for (int64_t p = r->row_start[k]; p < r->row_start[k + 1]; ++p)
            c.linearTerms.push_back({r->row_index[p], r->row_value[p]});
        red.constraints.push_back(std::move(c));
    }

    auto original = [](int64_t i) {
        return i < 0 ? presolve::INVALID_ORIGINAL_INDEX : static_cast<std::size_t>(i);
    };
    out.transformations.reserve(static_cast<std::size_t>(r->num_transformations));
    for (int64_t k = 0; k < r->num_transformations; ++k) {
        presolve::Transformation t;
        t.type = static_cast<presolve::TransformationType>(r->tr_type[k]);
        t.index = static_cast<std::size_t>(r->tr_index[k]);
        t.originalVariableIndex = original(r->tr_variable[k]);
        t.originalConstraintIndex = original(r->tr_constraint[k]);
        t.oldValue = r->tr_old_value[k];
        t.newValue = r->tr_new_value[k];
        t.reason = pdlpgpu_presolve_reason_string(r->tr_reason[k]);
        t.entityName = t.type == presolve::TransformationType::RemoveConstraint
                           ? input.constraints[static_cast<std::size_t>(r->tr_constraint[k])].name
                           : input.variables[static_cast<std::size_t>(r->tr_variable[k])].name;
        t.offsetChange = r->tr_offset_change[k];
        out.transformations.push_back(std::move(t));
    }

    presolve::PostsolveMetadata& ps = out.postsolve;
    ps.initialObjectiveOffset = r->initial_objective_offset;
    ps.presolvedObjectiveOffset = r->presolved_objective_offset;
    for (int64_t k = 0; k < r->num_fixed; ++k) {
        presolve::FixedVariableRecord f;
        const auto& var = input.variables[static_cast<std::size_t>(r->fixed_origin[k])];
        f.originalIndex = static_cast<std::size_t>(r->fixed_origin[k]);
        f.name = var.name;
        f.fixedValue = r->fixed_value[k];
        f.type = var.type;
        f.linearObjectiveContribution = r->fixed_linear[k];
        f.quadraticDiagonalContribution = r->fixed_quadratic_diagonal[k];
        for (int64_t e = r->fixed_cross_start[k]; e < r->fixed_cross_start[k + 1]; ++e)
            f.quadraticCrossContributions[static_cast<std::size_t>(r->fixed_cross_variable[e])] =
                r->fixed_cross_value[e];
        ps.fixedVariables.push_back(std::move(f));
    }
    for (int64_t k = 0; k < r->num_removed; ++k) {
        presolve::RemovedConstraintRecord c;
        c.originalIndex = static_cast<std::size_t>(r->removed_origin[k]);
        c.name = input.constraints[c.originalIndex].name;
        c.lowerBound = r->removed_lower[k];
        c.upperBound = r->removed_upper[k];
        c.reason = pdlpgpu_presolve_reason_string(r->removed_reason[k]);
        c.wasSingleton = r->removed_singleton[k] != 0;
        c.singletonOriginalVarIndex = static_cast<std::size_t>(r->removed_singleton_variable[k]);
        c.singletonCoefficient = r->removed_singleton_coefficient[k];
        c.wasDuplicate = r->removed_duplicate[k] != 0;
        c.duplicateOfOriginalIndex = static_cast<std::size_t>(r->removed_duplicate_of[k]);
        c.scale = r->removed_scale[k];
        ps.removedConstraints.push_back(std::move(c));
    }
    if (r->has_maps) {
        ps.presolvedToOriginalVar.assign(r->variable_origin,
                                         r->variable_origin + r->presolved_variables);
        ps.originalToPresolvedVar.assign(n, -1);
        for (int64_t k = 0; k < r->presolved_variables; ++k)
            ps.originalToPresolvedVar[static_cast<std::size_t>(r->variable_origin[k])] =
                static_cast<int>(k);
        ps.presolvedToOriginalConstraint.assign(r->constraint_origin,
                                                r->constraint_origin + r->presolved_constraints);
        ps.originalToPresolvedConstraint.assign(m, -1);
        for (int64_t k = 0; k < r->presolved_constraints; ++k)
            ps.originalToPresolvedConstraint[static_cast<std::size_t>(r->constraint_origin[k])] =
                static_cast<int>(k);
    }
    pdlpgpu_presolve_free(r);
    return out;
}

}  // namespace pdlpgpu

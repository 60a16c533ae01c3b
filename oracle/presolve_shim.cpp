// presolve_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's presolve::Presolver::run (src/presolve/presolver.cpp,
// compiled from the reference's sources where they lie) and this library's
// pdlpgpu::presolve_model (include/pdlpgpu_presolve.hpp over
// pdlpgpu_presolve) on the same model::Model and compares the two
// PresolveResults field by field, doubles by their bits. oracle/Makefile
// links it as oracle/_ref/libpresolve_cmp.so; only the ps_* functions are
// exported. Models come in as pdlpgpu_presolve_model arrays (variables named
// x<i>, rows c<i>) or as MPS files read by the reference's MpsReader.
#include "model/model.h"
#include "mps/mps_reader.h"
#include "pdlpgpu_presolve.hpp"
#include "presolve/presolver.h"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <sstream>
#include <string>

#define PS_API extern "C" __attribute__((visibility("default")))

namespace {

void put(char* dst, int len, const std::string& s) {
    if (dst == nullptr || len <= 0) return;
    const std::size_t k = std::min<std::size_t>(s.size(), static_cast<std::size_t>(len - 1));
    std::memcpy(dst, s.data(), k);
    dst[k] = '\0';
}

model::Model to_model(const pdlpgpu_presolve_model& in) {
    model::Model m;
    m.name = "presolve_case";
    m.objective.offset = in.objective_offset;
    for (int64_t v = 0; v < in.num_variables; ++v) {
        model::Variable var;
        var.name = "x" + std::to_string(v);
        var.type = static_cast<model::VariableType>(in.var_type[v]);
        var.lowerBound = in.var_lower[v];
        var.upperBound = in.var_upper[v];
        m.variables.push_back(var);
    }
    for (int64_t r = 0; r < in.num_constraints; ++r) {
        model::Constraint c;
        c.name = "c" + std::to_string(r);
        c.lowerBound = in.row_lower[r];
        c.upperBound = in.row_upper[r];
        for (int64_t p = in.row_start[r]; p < in.row_start[r + 1]; ++p)
            c.linearTerms.push_back({in.row_index[p], in.row_value[p]});
        m.constraints.push_back(std::move(c));
    }
    for (int64_t k = 0; k < in.num_objective_terms; ++k)
        m.objective.linearTerms.push_back({in.objective_index[k], in.objective_value[k]});
    for (int64_t k = 0; k < in.num_quadratic_terms; ++k)
        m.objective.quadraticTerms.push_back(
            {in.quadratic_index1[k], in.quadratic_index2[k], in.quadratic_value[k]});
    return m;
}

struct Diff {
    std::ostringstream where;
    bool found = false;
    template <class T>
    bool same(const char* what, const T& a, const T& b) {
        if (found || a == b) return !found;
        found = true;
        where << what << ": reference " << a << ", fast " << b;
        return false;
    }
    bool bits(const std::string& what, double a, double b) {
        if (found || std::memcmp(&a, &b, sizeof(double)) == 0) return !found;
        found = true;
        where.precision(17);
        where << what << ": reference " << a << ", fast " << b;
        return false;
    }
};

std::string at(const char* what, std::size_t k, const char* field) {
    return std::string(what) + "[" + std::to_string(k) + "]." + field;
}

void compare_models(Diff& d, const model::Model& a, const model::Model& b) {
    d.same("model.name", a.name, b.name);
    d.same("objective.sense", static_cast<int>(a.objective.sense), static_cast<int>(b.objective.sense));
    d.bits("objective.offset", a.objective.offset, b.objective.offset);
    d.same("objective.linearTerms.size", a.objective.linearTerms.size(), b.objective.linearTerms.size());
    for (std::size_t k = 0; !d.found && k < a.objective.linearTerms.size(); ++k) {
        d.same(at("objective.linearTerms", k, "variableIndex").c_str(),
               a.objective.linearTerms[k].variableIndex, b.objective.linearTerms[k].variableIndex);
        d.bits(at("objective.linearTerms", k, "value"), a.objective.linearTerms[k].value,
               b.objective.linearTerms[k].value);
    }
    d.same("objective.quadraticTerms.size", a.objective.quadraticTerms.size(),
           b.objective.quadraticTerms.size());
    for (std::size_t k = 0; !d.found && k < a.objective.quadraticTerms.size(); ++k) {
        const auto &x = a.objective.quadraticTerms[k], &y = b.objective.quadraticTerms[k];
        d.same(at("objective.quadraticTerms", k, "variableIndex1").c_str(), x.variableIndex1,
               y.variableIndex1);
        d.same(at("objective.quadraticTerms", k, "variableIndex2").c_str(), x.variableIndex2,
               y.variableIndex2);
        d.bits(at("objective.quadraticTerms", k, "value"), x.value, y.value);
    }
    d.same("variables.size", a.variables.size(), b.variables.size());
    for (std::size_t k = 0; !d.found && k < a.variables.size(); ++k) {
        d.same(at("variables", k, "name").c_str(), a.variables[k].name, b.variables[k].name);
        d.same(at("variables", k, "type").c_str(), static_cast<int>(a.variables[k].type),
               static_cast<int>(b.variables[k].type));
        d.bits(at("variables", k, "lowerBound"), a.variables[k].lowerBound, b.variables[k].lowerBound);
        d.bits(at("variables", k, "upperBound"), a.variables[k].upperBound, b.variables[k].upperBound);
    }
    d.same("constraints.size", a.constraints.size(), b.constraints.size());
    for (std::size_t k = 0; !d.found && k < a.constraints.size(); ++k) {
        const auto &x = a.constraints[k], &y = b.constraints[k];
        d.same(at("constraints", k, "name").c_str(), x.name, y.name);
        d.bits(at("constraints", k, "lowerBound"), x.lowerBound, y.lowerBound);
        d.bits(at("constraints", k, "upperBound"), x.upperBound, y.upperBound);
        d.same(at("constraints", k, "linearTerms.size").c_str(), x.linearTerms.size(),
               y.linearTerms.size());
        for (std::size_t t = 0; !d.found && t < x.linearTerms.size(); ++t) {
            d.same((at("constraints", k, "linearTerms[") + std::to_string(t) + "].variableIndex").c_str(),
                   x.linearTerms[t].variableIndex, y.linearTerms[t].variableIndex);
            d.bits(at("constraints", k, "linearTerms[") + std::to_string(t) + "].value",
                   x.linearTerms[t].value, y.linearTerms[t].value);
        }
    }
}

std::string compare(const presolve::PresolveResult& a, const presolve::PresolveResult& b) {
    Diff d;
    d.same("infeasible", a.infeasible, b.infeasible);
    d.same("converged", a.converged, b.converged);
    d.same("originalVariables", a.originalVariables, b.originalVariables);
    d.same("originalConstraints", a.originalConstraints, b.originalConstraints);
    d.same("presolvedVariables", a.presolvedVariables, b.presolvedVariables);
    d.same("presolvedConstraints", a.presolvedConstraints, b.presolvedConstraints);
    compare_models(d, a.model, b.model);
    d.same("transformations.size", a.transformations.size(), b.transformations.size());
    for (std::size_t k = 0; !d.found && k < a.transformations.size(); ++k) {
        const auto &x = a.transformations[k], &y = b.transformations[k];
        d.same(at("transformations", k, "type").c_str(), static_cast<int>(x.type), static_cast<int>(y.type));
        d.same(at("transformations", k, "index").c_str(), x.index, y.index);
        d.same(at("transformations", k, "originalVariableIndex").c_str(), x.originalVariableIndex,
               y.originalVariableIndex);
        d.same(at("transformations", k, "originalConstraintIndex").c_str(),
               x.originalConstraintIndex, y.originalConstraintIndex);
        d.bits(at("transformations", k, "oldValue"), x.oldValue, y.oldValue);
        d.bits(at("transformations", k, "newValue"), x.newValue, y.newValue);
        d.same(at("transformations", k, "reason").c_str(), x.reason, y.reason);
        d.same(at("transformations", k, "entityName").c_str(), x.entityName, y.entityName);
        d.bits(at("transformations", k, "offsetChange"), x.offsetChange, y.offsetChange);
    }
    const auto &p = a.postsolve, &q = b.postsolve;
    d.same("originalToPresolvedVar", p.originalToPresolvedVar == q.originalToPresolvedVar, true);
    d.same("presolvedToOriginalVar", p.presolvedToOriginalVar == q.presolvedToOriginalVar, true);
    d.same("originalToPresolvedConstraint",
           p.originalToPresolvedConstraint == q.originalToPresolvedConstraint, true);
    d.same("presolvedToOriginalConstraint",
           p.presolvedToOriginalConstraint == q.presolvedToOriginalConstraint, true);
    d.bits("initialObjectiveOffset", p.initialObjectiveOffset, q.initialObjectiveOffset);
    d.bits("presolvedObjectiveOffset", p.presolvedObjectiveOffset, q.presolvedObjectiveOffset);
    d.same("fixedVariables.size", p.fixedVariables.size(), q.fixedVariables.size());
    for (std::size_t k = 0; !d.found && k < p.fixedVariables.size(); ++k) {
        const auto &x = p.fixedVariables[k], &y = q.fixedVariables[k];
        d.same(at("fixedVariables", k, "originalIndex").c_str(), x.originalIndex, y.originalIndex);
        d.same(at("fixedVariables", k, "name").c_str(), x.name, y.name);
        d.bits(at("fixedVariables", k, "fixedValue"), x.fixedValue, y.fixedValue);
        d.same(at("fixedVariables", k, "type").c_str(), static_cast<int>(x.type), static_cast<int>(y.type));
        d.bits(at("fixedVariables", k, "linearObjectiveContribution"), x.linearObjectiveContribution,
               y.linearObjectiveContribution);
        d.bits(at("fixedVariables", k, "quadraticDiagonalContribution"),
               x.quadraticDiagonalContribution, y.quadraticDiagonalContribution);
        d.same(at("fixedVariables", k, "quadraticCrossContributions.size").c_str(),
               x.quadraticCrossContributions.size(), y.quadraticCrossContributions.size());
        auto i = x.quadraticCrossContributions.begin();
        auto j = y.quadraticCrossContributions.begin();
        for (; !d.found && i != x.quadraticCrossContributions.end(); ++i, ++j) {
            d.same(at("fixedVariables", k, "quadraticCrossContributions.key").c_str(), i->first, j->first);
            d.bits(at("fixedVariables", k, "quadraticCrossContributions.value"), i->second, j->second);
        }
    }
    d.same("removedConstraints.size", p.removedConstraints.size(), q.removedConstraints.size());
    for (std::size_t k = 0; !d.found && k < p.removedConstraints.size(); ++k) {
        const auto &x = p.removedConstraints[k], &y = q.removedConstraints[k];
        d.same(at("removedConstraints", k, "originalIndex").c_str(), x.originalIndex, y.originalIndex);
        d.same(at("removedConstraints", k, "name").c_str(), x.name, y.name);
        d.bits(at("removedConstraints", k, "lowerBound"), x.lowerBound, y.lowerBound);
        d.bits(at("removedConstraints", k, "upperBound"), x.upperBound, y.upperBound);
        d.same(at("removedConstraints", k, "reason").c_str(), x.reason, y.reason);
        d.same(at("removedConstraints", k, "wasSingleton").c_str(), x.wasSingleton, y.wasSingleton);
        d.same(at("removedConstraints", k, "singletonOriginalVarIndex").c_str(),
               x.singletonOriginalVarIndex, y.singletonOriginalVarIndex);
        d.bits(at("removedConstraints", k, "singletonCoefficient"), x.singletonCoefficient,
               y.singletonCoefficient);
        d.same(at("removedConstraints", k, "wasDuplicate").c_str(), x.wasDuplicate, y.wasDuplicate);
        d.same(at("removedConstraints", k, "duplicateOfOriginalIndex").c_str(),
               x.duplicateOfOriginalIndex, y.duplicateOfOriginalIndex);
        d.bits(at("removedConstraints", k, "scale"), x.scale, y.scale);
    }
    return d.found ? d.where.str() : std::string();
}

// summary[6] = {infeasible, converged, presolved variables, presolved
// constraints, transformations, removed constraints}
void summarise(const presolve::PresolveResult& r, int64_t* summary) {
    if (summary == nullptr) return;
    summary[0] = r.infeasible ? 1 : 0;
    summary[1] = r.converged ? 1 : 0;
    summary[2] = static_cast<int64_t>(r.presolvedVariables);
    summary[3] = static_cast<int64_t>(r.presolvedConstraints);
    summary[4] = static_cast<int64_t>(r.transformations.size());
    summary[5] = static_cast<int64_t>(r.postsolve.removedConstraints.size());
}

int run_compare(const model::Model& m, char* report, int len, int64_t* summary) {
    const presolve::PresolveResult ref = presolve::Presolver().run(m);
    const presolve::PresolveResult fast = pdlpgpu::presolve_model(m);
    summarise(ref, summary);
    const std::string diff = compare(ref, fast);
    put(report, len, diff);
    return diff.empty() ? 0 : 1;
}

}  // namespace

// 0: identical results; 1: they differ (report names the first field);
// -1: an exception (report holds it).
PS_API int ps_compare(const pdlpgpu_presolve_model* in, char* report, int len, int64_t* summary) {
    try {
        return run_compare(to_model(*in), report, len, summary);
    } catch (const std::exception& e) {
        put(report, len, e.what());
        return -1;
    }
}

PS_API int ps_compare_mps(const char* path, char* report, int len, int64_t* summary) {
    try {
        mps::MpsReader reader;
        return run_compare(reader.read(path), report, len, summary);
    } catch (const std::exception& e) {
        put(report, len, e.what());
        return -1;
    }
}

// Wall time of one presolve of the model: which = 0 the reference's
// Presolver::run, 1 pdlpgpu::presolve_model (with its conversions).
PS_API int ps_time(const pdlpgpu_presolve_model* in, int which, double* seconds, int64_t* summary) {
    try {
        const model::Model m = to_model(*in);
        const auto t0 = std::chrono::steady_clock::now();
        const presolve::PresolveResult r =
            which == 0 ? presolve::Presolver().run(m) : pdlpgpu::presolve_model(m);
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        summarise(r, summary);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

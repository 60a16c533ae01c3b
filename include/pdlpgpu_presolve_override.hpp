// pdlpgpu_presolve_override.hpp -- the link-time drop-in for presolve.
//
// Defines the reference's own presolve::Presolver::run
// (include/presolve/presolver.h:11) on pdlpgpu::presolve_model. A build of
// the reference that links one translation unit including this header in
// place of src/presolve/presolver.cpp runs the fast presolve inside
// solver::solve (src/solver/orchestrator.cpp:596-597) with no source line
// changed; the result is the one the reference's presolver returns.
//
// Include it in exactly one translation unit; linking presolver.cpp as well is
// a duplicate-symbol error, by design.
#pragma once

#include "pdlpgpu_presolve.hpp"
#include "presolve/presolver.h"

namespace presolve {

PresolveResult Presolver::run(const model::Model& input) { return pdlpgpu::presolve_model(input); }

}  // namespace presolve

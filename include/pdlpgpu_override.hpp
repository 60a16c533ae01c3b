// pdlpgpu_override.hpp -- the link-time drop-in.
//
// Defines the reference's own pdlp::PdlpSolver::solve
// (pdlp_engine/include/pdlp/pdlp_solver.h:9-15) and pdlp::toString(PdlpStatus)
// (pdlp_engine/include/pdlp/pdlp_result.h:64) in terms of this engine. A build
// of the reference that links one translation unit including this header in
// place of pdlp_engine/src/pdlp_solver.cpp sends every PdlpSolver call --
// solver::runPdlp (src/solver/orchestrator.cpp:337) among them -- to the GPU
// without changing a line of the reference's sources. Everything else of
// pdlp_engine (CompiledLp, SparseMatrix, the options and result types) is
// still the reference's.
//
// Include it in exactly one translation unit; linking pdlp_solver.cpp as well
// is a duplicate-symbol error, by design.
//
// The engine runs the reference's FP64 arithmetic on device 0 unless the
// environment says otherwise when the first solve starts:
//   PDLPGPU_PRECISION = fp64 | mixed   (mixed: FP32 iterations, FP64 checks)
//   PDLPGPU_DEVICE    = CUDA device ordinal
#pragma once

#include "pdlp/pdlp_result.h"
#include "pdlp/pdlp_solver.h"
#include "pdlpgpu.hpp"

#include <cstdlib>
#include <cstring>

namespace pdlpgpu_override_detail {

inline int32_t env_precision() {
    const char* v = std::getenv("PDLPGPU_PRECISION");
    return v != nullptr && std::strcmp(v, "mixed") == 0 ? PDLPGPU_PRECISION_MIXED
                                                         : PDLPGPU_PRECISION_FP64;
}

inline int32_t env_device() {
    const char* v = std::getenv("PDLPGPU_DEVICE");
    return v != nullptr ? static_cast<int32_t>(std::atoi(v)) : 0;
}

}  // namespace pdlpgpu_override_detail

namespace pdlp {

const char* toString(PdlpStatus status) noexcept {
    return pdlpgpu_status_string(static_cast<int32_t>(status));
}

PdlpResult PdlpSolver::solve(const CompiledLp& problem, const PdlpOptions& options) const {
    static const int32_t precision = pdlpgpu_override_detail::env_precision();
    static const int32_t device = pdlpgpu_override_detail::env_device();
    return pdlpgpu::PdlpSolver(precision, device).solve(problem, options);
}

}  // namespace pdlp

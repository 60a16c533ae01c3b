// presolve_override.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's presolve::Presolver::run defined on the library's fast
// presolve (include/pdlpgpu_presolve_override.hpp). oracle/Makefile links it
// into libpipeline_fastpre.so ahead of the reference's objects, so that
// solver::solve (src/solver/orchestrator.cpp:596-597) presolves through it
// while every other part of the pipeline is the reference's own.
#include "pdlpgpu_presolve_override.hpp"

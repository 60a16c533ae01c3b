// TEST INFRASTRUCTURE ONLY. The one translation unit a build of the reference
// adds in place of pdlp_engine/src/pdlp_solver.cpp so that every
// pdlp::PdlpSolver::solve call runs on the GPU engine (see the header).
#include "pdlpgpu_override.hpp"

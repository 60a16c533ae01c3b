// mps_override.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's mps::MpsReader::read defined on the library's fast reader
// (include/pdlpgpu_mps_override.hpp). oracle/Makefile links it in place of
// src/mps/mps_reader.cpp into the reference's own MPS reader tests and its
// command-line program, which then read files through the fast reader.
#include "pdlpgpu_mps_override.hpp"

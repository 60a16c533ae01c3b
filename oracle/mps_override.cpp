// mps_override.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's mps::MpsReader::read (include/mps/mps_reader.h:58-70)
// defined on the library's fast reader (include/pdlpgpu_mps.hpp), warnings
// included. oracle/Makefile links it in place of src/mps/mps_reader.cpp into
// the reference's own MPS reader tests, which then run against the fast
// reader.
#include "mps/mps_reader.h"
#include "pdlpgpu_mps.hpp"

namespace mps {

model::Model MpsReader::read(const std::string& filepath) {
    pdlpgpu::MpsReader fast;
    model::Model m = fast.read(filepath);
    warnings_ = fast.warnings();
    return m;
}

}  // namespace mps

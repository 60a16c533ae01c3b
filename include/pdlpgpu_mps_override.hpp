// pdlpgpu_mps_override.hpp -- the link-time drop-in for MPS reading.
//
// Defines the reference's own mps::MpsReader::read
// (include/mps/mps_reader.h:58-70) on the fast reader
// (include/pdlpgpu_mps.hpp): the same model::Model, the same warnings (left
// in the reader, where its warnings() returns them) and the same
// std::runtime_error messages. A build of the reference that links one
// translation unit including this header in place of src/mps/mps_reader.cpp
// reads files this way -- its command-line program and its solver included --
// with no source line changed. Terms of a row come in increasing column order
// (the reference's order is that of its hash map, which carries no meaning).
//
// Include it in exactly one translation unit; linking mps_reader.cpp as well
// is a duplicate-symbol error, by design.
#pragma once

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

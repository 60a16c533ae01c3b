// pdlpgpu_mps.hpp -- header-only C++ facade of the fast MPS reader with the
// reference reader's interface:
//
//   model::Model pdlpgpu::MpsReader::read(const std::string& filepath);
//   const std::vector<std::string>& pdlpgpu::MpsReader::warnings() const noexcept;
//
// It replaces mps::MpsReader (include/mps/mps_reader.h:58-77) wherever the
// reference reads a file (its CLI, its benchmark tools) by changing only the
// namespace: the same model::Model, the same warnings, and a std::runtime_error
// with the same message for every file the reference refuses. Include it where
// the reference's model headers are on the include path and link
// libpdlpgpu.so.
#pragma once

#include "model/model.h"
#include "pdlpgpu_mps.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace pdlpgpu {

class MpsReader {
public:
    model::Model read(const std::string& filepath) {
        warnings_.clear();
        pdlpgpu_mps* m = nullptr;
        if (pdlpgpu_mps_read(filepath.c_str(), &m) != 0) throw std::runtime_error(pdlpgpu_last_error());
        struct Release {
            pdlpgpu_mps* m;
            ~Release() { pdlpgpu_mps_free(m); }
        } release{m};
        int64_t sizes[8];
        pdlpgpu_mps_sizes(m, sizes);
        const std::size_t nv = static_cast<std::size_t>(sizes[0]), nc = static_cast<std::size_t>(sizes[1]);
        const std::size_t no = static_cast<std::size_t>(sizes[2]), nr = static_cast<std::size_t>(sizes[3]);
        const std::size_t nq = static_cast<std::size_t>(sizes[4]), nw = static_cast<std::size_t>(sizes[5]);
        double offset = 0.0;
        std::vector<int32_t> oi(no), vt(nv), ri(nr), qi(nq), qj(nq);
        std::vector<double> ov(no), vl(nv), vu(nv), rl(nc), ru(nc), rv(nr), qv(nq);
        std::vector<int64_t> rs(nc + 1);
        pdlpgpu_mps_model(m, &offset, oi.data(), ov.data(), vt.data(), vl.data(), vu.data(), rl.data(),
                          ru.data(), rs.data(), ri.data(), rv.data(), qi.data(), qj.data(), qv.data());
        model::Model out;
        out.name = pdlpgpu_mps_name(m, 0, 0);
        out.objective.sense = sizes[6] ? model::ObjectiveSense::Maximize : model::ObjectiveSense::Minimize;
        out.objective.offset = offset;
        out.objective.linearTerms.reserve(no);
        for (std::size_t k = 0; k < no; ++k) out.objective.linearTerms.push_back({oi[k], ov[k]});
        for (std::size_t k = 0; k < nq; ++k) out.objective.quadraticTerms.push_back({qi[k], qj[k], qv[k]});
        out.variables.resize(nv);
        for (std::size_t j = 0; j < nv; ++j) {
            model::Variable& v = out.variables[j];
            v.name = pdlpgpu_mps_name(m, 1, static_cast<int64_t>(j));
            v.type = static_cast<model::VariableType>(vt[j]);
            v.lowerBound = vl[j];
            v.upperBound = vu[j];
        }
        out.constraints.resize(nc);
        for (std::size_t i = 0; i < nc; ++i) {
            model::Constraint& c = out.constraints[i];
            c.name = pdlpgpu_mps_name(m, 2, static_cast<int64_t>(i));
            c.lowerBound = rl[i];
            c.upperBound = ru[i];
            c.linearTerms.reserve(static_cast<std::size_t>(rs[i + 1] - rs[i]));
            for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
                c.linearTerms.push_back({ri[static_cast<std::size_t>(k)], rv[static_cast<std::size_t>(k)]});
        }
        for (std::size_t k = 0; k < nw; ++k) warnings_.emplace_back(pdlpgpu_mps_name(m, 3, static_cast<int64_t>(k)));
        return out;
    }

    [[nodiscard]] const std::vector<std::string>& warnings() const noexcept { return warnings_; }

private:
    std::vector<std::string> warnings_;
};

}  // namespace pdlpgpu

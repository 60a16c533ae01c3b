// layout.hpp -- host-side construction of the device layout (no CUDA calls).
#pragma once

#include "common.cuh"
#include "pdlpgpu.h"

#include <cstdint>
#include <string>
#include <vector>

namespace pdlpgpu {

// Canonical CSR (what pdlp::SparseMatrix holds).
struct HostCsr {
    int32_t rows = 0;
    int32_t cols = 0;
    std::vector<int64_t> start;
    std::vector<int32_t> index;
    std::vector<double> value;
    int64_t nnz() const { return static_cast<int64_t>(value.size()); }
};

// SparseMatrix::fromTriplets semantics applied to a caller's CSR
// (pdlp_engine/src/sparse_matrix.cpp:76-201): entries ordered by column within
// each row, duplicates summed in input order, exact zeros dropped. Returns an
// empty string, or the reference's exception message for invalid input.
std::string canonicalize(const pdlpgpu_lp& lp, HostCsr& out);

// CompiledLp::validate (pdlp_engine/include/pdlp/compiled_lp.h:32-62) on the
// vectors. Returns an empty string or the reference's message.
std::string validate_vectors(const pdlpgpu_lp& lp);

struct Tuning {
    int lane_elements = 8;   // target entries per lane before the lane group doubles
    int vector_width = 1;    // 1, 2 or 4 entries per lane load
};

// One side of one matrix in the SELL-G layout.
struct SideLayout {
    std::vector<SliceDesc> slices;   // data_off relative to this side's first slot
    std::vector<int32_t> idx;        // slots; local indices into the other space
    std::vector<double> val;         // slots; original coefficients, 0 on padding
    std::vector<int32_t> line_len;   // entries per line, internal order
    int64_t entries = 0;             // real (non-padding) entries
    int64_t slots() const { return static_cast<int64_t>(idx.size()); }
};

struct MatrixLayout {
    int32_t m = 0, n = 0;
    std::vector<int32_t> row_perm;   // internal row -> original row
    std::vector<int32_t> col_perm;   // internal column -> original column
    SideLayout a;                    // lines = rows, gathers over columns
    SideLayout at;                   // lines = columns, gathers over rows
};

// Renumbers rows by decreasing length and columns by decreasing degree (ties
// by original index), then builds both sides.
MatrixLayout build_layout(const HostCsr& a, const Tuning& t);

// Splits the slices of each instance into CTAs of roughly `target_slots`
// slots (never crossing an instance). Appends to `out`; returns the count.
int append_cta_map(const SideLayout& side, int32_t instance, int32_t slice_base,
                   int64_t target_slots, std::vector<CtaWork>& out);

// Elementwise map: chunks of kVecChunk columns then rows of one instance.
int append_vec_map(int32_t instance, int32_t m, int32_t n, std::vector<VecWork>& out);

// Choice of slots per CTA for a total of `slots` over `sms` multiprocessors.
int64_t cta_target_slots(int64_t slots, int sms);

// Autotuning heuristic for a matrix: lane target and vector width.
Tuning choose_tuning(const HostCsr& a, bool fp32);

}  // namespace pdlpgpu

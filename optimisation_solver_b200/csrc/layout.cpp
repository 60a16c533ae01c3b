// layout.cpp -- host-side construction of the SELL-G device layout.
#include "layout.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace pdlpgpu {

std::string canonicalize(const pdlpgpu_lp& lp, HostCsr& out) {
    if (lp.num_rows < 0 || lp.num_cols < 0) return "Sparse matrix dimensions must be nonnegative";
    if (lp.row_start == nullptr) return "CompiledLp contains an invalid sparse matrix";
    const int32_t m = lp.num_rows, n = lp.num_cols;
    if (lp.row_start[0] != 0) return "CompiledLp contains an invalid sparse matrix";
    for (int32_t i = 0; i < m; ++i) {
        if (lp.row_start[i + 1] < lp.row_start[i]) return "CompiledLp contains an invalid sparse matrix";
    }
    const int64_t count = lp.row_start[m];
    if (count > 0 && (lp.col_index == nullptr || lp.values == nullptr))
        return "CompiledLp contains an invalid sparse matrix";
    for (int64_t k = 0; k < count; ++k) {
        if (lp.col_index[k] < 0 || lp.col_index[k] >= n) return "Sparse matrix triplet index is out of range";
        if (!std::isfinite(lp.values[k])) return "Sparse matrix coefficient must be finite";
    }
    out.rows = m;
    out.cols = n;
    out.start.assign(static_cast<size_t>(m) + 1, 0);
    out.index.clear();
    out.value.clear();
    out.index.reserve(static_cast<size_t>(count));
    out.value.reserve(static_cast<size_t>(count));
    std::vector<std::pair<int32_t, int64_t>> row;   // (column, input position)
    for (int32_t i = 0; i < m; ++i) {
        const int64_t b = lp.row_start[i], e = lp.row_start[i + 1];
        bool canonical = true;
        for (int64_t k = b; k < e; ++k) {
            if (lp.values[k] == 0.0 || (k > b && lp.col_index[k] <= lp.col_index[k - 1])) {
                canonical = false;
                break;
            }
        }
        if (canonical) {
            out.index.insert(out.index.end(), lp.col_index + b, lp.col_index + e);
            out.value.insert(out.value.end(), lp.values + b, lp.values + e);
        } else {
            row.clear();
            for (int64_t k = b; k < e; ++k) row.emplace_back(lp.col_index[k], k);
            std::sort(row.begin(), row.end());   // by column, then input position
            for (size_t k = 0; k < row.size();) {
                const int32_t col = row[k].first;
                double acc = lp.values[row[k].second];
                ++k;
                while (k < row.size() && row[k].first == col) {
                    acc += lp.values[row[k].second];
                    ++k;
                }
                if (acc != 0.0) {
                    out.index.push_back(col);
                    out.value.push_back(acc);
                }
            }
        }
        out.start[static_cast<size_t>(i) + 1] = static_cast<int64_t>(out.value.size());
    }
    return std::string();
}

std::string validate_vectors(const pdlpgpu_lp& lp) {
    const int32_t m = lp.num_rows, n = lp.num_cols;
    if ((n > 0 && (lp.objective == nullptr || lp.var_lower == nullptr || lp.var_upper == nullptr)))
        return "CompiledLp column vector dimensions do not match A";
    if (m > 0 && (lp.row_lower == nullptr || lp.row_upper == nullptr))
        return "CompiledLp row vector dimensions do not match A";
    if (!std::isfinite(lp.objective_offset)) return "Objective offset must be finite";
    for (int32_t j = 0; j < n; ++j) {
        const double l = lp.var_lower[j], u = lp.var_upper[j];
        if (!std::isfinite(lp.objective[j]) || std::isnan(l) || std::isnan(u) || l > u)
            return "Invalid objective coefficient or variable bounds";
    }
    for (int32_t i = 0; i < m; ++i) {
        const double l = lp.row_lower[i], u = lp.row_upper[i];
        if (std::isnan(l) || std::isnan(u) || l > u) return "Invalid row bounds";
    }
    return std::string();
}

namespace {

// Lines by decreasing length, ties by index: a stable counting sort.
std::vector<int32_t> order_by_length(const std::vector<int64_t>& start, int32_t lines) {
    std::vector<int32_t> perm(static_cast<size_t>(lines));
    int64_t longest = 0;
    for (int32_t x = 0; x < lines; ++x) longest = std::max(longest, start[x + 1] - start[x]);
    std::vector<int64_t> at(static_cast<size_t>(longest) + 2, 0);   // at[longest - len + 1]: count
    for (int32_t x = 0; x < lines; ++x) ++at[static_cast<size_t>(longest - (start[x + 1] - start[x])) + 1];
    for (size_t k = 1; k < at.size(); ++k) at[k] += at[k - 1];
    for (int32_t x = 0; x < lines; ++x) perm[at[static_cast<size_t>(longest - (start[x + 1] - start[x]))]++] = x;
    return perm;
}

int lane_group(int64_t len, int target) {
    if (len <= target) return 1;
    const int64_t need = (len + target - 1) / target;
    int g = 1;
    while (g < need && g < 32) g <<= 1;
    return g;
}

// Slice shapes of one side from its line lengths (internal order), and for
// every line where its entries go: entry k of line i lands in slot
// base[i] + (s / V) * 32 * V + (lane0[i] + (k & (G - 1))) * V + s % V with
// s = k >> glog[i], G = 1 << glog[i].
struct SlotMap {
    std::vector<int64_t> base;
    std::vector<int32_t> lane0;
    std::vector<uint8_t> glog;
    int vlog = 0;   // V = 1 << vlog
    int64_t slot(int32_t line, int64_t k) const {
        const int gl = glog[static_cast<size_t>(line)];
        const int64_t s = k >> gl;
        const int64_t lane = lane0[static_cast<size_t>(line)] + (k & ((int64_t(1) << gl) - 1));
        return base[static_cast<size_t>(line)] + (((s >> vlog) * 32 + lane) << vlog) + (s & ((1 << vlog) - 1));
    }
};

SlotMap plan_side(std::vector<int32_t> line_len, const Tuning& t, SideLayout& side) {
    const int V = t.vector_width;
    const int32_t L = static_cast<int32_t>(line_len.size());
    side.slices.clear();
    side.entries = 0;
    for (int32_t len : line_len) side.entries += len;
    SlotMap map;
    while ((1 << map.vlog) < V) ++map.vlog;
    map.base.resize(static_cast<size_t>(L));
    map.lane0.resize(static_cast<size_t>(L));
    map.glog.resize(static_cast<size_t>(L));
    int64_t slots = 0;
    for (int32_t i = 0; i < L;) {
        const int64_t len0 = line_len[i];
        const int G = lane_group(len0, t.lane_elements);
        int glog = 0;
        while ((1 << glog) < G) ++glog;
        const int R = 32 >> glog;
        const int nl = std::min<int32_t>(R, L - i);
        int64_t steps = (len0 + G - 1) / G;
        steps = (steps + V - 1) / V * V;
        SliceDesc sd;
        sd.data_off = static_cast<int32_t>(slots / 32);
        sd.line0 = i;
        sd.steps = static_cast<int32_t>(steps);
        sd.meta = glog | (nl << 8);
        side.slices.push_back(sd);
        for (int r = 0; r < nl; ++r) {
            map.base[static_cast<size_t>(i + r)] = slots;
            map.lane0[static_cast<size_t>(i + r)] = r * G;
            map.glog[static_cast<size_t>(i + r)] = static_cast<uint8_t>(glog);
        }
        slots += steps * 32;
        i += nl;
    }
    side.line_len = std::move(line_len);
    side.idx.assign(static_cast<size_t>(slots), 0);
    side.val.assign(static_cast<size_t>(slots), 0.0);
    return map;
}

}  // namespace

// One pass over the rows of A in internal order: each row's entries are
// renumbered to internal columns and sorted (rows are short), written to
// their A-side slots, and appended to their columns' A^T-side slots. Rows
// are visited in increasing internal order, so every column receives its
// entries in increasing internal row order -- no transpose of A and no
// intermediate copy.
MatrixLayout build_layout(const HostCsr& a, const Tuning& t) {
    MatrixLayout L;
    const int32_t m = a.rows, n = a.cols;
    L.m = m;
    L.n = n;
    L.row_perm = order_by_length(a.start, m);
    std::vector<int64_t> col_start(static_cast<size_t>(n) + 1, 0);
    for (int32_t j : a.index) ++col_start[static_cast<size_t>(j) + 1];
    for (int32_t j = 0; j < n; ++j) col_start[j + 1] += col_start[j];
    L.col_perm = order_by_length(col_start, n);
    std::vector<int32_t> inv_col(static_cast<size_t>(n));
    std::vector<int32_t> row_len(static_cast<size_t>(m)), col_len(static_cast<size_t>(n));
    for (int32_t c = 0; c < n; ++c) {
        const int32_t j = L.col_perm[c];
        inv_col[j] = c;
        col_len[c] = static_cast<int32_t>(col_start[j + 1] - col_start[j]);
    }
    for (int32_t r = 0; r < m; ++r) {
        const int32_t i = L.row_perm[r];
        row_len[r] = static_cast<int32_t>(a.start[i + 1] - a.start[i]);
    }
    const SlotMap rows = plan_side(std::move(row_len), t, L.a);
    const SlotMap cols = plan_side(std::move(col_len), t, L.at);
    std::vector<int64_t> fill(static_cast<size_t>(n), 0);   // entries placed per column
    std::vector<std::pair<int32_t, double>> line;
    for (int32_t r = 0; r < m; ++r) {
        const int32_t i = L.row_perm[r];
        line.clear();
        for (int64_t k = a.start[i]; k < a.start[i + 1]; ++k) line.emplace_back(inv_col[a.index[k]], a.value[k]);
        std::sort(line.begin(), line.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t k = 0; k < line.size(); ++k) {
            const int32_t c = line[k].first;
            const double v = line[k].second;
            const int64_t p = rows.slot(r, static_cast<int64_t>(k));
            L.a.idx[static_cast<size_t>(p)] = c;
            L.a.val[static_cast<size_t>(p)] = v;
            const int64_t q = cols.slot(c, fill[static_cast<size_t>(c)]++);
            L.at.idx[static_cast<size_t>(q)] = r;
            L.at.val[static_cast<size_t>(q)] = v;
        }
    }
    return L;
}

int append_cta_map(const SideLayout& side, int32_t instance, int32_t slice_base,
                   int64_t target_slots, std::vector<CtaWork>& out) {
    const int before = static_cast<int>(out.size());
    const int32_t S = static_cast<int32_t>(side.slices.size());
    int32_t s = 0;
    while (s < S) {
        int64_t acc = 0;
        const int32_t b = s;
        // Per-line work (epilogue, vector reads) counts as a few slots.
        while (s < S && (s == b || acc + 32LL * side.slices[s].steps + 64 <= target_slots)) {
            acc += 32LL * side.slices[s].steps + 64;
            ++s;
        }
        out.push_back(CtaWork{instance, slice_base + b, slice_base + s, 0});
    }
    if (static_cast<int>(out.size()) == before) out.push_back(CtaWork{instance, slice_base, slice_base, 0});
    return static_cast<int>(out.size()) - before;
}

int append_vec_map(int32_t instance, int32_t m, int32_t n, std::vector<VecWork>& out) {
    const int before = static_cast<int>(out.size());
    for (int32_t b = 0; b < n; b += kVecChunk) out.push_back(VecWork{instance, 0, b, std::min(n, b + kVecChunk)});
    for (int32_t b = 0; b < m; b += kVecChunk) out.push_back(VecWork{instance, 1, b, std::min(m, b + kVecChunk)});
    if (static_cast<int>(out.size()) == before) out.push_back(VecWork{instance, 0, 0, 0});
    return static_cast<int>(out.size()) - before;
}

int64_t cta_target_slots(int64_t slots, int sms) {
    const int64_t per = slots / (static_cast<int64_t>(sms) * 8);
    return std::max<int64_t>(256, std::min<int64_t>(per, 32768));
}

Tuning choose_tuning(const HostCsr& a, bool fp32) {
    Tuning t;
    const double mean_a = a.rows ? static_cast<double>(a.nnz()) / a.rows : 0.0;
    const double mean_at = a.cols ? static_cast<double>(a.nnz()) / a.cols : 0.0;
    const double mean = std::min(mean_a, mean_at);
    t.lane_elements = 8;
    if (fp32) t.vector_width = mean >= 24.0 ? 4 : (mean >= 12.0 ? 2 : 1);
    else t.vector_width = mean >= 16.0 ? 2 : 1;
    return t;
}

}  // namespace pdlpgpu

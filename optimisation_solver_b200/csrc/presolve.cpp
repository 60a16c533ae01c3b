// presolve.cpp -- presolve::Presolver::run (src/presolve/presolver.cpp:1045-1155)
// with the reference's results and without its quadratic costs.
//
// State: variables and rows keep their original index as a stable id with an
// alive flag; a row's terms stay in the input arrays with a per-term alive
// flag, so the order of the surviving terms is the order the reference keeps
// after its erasures; column lists give each variable's term positions. The
// local indices the reference's log records are prefix counts of alive ids.
// Every floating-point expression below is evaluated as the reference writes
// it, in the same order, so bounds, offsets and scales agree bit for bit.
#include "pdlpgpu_presolve.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

extern "C" void pdlpgpu_internal_set_error(const char* message);

namespace {

constexpr double kEps = 1e-9;  // presolver.cpp:14
constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr int8_t kInteger = 1;
constexpr int8_t kBinary = 2;

inline bool approx_equal(double a, double b) {  // presolver.cpp:16-21
    if (std::isinf(a) || std::isinf(b)) return a == b;
    return std::abs(a - b) <= kEps;
}
inline bool integral(int8_t t) { return t == kInteger || t == kBinary; }
inline double round_lower(double b, int8_t t) {  // presolver.cpp:25-31
    if (!std::isfinite(b)) return b;
    return integral(t) ? std::ceil(b - kEps) : b;
}
inline double round_upper(double b, int8_t t) {  // presolver.cpp:33-39
    if (!std::isfinite(b)) return b;
    return integral(t) ? std::floor(b + kEps) : b;
}

// Counts of alive ids below a position, under removals (duplicate rows are
// removed out of index order, so their local index needs a live count).
struct Fenwick {
    std::vector<int64_t> t;
    explicit Fenwick(int64_t n) : t(static_cast<std::size_t>(n) + 1, 0) {}
    void add(int64_t i, int64_t d) {
        for (++i; i < static_cast<int64_t>(t.size()); i += i & -i) t[i] += d;
    }
    int64_t below(int64_t i) const {  // sum over [0, i)
        int64_t s = 0;
        for (; i > 0; i -= i & -i) s += t[i];
        return s;
    }
};

// Host threads the read-only steps may use: PDLPGPU_PRESOLVE_THREADS when set
// to a positive number (1 runs everything on the calling thread), else the
// host's hardware threads; at most 16 either way.
unsigned presolve_threads() {
    if (const char* v = std::getenv("PDLPGPU_PRESOLVE_THREADS")) {
        const long k = std::strtol(v, nullptr, 10);
        if (k > 0) return static_cast<unsigned>(std::min(k, 16L));
    }
    return std::min(std::max(1u, std::thread::hardware_concurrency()), 16u);
}

// Runs body(begin, end) over [0, n) in contiguous pieces of at least 4096 on
// presolve_threads() threads. Used only for work that reads shared state and
// writes disjoint outputs, so the results do not depend on the split.
template <class Body>
void parallel_for(int64_t n, const Body& body) {
    const int64_t pieces = std::min<int64_t>({static_cast<int64_t>(presolve_threads()),
                                              (n + 4095) / 4096, n});
    if (pieces <= 1) {
        if (n > 0) body(int64_t{0}, n);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(static_cast<std::size_t>(pieces - 1));
    for (int64_t k = 1; k < pieces; ++k)
        pool.emplace_back([&, k] { body(n * k / pieces, n * (k + 1) / pieces); });
    body(int64_t{0}, n / pieces);
    for (std::thread& t : pool) t.join();
}

struct FixedRecord {
    int64_t origin = 0;
    double value = 0.0, linear = 0.0, diagonal = 0.0;
    std::map<int64_t, double> cross;
};

struct RemovedRecord {
    int64_t origin = 0;
    double lower = 0.0, upper = 0.0;
    int32_t reason = 0;
    int8_t singleton = 0, duplicate = 0;
    int64_t singleton_var = 0, duplicate_of = 0;
    double coefficient = 0.0, scale = 1.0;
};

struct Out : pdlpgpu_presolve_result {
    std::vector<int64_t> var_origin, con_origin, rs;
    std::vector<double> vlo, vhi, rlo, rhi, rv, ov, qv;
    std::vector<int32_t> ri, oi, qi, qj;
    std::vector<int32_t> tr_type_v, tr_reason_v;
    std::vector<int64_t> tr_index_v, tr_var_v, tr_con_v;
    std::vector<double> tr_old_v, tr_new_v, tr_off_v;
    std::vector<int64_t> fx_origin, fx_cross_start, fx_cross_var;
    std::vector<double> fx_value, fx_linear, fx_diag, fx_cross_val;
    std::vector<int64_t> rm_origin, rm_svar, rm_dup_of;
    std::vector<double> rm_lo, rm_hi, rm_coef, rm_scale;
    std::vector<int32_t> rm_reason;
    std::vector<int8_t> rm_single, rm_dup;
};

class Presolve {
public:
    explicit Presolve(const pdlpgpu_presolve_model& in);
    void run();
    void emit(Out& out);  // moves the log out: call once, last

private:
    // variables
    int64_t n_;
    // Each variable's bounds side by side ({lower, upper}): bound tightening
    // reads both for every term it gathers, so they share a cache line.
    // lb_[v] and ub_[v] name the two halves.
    template <int Side>
    struct BoundView {
        std::vector<std::array<double, 2>>* store;
        double& operator[](int64_t v) const { return (*store)[static_cast<std::size_t>(v)][Side]; }
    };
    std::vector<std::array<double, 2>> bounds_;
    BoundView<0> lb_{&bounds_};
    BoundView<1> ub_{&bounds_};
    std::vector<int8_t> type_;
    std::vector<char> var_alive_;
    std::vector<int64_t> var_rank_;
    // rows
    int64_t m_;
    std::vector<int64_t> rs_;
    std::vector<int32_t> ri_;
    std::vector<double> rv_, lo_, hi_;
    std::vector<char> term_alive_, row_alive_;
    std::vector<int64_t> row_count_;
    std::vector<char> row_repeats_;  // the row names some variable twice
    std::vector<double> act_min_, act_max_;
    bool row_zeros_done_ = false;
    // a row lost a term or moved a bound since the duplicate pass last ran
    bool rows_touched_ = true;
    // Bound tightening's record of its sweeps: a counter of bound changes,
    // the count at each variable's last change and at each row's last sweep,
    // whether that sweep moved nothing, and whether the row's own terms or
    // bounds changed since.
    int64_t bound_changes_ = 0;
    std::vector<int64_t> var_changed_, row_swept_;
    std::vector<char> row_quiet_, row_dirty_;
    // tightening targets settled by their brackets, and those summed exactly
    int64_t bracketed_ = 0, summed_ = 0;
    void bound_moved(int64_t v) { var_changed_[v] = ++bound_changes_; }
    // column lists: term positions of each variable, by row then position
    std::vector<int64_t> cs_, cterm_;
    std::vector<int64_t> term_row_;
    // objective
    double offset_;
    std::vector<int32_t> oi_;
    std::vector<double> ov_;
    std::vector<char> oalive_;
    std::vector<int64_t> os_, opos_;
    std::unordered_map<int32_t, std::vector<int64_t>> oextra_;
    std::vector<int32_t> qi_, qj_;
    std::vector<double> qv_;
    std::vector<char> qalive_;
    // result
    bool infeasible_ = false, converged_ = true, has_maps_ = false;
    double initial_offset_;
    std::vector<FixedRecord> fixed_;
    std::vector<RemovedRecord> removed_;
    Out logbuf_;  // the transformation log's columns

    void log(int32_t type, int32_t reason, int64_t index, int64_t var, int64_t con,
             double old_value = 0.0, double new_value = 0.0, double offset = 0.0) {
        Out& L = logbuf_;
        L.tr_type_v.push_back(type);
        L.tr_reason_v.push_back(reason);
        L.tr_index_v.push_back(index);
        L.tr_var_v.push_back(var);
        L.tr_con_v.push_back(con);
        L.tr_old_v.push_back(old_value);
        L.tr_new_v.push_back(new_value);
        L.tr_off_v.push_back(offset);
    }
    void remove_row(int64_t r, int32_t reason) {
        RemovedRecord rec;
        rec.origin = r;
        rec.lower = lo_[r];
        rec.upper = hi_[r];
        rec.reason = reason;
        removed_.push_back(rec);
        row_alive_[r] = 0;
    }
    void rank_variables() {
        var_rank_.assign(static_cast<std::size_t>(n_), -1);
        int64_t k = 0;
        for (int64_t v = 0; v < n_; ++v)
            if (var_alive_[v]) var_rank_[v] = k++;
    }
    int64_t alive_rows() const {
        int64_t k = 0;
        for (int64_t r = 0; r < m_; ++r) k += row_alive_[r] ? 1 : 0;
        return k;
    }
    // minConstraintActivity / maxConstraintActivity (presolver.cpp:330-381):
    // the sums in term order, or -inf / +inf at the first unbounded term.
    void activities(int64_t r, double& mn, double& mx) const {
        double a_min = 0.0, a_max = 0.0;
        bool inf_min = false, inf_max = false;
        for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p) {
            if (!term_alive_[p]) continue;
            const int32_t v = ri_[p];
            const double a = rv_[p];
            if (a > 0.0) {
                if (!inf_min) {
                    if (!std::isfinite(lb_[v])) inf_min = true;
                    else a_min += a * lb_[v];
                }
                if (!inf_max) {
                    if (!std::isfinite(ub_[v])) inf_max = true;
                    else a_max += a * ub_[v];
                }
            } else if (a < 0.0) {
                if (!inf_min) {
                    if (!std::isfinite(ub_[v])) inf_min = true;
                    else a_min += a * ub_[v];
                }
                if (!inf_max) {
                    if (!std::isfinite(lb_[v])) inf_max = true;
                    else a_max += a * lb_[v];
                }
            }
        }
        mn = inf_min ? -kInf : a_min;
        mx = inf_max ? kInf : a_max;
    }

    bool remove_zero_coefficients();
    bool detect_simple_infeasibility() const;
    bool empty_rows();
    bool fixed_variables();
    bool fix_variable(int64_t v, double value, int64_t rank);
    bool singleton_rows();
    bool singleton_row(int64_t r, int64_t rank);
    bool tighten_bounds();
    bool redundant_rows();
    bool duplicate_rows();
};

Presolve::Presolve(const pdlpgpu_presolve_model& in)
    : n_(in.num_variables), m_(in.num_constraints), offset_(in.objective_offset),
      initial_offset_(in.objective_offset) {
    const std::size_t n = static_cast<std::size_t>(n_), m = static_cast<std::size_t>(m_);
    bounds_.resize(n);
    for (std::size_t v = 0; v < n; ++v) bounds_[v] = {in.var_lower[v], in.var_upper[v]};
    type_.assign(in.var_type, in.var_type + n);
    var_alive_.assign(n, 1);
    rs_.assign(in.row_start, in.row_start + m + 1);
    const std::size_t nnz = static_cast<std::size_t>(rs_[m]);
    ri_.assign(in.row_index, in.row_index + nnz);
    rv_.assign(in.row_value, in.row_value + nnz);
    lo_.assign(in.row_lower, in.row_lower + m);
    hi_.assign(in.row_upper, in.row_upper + m);
    term_alive_.assign(nnz, 1);
    row_alive_.assign(m, 1);
    row_count_.resize(m);
    term_row_.resize(nnz);
    row_repeats_.assign(m, 0);
    var_changed_.assign(n, 0);
    row_swept_.assign(m, 0);
    row_quiet_.assign(m, 0);
    row_dirty_.assign(m, 1);
    {
        std::vector<int64_t> stamp(n, -1);
        for (std::size_t r = 0; r < m; ++r) {
            row_count_[r] = rs_[r + 1] - rs_[r];
            for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p) {
                term_row_[p] = static_cast<int64_t>(r);
                if (stamp[ri_[p]] == static_cast<int64_t>(r)) row_repeats_[r] = 1;
                stamp[ri_[p]] = static_cast<int64_t>(r);
            }
        }
    }
    // column lists (counting sort keeps row-then-position order)
    cs_.assign(n + 1, 0);
    for (std::size_t p = 0; p < nnz; ++p) cs_[ri_[p] + 1]++;
    for (std::size_t v = 0; v < n; ++v) cs_[v + 1] += cs_[v];
    cterm_.resize(nnz);
    {
        std::vector<int64_t> fill(cs_.begin(), cs_.end() - 1);
        for (std::size_t p = 0; p < nnz; ++p) cterm_[fill[ri_[p]]++] = static_cast<int64_t>(p);
    }
    const std::size_t no = static_cast<std::size_t>(in.num_objective_terms);
    oi_.assign(in.objective_index, in.objective_index + no);
    ov_.assign(in.objective_value, in.objective_value + no);
    oalive_.assign(no, 1);
    os_.assign(n + 1, 0);
    for (std::size_t k = 0; k < no; ++k) os_[oi_[k] + 1]++;
    for (std::size_t v = 0; v < n; ++v) os_[v + 1] += os_[v];
    opos_.resize(no);
    {
        std::vector<int64_t> fill(os_.begin(), os_.end() - 1);
        for (std::size_t k = 0; k < no; ++k) opos_[fill[oi_[k]]++] = static_cast<int64_t>(k);
    }
    const std::size_t nq = static_cast<std::size_t>(in.num_quadratic_terms);
    qi_.assign(in.quadratic_index1, in.quadratic_index1 + nq);
    qj_.assign(in.quadratic_index2, in.quadratic_index2 + nq);
    qv_.assign(in.quadratic_value, in.quadratic_value + nq);
    qalive_.assign(nq, 1);
}

// removeZeroCoefficients (presolver.cpp:128-171). Row coefficients never
// change after the first pass, so their sweep runs once.
bool Presolve::remove_zero_coefficients() {
    bool changed = false;
    for (std::size_t k = 0; k < ov_.size(); ++k)
        if (oalive_[k] && std::abs(ov_[k]) <= kEps) {
            oalive_[k] = 0;
            changed = true;
        }
    for (std::size_t k = 0; k < qv_.size(); ++k)
        if (qalive_[k] && std::abs(qv_[k]) <= kEps) {
            qalive_[k] = 0;
            changed = true;
        }
    if (!row_zeros_done_) {
        for (int64_t r = 0; r < m_; ++r) {
            if (!row_alive_[r]) continue;
            for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p)
                if (term_alive_[p] && std::abs(rv_[p]) <= kEps) {
                    term_alive_[p] = 0;
                    row_count_[r]--;
                    changed = true;
                    rows_touched_ = true;
                }
        }
        row_zeros_done_ = true;
    }
    return changed;
}

// detectSimpleInfeasibility (presolver.cpp:512-565).
bool Presolve::detect_simple_infeasibility() const {
    for (int64_t v = 0; v < n_; ++v) {
        if (!var_alive_[v]) continue;
        const double l = lb_[v], u = ub_[v];
        if (std::isnan(l) || std::isnan(u)) return true;
        if (l > u + kEps) return true;
        if (type_[v] == kBinary && (l > 1.0 + kEps || u < -kEps)) return true;
        if (integral(type_[v]) && std::isfinite(l) && std::isfinite(u) &&
            std::ceil(l - kEps) > std::floor(u + kEps))
            return true;
    }
    // rows: every test reads the model only, so pieces of rows run apart and
    // the answer is whether any row fails
    std::atomic<bool> failed{false};
    parallel_for(m_, [&](int64_t begin, int64_t end) {
        bool fail = false;
        for (int64_t r = begin; r < end && !fail; ++r) {
            if (!row_alive_[r]) continue;
            const double l = lo_[r], u = hi_[r];
            if (std::isnan(l) || std::isnan(u) || l > u + kEps) {
                fail = true;
                break;
            }
            if (row_count_[r] == 0) {
                if (l > kEps || u < -kEps) fail = true;
                continue;
            }
            double mn, mx;
            activities(r, mn, mx);
            if ((std::isfinite(l) && std::isfinite(mx) && mx < l - kEps) ||
                (std::isfinite(u) && std::isfinite(mn) && mn > u + kEps))
                fail = true;
        }
        if (fail) failed.store(true, std::memory_order_relaxed);
    });
    return failed.load();
}

// Empty rows (presolver.cpp:1084-1117): highest local index first.
bool Presolve::empty_rows() {
    bool changed = false;
    int64_t k = alive_rows();
    for (int64_t r = m_ - 1; r >= 0; --r) {
        if (!row_alive_[r]) continue;
        --k;  // local index of r: alive rows below it
        if (row_count_[r] != 0) continue;
        if (lo_[r] <= kEps && hi_[r] >= -kEps) {
            log(PDLPGPU_TR_REMOVE_CONSTRAINT, PDLPGPU_PR_EMPTY_ROW, k, -1, r);
            remove_row(r, PDLPGPU_PR_EMPTY_ROW);
            changed = true;
        } else {
            infeasible_ = true;
            log(PDLPGPU_TR_REMOVE_CONSTRAINT, PDLPGPU_PR_EMPTY_ROW_INFEASIBLE, k, -1, r);
            break;
        }
    }
    return changed;
}

// fixVariable (presolver.cpp:177-307). Rows that do not hold the variable are
// not visited: the reference's per-row infeasibility tests cannot fire on them,
// because every alive row passed the same tests when this pass's first
// infeasibility test ran and the empty rows were removed, and a row changes
// here only when it holds the variable being fixed.
bool Presolve::fix_variable(int64_t v, double value, int64_t rank) {
    FixedRecord rec;
    rec.origin = v;
    rec.value = value;
    // 1. objective terms of v, in list order
    auto take_objective = [&](int64_t pos) {
        if (!oalive_[pos]) return;
        const double contribution = ov_[pos] * value;
        rec.linear += contribution;
        offset_ += contribution;
        oalive_[pos] = 0;
    };
    for (int64_t e = os_[v]; e < os_[v + 1]; ++e) take_objective(opos_[e]);
    auto extra = oextra_.find(static_cast<int32_t>(v));
    if (extra != oextra_.end())
        for (int64_t pos : extra->second) take_objective(pos);
    // 2. quadratic terms
    std::map<int32_t, double> linear_contributions;
    for (std::size_t q = 0; q < qv_.size(); ++q) {
        if (!qalive_[q]) continue;
        if (qi_[q] == v && qj_[q] == v) {
            const double diag = qv_[q] * value * value;
            rec.diagonal += diag;
            offset_ += diag;
            qalive_[q] = 0;
        } else if (qi_[q] == v || qj_[q] == v) {
            const int32_t other = qi_[q] == v ? qj_[q] : qi_[q];
            const double cross = qv_[q] * value;
            rec.cross[other] += cross;
            linear_contributions[other] += cross;
            qalive_[q] = 0;
        }
    }
    for (const auto& [other, coeff] : linear_contributions) {
        if (std::abs(coeff) <= kEps) continue;
        // the first alive objective term of `other`, in list order
        int64_t first = -1;
        for (int64_t e = os_[other]; e < os_[other + 1] && first < 0; ++e)
            if (oalive_[opos_[e]]) first = opos_[e];
        auto ex = oextra_.find(other);
        if (first < 0 && ex != oextra_.end())
            for (int64_t pos : ex->second)
                if (oalive_[pos]) {
                    first = pos;
                    break;
                }
        if (first >= 0) {
            ov_[first] += coeff;
        } else {
            oextra_[other].push_back(static_cast<int64_t>(ov_.size()));
            oi_.push_back(other);
            ov_.push_back(coeff);
            oalive_.push_back(1);
        }
    }
    // 3. rows holding v, in row order; each row tested after all its terms of v
    for (int64_t e = cs_[v]; e < cs_[v + 1];) {
        const int64_t r = term_row_[cterm_[e]];
        for (; e < cs_[v + 1] && term_row_[cterm_[e]] == r; ++e) {
            const int64_t p = cterm_[e];
            if (!row_alive_[r] || !term_alive_[p]) continue;
            const double contribution = rv_[p] * value;
            if (std::isfinite(lo_[r])) lo_[r] -= contribution;
            if (std::isfinite(hi_[r])) hi_[r] -= contribution;
            term_alive_[p] = 0;
            row_count_[r]--;
            rows_touched_ = true;
            row_dirty_[r] = 1;
        }
        if (!row_alive_[r]) continue;
        if (lo_[r] > hi_[r] + kEps) {
            infeasible_ = true;
            return false;
        }
        if (row_count_[r] == 0 && (lo_[r] > kEps || hi_[r] < -kEps)) {
            infeasible_ = true;
            return false;
        }
    }
    log(PDLPGPU_TR_FIX_VARIABLE, PDLPGPU_PR_FIXED_BY_BOUNDS, rank, v, -1, value, value,
        rec.linear + rec.diagonal);
    fixed_.push_back(std::move(rec));
    var_alive_[v] = 0;
    return true;
}

// Fixed variables (presolver.cpp:1120-1131): highest local index first.
bool Presolve::fixed_variables() {
    bool changed = false;
    int64_t k = 0;
    for (int64_t v = 0; v < n_; ++v) k += var_alive_[v] ? 1 : 0;
    for (int64_t v = n_ - 1; v >= 0; --v) {
        if (!var_alive_[v]) continue;
        --k;
        if (!approx_equal(lb_[v], ub_[v])) continue;
        if (!fix_variable(v, lb_[v], k)) {
            infeasible_ = true;
            break;
        }
        changed = true;
    }
    return changed;
}

// processSingletonRow (presolver.cpp:387-506).
bool Presolve::singleton_row(int64_t r, int64_t rank) {
    int64_t p = rs_[r];
    while (!term_alive_[p]) ++p;
    const int32_t v = ri_[p];
    const double a = rv_[p];
    if (std::abs(a) <= kEps) return false;
    const double lo = lo_[r], hi = hi_[r];
    double cand_lower = -kInf, cand_upper = kInf;
    if (a > 0.0) {
        if (std::isfinite(lo)) cand_lower = lo / a;
        if (std::isfinite(hi)) cand_upper = hi / a;
    } else {
        if (std::isfinite(hi)) cand_lower = hi / a;
        if (std::isfinite(lo)) cand_upper = lo / a;
    }
    cand_lower = round_lower(cand_lower, type_[v]);
    cand_upper = round_upper(cand_upper, type_[v]);
    if (cand_lower > cand_upper + kEps) {
        infeasible_ = true;
        return false;
    }
    double new_lower = std::max(lb_[v], cand_lower);
    double new_upper = std::min(ub_[v], cand_upper);
    if (type_[v] == kBinary) {
        new_lower = std::max(0.0, new_lower);
        new_upper = std::min(1.0, new_upper);
    }
    if (new_lower > new_upper + kEps) {
        infeasible_ = true;
        return false;
    }
    if (integral(type_[v]) && std::isfinite(new_lower) && std::isfinite(new_upper) &&
        std::ceil(new_lower - kEps) > std::floor(new_upper + kEps)) {
        infeasible_ = true;
        return false;
    }
    const bool lower_changed = !approx_equal(lb_[v], new_lower);
    const bool upper_changed = !approx_equal(ub_[v], new_upper);
    if (lower_changed || upper_changed) bound_moved(v);
    if (lower_changed) {
        log(PDLPGPU_TR_TIGHTEN_LOWER, PDLPGPU_PR_SINGLETON_LOWER, var_rank_[v], v, r, lb_[v],
            new_lower);
        lb_[v] = new_lower;
    }
    if (upper_changed) {
        log(PDLPGPU_TR_TIGHTEN_UPPER, PDLPGPU_PR_SINGLETON_UPPER, var_rank_[v], v, r, ub_[v],
            new_upper);
        ub_[v] = new_upper;
    }
    RemovedRecord rec;
    rec.origin = r;
    rec.lower = lo;
    rec.upper = hi;
    rec.reason = PDLPGPU_PR_SINGLETON_ROW;
    rec.singleton = 1;
    rec.singleton_var = v;
    rec.coefficient = a;
    removed_.push_back(rec);
    log(PDLPGPU_TR_REMOVE_CONSTRAINT, PDLPGPU_PR_SINGLETON_ROW, rank, v, r);
    row_alive_[r] = 0;
    return true;
}

// Singleton rows (presolver.cpp:1134-1143): highest local index first.
bool Presolve::singleton_rows() {
    bool changed = false;
    int64_t k = alive_rows();
    for (int64_t r = m_ - 1; r >= 0; --r) {
        if (!row_alive_[r]) continue;
        --k;
        if (row_count_[r] != 1) continue;
        if (singleton_row(r, k)) changed = true;
        if (infeasible_) break;
    }
    return changed;
}

// tightenBounds (presolver.cpp:571-762). For each term of a row, in order, the
// activity of the row's other terms (all terms of other variables, summed in
// row order) bounds the term's variable; bounds move as the sweep goes, and
// later terms and rows see the moved bounds. Each row's terms are gathered
// once with their contributions to the row's least and greatest activity
// (coefficient times the bound the reference multiplies, the same product)
// and a count of the terms unbounded on each side: a side with an unbounded
// other term is not finite whatever it adds. The finite sums are bracketed
// (below) and formed, in row order, only where the bracket leaves the outcome
// open. A term's entries are refreshed after its own bounds may have moved.
// Rows that name a variable twice, or hold a zero coefficient, take the
// reference's loop as it stands.
bool Presolve::tighten_bounds() {
    bool changed = false;
    std::vector<int32_t> tv;
    std::vector<double> ta, cmn, cmx;
    std::vector<char> imn, imx;
    for (int64_t r = 0; r < m_; ++r) {
        // A sweep of a row is a function of the row's terms and bounds and of
        // its variables' bounds; one that moved nothing, from the same state,
        // moves nothing again, so such rows are passed over.
        if (!row_alive_[r]) continue;
        if (row_quiet_[r] && !row_dirty_[r]) {
            bool fresh = false;
            for (int64_t p = rs_[r]; p < rs_[r + 1] && !fresh; ++p)
                fresh = term_alive_[p] && var_changed_[ri_[p]] > row_swept_[r];
            if (!fresh) continue;
        }
        row_dirty_[r] = 0;
        row_swept_[r] = bound_changes_;
        const int64_t changes_before = bound_changes_;
        tv.clear();
        ta.clear();
        bool plain = !row_repeats_[r];
        for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p) {
            if (!term_alive_[p]) continue;
            tv.push_back(ri_[p]);
            ta.push_back(rv_[p]);
            if (rv_[p] == 0.0) plain = false;
        }
        const std::size_t L = tv.size();
        const double lo = lo_[r], hi = hi_[r];
        cmn.resize(L);
        cmx.resize(L);
        imn.resize(L);
        imx.resize(L);
        int64_t n_min_inf = 0, n_max_inf = 0;
        auto contribute = [&](std::size_t k) {
            const double c = ta[k];
            const double bmin = c > 0.0 ? lb_[tv[k]] : ub_[tv[k]];
            const double bmax = c > 0.0 ? ub_[tv[k]] : lb_[tv[k]];
            imn[k] = !std::isfinite(bmin);
            imx[k] = !std::isfinite(bmax);
            cmn[k] = imn[k] ? 0.0 : c * bmin;
            cmx[k] = imx[k] ? 0.0 : c * bmax;
            n_min_inf += imn[k];
            n_max_inf += imx[k];
        };
        if (plain)
            for (std::size_t k = 0; k < L; ++k) contribute(k);
        // The reference's sum for target t, (((0 + c_0) + c_1) ... + c_{t-1}) +
        // c_{t+1} ... + c_{L-1}, is the running prefix of the terms before t
        // (kept exact as the sweep goes, with each term's entry as it stands
        // after its own turn) continued over the terms after t.
        double prefix_min = 0.0, prefix_max = 0.0;  // exact, terms 0 .. t-1
        // A target's two sums are bracketed instead of formed. The
        // reference's sequential sum S of the other entries lies within
        // gamma_(L-2) * sum |c_k| of their exact sum (recursive summation,
        // round to nearest), and that exact sum is the row's total less the
        // target's own entry, both taken in extended precision; the bracket
        // below is wider than that bound by a factor of more than four.
        // Rounding is monotone, so every candidate the reference can compute
        // from an S in the bracket lies between the candidates computed from
        // the bracket's ends: where the extreme one neither moves a bound nor
        // proves infeasibility, the target does neither, and its sums are not
        // needed. Otherwise they are formed exactly (the exact prefix
        // continued over the later entries). The totals are redone whenever
        // an entry changes. About one target in twenty moves a bound in a
        // pass of the large configurations; the others cost O(1).
        long double total_min = 0.0L, total_max = 0.0L;
        double abs_min = 0.0, abs_max = 0.0;
        auto totals = [&]() {
            total_min = total_max = 0.0L;
            abs_min = abs_max = 0.0;
            for (std::size_t k = 0; k < L; ++k) {
                total_min += cmn[k];
                total_max += cmx[k];
                abs_min += std::abs(cmn[k]);
                abs_max += std::abs(cmx[k]);
            }
        };
        if (plain) totals();
        const double bracket_scale = (static_cast<double>(L) + 8.0) * 0x1p-52;
        auto bracket = [&](long double total, double absolute, double own, double& s1, double& s2) {
            const double est = static_cast<double>(total - static_cast<long double>(own));
            const double b = bracket_scale * (absolute + std::abs(est) + std::abs(own)) + 1e-300;
            s1 = est - 2.0 * b;
            s2 = est + 2.0 * b;
        };
        for (std::size_t t = 0; t < L; ++t) {
            const int32_t v = tv[t];
            const double a = ta[t];
            if (std::abs(a) <= kEps) {
                if (plain) {
                    prefix_min += cmn[t];
                    prefix_max += cmx[t];
                }
                continue;
            }
            double other_min = 0.0, other_max = 0.0;
            bool min_finite = true, max_finite = true;
            bool quiet = false;  // proven to move no bound and prove nothing
            if (plain) {
                min_finite = n_min_inf - imn[t] == 0;
                max_finite = n_max_inf - imx[t] == 0;
                const bool need_min = min_finite && std::isfinite(hi);
                const bool need_max = max_finite && std::isfinite(lo);
                const double l = lb_[v], u = ub_[v];
                const int8_t ty = type_[v];
                quiet = true;
                if (need_max) {  // candidate (lo - S_max) / a, extreme at S_max's low end
                    double s1, s2;
                    bracket(total_max, abs_max, cmx[t], s1, s2);
                    if (a > 0.0) {
                        const double c = round_lower((lo - s1) / a, ty);
                        quiet = std::isfinite(c) && !(c > u + kEps) && !(c > l + kEps);
                    } else {
                        const double c = round_upper((lo - s1) / a, ty);
                        quiet = std::isfinite(c) && !(c < l - kEps) && !(c < u - kEps);
                    }
                }
                if (quiet && need_min) {  // candidate (hi - S_min) / a, extreme at S_min's high end
                    double s1, s2;
                    bracket(total_min, abs_min, cmn[t], s1, s2);
                    if (a > 0.0) {
                        const double c = round_upper((hi - s2) / a, ty);
                        quiet = std::isfinite(c) && !(c < l - kEps) && !(c < u - kEps);
                    } else {
                        const double c = round_lower((hi - s2) / a, ty);
                        quiet = std::isfinite(c) && !(c > u + kEps) && !(c > l + kEps);
                    }
                }
                ++(quiet ? bracketed_ : summed_);
                if (!quiet) {
                    other_min = prefix_min;
                    other_max = prefix_max;
                    for (std::size_t k = t + 1; k < L; ++k) {
                        other_min += cmn[k];
                        other_max += cmx[k];
                    }
                }
            } else {
                for (std::size_t k = 0; k < L; ++k) {
                    const int32_t u = tv[k];
                    if (u == v) continue;
                    const double c = ta[k];
                    if (c > 0.0) {
                        if (std::isfinite(lb_[u])) other_min += c * lb_[u];
                        else min_finite = false;
                        if (std::isfinite(ub_[u])) other_max += c * ub_[u];
                        else max_finite = false;
                    } else if (c < 0.0) {
                        if (std::isfinite(ub_[u])) other_min += c * ub_[u];
                        else min_finite = false;
                        if (std::isfinite(lb_[u])) other_max += c * lb_[u];
                        else max_finite = false;
                    }
                }
            }
            const int8_t type = type_[v];
            const int64_t rank = var_rank_[v];
            const double lb_before = lb_[v], ub_before = ub_[v];
            if (!quiet && std::isfinite(lo) && max_finite) {
                double candidate = (lo - other_max) / a;
                if (a > 0.0) {
                    candidate = round_lower(candidate, type);
                    if (candidate > ub_[v] + kEps) {
                        infeasible_ = true;
                        return false;
                    }
                    if (candidate > lb_[v] + kEps) {
                        log(PDLPGPU_TR_TIGHTEN_LOWER, PDLPGPU_PR_TIGHTENED_LOWER, rank, v, r, lb_[v],
                            candidate);
                        lb_[v] = candidate;
                        changed = true;
                    }
                } else {
                    candidate = round_upper(candidate, type);
                    if (candidate < lb_[v] - kEps) {
                        infeasible_ = true;
                        return false;
                    }
                    if (candidate < ub_[v] - kEps) {
                        log(PDLPGPU_TR_TIGHTEN_UPPER, PDLPGPU_PR_TIGHTENED_UPPER, rank, v, r, ub_[v],
                            candidate);
                        ub_[v] = candidate;
                        changed = true;
                    }
                }
            }
            if (!quiet && std::isfinite(hi) && min_finite) {
                double candidate = (hi - other_min) / a;
                if (a > 0.0) {
                    candidate = round_upper(candidate, type);
                    if (candidate < lb_[v] - kEps) {
                        infeasible_ = true;
                        return false;
                    }
                    if (candidate < ub_[v] - kEps) {
                        log(PDLPGPU_TR_TIGHTEN_UPPER, PDLPGPU_PR_TIGHTENED_UPPER, rank, v, r, ub_[v],
                            candidate);
                        ub_[v] = candidate;
                        changed = true;
                    }
                } else {
                    candidate = round_lower(candidate, type);
                    if (candidate > ub_[v] + kEps) {
                        infeasible_ = true;
                        return false;
                    }
                    if (candidate > lb_[v] + kEps) {
                        log(PDLPGPU_TR_TIGHTEN_LOWER, PDLPGPU_PR_TIGHTENED_LOWER, rank, v, r, lb_[v],
                            candidate);
                        lb_[v] = candidate;
                        changed = true;
                    }
                }
            }
            if (type == kBinary) {
                lb_[v] = std::max(0.0, lb_[v]);
                ub_[v] = std::min(1.0, ub_[v]);
            }
            if (lb_[v] > ub_[v] + kEps) {
                infeasible_ = true;
                return false;
            }
            if (integral(type) && std::isfinite(lb_[v]) && std::isfinite(ub_[v]) &&
                std::ceil(lb_[v] - kEps) > std::floor(ub_[v] + kEps)) {
                infeasible_ = true;
                return false;
            }
            if (std::memcmp(&lb_before, &lb_[v], sizeof(double)) != 0 ||
                std::memcmp(&ub_before, &ub_[v], sizeof(double)) != 0)
                bound_moved(v);
            if (plain) {
                const double old_min = cmn[t], old_max = cmx[t];
                n_min_inf -= imn[t];
                n_max_inf -= imx[t];
                contribute(t);
                if (std::memcmp(&old_min, &cmn[t], sizeof(double)) != 0 ||
                    std::memcmp(&old_max, &cmx[t], sizeof(double)) != 0)
                    totals();
                prefix_min += cmn[t];
                prefix_max += cmx[t];
            }
        }
        row_quiet_[r] = bound_changes_ == changes_before;
    }
    return changed;
}

// removeRedundantConstraints (presolver.cpp:768-836): highest local index first.
bool Presolve::redundant_rows() {
    bool changed = false;
    // no bound moves during this pass: the activities are computed first, in
    // parallel, then the rows are decided in the reference's order
    act_min_.resize(static_cast<std::size_t>(m_));
    act_max_.resize(static_cast<std::size_t>(m_));
    parallel_for(m_, [&](int64_t begin, int64_t end) {
        for (int64_t r = begin; r < end; ++r)
            if (row_alive_[r]) activities(r, act_min_[r], act_max_[r]);
    });
    int64_t k = alive_rows();
    for (int64_t r = m_ - 1; r >= 0; --r) {
        if (!row_alive_[r]) continue;
        --k;
        const double mn = act_min_[r], mx = act_max_[r];
        const double lo = lo_[r], hi = hi_[r];
        if (std::isfinite(lo) && std::isfinite(mx) && mx < lo - kEps) {
            infeasible_ = true;
            return false;
        }
        if (std::isfinite(hi) && std::isfinite(mn) && mn > hi + kEps) {
            infeasible_ = true;
            return false;
        }
        bool redundant = true;
        if (std::isfinite(lo) && (!std::isfinite(mn) || mn < lo - kEps)) redundant = false;
        if (std::isfinite(hi) && (!std::isfinite(mx) || mx > hi + kEps)) redundant = false;
        if (!redundant) continue;
        remove_row(r, PDLPGPU_PR_REDUNDANT);
        log(PDLPGPU_TR_REMOVE_CONSTRAINT, PDLPGPU_PR_REDUNDANT, k, -1, r);
        changed = true;
    }
    return changed;
}

// removeDuplicateAndParallelRows (presolver.cpp:895-981). The reference
// compares every pair (i ascending, j descending from the end) with
// coefficient maps (buildCoefficientMap, presolver.cpp:41-57): only rows with
// the same support can be parallel, so rows are grouped by their exact
// support and each group replays the reference's pair order on its own;
// groups do not interact (a removal changes only pairs of its own group). The
// removals of all groups are then applied in the reference's global order,
// up to the first contradictory pair, with live local indices.
bool Presolve::duplicate_rows() {
    // coefficient maps: support ascending, duplicates summed in term order,
    // |value| <= eps dropped before and after summing
    std::vector<int64_t> ms(static_cast<std::size_t>(m_) + 1, 0);
    std::vector<int32_t> mvar;
    std::vector<double> mval;
    std::vector<std::pair<int32_t, int64_t>> buf;
    for (int64_t r = 0; r < m_; ++r) {
        ms[r] = static_cast<int64_t>(mvar.size());
        if (!row_alive_[r]) continue;
        buf.clear();
        for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p)
            if (term_alive_[p] && std::abs(rv_[p]) > kEps) buf.emplace_back(ri_[p], p);
        std::stable_sort(buf.begin(), buf.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        for (std::size_t k = 0; k < buf.size();) {
            const int32_t v = buf[k].first;
            double s = 0.0;
            for (; k < buf.size() && buf[k].first == v; ++k) s += rv_[buf[k].second];
            if (std::abs(s) > kEps) {
                mvar.push_back(v);
                mval.push_back(s);
            }
        }
    }
    ms[m_] = static_cast<int64_t>(mvar.size());
    // group alive rows with a non-empty map by exact support
    std::vector<std::pair<uint64_t, int64_t>> keyed;
    for (int64_t r = 0; r < m_; ++r) {
        if (!row_alive_[r] || ms[r + 1] == ms[r]) continue;
        uint64_t h = 1469598103934665603ull ^ static_cast<uint64_t>(ms[r + 1] - ms[r]);
        for (int64_t k = ms[r]; k < ms[r + 1]; ++k) {
            h ^= static_cast<uint64_t>(static_cast<uint32_t>(mvar[k])) + 0x9e3779b97f4a7c15ull +
                 (h << 6) + (h >> 2);
            h *= 1099511628211ull;
        }
        keyed.emplace_back(h, r);
    }
    std::sort(keyed.begin(), keyed.end());
    auto same_support = [&](int64_t a, int64_t b) {
        const int64_t la = ms[a + 1] - ms[a], lb = ms[b + 1] - ms[b];
        return la == lb && std::equal(mvar.begin() + ms[a], mvar.begin() + ms[a + 1],
                                      mvar.begin() + ms[b]);
    };
    struct Event {
        int64_t i, j;
        double scale;
    };
    auto before = [](int64_t i1, int64_t j1, int64_t i2, int64_t j2) {
        return i1 < i2 || (i1 == i2 && j1 > j2);
    };
    std::vector<Event> events;
    bool have_trigger = false;
    int64_t trig_i = 0, trig_j = 0;
    std::vector<int64_t> members;
    std::vector<char> gone;
    std::vector<char> used;
    for (std::size_t s = 0; s < keyed.size();) {
        std::size_t e = s;
        while (e < keyed.size() && keyed[e].first == keyed[s].first) ++e;
        // split a hash run into exact-support groups (rows ascending)
        used.assign(e - s, 0);
        for (std::size_t a = s; a < e; ++a) {
            if (used[a - s]) continue;
            members.clear();
            for (std::size_t b = a; b < e; ++b)
                if (!used[b - s] && same_support(keyed[a].second, keyed[b].second)) {
                    used[b - s] = 1;
                    members.push_back(keyed[b].second);
                }
            if (members.size() < 2) continue;
            std::sort(members.begin(), members.end());
            const std::size_t g = members.size();
            gone.assign(g, 0);
            bool stop = false;
            for (std::size_t ii = 0; ii < g && !stop; ++ii) {
                if (gone[ii]) continue;
                const int64_t i = members[ii];
                const double* va = mval.data() + ms[i];
                const int64_t len = ms[i + 1] - ms[i];
                for (std::size_t jj = g; jj-- > ii + 1;) {
                    if (gone[jj]) continue;
                    const int64_t j = members[jj];
                    const double* vb = mval.data() + ms[j];
                    // constraintsParallel (presolver.cpp:862-893)
                    const double first = vb[0] / va[0];
                    bool parallel = true;
                    for (int64_t k = 1; k < len && parallel; ++k)
                        if (!approx_equal(vb[k] / va[k], first)) parallel = false;
                    if (!parallel || !(std::abs(first) > kEps)) continue;
                    const double scale = first;
                    double norm_lower = -kInf, norm_upper = kInf;
                    if (scale > 0.0) {
                        if (std::isfinite(lo_[j])) norm_lower = lo_[j] / scale;
                        if (std::isfinite(hi_[j])) norm_upper = hi_[j] / scale;
                    } else {
                        if (std::isfinite(hi_[j])) norm_lower = hi_[j] / scale;
                        if (std::isfinite(lo_[j])) norm_upper = lo_[j] / scale;
                    }
                    const double eff_lower = std::max(lo_[i], norm_lower);
                    const double eff_upper = std::min(hi_[i], norm_upper);
                    if (eff_lower > eff_upper + kEps) {
                        if (!have_trigger || before(i, j, trig_i, trig_j)) {
                            have_trigger = true;
                            trig_i = i;
                            trig_j = j;
                        }
                        stop = true;
                        break;
                    }
                    if (approx_equal(lo_[i], norm_lower) && approx_equal(hi_[i], norm_upper)) {
                        events.push_back({i, j, scale});
                        gone[jj] = 1;
                    }
                }
            }
        }
        s = e;
    }
    std::sort(events.begin(), events.end(),
              [&](const Event& x, const Event& y) { return before(x.i, x.j, y.i, y.j); });
    bool changed = false;
    Fenwick alive(m_);
    if (!events.empty())
        for (int64_t r = 0; r < m_; ++r)
            if (row_alive_[r]) alive.add(r, 1);
    for (const Event& ev : events) {
        if (have_trigger && !before(ev.i, ev.j, trig_i, trig_j)) break;
        RemovedRecord rec;
        rec.origin = ev.j;
        rec.lower = lo_[ev.j];
        rec.upper = hi_[ev.j];
        rec.reason = PDLPGPU_PR_DUPLICATE;
        rec.duplicate = 1;
        rec.duplicate_of = ev.i;
        rec.scale = ev.scale;
        removed_.push_back(rec);
        log(PDLPGPU_TR_REMOVE_CONSTRAINT, PDLPGPU_PR_DUPLICATE, alive.below(ev.j), -1, ev.j);
        row_alive_[ev.j] = 0;
        alive.add(ev.j, -1);
        changed = true;
    }
    if (have_trigger) infeasible_ = true;
    return changed;
}

// Presolver::run (presolver.cpp:1045-1155).
void Presolve::run() {
    if (detect_simple_infeasibility()) {
        infeasible_ = true;
        return;  // the reference returns before it fills the index maps
    }
    constexpr int kMaxPasses = 50;
    bool fixed_point = false;
    // PDLPGPU_PRESOLVE_TRACE=1: one line per pass on stderr with the time
    // of each step (ms) and the log's length after it.
    const bool trace = std::getenv("PDLPGPU_PRESOLVE_TRACE") != nullptr;
    using clock = std::chrono::steady_clock;
    clock::time_point t0 = clock::now();
    auto lap = [&](const char* step) {
        if (!trace) return;
        const clock::time_point t1 = clock::now();
        std::fprintf(stderr, " %s %.2f/%zu", step,
                     std::chrono::duration<double, std::milli>(t1 - t0).count(),
                     logbuf_.tr_type_v.size());
        t0 = t1;
    };
    for (int pass = 0; pass < kMaxPasses; ++pass) {
        if (infeasible_) break;
        if (trace) std::fprintf(stderr, "presolve pass %d:", pass);
        bool changed = false;
        if (remove_zero_coefficients()) changed = true;
        if (detect_simple_infeasibility()) {
            infeasible_ = true;
            break;
        }
        lap("zeros+test");
        if (empty_rows()) changed = true;
        if (infeasible_) break;
        if (fixed_variables()) changed = true;
        if (infeasible_) break;
        rank_variables();
        if (singleton_rows()) changed = true;
        if (infeasible_) break;
        lap("empty+fixed+singleton");
        if (tighten_bounds()) changed = true;
        if (infeasible_) break;
        lap("tighten");
        if (redundant_rows()) changed = true;
        if (infeasible_) break;
        lap("redundant");
        // The duplicate pass examined every pair of the rows alive now when it
        // last ran and acted on none; the pairs' outcome depends on the rows'
        // terms and bounds only, so unless one of those changed since, it
        // would act on none again.
        if (rows_touched_) {
            rows_touched_ = false;
            if (duplicate_rows()) changed = true;
            if (infeasible_) break;
        }
        lap("duplicate");
        if (trace)
            std::fprintf(stderr, " targets bracketed/summed %lld/%lld\n",
                         static_cast<long long>(bracketed_),
                         static_cast<long long>(summed_));
        if (!changed) {
            fixed_point = true;
            break;
        }
    }
    if (!infeasible_ && !fixed_point) converged_ = false;
    if (!infeasible_ && detect_simple_infeasibility()) infeasible_ = true;
    has_maps_ = true;
}

void Presolve::emit(Out& o) {
    std::vector<int32_t> rank(static_cast<std::size_t>(n_), -1);
    for (int64_t v = 0; v < n_; ++v)
        if (var_alive_[v]) {
            rank[v] = static_cast<int32_t>(o.var_origin.size());
            o.var_origin.push_back(v);
            o.vlo.push_back(lb_[v]);
            o.vhi.push_back(ub_[v]);
        }
    o.rs.push_back(0);
    for (int64_t r = 0; r < m_; ++r) {
        if (!row_alive_[r]) continue;
        o.con_origin.push_back(r);
        o.rlo.push_back(lo_[r]);
        o.rhi.push_back(hi_[r]);
        for (int64_t p = rs_[r]; p < rs_[r + 1]; ++p)
            if (term_alive_[p]) {
                o.ri.push_back(rank[ri_[p]]);
                o.rv.push_back(rv_[p]);
            }
        o.rs.push_back(static_cast<int64_t>(o.ri.size()));
    }
    for (std::size_t k = 0; k < ov_.size(); ++k)
        if (oalive_[k]) {
            o.oi.push_back(rank[oi_[k]]);
            o.ov.push_back(ov_[k]);
        }
    for (std::size_t k = 0; k < qv_.size(); ++k)
        if (qalive_[k]) {
            o.qi.push_back(rank[qi_[k]]);
            o.qj.push_back(rank[qj_[k]]);
            o.qv.push_back(qv_[k]);
        }
    // the log moves into the result (emit is the last use of this object)
    Out& L = logbuf_;
    o.tr_type_v = std::move(L.tr_type_v);
    o.tr_reason_v = std::move(L.tr_reason_v);
    o.tr_index_v = std::move(L.tr_index_v);
    o.tr_var_v = std::move(L.tr_var_v);
    o.tr_con_v = std::move(L.tr_con_v);
    o.tr_old_v = std::move(L.tr_old_v);
    o.tr_new_v = std::move(L.tr_new_v);
    o.tr_off_v = std::move(L.tr_off_v);
    o.fx_cross_start.push_back(0);
    for (const FixedRecord& f : fixed_) {
        o.fx_origin.push_back(f.origin);
        o.fx_value.push_back(f.value);
        o.fx_linear.push_back(f.linear);
        o.fx_diag.push_back(f.diagonal);
        for (const auto& [other, c] : f.cross) {
            o.fx_cross_var.push_back(other);
            o.fx_cross_val.push_back(c);
        }
        o.fx_cross_start.push_back(static_cast<int64_t>(o.fx_cross_var.size()));
    }
    for (const RemovedRecord& rr : removed_) {
        o.rm_origin.push_back(rr.origin);
        o.rm_lo.push_back(rr.lower);
        o.rm_hi.push_back(rr.upper);
        o.rm_reason.push_back(rr.reason);
        o.rm_single.push_back(rr.singleton);
        o.rm_svar.push_back(rr.singleton_var);
        o.rm_coef.push_back(rr.coefficient);
        o.rm_dup.push_back(rr.duplicate);
        o.rm_dup_of.push_back(rr.duplicate_of);
        o.rm_scale.push_back(rr.scale);
    }

    o.infeasible = infeasible_ ? 1 : 0;
    o.converged = converged_ ? 1 : 0;
    o.has_maps = has_maps_ ? 1 : 0;
    o.original_variables = n_;
    o.original_constraints = m_;
    o.presolved_variables = static_cast<int64_t>(o.var_origin.size());
    o.presolved_constraints = static_cast<int64_t>(o.con_origin.size());
    o.initial_objective_offset = initial_offset_;
    o.presolved_objective_offset = offset_;
    o.variable_origin = o.var_origin.data();
    o.var_lower = o.vlo.data();
    o.var_upper = o.vhi.data();
    o.constraint_origin = o.con_origin.data();
    o.row_lower = o.rlo.data();
    o.row_upper = o.rhi.data();
    o.row_start = o.rs.data();
    o.row_index = o.ri.data();
    o.row_value = o.rv.data();
    o.num_objective_terms = static_cast<int64_t>(o.oi.size());
    o.objective_index = o.oi.data();
    o.objective_value = o.ov.data();
    o.num_quadratic_terms = static_cast<int64_t>(o.qv.size());
    o.quadratic_index1 = o.qi.data();
    o.quadratic_index2 = o.qj.data();
    o.quadratic_value = o.qv.data();
    o.num_transformations = static_cast<int64_t>(o.tr_type_v.size());
    o.tr_type = o.tr_type_v.data();
    o.tr_reason = o.tr_reason_v.data();
    o.tr_index = o.tr_index_v.data();
    o.tr_variable = o.tr_var_v.data();
    o.tr_constraint = o.tr_con_v.data();
    o.tr_old_value = o.tr_old_v.data();
    o.tr_new_value = o.tr_new_v.data();
    o.tr_offset_change = o.tr_off_v.data();
    o.num_fixed = static_cast<int64_t>(o.fx_origin.size());
    o.fixed_origin = o.fx_origin.data();
    o.fixed_value = o.fx_value.data();
    o.fixed_linear = o.fx_linear.data();
    o.fixed_quadratic_diagonal = o.fx_diag.data();
    o.fixed_cross_start = o.fx_cross_start.data();
    o.fixed_cross_variable = o.fx_cross_var.data();
    o.fixed_cross_value = o.fx_cross_val.data();
    o.num_removed = static_cast<int64_t>(o.rm_origin.size());
    o.removed_origin = o.rm_origin.data();
    o.removed_lower = o.rm_lo.data();
    o.removed_upper = o.rm_hi.data();
    o.removed_reason = o.rm_reason.data();
    o.removed_singleton = o.rm_single.data();
    o.removed_singleton_variable = o.rm_svar.data();
    o.removed_singleton_coefficient = o.rm_coef.data();
    o.removed_duplicate = o.rm_dup.data();
    o.removed_duplicate_of = o.rm_dup_of.data();
    o.removed_scale = o.rm_scale.data();
}

const char* check(const pdlpgpu_presolve_model& m) {
    if (m.num_variables < 0 || m.num_constraints < 0 || m.num_objective_terms < 0 ||
        m.num_quadratic_terms < 0)
        return "presolve: negative count";
    if (m.num_variables > INT32_MAX) return "presolve: more variables than 32-bit indices hold";
    if (m.num_variables > 0 && (!m.var_lower || !m.var_upper || !m.var_type))
        return "presolve: NULL variable array";
    if (!m.row_start) return "presolve: NULL row_start";
    if (m.num_constraints > 0 && (!m.row_lower || !m.row_upper))
        return "presolve: NULL row bound array";
    if (m.row_start[0] != 0) return "presolve: row_start[0] must be 0";
    for (int64_t r = 0; r < m.num_constraints; ++r)
        if (m.row_start[r + 1] < m.row_start[r]) return "presolve: row_start decreases";
    const int64_t nnz = m.row_start[m.num_constraints];
    if (nnz > 0 && (!m.row_index || !m.row_value)) return "presolve: NULL row term array";
    for (int64_t p = 0; p < nnz; ++p) {
        if (m.row_index[p] < 0 || m.row_index[p] >= m.num_variables)
            return "presolve: a constraint term names no variable";
        if (!std::isfinite(m.row_value[p])) return "presolve: non-finite constraint coefficient";
    }
    if (m.num_objective_terms > 0 && (!m.objective_index || !m.objective_value))
        return "presolve: NULL objective array";
    for (int64_t k = 0; k < m.num_objective_terms; ++k) {
        if (m.objective_index[k] < 0 || m.objective_index[k] >= m.num_variables)
            return "presolve: an objective term names no variable";
        if (!std::isfinite(m.objective_value[k])) return "presolve: non-finite objective coefficient";
    }
    if (m.num_quadratic_terms > 0 &&
        (!m.quadratic_index1 || !m.quadratic_index2 || !m.quadratic_value))
        return "presolve: NULL quadratic array";
    for (int64_t k = 0; k < m.num_quadratic_terms; ++k) {
        if (m.quadratic_index1[k] < 0 || m.quadratic_index1[k] >= m.num_variables ||
            m.quadratic_index2[k] < 0 || m.quadratic_index2[k] >= m.num_variables)
            return "presolve: a quadratic term names no variable";
        if (!std::isfinite(m.quadratic_value[k])) return "presolve: non-finite quadratic coefficient";
    }
    for (int64_t v = 0; v < m.num_variables; ++v)
        if (m.var_type[v] < 0 || m.var_type[v] > 2) return "presolve: unknown variable type";
    return nullptr;
}

}  // namespace

extern "C" int32_t pdlpgpu_presolve(const pdlpgpu_presolve_model* model,
                                    pdlpgpu_presolve_result** result) {
    if (result == nullptr || model == nullptr) {
        pdlpgpu_internal_set_error("presolve: NULL argument");
        return -1;
    }
    *result = nullptr;
    if (const char* why = check(*model)) {
        pdlpgpu_internal_set_error(why);
        return -1;
    }
    try {
        Presolve p(*model);
        p.run();
        Out* out = new Out();
        p.emit(*out);
        *result = out;
        return 0;
    } catch (const std::bad_alloc&) {
        pdlpgpu_internal_set_error("presolve: out of host memory");
        return -1;
    } catch (const std::exception& e) {
        pdlpgpu_internal_set_error((std::string("presolve: ") + e.what()).c_str());
        return -1;
    } catch (...) {
        pdlpgpu_internal_set_error("presolve: unknown error");
        return -1;
    }
}

extern "C" void pdlpgpu_presolve_free(pdlpgpu_presolve_result* result) {
    delete static_cast<Out*>(result);
}

extern "C" const char* pdlpgpu_presolve_reason_string(int32_t reason) {
    switch (reason) {  // the reference's reason strings, presolver.cpp
        case PDLPGPU_PR_FIXED_BY_BOUNDS: return "Variable is fixed by equal lower and upper bounds";
        case PDLPGPU_PR_SINGLETON_LOWER: return "Singleton row tightened variable lower bound";
        case PDLPGPU_PR_SINGLETON_UPPER: return "Singleton row tightened variable upper bound";
        case PDLPGPU_PR_SINGLETON_ROW: return "Singleton row converted to variable bounds";
        case PDLPGPU_PR_TIGHTENED_LOWER: return "Constraint tightened variable lower bound";
        case PDLPGPU_PR_TIGHTENED_UPPER: return "Constraint tightened variable upper bound";
        case PDLPGPU_PR_REDUNDANT: return "Constraint is redundant given variable bounds";
        case PDLPGPU_PR_DUPLICATE: return "Duplicate/parallel equivalent constraint removed";
        case PDLPGPU_PR_EMPTY_ROW: return "Empty row is redundant";
        case PDLPGPU_PR_EMPTY_ROW_INFEASIBLE: return "Empty row makes model infeasible";
        default: return "";
    }
}

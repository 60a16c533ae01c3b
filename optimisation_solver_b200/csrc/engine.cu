// engine.cu -- host side of the device PDLP engine: validation, layout,
// device arena, setup kernels, the graph-captured iteration loop and result
// extraction. Restates the control of PdlpSolver::solve
// (pdlp_engine/src/pdlp_solver.cpp:116-548) for a batch of instances whose
// per-iteration decisions all happen on the device.
#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

namespace pdlpgpu {

const char* message_text(int32_t id) {
    switch (id) {
        case kMsgInitialOptimal: return "Initial point satisfies the requested tolerances";
        case kMsgNonFinite: return "PDHG generated a non-finite iterate";
        case kMsgLinesearch: return "Adaptive linesearch failed to accept a step";
        case kMsgInfeasible: return "Primal infeasible: Farkas ray found";
        case kMsgUnbounded: return "Unbounded: improving ray found";
        case kMsgOptimal: return "Primal, dual, and gap tolerances satisfied";
        case kMsgPolishOptimal: return "Tolerances satisfied after refinement polishing";
        case kMsgIterationLimit: return "Iteration limit reached";
        case kMsgTimeLimit: return "Time limit reached";
        default: return "";
    }
}

namespace {

struct ArenaPlan {
    struct Req { void** ptr; size_t bytes; };
    std::vector<Req> reqs;
    template <class T>
    void add(T*& p, int64_t count) {
        reqs.push_back(Req{reinterpret_cast<void**>(&p), static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(T)});
    }
    template <class T>
    void add(const T*& p, int64_t count) {
        reqs.push_back(Req{reinterpret_cast<void**>(const_cast<T**>(&p)), static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(T)});
    }
    size_t total() const {
        size_t t = 0;
        for (const Req& r : reqs) t += (r.bytes + 255) & ~size_t(255);
        return t;
    }
    void assign(char* base) const {
        size_t off = 0;
        for (const Req& r : reqs) {
            *r.ptr = base + off;
            off += (r.bytes + 255) & ~size_t(255);
        }
    }
};

double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }

// TerminationChecker's normalisers (termination.cpp:14-62), in the
// reference's summation order.
void normalisers(const pdlpgpu_lp& lp, double& pnorm, double& dnorm) {
    double sum = 0.0;
    for (int32_t i = 0; i < lp.num_rows; ++i) {
        const double l = lp.row_lower[i], u = lp.row_upper[i];
        if (std::isfinite(l)) sum += l * l;
        if (std::isfinite(u) && u != l) sum += u * u;
    }
    pnorm = 1.0 + std::sqrt(sum);
    double cs = 0.0;
    for (int32_t j = 0; j < lp.num_cols; ++j) cs += lp.objective[j] * lp.objective[j];
    dnorm = 1.0 + std::sqrt(cs);
}

template <class T>
void fill_value(std::vector<T>& v, size_t n, T x) { v.assign(n, x); }

// f(k) for k in [0, count), spread over the host's hardware threads.
template <class F>
void parallel_for(int count, F f) {
    const int threads = std::min<int>(count, std::max(1u, std::thread::hardware_concurrency()));
    if (threads <= 1) {
        for (int k = 0; k < count; ++k) f(k);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] { for (int k = t; k < count; k += threads) f(k); });
    for (auto& th : pool) th.join();
}

// f(k) for k in [0, count), each k to the next free host thread.
template <class F>
void parallel_dynamic(int count, F f) {
    const int threads = std::min<int>(count, std::max(1u, std::thread::hardware_concurrency()));
    if (threads <= 1) {
        for (int k = 0; k < count; ++k) f(k);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (int k = next++; k < count; k = next++) f(k);
        });
    for (auto& th : pool) th.join();
}

}  // namespace

Engine::Engine(int device) : device_(device) {}

void Engine::mark(const char* phase) {
    static const bool on = [] {
        const char* v = std::getenv("PDLPGPU_TRACE");
        return v != nullptr && v[0] == '1';
    }();
    if (!on) return;
    trace_.emplace_back(phase, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count());
}

namespace {
constexpr size_t kPinnedChunk = size_t(64) << 20;   // bytes per staging buffer
constexpr size_t kPinnedDirect = size_t(4) << 20;   // smaller uploads go as they are
constexpr size_t kCopyJob = size_t(2) << 20;        // host memcpy piece per thread
}  // namespace

bool Engine::ensure_pinned() {
    for (int b = 0; b < 2; ++b) {
        if (pinned_[b] == nullptr &&
            !check(cudaHostAlloc(reinterpret_cast<void**>(&pinned_[b]), kPinnedChunk, cudaHostAllocDefault), "cudaHostAlloc"))
            return false;
        if (pinned_done_[b] == nullptr &&
            !check(cudaEventCreateWithFlags(&pinned_done_[b], cudaEventDisableTiming), "cudaEventCreate"))
            return false;
    }
    return true;
}

// The reverse path: the DMA of the next chunk into one pinned buffer runs
// while all host threads copy the previous chunk out of the other.
bool Engine::download(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return true;
    if (bytes < kPinnedDirect)
        return check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_), "download") &&
               check(cudaStreamSynchronize(stream_), "download");
    if (!ensure_pinned()) return false;
    const size_t chunks = (bytes + kPinnedChunk - 1) / kPinnedChunk;
    auto enqueue = [&](size_t c) {
        const size_t off = c * kPinnedChunk, n = std::min(kPinnedChunk, bytes - off);
        return check(cudaMemcpyAsync(pinned_[c & 1], static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, stream_), "download") &&
               check(cudaEventRecord(pinned_done_[c & 1], stream_), "download");
    };
    if (!enqueue(0)) return false;
    for (size_t c = 0; c < chunks; ++c) {
        if (c + 1 < chunks && !enqueue(c + 1)) return false;
        if (!check(cudaEventSynchronize(pinned_done_[c & 1]), "download")) return false;
        const size_t off = c * kPinnedChunk, n = std::min(kPinnedChunk, bytes - off);
        const int jobs = static_cast<int>((n + kCopyJob - 1) / kCopyJob);
        const char* from = pinned_[c & 1];
        char* to = static_cast<char*>(dst) + off;
        parallel_for(jobs, [&](int j) {
            const size_t a = static_cast<size_t>(j) * kCopyJob;
            std::memcpy(to + a, from + a, std::min(kCopyJob, n - a));
        });
    }
    return true;
}

// A copy from pageable memory is staged by the driver through its own small
// pinned buffers, one thread, and returns only when it is done: for the
// gigabytes of a large batch's matrices that runs at a fraction of the host
// link. Large uploads here go through two 64 MiB pinned buffers instead: all
// host threads fill one while the other's DMA is in flight.
bool Engine::upload(void* dst, const std::vector<HostPiece>& pieces) {
    size_t total = 0;
    for (const HostPiece& q : pieces) total += q.bytes;
    if (total == 0) return true;
    char* out = static_cast<char*>(dst);
    if (total < kPinnedDirect) {
        for (const HostPiece& q : pieces) {
            if (q.bytes && !check(cudaMemcpyAsync(out, q.src, q.bytes, cudaMemcpyHostToDevice, stream_), "upload"))
                return false;
            out += q.bytes;
        }
        return true;
    }
    if (!ensure_pinned()) return false;
    struct Job {
        size_t at;          // offset in the staging buffer
        const char* src;
        size_t bytes;
    };
    std::vector<Job> jobs;
    size_t piece = 0, in_piece = 0;   // read position
    for (int chunk = 0; piece < pieces.size(); ++chunk) {
        const int b = chunk & 1;
        // Jobs of this chunk: up to kPinnedChunk bytes of the pieces, cut
        // into at most kCopyJob bytes each.
        jobs.clear();
        size_t fill = 0;
        while (fill < kPinnedChunk && piece < pieces.size()) {
            const HostPiece& q = pieces[piece];
            const size_t n = std::min({q.bytes - in_piece, kPinnedChunk - fill, kCopyJob});
            if (n > 0) jobs.push_back({fill, static_cast<const char*>(q.src) + in_piece, n});
            fill += n;
            in_piece += n;
            if (in_piece == q.bytes) {
                ++piece;
                in_piece = 0;
            }
        }
        if (fill == 0) break;
        // The buffer's previous copy must have finished before it is refilled.
        if (!check(cudaEventSynchronize(pinned_done_[b]), "upload")) return false;
        char* stage = pinned_[b];
        parallel_for(static_cast<int>(jobs.size()),
                     [&](int j) { std::memcpy(stage + jobs[j].at, jobs[j].src, jobs[j].bytes); });
        if (!check(cudaMemcpyAsync(out, stage, fill, cudaMemcpyHostToDevice, stream_), "upload") ||
            !check(cudaEventRecord(pinned_done_[b], stream_), "upload"))
            return false;
        out += fill;
    }
    return true;
}

Engine::~Engine() {
    for (cudaEvent_t e : tev_)
        if (e) cudaEventDestroy(e);
    if (caller_done_) cudaEventDestroy(caller_done_);
    for (void* q : extra_) cudaFree(q);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (graph64_) cudaGraphExecDestroy(graph64_);
    if (arena_) cudaFree(arena_);
    if (h_active_) cudaFreeHost(h_active_);
    for (int b = 0; b < 2; ++b) {
        if (pinned_done_[b]) cudaEventDestroy(pinned_done_[b]);
        if (pinned_[b]) cudaFreeHost(pinned_[b]);
    }
    if (stream_) cudaStreamDestroy(stream_);
}

bool Engine::check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    if (error_.empty()) error_ = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

template <class V>
void Engine::to_internal_cols(const V* src, std::vector<V>& dst, int b) const {
    const MatrixLayout& L = layouts_[spec_.shared_matrix ? 0 : b];
    dst.resize(L.col_perm.size());
    for (size_t c = 0; c < L.col_perm.size(); ++c) dst[c] = src[L.col_perm[c]];
}

template <class V>
void Engine::to_internal_rows(const V* src, std::vector<V>& dst, int b) const {
    const MatrixLayout& L = layouts_[spec_.shared_matrix ? 0 : b];
    dst.resize(L.row_perm.size());
    for (size_t r = 0; r < L.row_perm.size(); ++r) dst[r] = src[L.row_perm[r]];
}

bool Engine::prepare(const SolveSpec& spec) {
    t0_ = std::chrono::steady_clock::now();
    spec_ = spec;
    const int nspec = static_cast<int>(spec.lps.size());
    invalid_.assign(static_cast<size_t>(nspec), std::string());
    device_of_.assign(static_cast<size_t>(nspec), -1);
    const pdlpgpu_options& o = spec.opt;
    mixed_ = spec.ext.precision == PDLPGPU_PRECISION_MIXED;

    // --- host validation (pdlp_solver.cpp:121-134) -----------------------
    std::vector<HostCsr> csr(static_cast<size_t>(spec.shared_matrix ? 1 : nspec));
    std::string shared_error;
    if (spec.shared_matrix && nspec > 0) shared_error = canonicalize(*spec.lps[0], csr[0]);
    parallel_for(nspec, [&](int i) {
        const pdlpgpu_lp& lp = *spec.lps[i];
        std::string err;
        if (spec.shared_matrix) {
            err = shared_error;
            if (err.empty() && (lp.num_rows != spec.lps[0]->num_rows || lp.num_cols != spec.lps[0]->num_cols))
                err = "CompiledLp row vector dimensions do not match A";
        } else {
            err = canonicalize(lp, csr[i]);
        }
        if (err.empty()) err = validate_vectors(lp);
        invalid_[i] = err;
    });
    const bool bad_options = o.iteration_limit < 0 || o.termination_check_frequency <= 0 ||
                             o.primal_tolerance < 0.0 || o.dual_tolerance < 0.0 ||
                             o.gap_tolerance < 0.0 || o.initial_step_safety <= 0.0 ||
                             o.minimum_primal_weight <= 0.0 ||
                             o.maximum_primal_weight < o.minimum_primal_weight;
    for (int i = 0; i < nspec; ++i) {
        if (invalid_[i].empty() && bad_options) invalid_[i] = "Invalid PDLP options";
        if (invalid_[i].empty()) device_of_[i] = count_++;
    }
    if (count_ == 0) {
        setup_ok_ = true;
        return true;
    }
    mark("validate");

    // --- device and tuning ------------------------------------------------
    if (!check(cudaSetDevice(device_), "cudaSetDevice")) return false;
    cudaDeviceProp prop;
    if (!check(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties")) return false;
    sms_ = prop.multiProcessorCount;
    if (!check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    for (cudaEvent_t& e : tev_)
        if (e == nullptr && !check(cudaEventCreate(&e), "cudaEventCreate")) return false;

    // Layouts: one per device instance, or one shared.
    std::vector<int> spec_of(static_cast<size_t>(count_));
    for (int i = 0; i < nspec; ++i) if (device_of_[i] >= 0) spec_of[device_of_[i]] = i;
    const int nlayouts = spec.shared_matrix ? 1 : count_;
    {
        int64_t nnz = 0, lines = 0, clines = 0;
        for (int k = 0; k < nlayouts; ++k) {
            const HostCsr& a = csr[spec.shared_matrix ? 0 : spec_of[k]];
            nnz += a.nnz();
            lines += a.rows;
            clines += a.cols;
        }
        HostCsr agg_a, agg_at;   // only the counts matter for the heuristic
        agg_a.rows = static_cast<int32_t>(std::min<int64_t>(lines, INT32_MAX));
        agg_at.rows = static_cast<int32_t>(std::min<int64_t>(clines, INT32_MAX));
        agg_a.value.resize(0);
        tuning_ = Tuning();
        const double mean_a = lines ? static_cast<double>(nnz) / lines : 0.0;
        const double mean_at = clines ? static_cast<double>(nnz) / clines : 0.0;
        const double mean = std::min(mean_a, mean_at);
        // Wider lane loads pay only when lines are long enough that rounding
        // each slice's steps up to the width adds little padding.
        if (mixed_) tuning_.vector_width = mean >= 24.0 ? 4 : (mean >= 12.0 ? 2 : 1);
        else tuning_.vector_width = mean >= 16.0 ? 2 : 1;
        if (spec.ext.lane_elements > 0) tuning_.lane_elements = spec.ext.lane_elements;
        if (spec.ext.vector_width == 1 || spec.ext.vector_width == 2 || spec.ext.vector_width == 4)
            tuning_.vector_width = spec.ext.vector_width;
    }
    layouts_.resize(static_cast<size_t>(nlayouts));
    {
        // Largest matrices first, each to the next free thread.
        std::vector<int> order(static_cast<size_t>(nlayouts));
        std::iota(order.begin(), order.end(), 0);
        auto nnz_of = [&](int k) { return csr[spec.shared_matrix ? 0 : spec_of[k]].nnz(); };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return nnz_of(x) > nnz_of(y); });
        parallel_dynamic(nlayouts, [&](int q) {
            const int k = order[static_cast<size_t>(q)];
            const HostCsr& a = csr[spec.shared_matrix ? 0 : spec_of[k]];
            layouts_[k] = build_layout(a, tuning_);
        });
    }
    if (!csr.empty()) csr0_ = std::move(csr[spec.shared_matrix ? 0 : spec_of[0]]);
    csr.clear();
    mark("layouts");

    // --- spaces, slices and CTA maps --------------------------------------
    info_.resize(static_cast<size_t>(count_));
    rows_total_ = cols_total_ = 0;
    a_slots_ = at_slots_ = 0;
    a_slices_ = at_slices_ = 0;
    for (int k = 0; k < nlayouts; ++k) {
        a_slots_ += layouts_[k].a.slots();
        at_slots_ += layouts_[k].at.slots();
        a_slices_ += static_cast<int32_t>(layouts_[k].a.slices.size());
        at_slices_ += static_cast<int32_t>(layouts_[k].at.slices.size());
    }
    int64_t target_a = cta_target_slots(spec.shared_matrix ? a_slots_ * count_ : a_slots_, sms_);
    int64_t target_at = cta_target_slots(spec.shared_matrix ? at_slots_ * count_ : at_slots_, sms_);
    if (spec.ext.cta_slots > 0) target_a = target_at = spec.ext.cta_slots;
    a_ctas_.clear();
    at_ctas_.clear();
    vec_.clear();
    int64_t a_data = 0, at_data = 0;
    int32_t a_sl = 0, at_sl = 0;
    for (int b = 0; b < count_; ++b) {
        const MatrixLayout& L = layouts_[spec.shared_matrix ? 0 : b];
        InstanceInfo& inf = info_[b];
        inf.m = L.m;
        inf.n = L.n;
        inf.row_off = rows_total_;
        inf.col_off = cols_total_;
        rows_total_ += L.m;
        cols_total_ += L.n;
        const bool own = !spec.shared_matrix || b == 0;
        inf.a_data_base = spec.shared_matrix ? 0 : a_data;
        inf.at_data_base = spec.shared_matrix ? 0 : at_data;
        inf.a_slice_base = spec.shared_matrix ? 0 : a_sl;
        inf.at_slice_base = spec.shared_matrix ? 0 : at_sl;
        inf.a_len_base = spec.shared_matrix ? 0 : inf.row_off;
        inf.at_len_base = spec.shared_matrix ? 0 : inf.col_off;
        if (own && !spec.shared_matrix) {
            a_data += L.a.slots();
            at_data += L.at.slots();
            a_sl += static_cast<int32_t>(L.a.slices.size());
            at_sl += static_cast<int32_t>(L.at.slices.size());
        }
        inf.a_cta_begin = static_cast<int32_t>(a_ctas_.size());
        append_cta_map(L.a, b, inf.a_slice_base, target_a, a_ctas_);
        inf.a_cta_end = static_cast<int32_t>(a_ctas_.size());
        inf.at_cta_begin = static_cast<int32_t>(at_ctas_.size());
        append_cta_map(L.at, b, inf.at_slice_base, target_at, at_ctas_);
        inf.at_cta_end = static_cast<int32_t>(at_ctas_.size());
        inf.vec_cta_begin = static_cast<int32_t>(vec_.size());
        append_vec_map(b, L.m, L.n, vec_);
        inf.vec_cta_end = static_cast<int32_t>(vec_.size());
    }
    first_a_ctas_ = info_[0].a_cta_end - info_[0].a_cta_begin;
    first_at_ctas_ = info_[0].at_cta_end - info_[0].at_cta_begin;
    first_vec_ = info_[0].vec_cta_end - info_[0].vec_cta_begin;

    // --- device arena ------------------------------------------------------
    const int64_t R = rows_total_, N = cols_total_;
    const int64_t slots = a_slots_ + at_slots_;
    const int64_t lens = spec.shared_matrix ? (layouts_[0].m + layouts_[0].n) : (R + N);
    bool any_warm = false;
    for (const auto* w : spec.warm) any_warm |= (w != nullptr && (w->primal || w->row_dual));
    ArenaPlan plan;
    SliceDesc* d_slices = nullptr;
    int32_t* d_idx = nullptr;
    double* d_val = nullptr;
    int32_t* d_len = nullptr;
    CtaWork* d_ctas = nullptr;
    VecWork* d_vec = nullptr;
    InstanceInfo* d_info = nullptr;
    double* warm_x = nullptr;
    double* warm_y = nullptr;
    plan.add(d_slices, a_slices_ + at_slices_);
    plan.add(d_idx, slots);
    plan.add(d_val, slots);
    plan.add(a_s64_, a_slots_);
    plan.add(at_s64_, at_slots_);
    if (mixed_) {
        plan.add(a_s32_, a_slots_);
        plan.add(at_s32_, at_slots_);
    }
    plan.add(d_len, lens);
    plan.add(d_ctas, static_cast<int64_t>(a_ctas_.size() + at_ctas_.size()));
    plan.add(d_vec, static_cast<int64_t>(vec_.size()));
    plan.add(d_info, count_);
    plan.add(g_.ctl, count_);
    for (double** p : {&g_.rs, &g_.row_tmp, &g_.y_o, &g_.ya_o, &g_.dy_o, &g_.best_y, &g_.dray}) plan.add(*p, R);
    for (double** p : {&g_.cs, &g_.col_tmp, &g_.x_o, &g_.xa_o, &g_.p_proj, &g_.best_x, &g_.pray}) plan.add(*p, N);
    plan.add(g_.c_orig, N);
    plan.add(g_.xl_orig, N);
    plan.add(g_.xu_orig, N);
    plan.add(g_.rl_orig, R);
    plan.add(g_.ru_orig, R);
    if (any_warm) {
        plan.add(warm_x, N);
        plan.add(warm_y, R);
    }
    plan.add(g_.part_primal, static_cast<int64_t>(at_ctas_.size()));
    plan.add(g_.part_dual, 2 * static_cast<int64_t>(a_ctas_.size()));
    plan.add(g_.part_prep, kPrepSlots * static_cast<int64_t>(vec_.size()));
    plan.add(g_.part_check, kCheckSlots * static_cast<int64_t>(a_ctas_.size() + at_ctas_.size()));
    plan.add(g_.count_dual, count_);
    plan.add(g_.count_check, count_);
    plan.add(d_active_, 2);
    if (spec.ext.restart_metric == PDLPGPU_RESTART_NORMALIZED_GAP)
        for (int k = 0; k < 2; ++k) {
            plan.add(g_.ndg_g[k], N);
            plan.add(g_.ndg_a[k], R);
        }
    auto plan_work = [&](auto& w, int64_t Rn, int64_t Nn) {
        for (int k = 0; k < 2; ++k) {
            plan.add(w.X[k], Nn);
            plan.add(w.Y[k], Rn);
            plan.add(w.AX[k], Rn);
        }
        for (auto** p : {&w.avg_x, &w.rx, &w.c, &w.xl, &w.xu, &w.tau, &w.itau}) plan.add(*p, Nn);
        for (auto** p : {&w.avg_y, &w.ry, &w.rl, &w.ru, &w.sigma, &w.isigma}) plan.add(*p, Rn);
    };
    plan_work(w64_, R, N);
    if (mixed_) plan_work(w32_, R, N);
    arena_bytes_ = plan.total();
    if (!check(cudaMalloc(&arena_, arena_bytes_), "cudaMalloc")) return false;
    plan.assign(arena_);
    g_.rx64 = w64_.rx;
    g_.ry64 = w64_.ry;
    g_.rx32 = mixed_ ? w32_.rx : nullptr;
    g_.ry32 = mixed_ ? w32_.ry : nullptr;
    if (!check(cudaMallocHost(&h_active_, 2 * sizeof(int32_t)), "cudaMallocHost")) return false;
    if (!check(cudaMemsetAsync(arena_, 0, arena_bytes_, stream_), "cudaMemset")) return false;
    mark("maps and arena");

    // --- host staging and upload ------------------------------------------
    auto up = [&](void* dst, const void* src, size_t bytes) { return upload(dst, src, bytes); };
    {
        std::vector<SliceDesc> slices;
        slices.reserve(static_cast<size_t>(a_slices_ + at_slices_));
        for (int k = 0; k < nlayouts; ++k)
            slices.insert(slices.end(), layouts_[k].a.slices.begin(), layouts_[k].a.slices.end());
        for (int k = 0; k < nlayouts; ++k)
            slices.insert(slices.end(), layouts_[k].at.slices.begin(), layouts_[k].at.slices.end());
        // Slot data of every layout, A side then A^T side, straight from the
        // layouts (which outlive the copies).
        std::vector<HostPiece> idx, val;
        for (int side = 0; side < 2; ++side)
            for (int k = 0; k < nlayouts; ++k) {
                const SideLayout& S = side == 0 ? layouts_[k].a : layouts_[k].at;
                idx.push_back({S.idx.data(), S.idx.size() * sizeof(int32_t)});
                val.push_back({S.val.data(), S.val.size() * sizeof(double)});
            }
        if (!up(d_slices, slices.data(), slices.size() * sizeof(SliceDesc))) return false;
        if (!upload(d_idx, idx) || !upload(d_val, val)) return false;
        std::vector<int32_t> len;
        len.reserve(static_cast<size_t>(lens));
        for (int k = 0; k < nlayouts; ++k) len.insert(len.end(), layouts_[k].a.line_len.begin(), layouts_[k].a.line_len.end());
        const size_t a_len_total = len.size();
        for (int k = 0; k < nlayouts; ++k) len.insert(len.end(), layouts_[k].at.line_len.begin(), layouts_[k].at.line_len.end());
        if (!up(d_len, len.data(), len.size() * sizeof(int32_t))) return false;
        std::vector<CtaWork> ctas(a_ctas_);
        ctas.insert(ctas.end(), at_ctas_.begin(), at_ctas_.end());
        if (!up(d_ctas, ctas.data(), ctas.size() * sizeof(CtaWork))) return false;
        if (!up(d_vec, vec_.data(), vec_.size() * sizeof(VecWork))) return false;
        if (!up(d_info, info_.data(), info_.size() * sizeof(InstanceInfo))) return false;
        // Wire the sides: A-side data first, then A^T-side data.
        g_.a.slices = d_slices;
        g_.at.slices = d_slices + a_slices_;
        g_.a.idx = d_idx;
        g_.at.idx = d_idx + a_slots_;
        g_.a.val_orig = d_val;
        g_.at.val_orig = d_val + a_slots_;
        g_.a.val_s64 = a_s64_;
        g_.at.val_s64 = at_s64_;
        g_.a.val_s32 = a_s32_;
        g_.at.val_s32 = at_s32_;
        g_.a.line_len = d_len;
        g_.at.line_len = d_len + a_len_total;
        g_.a.ctas = d_ctas;
        g_.at.ctas = d_ctas + a_ctas_.size();
        g_.a.num_ctas = static_cast<int32_t>(a_ctas_.size());
        g_.at.num_ctas = static_cast<int32_t>(at_ctas_.size());
        g_.vec = d_vec;
        g_.num_vec = static_cast<int32_t>(vec_.size());
        g_.info = d_info;
        g_.shared_matrix = spec.shared_matrix ? 1 : 0;
        g_.mixed = mixed_ ? 1 : 0;
        g_.warm_x = nullptr;
        g_.warm_y = nullptr;
        // A^T-side data bases, slice indices and line bases in info_ and in the
        // CTA map are relative to the g_.at pointers.
    }
    mark("matrix upload");
    {
        // Original-problem vectors in internal order.
        // Every element is written below (the instances tile both spaces).
        std::unique_ptr<double[]> cvec(new double[static_cast<size_t>(std::max<int64_t>(N, 1))]);
        std::unique_ptr<double[]> xl(new double[static_cast<size_t>(std::max<int64_t>(N, 1))]);
        std::unique_ptr<double[]> xu(new double[static_cast<size_t>(std::max<int64_t>(N, 1))]);
        std::unique_ptr<double[]> rl(new double[static_cast<size_t>(std::max<int64_t>(R, 1))]);
        std::unique_ptr<double[]> ru(new double[static_cast<size_t>(std::max<int64_t>(R, 1))]);
        std::vector<double> wx, wy;
        if (any_warm) {
            wx.assign(static_cast<size_t>(N), std::nan(""));
            wy.assign(static_cast<size_t>(R), std::nan(""));
        }
        parallel_for(nspec, [&](int i) {
            const int b = device_of_[i];
            if (b < 0) return;
            std::vector<double> tmp;
            const pdlpgpu_lp& lp = *spec.lps[i];
            const InstanceInfo& inf = info_[b];
            to_internal_cols(lp.objective, tmp, b);
            std::copy(tmp.begin(), tmp.end(), cvec.get() + inf.col_off);
            to_internal_cols(lp.var_lower, tmp, b);
            std::copy(tmp.begin(), tmp.end(), xl.get() + inf.col_off);
            to_internal_cols(lp.var_upper, tmp, b);
            std::copy(tmp.begin(), tmp.end(), xu.get() + inf.col_off);
            to_internal_rows(lp.row_lower, tmp, b);
            std::copy(tmp.begin(), tmp.end(), rl.get() + inf.row_off);
            to_internal_rows(lp.row_upper, tmp, b);
            std::copy(tmp.begin(), tmp.end(), ru.get() + inf.row_off);
            const pdlpgpu_warmstart* w = (i < static_cast<int>(spec.warm.size())) ? spec.warm[i] : nullptr;
            if (w && w->primal) {
                to_internal_cols(w->primal, tmp, b);
                std::copy(tmp.begin(), tmp.end(), wx.begin() + inf.col_off);
            }
            if (w && w->row_dual) {
                to_internal_rows(w->row_dual, tmp, b);
                std::copy(tmp.begin(), tmp.end(), wy.begin() + inf.row_off);
            }
        });
        const size_t nb = static_cast<size_t>(N) * 8, rb = static_cast<size_t>(R) * 8;
        if (!up(const_cast<double*>(g_.c_orig), cvec.get(), nb)) return false;
        if (!up(const_cast<double*>(g_.xl_orig), xl.get(), nb)) return false;
        if (!up(const_cast<double*>(g_.xu_orig), xu.get(), nb)) return false;
        if (!up(const_cast<double*>(g_.rl_orig), rl.get(), rb)) return false;
        if (!up(const_cast<double*>(g_.ru_orig), ru.get(), rb)) return false;
        if (any_warm) {
            // NaN marks "no warm value": k_setup_vectors falls back to the cold point.
            if (!up(warm_x, wx.data(), wx.size() * 8)) return false;
            if (!up(warm_y, wy.data(), wy.size() * 8)) return false;
            g_.warm_x = warm_x;
            g_.warm_y = warm_y;
        }
        // Unit scales and the preconditioner defaults (disabled
        // preconditioning keeps these).
        for (double* p : {g_.rs, w64_.sigma, w64_.isigma}) launch_fill<double>(p, R, 1.0, stream_);
        for (double* p : {g_.cs, w64_.tau, w64_.itau}) launch_fill<double>(p, N, 1.0, stream_);
        if (mixed_) {
            for (float* p : {w32_.sigma, w32_.isigma}) launch_fill<float>(p, R, 1.0f, stream_);
            for (float* p : {w32_.tau, w32_.itau}) launch_fill<float>(p, N, 1.0f, stream_);
        }
        if (!check(cudaGetLastError(), "fill")) return false;
    }

    // --- options and per-instance control ---------------------------------
    dopt_.iteration_limit = o.iteration_limit;
    dopt_.check_frequency = o.termination_check_frequency;
    dopt_.max_trials = std::max(o.maximum_step_trials, 1);
    dopt_.adaptive = o.use_adaptive_linesearch != 0;
    dopt_.averaging = o.use_averaging != 0;
    dopt_.restarts = o.use_restarts != 0;
    dopt_.detect_infeasibility = o.detect_infeasibility != 0;
    dopt_.polishing = o.use_feasibility_polishing != 0;
    dopt_.polishing_iterations = o.polishing_iterations;
    dopt_.min_restart = o.minimum_restart_iterations;
    dopt_.max_restart = o.maximum_restart_iterations;
    dopt_.mixed = mixed_ ? 1 : 0;
    dopt_.fp32_stall_checks = spec.ext.fp32_stall_checks > 0 ? spec.ext.fp32_stall_checks : 8;
    // FP32 stalls far above the tolerance, or above the relative KKT level
    // FP32 iterates reach without difficulty (1e-5), are the method's, not
    // the precision's: the FP64 stage is considered only below both.
    dopt_.fp32_switch_kkt = std::min(
        1e-5, (spec.ext.fp32_switch_factor > 0 ? spec.ext.fp32_switch_factor : 1000) *
                  std::max({spec.opt.primal_tolerance, spec.opt.dual_tolerance, spec.opt.gap_tolerance}));
    dopt_.primal_tol = o.primal_tolerance;
    dopt_.dual_tol = o.dual_tolerance;
    dopt_.gap_tol = o.gap_tolerance;
    dopt_.min_step_scale = o.minimum_step_scale;
    dopt_.w_min = o.minimum_primal_weight;
    dopt_.w_max = o.maximum_primal_weight;
    dopt_.smoothing = o.primal_weight_smoothing;
    dopt_.initial_step_safety = o.initial_step_safety;
    dopt_.sufficient = o.restart_sufficient_decay;
    dopt_.necessary = o.restart_necessary_decay;
    dopt_.artificial = o.restart_artificial_fraction;
    dopt_.infeasibility_tol = o.infeasibility_tolerance;
    dopt_.time_limit = o.time_limit_seconds;
    dopt_.ndg_restarts = spec.ext.restart_metric == PDLPGPU_RESTART_NORMALIZED_GAP ? 1 : 0;
    {
        // Step factors for every iteration index a solve can reach (main loop
        // and polishing), at most 2^20 of them (16 MiB).
        const int64_t reach = std::max<int64_t>(o.iteration_limit, o.polishing_iterations) + 2;
        const int64_t entries = std::min<int64_t>(std::max<int64_t>(reach, 1), int64_t(1) << 20);
        void* t = nullptr;
        if (!check(cudaMalloc(&t, static_cast<size_t>(entries) * 2 * sizeof(double)), "cudaMalloc")) return false;
        extra_.push_back(t);
        launch_step_pow(static_cast<double*>(t), entries, stream_);
        dopt_.step_pow = static_cast<const double*>(t);
        dopt_.step_pow_entries = entries;
    }
    setup_ok_ = true;
    mark("vector upload");
    return true;
}


// ---------------------------------------------------------------------------
// Control state, setup kernels, initial check
// ---------------------------------------------------------------------------
bool Engine::init_control() {
    const pdlpgpu_options& o = spec_.opt;
    std::vector<InstanceCtl> ctl(static_cast<size_t>(count_));
    for (size_t i = 0; i < spec_.lps.size(); ++i) {
        const int b = device_of_[i];
        if (b < 0) continue;
        const pdlpgpu_lp& lp = *spec_.lps[i];
        InstanceCtl c;
        std::memset(&c, 0, sizeof(c));
        c.phase = kPhaseMain;
        c.stage = kStageCheck;
        c.check_kind = kCheckInitial;
        c.need_refresh = 1;
        c.fp64_stage = mixed_ ? 0 : 1;
        c.status = -1;
        c.limit_status = 3;
        const pdlpgpu_warmstart* w = i < spec_.warm.size() ? spec_.warm[i] : nullptr;
        const bool warm = w != nullptr && (w->primal != nullptr || w->row_dual != nullptr);
        c.have_avg_at_check = warm ? 1 : 0;
        // StepController (step_controller.cpp:17-28) with the preconditioned
        // static bound 0.99 (pdlp_solver.cpp:188); the power iteration
        // replaces it when preconditioning is off.
        c.eta_max = 0.99;
        c.eta = clampd(o.initial_step_safety * c.eta_max, o.minimum_step_scale * c.eta_max, c.eta_max);
        c.omega = 1.0;
        auto set_w = [&](double v) {
            if (v > 0.0 && std::isfinite(v)) c.omega = clampd(v, o.minimum_primal_weight, o.maximum_primal_weight);
        };
        set_w(o.initial_primal_weight);
        if (w != nullptr && w->primal_weight > 0.0) set_w(w->primal_weight);
        c.trial_eta = c.eta;
        c.trial_omega = c.omega;
        c.ctl_eta = c.eta;
        c.ctl_omega = c.omega;
        c.best_pobj = std::nan("");
        c.best_dobj = -INFINITY;
        c.best_pres = c.best_dres = c.best_gap = c.best_kkt = INFINITY;
        c.restart_baseline = INFINITY;
        c.prev_candidate = INFINITY;
        normalisers(lp, c.pnorm, c.dnorm);
        c.objective_offset = lp.objective_offset;
        ctl[static_cast<size_t>(b)] = c;
    }
    return check(cudaMemcpyAsync(g_.ctl, ctl.data(), ctl.size() * sizeof(InstanceCtl),
                                 cudaMemcpyHostToDevice, stream_), "upload control");
}

bool Engine::setup_kernels() {
    const pdlpgpu_options& o = spec_.opt;
    const int a_n = spec_.shared_matrix ? first_a_ctas_ : g_.a.num_ctas;
    const int at_n = spec_.shared_matrix ? first_at_ctas_ : g_.at.num_ctas;
    const int vec_n = spec_.shared_matrix ? first_vec_ : g_.num_vec;
    const int V = tuning_.vector_width;
    if (!spec_.working_given && o.use_ruiz_scaling && o.ruiz_iterations > 0) {
        for (int pass = 0; pass < o.ruiz_iterations; ++pass) {
            launch_ruiz_max(g_, V, a_n, at_n, stream_);
            launch_ruiz_update(g_, vec_n, stream_);
        }
    }
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, a_n, at_n, stream_);
    if (spec_.shared_matrix) launch_broadcast_scales(g_, info_[0], count_, info_[0].m, info_[0].n, stream_);
    if (o.use_diagonal_preconditioning) {
        launch_precondition<double>(g_, w64_, 1, V, a_n, at_n, stream_);
        if (mixed_) launch_precondition<float>(g_, w32_, 1, V, a_n, at_n, stream_);
        if (spec_.shared_matrix) {
            launch_broadcast_precond<double>(w64_, info_[0], count_, info_[0].m, info_[0].n, stream_);
            if (mixed_) launch_broadcast_precond<float>(w32_, info_[0], count_, info_[0].m, info_[0].n, stream_);
        }
    }
    launch_setup_vectors<double>(g_, w64_, stream_);
    if (mixed_) launch_setup_vectors<float>(g_, w32_, stream_);
    return check(cudaGetLastError(), "setup kernels");
}

// Power iteration on the scaled FP64 matrix (preconditioner.cpp:82-140). The
// starting vector is the reference's: mt19937 seeded with 1, uniform on [-1, 1),
// drawn in original column order.
bool Engine::power_iteration() {
    const pdlpgpu_options& o = spec_.opt;
    std::vector<double> z(static_cast<size_t>(cols_total_));
    std::vector<double> draw;
    for (size_t i = 0; i < spec_.lps.size(); ++i) {
        const int b = device_of_[i];
        if (b < 0) continue;
        const int32_t n = info_[b].n;
        // MT19937 (Matsumoto and Nishimura, 1998); libstdc++ maps two draws
        // to a double in [0, 1) before the affine map to [a, b).
        uint32_t st[624];
        st[0] = 1u;
        for (int k = 1; k < 624; ++k) st[k] = 1812433253u * (st[k - 1] ^ (st[k - 1] >> 30)) + static_cast<uint32_t>(k);
        int pos = 624;
        auto next = [&]() {
            if (pos >= 624) {
                for (int k = 0; k < 624; ++k) {
                    const uint32_t y = (st[k] & 0x80000000u) | (st[(k + 1) % 624] & 0x7fffffffu);
                    st[k] = st[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
                }
                pos = 0;
            }
            uint32_t y = st[pos++];
            y ^= y >> 11;
            y ^= (y << 7) & 0x9d2c5680u;
            y ^= (y << 15) & 0xefc60000u;
            y ^= y >> 18;
            return y;
        };
        draw.resize(static_cast<size_t>(n));
        for (int32_t j = 0; j < n; ++j) {
            double sum = 0.0, sc = 1.0;
            for (int k = 0; k < 2; ++k) {
                sum += static_cast<double>(next()) * sc;
                sc *= 4294967296.0;
            }
            double r = sum / sc;
            if (r >= 1.0) r = std::nextafter(1.0, 0.0);
            draw[j] = r * 2.0 - 1.0;
        }
        std::vector<double> internal;
        to_internal_cols(draw.data(), internal, b);
        std::copy(internal.begin(), internal.end(), z.begin() + info_[b].col_off);
    }
    double* x = g_.x_o;
    double* y = g_.y_o;
    double* zd = g_.xa_o;
    if (!check(cudaMemcpyAsync(zd, z.data(), z.size() * 8, cudaMemcpyHostToDevice, stream_), "upload power start"))
        return false;
    const int V = tuning_.vector_width;
    launch_power_dot(g_, zd, zd, stream_);
    launch_power_step(g_, count_, 1, 0, 1, stream_);
    launch_power_scale(g_, x, zd, stream_);
    const int budget = std::max(o.power_iteration_count, 1);
    for (int it = 0; it < budget; ++it) {
        launch_spmv<double>(g_, 0, 1, x, y, V, stream_);
        launch_spmv<double>(g_, 1, 1, y, zd, V, stream_);
        launch_power_dot(g_, x, zd, stream_);
        launch_power_step(g_, count_, 0, it, budget, stream_);
        launch_power_scale(g_, x, zd, stream_);
    }
    launch_power_finish(g_, count_, o.initial_step_safety, o.minimum_step_scale, stream_);
    return check(cudaGetLastError(), "power iteration");
}

// A time limit as the device clocks it: nanoseconds, 0 for none. A positive
// limit is at least 1 ns (so 1e-30 s is a limit that has passed when the
// first loop top is reached, as in the reference, pdlp_solver.cpp:277-285);
// one beyond the int64 range is none.
static int64_t deadline_ns_of(double seconds) {
    if (!(seconds > 0.0)) return 0;
    const double ns = seconds * 1e9;
    if (!(ns < 9.0e18)) return 0;
    return std::max<int64_t>(1, static_cast<int64_t>(ns));
}

bool Engine::start() {
    if (!setup_ok_) return false;
    if (count_ == 0) return true;
    if (!init_control()) return false;
    if (!setup_kernels()) return false;
    if (!spec_.opt.use_diagonal_preconditioning && !power_iteration()) return false;
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    const double limit = spec_.opt.time_limit_seconds;
    launch_stamp_clock(g_, count_, static_cast<int64_t>(elapsed * 1e9), deadline_ns_of(limit), stream_);
    // Initial A x (refresh is gated on need_refresh, set by init_control),
    // then the initial score (pdlp_solver.cpp:239-264).
    if (mixed_) launch_refresh<float>(g_, w32_, dopt_, tuning_.vector_width, stream_);
    launch_refresh<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
    enqueue_check_stage();
    mark("start");
    return check(cudaGetLastError(), "initial check");
}

// ---------------------------------------------------------------------------
// The iteration loop
// ---------------------------------------------------------------------------
template <class T>
void Engine::enqueue_trial(const Work<T>& w) {
    launch_primal<T>(g_, w, dopt_, tuning_.vector_width, stream_);
    launch_dual<T>(g_, w, dopt_, tuning_.vector_width, stream_);
    launches_ += 2;
}

void Engine::enqueue_check_stage(bool il_sync) {
    const int V = tuning_.vector_width;
    const bool sync = il_sync && il_;
    if (sync) il_move_iterates(true, kIlAtCheck, nullptr);
    if (mixed_) launch_check_prep<float>(g_, w32_, dopt_, stream_);
    launch_check_prep<double>(g_, w64_, dopt_, stream_);
    launch_check_spmv(g_, dopt_, V, stream_);
    launch_check_ndg(g_, dopt_, count_, stream_);
    if (mixed_) launch_check_apply<float>(g_, w32_, dopt_, stream_);
    launch_check_apply<double>(g_, w64_, dopt_, stream_);
    // Mixed: instances the check moves to the FP64 stage take their last
    // FP32 restart point as the FP64 iterate (its A x is refreshed next).
    if (mixed_) launch_switch_fp64(g_, w32_, w64_, stream_);
    if (mixed_) launch_refresh<float>(g_, w32_, dopt_, V, stream_);
    launch_refresh<double>(g_, w64_, dopt_, V, stream_);
    if (sync) il_move_iterates(false, kIlSynced, nullptr);
    cudaMemsetAsync(d_active_, 0, 2 * sizeof(int32_t), stream_);
    launch_finalize(g_, count_, d_active_, stream_);
    launches_ += check_stage_launches(il_sync);
}

void Engine::record_timing(int k) {
    // Event nodes in the captured graph (plain records when not capturing).
    cudaEventRecordWithFlags(tev_[k], stream_, cudaEventRecordExternal);
}

int Engine::timed_position(int k, int slots) const {
    // First, second, middle and last slot of the chunk (distinct slots only).
    const int pos[kTimedSlots] = {0, 1, slots / 2, slots - 1};
    for (int p = 0; p < kTimedSlots; ++p) {
        bool dup = false;
        for (int q = 0; q < p; ++q) dup = dup || pos[q] == pos[p];
        if (!dup && pos[p] == k) return p;
    }
    return -1;
}

// Small instances run the trials of a check interval in one cluster launch
// per precision (k_fused) instead of two launches per trial slot: up to 16
// instances whose slices' warp sums fit a CTA's shared memory, when the
// device can hold such a cluster. When the cluster has a warp for every
// slice and the warps' slices fit beside the sums, the slices are staged in
// shared memory for the launch, and when x and y fit beside them too, every
// CTA keeps copies of them and no trial touches global memory.
void Engine::choose_fused() {
    fused_cluster_ = 0;
    fused_shape32_ = fused_shape64_ = FusedShape{};
    if (il_ || spec_.ext.two_kernel_trials == 1 || count_ <= 0 || count_ > 16) return;
    // The fused kernel adds an entry's slice sums in slice order; that
    // equals the two-kernel path's block sum (one slice per warp, warps in
    // order) only while no entry has more slices than a CTA has warps.
    bool multi = false;
    for (const auto* side : {&a_ctas_, &at_ctas_})
        for (const CtaWork& cw : *side) {
            if (cw.slice_end - cw.slice_begin > kThreads / 32) return;
            multi = multi || cw.slice_end - cw.slice_begin != 1;
        }
    // An instance's slices are contiguous in its CTA map.
    auto first = [](const std::vector<CtaWork>& side, int e0) { return side[static_cast<size_t>(e0)].slice_begin; };
    auto last = [](const std::vector<CtaWork>& side, int e1) { return side[static_cast<size_t>(e1 - 1)].slice_end; };
    FusedShape sh{};
    sh.multi = multi ? 1 : 0;
    sh.elem = static_cast<int32_t>(sizeof(double));
    for (int b = 0; b < count_; ++b) {
        const InstanceInfo& inf = info_[static_cast<size_t>(b)];
        sh.slices_p = std::max(sh.slices_p, last(at_ctas_, inf.at_cta_end) - first(at_ctas_, inf.at_cta_begin));
        sh.slices_d = std::max(sh.slices_d, last(a_ctas_, inf.a_cta_end) - first(a_ctas_, inf.a_cta_begin));
        sh.entries_p = std::max(sh.entries_p, inf.at_cta_end - inf.at_cta_begin);
        sh.entries_d = std::max(sh.entries_d, inf.a_cta_end - inf.a_cta_begin);
    }
    if (fused_smem_bytes(sh) > kFusedMaxSmemHost) return;
    const int warps_per_cta = kFusedCtaThreads / 32;
    const int V = tuning_.vector_width;
    auto resident = [&](int cluster, const FusedShape& f) {
        return mixed_ ? std::min(fused_max_clusters<float>(V, cluster, f), fused_max_clusters<double>(V, cluster, f))
                      : fused_max_clusters<double>(V, cluster, f);
    };
    // The smallest cluster with a warp for every slice, up to 16 CTAs (8
    // where the device cannot hold 16).
    int cluster = 1;
    while (cluster < 16 && cluster * warps_per_cta < std::max(sh.slices_p, sh.slices_d)) cluster *= 2;
    if (cluster == 16 && resident(16, sh) <= 0) cluster = 8;
    if (resident(cluster, sh) <= 0) return;
    // Staging: CTA rank r's warp q takes slice r * 16 + q of each side; its
    // bytes at element size `elem`, with or without the lines' own iterates.
    auto stage_bytes = [&](int own_p, int own_d, int elem) {
        int64_t stage = 0;
        for (int b = 0; b < count_; ++b) {
            const InstanceInfo& inf = info_[static_cast<size_t>(b)];
            const MatrixLayout& L = layouts_[spec_.shared_matrix ? 0 : b];
            const int ps0 = first(at_ctas_, inf.at_cta_begin) - inf.at_slice_base;
            const int ps1 = last(at_ctas_, inf.at_cta_end) - inf.at_slice_base;
            const int ds0 = first(a_ctas_, inf.a_cta_begin) - inf.a_slice_base;
            const int ds1 = last(a_ctas_, inf.a_cta_end) - inf.a_slice_base;
            for (int r = 0; r < cluster; ++r) {
                int64_t cta = 0;
                for (int q = 0; q < warps_per_cta; ++q) {
                    const int k = r * warps_per_cta + q;
                    if (ps0 + k < ps1)
                        cta += fused_slice_bytes(L.at.slices[static_cast<size_t>(ps0 + k)].steps,
                                                 kFusedPrimalConsts + own_p, elem);
                    if (ds0 + k < ds1)
                        cta += fused_slice_bytes(L.a.slices[static_cast<size_t>(ds0 + k)].steps,
                                                 kFusedDualConsts + own_d, elem);
                }
                stage = std::max(stage, cta);
            }
        }
        // Never zero when staged (the kernel tells the modes apart by it).
        return static_cast<int32_t>(std::max<int64_t>(16, std::min<int64_t>(stage, INT32_MAX)));
    };
    int32_t lines = 0;
    for (int b = 0; b < count_; ++b)
        lines = std::max(lines, info_[static_cast<size_t>(b)].m + info_[static_cast<size_t>(b)].n);
    // Per working precision: copies of x and y if they fit, else the staged
    // slices if they fit, else neither.
    auto best = [&](int elem, auto fits) {
        FusedShape out = sh;
        out.elem = elem;
        if (cluster * warps_per_cta < std::max(sh.slices_p, sh.slices_d)) return out;
        FusedShape copies = out;
        copies.stage_bytes = stage_bytes(kFusedPrimalOwn, kFusedDualOwn, elem);
        copies.lines = lines;
        FusedShape staged = out;
        staged.stage_bytes = stage_bytes(0, 0, elem);
        if (fused_smem_bytes(copies) <= kFusedMaxSmemHost && fits(copies)) return copies;
        if (fused_smem_bytes(staged) <= kFusedMaxSmemHost && fits(staged)) return staged;
        return out;
    };
    fused_shape64_ = best(static_cast<int>(sizeof(double)),
                          [&](const FusedShape& f) { return fused_max_clusters<double>(V, cluster, f) > 0; });
    if (mixed_)
        fused_shape32_ = best(static_cast<int>(sizeof(float)),
                              [&](const FusedShape& f) { return fused_max_clusters<float>(V, cluster, f) > 0; });
    fused_cluster_ = cluster;
}

void Engine::enqueue_chunk(int slots, bool fp64_stage) {
    if (fused_cluster_ > 0) {
        // One launch runs every instance's trials of the interval.
        const int V = tuning_.vector_width;
        record_timing(0);
        if (mixed_) launch_fused<float>(g_, w32_, dopt_, V, count_, fused_cluster_, slots, fused_shape32_, stream_);
        else launch_fused<double>(g_, w64_, dopt_, V, count_, fused_cluster_, slots, fused_shape64_, stream_);
        launches_ += 1;
        if (mixed_ && fp64_stage) {
            launch_fused<double>(g_, w64_, dopt_, V, count_, fused_cluster_, slots, fused_shape64_, stream_);
            launches_ += 1;
        }
        record_timing(1);
        enqueue_check_stage(true);
        record_timing(2);
        return;
    }
    // A mixed solve iterates in FP32; while some instance is in its FP64
    // stage, each slot also launches the per-instance FP64 trial kernels
    // (each kernel runs only the instances of its precision). Four slots'
    // kernels are bracketed by timing events.
    record_timing(0);
    for (int k = 0; k < slots; ++k) {
        const int p = timed_position(k, slots);
        if (p >= 0) record_timing(3 + 3 * p);
        if (il_) {
            if (mixed_) launch_il_primal<float>(il32_, g_.ctl, 0, k, stream_);
            else launch_il_primal<double>(il64_, g_.ctl, 0, k, stream_);
            if (p >= 0) record_timing(4 + 3 * p);
            if (mixed_) launch_il_dual<float>(il32_, g_.ctl, dopt_, 0, k, stream_);
            else launch_il_dual<double>(il64_, g_.ctl, dopt_, 0, k, stream_);
        } else if (mixed_) {
            launch_primal<float>(g_, w32_, dopt_, tuning_.vector_width, stream_);
            if (p >= 0) record_timing(4 + 3 * p);
            launch_dual<float>(g_, w32_, dopt_, tuning_.vector_width, stream_);
        } else {
            launch_primal<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
            if (p >= 0) record_timing(4 + 3 * p);
            launch_dual<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
        }
        launches_ += 2;
        if (p >= 0) record_timing(5 + 3 * p);
        if (mixed_ && fp64_stage) {
            launch_primal<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
            launch_dual<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
            launches_ += 2;
        }
    }
    record_timing(1);
    enqueue_check_stage(true);
    record_timing(2);
}

void Engine::timing_reset() {
    for (int p = 0; p < kTimedSlots; ++p) t_primal_[p] = t_dual_[p] = 0.0;
    t_chunk_ = t_check_ = 0.0;
    t_samples_ = t_chunks_ = 0;
}

void Engine::timing_collect(int slots) {
    float c = 0.f, d = 0.f;
    if (cudaEventElapsedTime(&c, tev_[0], tev_[2]) != cudaSuccess ||
        cudaEventElapsedTime(&d, tev_[1], tev_[2]) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    t_chunk_ += c;
    t_check_ += d;
    ++t_chunks_;
    bool all = true;
    float a[kTimedSlots] = {}, b[kTimedSlots] = {};
    for (int k = 0; k < slots; ++k) {
        const int p = timed_position(k, slots);
        if (p < 0) continue;
        all = all && cudaEventElapsedTime(&a[p], tev_[3 + 3 * p], tev_[4 + 3 * p]) == cudaSuccess &&
              cudaEventElapsedTime(&b[p], tev_[4 + 3 * p], tev_[5 + 3 * p]) == cudaSuccess;
    }
    cudaGetLastError();
    if (!all || slots < kTimedSlots) return;
    for (int p = 0; p < kTimedSlots; ++p) {
        t_primal_[p] += a[p];
        t_dual_[p] += b[p];
    }
    ++t_samples_;
}

void Engine::loop_timing(double* out) const {
    double p = 0.0, d = 0.0;
    for (int k = 0; k < kTimedSlots; ++k) {
        p += t_primal_[k];
        d += t_dual_[k];
    }
    const double n = static_cast<double>(t_samples_) * kTimedSlots;
    out[0] = t_samples_ ? p / n : 0.0;
    out[1] = t_samples_ ? d / n : 0.0;
    out[2] = static_cast<double>(t_samples_ * kTimedSlots);
    out[3] = t_chunks_ ? t_chunk_ / t_chunks_ : 0.0;
    out[4] = static_cast<double>(t_chunks_);
    out[5] = device_seconds_;
    out[6] = t_chunks_ ? t_check_ / t_chunks_ : 0.0;
    for (int k = 0; k < kTimedSlots; ++k) {
        out[7 + 2 * k] = t_samples_ ? t_primal_[k] / t_samples_ : 0.0;
        out[8 + 2 * k] = t_samples_ ? t_dual_[k] / t_samples_ : 0.0;
    }
}

bool Engine::build_graph(int slots, bool fp64_stage) {
    cudaGraph_t graph = nullptr;
    if (!check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture"))
        return false;
    const int64_t before = launches_;
    enqueue_chunk(slots, fp64_stage);
    launches_ = before;
    if (!check(cudaStreamEndCapture(stream_, &graph), "end capture")) return false;
    const bool ok = check(cudaGraphInstantiate(fp64_stage ? &graph64_ : &graph_, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    graph_slots_ = slots;
    graph_family_ = il_family_;
    return ok;
}

bool Engine::launch_chunk(int slots) {
    // h_active_[1]: instances in the FP64 stage at the last poll.
    const bool fp64 = mixed_ && h_active_[1] > 0;
    const int trial_launches = fused_cluster_ > 0 ? (fp64 ? 2 : 1) : 2 * slots * (fp64 ? 2 : 1);
    const int per_chunk = trial_launches + check_stage_launches(true);
    if (spec_.ext.disable_graphs) {
        enqueue_chunk(slots, fp64);
        return check(cudaGetLastError(), "chunk launch");
    }
    cudaGraphExec_t& g = fp64 ? graph64_ : graph_;
    if (g == nullptr && !build_graph(slots, fp64)) return false;
    launches_ += per_chunk;
    return check(cudaGraphLaunch(g, stream_), "graph launch");
}

bool Engine::run() {
    if (!setup_ok_ || count_ == 0) return setup_ok_;
    const pdlpgpu_options& o = spec_.opt;
    if (!check(cudaMemcpyAsync(h_active_, d_active_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_), "poll"))
        return false;
    if (!check(cudaStreamSynchronize(stream_), "setup")) return false;
    mark("device setup");
    choose_fused();
    const int slack = spec_.ext.chunk_slack > 0 ? spec_.ext.chunk_slack : 4;
    const int slots = chunk_slots();
    const int64_t trials_bound =
        (std::max<int64_t>(o.iteration_limit, 0) + std::max(o.polishing_iterations, 0) + 2) *
        std::max(o.maximum_step_trials, 1);
    const int64_t max_chunks = trials_bound / std::max(1, slots - slack) + 64;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream_);
    timing_reset();
    int64_t chunks = 0;
    while (*h_active_ != 0) {
        if (chunks >= max_chunks) {
            error_ = "device loop exceeded its chunk bound";
            break;
        }
        if (!launch_chunk(slots)) break;
        ++chunks;
        cudaMemcpyAsync(h_active_, d_active_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
        if (!check(cudaStreamSynchronize(stream_), "iteration loop")) break;
        timing_collect(slots);
    }
    cudaEventRecord(e1, stream_);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    device_seconds_ = 1e-3 * ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ran_ = true;
    mark("iterations");
    return error_.empty();
}

void Engine::results(std::vector<pdlpgpu_result*>& out) {
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    std::vector<InstanceCtl> ctl(static_cast<size_t>(count_));
    // Best points always, rays only when some instance ends with one (no
    // zero fill: every element read is downloaded).
    std::unique_ptr<double[]> bx, by, dr, pr;
    bool have = false;
    if (count_ > 0 && stream_ != nullptr && arena_ != nullptr) {
        const size_t R = static_cast<size_t>(rows_total_), N = static_cast<size_t>(cols_total_);
        bx.reset(new double[std::max<size_t>(N, 1)]);
        by.reset(new double[std::max<size_t>(R, 1)]);
        have = download(ctl.data(), g_.ctl, ctl.size() * sizeof(InstanceCtl)) &&
               download(bx.get(), g_.best_x, N * 8) && download(by.get(), g_.best_y, R * 8);
        bool rays = false;
        for (const InstanceCtl& c : ctl) rays = rays || c.ray_kind != 0;
        mark("download");
        if (have && rays) {
            dr.reset(new double[std::max<size_t>(R, 1)]);
            pr.reset(new double[std::max<size_t>(N, 1)]);
            have = download(dr.get(), g_.dray, R * 8) && download(pr.get(), g_.pray, N * 8);
        }
    }
    out.assign(spec_.lps.size(), nullptr);
    parallel_for(static_cast<int>(spec_.lps.size()), [&](int i) {
        const pdlpgpu_lp& lp = *spec_.lps[i];
        auto* r = static_cast<pdlpgpu_result*>(std::calloc(1, sizeof(pdlpgpu_result)));
        r->num_rows = lp.num_rows;
        r->num_cols = lp.num_cols;
        r->primal_objective = std::nan("");
        r->dual_objective = -INFINITY;
        r->primal_residual = r->dual_residual = r->relative_gap = INFINITY;
        r->final_primal_weight = 1.0;
        r->solve_time_seconds = elapsed;
        const int b = device_of_[i];
        if (b < 0) {
            r->status = PDLPGPU_INVALID_PROBLEM;
            std::snprintf(r->status_message, sizeof(r->status_message), "%s", invalid_[i].c_str());
            out[i] = r;
            return;
        }
        const InstanceCtl& c = ctl[static_cast<size_t>(b)];
        if (!have || c.phase != kPhaseDone || c.status < 0) {
            r->status = PDLPGPU_NUMERICAL_FAILURE;
            std::snprintf(r->status_message, sizeof(r->status_message), "%s",
                          error_.empty() ? "device loop did not complete" : error_.c_str());
            out[i] = r;
            return;
        }
        const MatrixLayout& L = layouts_[spec_.shared_matrix ? 0 : b];
        const InstanceInfo& inf = info_[b];
        r->status = c.status;
        std::snprintf(r->status_message, sizeof(r->status_message), "%s", message_text(c.message));
        r->primal = static_cast<double*>(std::malloc(sizeof(double) * std::max(1, lp.num_cols)));
        r->row_dual = static_cast<double*>(std::malloc(sizeof(double) * std::max(1, lp.num_rows)));
        for (int32_t k = 0; k < inf.n; ++k) r->primal[L.col_perm[k]] = bx[static_cast<size_t>(inf.col_off) + k];
        for (int32_t k = 0; k < inf.m; ++k) r->row_dual[L.row_perm[k]] = by[static_cast<size_t>(inf.row_off) + k];
        if (c.status == PDLPGPU_INFEASIBLE && c.ray_kind == 1 && dr) {
            r->dual_ray = static_cast<double*>(std::malloc(sizeof(double) * std::max(1, lp.num_rows)));
            for (int32_t k = 0; k < inf.m; ++k) r->dual_ray[L.row_perm[k]] = dr[static_cast<size_t>(inf.row_off) + k];
        }
        if (c.status == PDLPGPU_UNBOUNDED && c.ray_kind == 2 && pr) {
            r->primal_ray = static_cast<double*>(std::malloc(sizeof(double) * std::max(1, lp.num_cols)));
            for (int32_t k = 0; k < inf.n; ++k) r->primal_ray[L.col_perm[k]] = pr[static_cast<size_t>(inf.col_off) + k];
        }
        r->primal_objective = c.best_pobj;
        r->dual_objective = c.best_dobj;
        r->primal_residual = c.best_pres;
        r->dual_residual = c.best_dres;
        r->relative_gap = c.best_gap;
        r->iterations = c.iteration;
        r->step_trials = c.step_trials;
        r->restart_count = c.restart_count;
        if (c.diagnostics) {
            r->final_step_size = c.eta;
            r->static_step_bound = c.eta_max;
            r->final_primal_weight = c.omega;
        }
        r->precision_used = mixed_ ? (c.fp64_stage ? 2 : 1) : 0;
        r->fp64_iterations = c.fp64_iterations;
        r->device_seconds = device_seconds_;
        out[i] = r;
    });
    mark("results");
    if (!trace_.empty()) {
        std::fprintf(stderr, "pdlpgpu:");
        double prev = 0.0;
        for (const auto& t : trace_) {
            std::fprintf(stderr, " %s %.3f s;", t.first, t.second - prev);
            prev = t.second;
        }
        std::fprintf(stderr, " total %.3f s\n", prev);
        trace_.clear();
    }
}

// ---------------------------------------------------------------------------
// Component tests
// ---------------------------------------------------------------------------
namespace {
template <class T>
std::vector<T> cast_vec(const std::vector<double>& v) {
    return std::vector<T>(v.begin(), v.end());
}
}  // namespace

bool Engine::component_spmv(int transpose, int values, const double* in, double* out) {
    if (!setup_ok_ || count_ != 1) return false;
    const int V = tuning_.vector_width;
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    std::vector<double> src;
    if (transpose) to_internal_rows(in, src, 0); else to_internal_cols(in, src, 0);
    const size_t out_n = transpose ? info_[0].n : info_[0].m;
    std::vector<double> res(out_n);
    if (values == 2) {
        if (!mixed_) return false;
        const std::vector<float> sf = cast_vec<float>(src);
        float* din = transpose ? w32_.Y[0] : w32_.X[0];
        float* dout = transpose ? w32_.X[1] : w32_.Y[1];
        if (!check(cudaMemcpyAsync(din, sf.data(), sf.size() * 4, cudaMemcpyHostToDevice, stream_), "upload")) return false;
        launch_spmv<float>(g_, transpose, 2, din, dout, V, stream_);
        std::vector<float> rf(out_n);
        if (!check(cudaMemcpyAsync(rf.data(), dout, out_n * 4, cudaMemcpyDeviceToHost, stream_), "download")) return false;
        if (!check(cudaStreamSynchronize(stream_), "spmv")) return false;
        for (size_t k = 0; k < out_n; ++k) res[k] = rf[k];
    } else {
        double* din = transpose ? g_.y_o : g_.x_o;
        double* dout = transpose ? g_.x_o : g_.y_o;
        if (!check(cudaMemcpyAsync(din, src.data(), src.size() * 8, cudaMemcpyHostToDevice, stream_), "upload")) return false;
        launch_spmv<double>(g_, transpose, values, din, dout, V, stream_);
        if (!check(cudaMemcpyAsync(res.data(), dout, out_n * 8, cudaMemcpyDeviceToHost, stream_), "download")) return false;
        if (!check(cudaStreamSynchronize(stream_), "spmv")) return false;
    }
    const MatrixLayout& L = layouts_[0];
    if (transpose) for (int32_t k = 0; k < L.n; ++k) out[L.col_perm[k]] = res[k];
    else for (int32_t k = 0; k < L.m; ++k) out[L.row_perm[k]] = res[k];
    return true;
}

bool Engine::component_ruiz(double* row_scale, double* col_scale, double* scaled_csr) {
    if (!setup_ok_ || count_ != 1) return false;
    const int V = tuning_.vector_width;
    const pdlpgpu_options& o = spec_.opt;
    for (int pass = 0; pass < o.ruiz_iterations; ++pass) {
        launch_ruiz_max(g_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
        launch_ruiz_update(g_, g_.num_vec, stream_);
    }
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    const MatrixLayout& L = layouts_[0];
    std::vector<double> rs(L.m), cs(L.n), slots(static_cast<size_t>(a_slots_));
    if (!check(cudaMemcpyAsync(rs.data(), g_.rs, rs.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaMemcpyAsync(cs.data(), g_.cs, cs.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaMemcpyAsync(slots.data(), a_s64_, slots.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaStreamSynchronize(stream_), "ruiz"))
        return false;
    for (int32_t k = 0; k < L.m; ++k) row_scale[L.row_perm[k]] = rs[k];
    for (int32_t k = 0; k < L.n; ++k) col_scale[L.col_perm[k]] = cs[k];
    if (scaled_csr != nullptr) {
        const int Vw = tuning_.vector_width;
        for (const SliceDesc& sd : L.a.slices) {
            const int glog = slice_glog(sd.meta), nl = slice_lines(sd.meta), G = 1 << glog;
            const int64_t base = static_cast<int64_t>(sd.data_off) * 32;
            for (int r = 0; r < nl; ++r) {
                const int32_t line = sd.line0 + r;
                const int32_t row = L.row_perm[line];
                for (int k = 0; k < L.a.line_len[line]; ++k) {
                    const int64_t s = k >> glog;
                    const int lane = r * G + (k & (G - 1));
                    const int64_t pos = base + (s / Vw) * 32 * Vw + lane * Vw + (s % Vw);
                    const int32_t col = L.col_perm[L.a.idx[pos]];
                    const int32_t* b = csr0_.index.data() + csr0_.start[row];
                    const int32_t* e = csr0_.index.data() + csr0_.start[row + 1];
                    const int32_t* f = std::lower_bound(b, e, col);
                    scaled_csr[f - csr0_.index.data()] = slots[pos];
                }
            }
        }
    }
    return true;
}

bool Engine::component_precondition(double* tau, double* tau_inv, double* sigma, double* sigma_inv) {
    if (!setup_ok_ || count_ != 1) return false;
    const int V = tuning_.vector_width;
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    launch_precondition<double>(g_, w64_, 1, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    const MatrixLayout& L = layouts_[0];
    std::vector<double> t(L.n), ti(L.n), sg(L.m), si(L.m);
    if (!check(cudaMemcpyAsync(t.data(), w64_.tau, t.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaMemcpyAsync(ti.data(), w64_.itau, ti.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaMemcpyAsync(sg.data(), w64_.sigma, sg.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaMemcpyAsync(si.data(), w64_.isigma, si.size() * 8, cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaStreamSynchronize(stream_), "precondition"))
        return false;
    for (int32_t k = 0; k < L.n; ++k) { tau[L.col_perm[k]] = t[k]; tau_inv[L.col_perm[k]] = ti[k]; }
    for (int32_t k = 0; k < L.m; ++k) { sigma[L.row_perm[k]] = sg[k]; sigma_inv[L.row_perm[k]] = si[k]; }
    return true;
}

namespace {
template <class T>
bool put(cudaStream_t s, T* dst, const std::vector<double>& src) {
    const std::vector<T> v(src.begin(), src.end());
    return cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess;
}
template <class T>
bool get(cudaStream_t s, const T* src, std::vector<double>& dst, size_t n) {
    std::vector<T> v(n);
    if (cudaMemcpyAsync(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, s) != cudaSuccess) return false;
    if (cudaStreamSynchronize(s) != cudaSuccess) return false;
    dst.assign(v.begin(), v.end());
    return true;
}
}  // namespace

bool Engine::component_trial(const double* tau, const double* tau_inv, const double* sigma,
                             const double* sigma_inv, const double* x, const double* y,
                             const double* ax, double step, double weight, double* x_out,
                             double* y_out, double* ax_out, double* reductions) {
    if (!setup_ok_ || count_ != 1) return false;
    const int V = tuning_.vector_width;
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    launch_setup_vectors<double>(g_, w64_, stream_);
    if (mixed_) launch_setup_vectors<float>(g_, w32_, stream_);
    std::vector<double> t, ti, sg, si, xv, yv, av;
    to_internal_cols(tau, t, 0);
    to_internal_cols(tau_inv, ti, 0);
    to_internal_rows(sigma, sg, 0);
    to_internal_rows(sigma_inv, si, 0);
    to_internal_cols(x, xv, 0);
    to_internal_rows(y, yv, 0);
    to_internal_rows(ax, av, 0);
    InstanceCtl c;
    std::memset(&c, 0, sizeof(c));
    c.phase = kPhaseMain;
    c.stage = kStageTrial;
    c.fp64_stage = mixed_ ? 0 : 1;
    c.eta = c.trial_eta = step;
    c.omega = c.trial_omega = weight;
    c.eta_max = 1.0;
    c.best_kkt = INFINITY;
    bool ok = check(cudaMemcpyAsync(g_.ctl, &c, sizeof(c), cudaMemcpyHostToDevice, stream_), "upload");
    std::vector<double> xo, yo, ao;
    const MatrixLayout& L = layouts_[0];
    if (mixed_) {
        ok = ok && put(stream_, w32_.tau, t) && put(stream_, w32_.itau, ti) && put(stream_, w32_.sigma, sg) &&
             put(stream_, w32_.isigma, si) && put(stream_, w32_.X[0], xv) && put(stream_, w32_.Y[0], yv) &&
             put(stream_, w32_.AX[0], av);
        if (!ok) return check(cudaErrorInvalidValue, "upload");
        launch_primal<float>(g_, w32_, dopt_, V, stream_);
        launch_dual<float>(g_, w32_, dopt_, V, stream_);
        ok = get(stream_, w32_.X[1], xo, L.n) && get(stream_, w32_.Y[1], yo, L.m) && get(stream_, w32_.AX[1], ao, L.m);
    } else {
        ok = ok && put(stream_, w64_.tau, t) && put(stream_, w64_.itau, ti) && put(stream_, w64_.sigma, sg) &&
             put(stream_, w64_.isigma, si) && put(stream_, w64_.X[0], xv) && put(stream_, w64_.Y[0], yv) &&
             put(stream_, w64_.AX[0], av);
        if (!ok) return check(cudaErrorInvalidValue, "upload");
        launch_primal<double>(g_, w64_, dopt_, V, stream_);
        launch_dual<double>(g_, w64_, dopt_, V, stream_);
        ok = get(stream_, w64_.X[1], xo, L.n) && get(stream_, w64_.Y[1], yo, L.m) && get(stream_, w64_.AX[1], ao, L.m);
    }
    if (!ok || !check(cudaGetLastError(), "trial")) return false;
    if (!check(cudaMemcpyAsync(&c, g_.ctl, sizeof(c), cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaStreamSynchronize(stream_), "trial"))
        return false;
    for (int32_t k = 0; k < L.n; ++k) x_out[L.col_perm[k]] = xo[k];
    for (int32_t k = 0; k < L.m; ++k) { y_out[L.row_perm[k]] = yo[k]; ax_out[L.row_perm[k]] = ao[k]; }
    reductions[0] = c.dbg[0];
    reductions[1] = c.dbg[1];
    reductions[2] = c.dbg[2];
    return true;
}

bool Engine::component_evaluate(const double* x, const double* y, const double* rx,
                                const double* ry, double* metrics, double* verdicts) {
    if (!setup_ok_ || count_ != 1) return false;
    const int V = tuning_.vector_width;
    launch_scale_values(g_, a_s64_, at_s64_, a_s32_, at_s32_, V, g_.a.num_ctas, g_.at.num_ctas, stream_);
    launch_setup_vectors<double>(g_, w64_, stream_);
    std::vector<double> xv, yv, rxv, ryv;
    to_internal_cols(x, xv, 0);
    to_internal_rows(y, yv, 0);
    to_internal_cols(rx, rxv, 0);
    to_internal_rows(ry, ryv, 0);
    InstanceCtl c;
    std::memset(&c, 0, sizeof(c));
    c.phase = kPhaseMain;
    c.stage = kStageCheck;
    c.check_kind = kCheckEvaluate;
    c.fp64_stage = 1;
    normalisers(*spec_.lps[0], c.pnorm, c.dnorm);
    c.objective_offset = spec_.lps[0]->objective_offset;
    c.best_kkt = INFINITY;
    bool ok = check(cudaMemcpyAsync(g_.ctl, &c, sizeof(c), cudaMemcpyHostToDevice, stream_), "upload") &&
              put(stream_, w64_.X[0], xv) && put(stream_, w64_.Y[0], yv) && put(stream_, w64_.rx, rxv) &&
              put(stream_, w64_.ry, ryv);
    if (!ok) return check(cudaErrorInvalidValue, "upload");
    launch_check_prep<double>(g_, w64_, dopt_, stream_);
    launch_check_spmv(g_, dopt_, V, stream_);
    launch_check_ndg(g_, dopt_, count_, stream_);
    if (!check(cudaMemcpyAsync(&c, g_.ctl, sizeof(c), cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaStreamSynchronize(stream_), "evaluate"))
        return false;
    metrics[0] = c.best_pobj;
    metrics[1] = c.best_dobj;
    metrics[2] = c.best_pres;
    metrics[3] = c.best_dres;
    metrics[4] = c.best_gap;
    metrics[5] = c.best_kkt;
    metrics[6] = c.best_finite;
    metrics[7] = c.best_valid;
    for (int q = 0; q < 6; ++q) verdicts[q] = c.dbg[3 + q];
    return true;
}


// ---------------------------------------------------------------------------
// Sessions
// ---------------------------------------------------------------------------
bool Engine::session_create(const pdlpgpu_lp& family, int32_t batch, const pdlpgpu_options& opt,
                            const pdlpgpu_ext_options& ext) {
    family_ = family;
    SolveSpec spec;
    spec.lps.assign(static_cast<size_t>(batch), &family_);
    spec.shared_matrix = true;
    spec.opt = opt;
    spec.ext = ext;
    if (!prepare(spec)) return false;
    if (count_ != batch) {
        error_ = invalid_.empty() ? "invalid session" : invalid_[0];
        return false;
    }
    const MatrixLayout& L = layouts_[0];
    auto dalloc = [&](auto*& p, size_t count) {
        void* q = nullptr;
        if (!check(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(*p)), "cudaMalloc")) return false;
        extra_.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        return true;
    };
    if (!dalloc(d_row_perm_, L.m) || !dalloc(d_col_perm_, L.n)) return false;
    for (int k = 0; k < 5; ++k) if (!dalloc(fam_[k], (k == 0 || k >= 3) ? L.n : L.m)) return false;
    if (!dalloc(warm_x_, static_cast<size_t>(cols_total_)) || !dalloc(warm_y_, static_cast<size_t>(rows_total_)) ||
        !dalloc(warm_w_, static_cast<size_t>(batch)))
        return false;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return bytes == 0 || check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
    };
    std::vector<double> v;
    bool ok = up(d_row_perm_, L.row_perm.data(), L.row_perm.size() * 4) &&
              up(d_col_perm_, L.col_perm.data(), L.col_perm.size() * 4);
    to_internal_cols(family.objective, v, 0);
    ok = ok && up(fam_[0], v.data(), v.size() * 8);
    to_internal_rows(family.row_lower, v, 0);
    ok = ok && up(fam_[1], v.data(), v.size() * 8);
    to_internal_rows(family.row_upper, v, 0);
    ok = ok && up(fam_[2], v.data(), v.size() * 8);
    to_internal_cols(family.var_lower, v, 0);
    ok = ok && up(fam_[3], v.data(), v.size() * 8);
    to_internal_cols(family.var_upper, v, 0);
    ok = ok && up(fam_[4], v.data(), v.size() * 8);
    if (!ok) return false;
    // Matrix-only setup, once: Ruiz scaling, scaled coefficients,
    // preconditioner, static step bound.
    if (!init_control() || !setup_kernels()) return false;
    if (!spec_.opt.use_diagonal_preconditioning) {
        if (!power_iteration()) return false;
        InstanceCtl c0;
        if (!check(cudaMemcpyAsync(&c0, g_.ctl, sizeof(c0), cudaMemcpyDeviceToHost, stream_), "download") ||
            !check(cudaStreamSynchronize(stream_), "power iteration"))
            return false;
        session_eta_max_ = c0.eta_max;
    }
    il_ = ext.layout == PDLPGPU_LAYOUT_INTERLEAVED || (ext.layout == PDLPGPU_LAYOUT_AUTO && batch >= 16);
    if (il_ && !(mixed_ ? il_build(il32_, w32_) : il_build(il64_, w64_))) return false;
    return check(cudaStreamSynchronize(stream_), "session setup");
}

// Device-pointer inputs are usually written just before the call by the
// caller's own kernels or copies, enqueued on the legacy default stream (the
// stream PyTorch and most callers use by default). The session's stream does
// not synchronise with it implicitly (it is non-blocking), so it waits for
// everything enqueued there so far.
bool Engine::wait_for_caller() {
    if (caller_done_ == nullptr &&
        !check(cudaEventCreateWithFlags(&caller_done_, cudaEventDisableTiming), "cudaEventCreate"))
        return false;
    return check(cudaEventRecord(caller_done_, cudaStreamLegacy), "cudaEventRecord") &&
           check(cudaStreamWaitEvent(stream_, caller_done_, 0), "cudaStreamWaitEvent");
}

bool Engine::session_load(bool on_device, const double* c, const double* rl, const double* ru,
                          const double* xl, const double* xu, const double* wx, const double* wy,
                          const double* ww) {
    const int64_t n = info_[0].n, m = info_[0].m;
    if (on_device && !wait_for_caller()) return false;
    auto load = [&](const double* src, double* dst, const double* fam, bool cols) {
        const int64_t len = cols ? n : m;
        if (src == nullptr) {
            launch_permute(fam, dst, nullptr, len, count_, 2, stream_);
            return true;
        }
        const double* dsrc = src;
        if (!on_device) {
            double* staging = cols ? g_.x_o : g_.y_o;
            if (!check(cudaMemcpyAsync(staging, src, static_cast<size_t>(len * count_) * 8,
                                       cudaMemcpyHostToDevice, stream_), "load"))
                return false;
            dsrc = staging;
        }
        launch_permute(dsrc, dst, cols ? d_col_perm_ : d_row_perm_, len, count_, 0, stream_);
        return true;
    };
    bool ok = load(c, const_cast<double*>(g_.c_orig), fam_[0], true) &&
              load(rl, const_cast<double*>(g_.rl_orig), fam_[1], false) &&
              load(ru, const_cast<double*>(g_.ru_orig), fam_[2], false) &&
              load(xl, const_cast<double*>(g_.xl_orig), fam_[3], true) &&
              load(xu, const_cast<double*>(g_.xu_orig), fam_[4], true);
    if (il_)
        il_set_family((c == nullptr ? 1 << kIlC : 0) | (rl == nullptr ? 1 << kIlRl : 0) |
                      (ru == nullptr ? 1 << kIlRu : 0) | (xl == nullptr ? 1 << kIlXl : 0) |
                      (xu == nullptr ? 1 << kIlXu : 0));
    g_.warm_x = nullptr;
    g_.warm_y = nullptr;
    if (wx != nullptr) ok = ok && load(wx, warm_x_, nullptr, true), g_.warm_x = warm_x_;
    if (wy != nullptr) ok = ok && load(wy, warm_y_, nullptr, false), g_.warm_y = warm_y_;
    session_warm_ = wx != nullptr || wy != nullptr;
    session_has_ww_ = ww != nullptr;
    if (ww != nullptr)
        ok = ok && check(cudaMemcpyAsync(warm_w_, ww, static_cast<size_t>(count_) * 8,
                                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                         stream_), "load");
    return ok && check(cudaGetLastError(), "session load");
}

bool Engine::session_solve(int32_t* optimal) {
    t0_ = std::chrono::steady_clock::now();
    const pdlpgpu_options& o = spec_.opt;
    launch_norm_parts(g_, stream_);
    double initial_weight = o.initial_primal_weight;
    launch_init_ctl(g_, dopt_, count_, mixed_ ? 1 : 0, session_warm_ ? 1 : 0,
                    session_has_ww_ ? warm_w_ : nullptr, session_eta_max_, initial_weight,
                    family_.objective_offset, stream_);
    launch_setup_vectors<double>(g_, w64_, stream_);
    if (mixed_) launch_setup_vectors<float>(g_, w32_, stream_);
    launch_stamp_clock(g_, count_, 0, deadline_ns_of(o.time_limit_seconds), stream_);
    if (mixed_) launch_refresh<float>(g_, w32_, dopt_, tuning_.vector_width, stream_);
    launch_refresh<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
    const int64_t before = launches_;
    enqueue_check_stage();
    if (il_) {
        il_move_statics(kIlAll, nullptr);
        il_move_iterates(false, kIlAll, nullptr);
    }
    launches_ = before;
    if (!check(cudaGetLastError(), "session start")) return false;
    launches_ = 0;
    if (!ensure_graph()) return false;
    if (!run()) return false;
    std::vector<InstanceCtl> ctl(static_cast<size_t>(count_));
    if (!check(cudaMemcpyAsync(ctl.data(), g_.ctl, ctl.size() * sizeof(InstanceCtl), cudaMemcpyDeviceToHost, stream_), "download") ||
        !check(cudaStreamSynchronize(stream_), "session solve"))
        return false;
    int32_t k = 0;
    for (const auto& c : ctl) k += (c.phase == kPhaseDone && c.status == 0) ? 1 : 0;
    *optimal = k;
    return true;
}

bool Engine::session_read(bool on_device, double* primal, double* dual, int32_t* status,
                          int64_t* iterations, double* stats) {
    const int64_t n = info_[0].n, m = info_[0].m;
    if (on_device && (primal != nullptr || dual != nullptr) && !wait_for_caller()) return false;
    if (primal != nullptr) {
        double* dst = on_device ? primal : g_.x_o;
        launch_permute(g_.best_x, dst, d_col_perm_, n, count_, 1, stream_);
        if (!on_device && !check(cudaMemcpyAsync(primal, g_.x_o, static_cast<size_t>(n * count_) * 8,
                                                 cudaMemcpyDeviceToHost, stream_), "read"))
            return false;
    }
    if (dual != nullptr) {
        double* dst = on_device ? dual : g_.y_o;
        launch_permute(g_.best_y, dst, d_row_perm_, m, count_, 1, stream_);
        if (!on_device && !check(cudaMemcpyAsync(dual, g_.y_o, static_cast<size_t>(m * count_) * 8,
                                                 cudaMemcpyDeviceToHost, stream_), "read"))
            return false;
    }
    if (status != nullptr || iterations != nullptr || stats != nullptr) {
        std::vector<InstanceCtl> ctl(static_cast<size_t>(count_));
        if (!check(cudaMemcpyAsync(ctl.data(), g_.ctl, ctl.size() * sizeof(InstanceCtl), cudaMemcpyDeviceToHost, stream_), "read") ||
            !check(cudaStreamSynchronize(stream_), "read"))
            return false;
        for (int32_t b = 0; b < count_; ++b) {
            const InstanceCtl& c = ctl[static_cast<size_t>(b)];
            if (status) status[b] = c.phase == kPhaseDone ? c.status : PDLPGPU_NUMERICAL_FAILURE;
            if (iterations) iterations[b] = c.iteration;
            if (stats) {
                double* st = stats + 8 * b;
                st[0] = c.best_pobj; st[1] = c.best_dobj; st[2] = c.best_pres;
                st[3] = c.best_dres; st[4] = c.best_gap; st[5] = static_cast<double>(c.step_trials);
                st[6] = c.omega; st[7] = static_cast<double>(c.restart_count);
            }
        }
    }
    return check(cudaStreamSynchronize(stream_), "read");
}

bool Engine::time_kernels(int reps, double* out) {
    Global gm = g_;
    gm.measure = 1;
    cudaEvent_t e[4];
    for (auto& ev : e) cudaEventCreate(&ev);
    const int V = tuning_.vector_width;
    // The interleaved kernels in timing mode write their trial buffers for
    // every lane, which may hold committed points: the iterates are undefined
    // afterwards (every solve starts from a fresh setup).
    auto primal = [&] {
        if (il_ && mixed_) launch_il_primal<float>(il32_, g_.ctl, 1, 0, stream_);
        else if (il_) launch_il_primal<double>(il64_, g_.ctl, 1, 0, stream_);
        else if (mixed_) launch_primal<float>(gm, w32_, dopt_, V, stream_);
        else launch_primal<double>(gm, w64_, dopt_, V, stream_);
    };
    auto dual = [&] {
        if (il_ && mixed_) launch_il_dual<float>(il32_, g_.ctl, dopt_, 1, 0, stream_);
        else if (il_) launch_il_dual<double>(il64_, g_.ctl, dopt_, 1, 0, stream_);
        else if (mixed_) launch_dual<float>(gm, w32_, dopt_, V, stream_);
        else launch_dual<double>(gm, w64_, dopt_, V, stream_);
    };
    primal();
    dual();
    cudaEventRecord(e[0], stream_);
    for (int r = 0; r < reps; ++r) primal();
    cudaEventRecord(e[1], stream_);
    for (int r = 0; r < reps; ++r) dual();
    cudaEventRecord(e[2], stream_);
    if (!check(cudaEventSynchronize(e[2]), "time kernels")) return false;
    float mp = 0.f, md = 0.f;
    cudaEventElapsedTime(&mp, e[0], e[1]);
    cudaEventElapsedTime(&md, e[1], e[2]);
    for (auto& ev : e) cudaEventDestroy(ev);
    // Algorithmic bytes: each nonzero once (value + index), every per-line
    // vector once, the gathered vector once; a shared matrix counts once.
    const double T = mixed_ ? 4.0 : 8.0;
    double e_at = 0, e_a = 0, s_at = 0, s_a = 0;
    for (const MatrixLayout& L : layouts_) {
        e_at += L.at.entries; e_a += L.a.entries;
        s_at += L.at.slots(); s_a += L.a.slots();
    }
    const double N = static_cast<double>(cols_total_), R = static_cast<double>(rows_total_);
    out[0] = mp / reps;
    out[1] = md / reps;
    if (il_) {
        // Per instance: the line's own vectors (x read, x' written, and each
        // problem vector loaded per instance) and the gathered vector once;
        // once for the batch: the matrix (value, index, row pointer) and the
        // broadcast vectors (preconditioner and family vectors).
        auto own = [&](int k) { return ((il_family_ >> k) & 1) ? 0.0 : 1.0; };
        const double B = count_, n = info_[0].n, m = info_[0].m, nnz = e_at;
        const double col_own = 2.0 + own(kIlC) + own(kIlXl) + own(kIlXu);
        const double col_fam = 2.0 + (3.0 - own(kIlC) - own(kIlXl) - own(kIlXu));
        const double row_own = 4.0 + own(kIlRl) + own(kIlRu);
        const double row_fam = 2.0 + (2.0 - own(kIlRl) - own(kIlRu));
        out[2] = B * n * col_own * T + n * col_fam * T + nnz * (T + 4.0) + (n + 1) * 8.0 + B * m * T;
        out[3] = B * m * row_own * T + m * row_fam * T + nnz * (T + 4.0) + (m + 1) * 8.0 + B * n * T;
        out[4] = 0.0;
        out[5] = 0.0;
        return true;
    }
    out[2] = e_at * (T + 4.0) + N * 7.0 * T + R * T;
    out[3] = e_a * (T + 4.0) + R * 8.0 * T + N * T;
    out[4] = s_at - e_at;
    out[5] = s_a - e_a;
    return true;
}


// ---------------------------------------------------------------------------
// Streams
// ---------------------------------------------------------------------------
bool Engine::ensure_graph() {
    if (il_ && graph_family_ != il_family_) {
        // The captured interleaved kernels address the family vectors of the
        // load they were captured with.
        for (cudaGraphExec_t* g : {&graph_, &graph64_}) {
            if (*g != nullptr) cudaGraphExecDestroy(*g);
            *g = nullptr;
        }
    }
    if (graph_ != nullptr || spec_.ext.disable_graphs) return true;
    return build_graph(chunk_slots(), false);
}

bool Engine::session_stream(bool on_device, int64_t N, const double* const in[5], const double* wx,
                            const double* wy, const double* ww, double* out_x, double* out_y,
                            int32_t* status, int64_t* iterations, double* stats) {
    t0_ = std::chrono::steady_clock::now();
    const int32_t B = count_;
    const int64_t n = info_[0].n, m = info_[0].m;
    const pdlpgpu_options& o = spec_.opt;
    if (on_device && !wait_for_caller()) return false;
    std::vector<void*> temp;   // per-call device buffers
    auto dalloc = [&](auto*& p, size_t count, std::vector<void*>& list) {
        void* q = nullptr;
        if (!check(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(*p)), "cudaMalloc")) return false;
        list.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        return true;
    };
    struct Free {
        std::vector<void*>& v;
        ~Free() { for (void* q : v) cudaFree(q); }
    } free_temp{temp};
    if (d_inst_ == nullptr) {
        if (!dalloc(d_inst_, B, extra_) || !dalloc(d_mask_, B, extra_) || !dalloc(d_done_, B, extra_) ||
            !dalloc(d_zero_perm_, 1, extra_))
            return false;
        if (!check(cudaMemsetAsync(d_zero_perm_, 0, sizeof(int32_t), stream_), "memset")) return false;
    }
    // Inputs and outputs on the device.
    const int64_t lens[5] = {n, m, m, n, n};
    const double* src[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    const double *swx = wx, *swy = wy, *sww = ww;
    double *dox = out_x, *doy = out_y;
    auto up = [&](const double* h, int64_t count, const double*& d) {
        double* q = nullptr;
        if (!dalloc(q, static_cast<size_t>(count), temp)) return false;
        d = q;
        return check(cudaMemcpyAsync(q, h, static_cast<size_t>(count) * 8, cudaMemcpyHostToDevice, stream_), "upload");
    };
    for (int k = 0; k < 5; ++k) {
        if (in[k] == nullptr) continue;
        if (on_device) src[k] = in[k];
        else if (!up(in[k], N * lens[k], src[k])) return false;
    }
    if (!on_device) {
        if (wx && !up(wx, N * n, swx)) return false;
        if (wy && !up(wy, N * m, swy)) return false;
        if (ww && !up(ww, N, sww)) return false;
        if (out_x && !dalloc(dox, static_cast<size_t>(N * n), temp)) return false;
        if (out_y && !dalloc(doy, static_cast<size_t>(N * m), temp)) return false;
    }
    const bool warm = wx != nullptr || wy != nullptr;
    if (il_) {
        int32_t family = 0;
        for (int k = 0; k < kIlVecs; ++k) family |= in[k] == nullptr ? 1 << k : 0;
        il_set_family(family);
    }
    if (!ensure_graph()) return false;

    launch_retire(g_, B, stream_);
    std::vector<int64_t> slot(static_cast<size_t>(B), -1);
    std::vector<int32_t> mask(static_cast<size_t>(B), 0), done(static_cast<size_t>(B), 0);
    std::vector<InstanceCtl> ctl(static_cast<size_t>(B));
    int64_t next = 0;
    const int slack = spec_.ext.chunk_slack > 0 ? spec_.ext.chunk_slack : 4;
    const int slots = graph_slots_ > 0 ? graph_slots_ : chunk_slots();
    launches_ = 0;

    auto upload_slots = [&]() {
        return check(cudaMemcpyAsync(d_inst_, slot.data(), slot.size() * 8, cudaMemcpyHostToDevice, stream_), "upload") &&
               check(cudaMemcpyAsync(d_mask_, mask.data(), mask.size() * 4, cudaMemcpyHostToDevice, stream_), "upload");
    };
    auto refill = [&]() {
        bool any = false;
        for (int32_t b = 0; b < B; ++b) {
            mask[b] = 0;
            if (slot[b] < 0 && next < N) {
                slot[b] = next++;
                mask[b] = 1;
                any = true;
            }
        }
        if (!any) return true;
        if (!upload_slots()) return false;
        double* dst[5] = {const_cast<double*>(g_.c_orig), const_cast<double*>(g_.rl_orig),
                          const_cast<double*>(g_.ru_orig), const_cast<double*>(g_.xl_orig),
                          const_cast<double*>(g_.xu_orig)};
        for (int k = 0; k < 5; ++k) {
            const bool cols = k == 0 || k >= 3;
            launch_gather_slots(src[k], fam_[k], dst[k], cols ? d_col_perm_ : d_row_perm_, d_inst_, d_mask_,
                                lens[k], B, stream_);
        }
        Global gm = g_;
        gm.slot_mask = d_mask_;
        gm.warm_x = nullptr;
        gm.warm_y = nullptr;
        if (swx) {
            launch_gather_slots(swx, nullptr, warm_x_, d_col_perm_, d_inst_, d_mask_, n, B, stream_);
            gm.warm_x = warm_x_;
        }
        if (swy) {
            launch_gather_slots(swy, nullptr, warm_y_, d_row_perm_, d_inst_, d_mask_, m, B, stream_);
            gm.warm_y = warm_y_;
        }
        if (sww) launch_gather_slots(sww, nullptr, warm_w_, d_zero_perm_, d_inst_, d_mask_, 1, B, stream_);
        launch_norm_parts(gm, stream_);
        launch_init_ctl(gm, dopt_, B, mixed_ ? 1 : 0, warm ? 1 : 0, sww ? warm_w_ : nullptr,
                        session_eta_max_, o.initial_primal_weight, family_.objective_offset, stream_);
        launch_setup_vectors<double>(gm, w64_, stream_);
        if (mixed_) launch_setup_vectors<float>(gm, w32_, stream_);
        const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
        (void)elapsed;
        launch_stamp_clock(gm, B, 0, deadline_ns_of(o.time_limit_seconds), stream_);
        if (mixed_) launch_refresh<float>(g_, w32_, dopt_, tuning_.vector_width, stream_);
        launch_refresh<double>(g_, w64_, dopt_, tuning_.vector_width, stream_);
        enqueue_check_stage();
        launches_ += 12;
        if (il_) {
            il_move_statics(kIlMasked, d_mask_);
            il_move_iterates(false, kIlMasked, d_mask_);
            launches_ += 2;
        }
        return check(cudaGetLastError(), "refill");
    };
    auto harvest = [&]() {
        bool any = false;
        for (int32_t b = 0; b < B; ++b) {
            mask[b] = (done[b] && slot[b] >= 0) ? 1 : 0;
            any = any || mask[b];
        }
        if (!any) return true;
        if (!upload_slots()) return false;
        if (dox) launch_scatter_slots(g_.best_x, dox, d_col_perm_, d_inst_, d_mask_, n, B, stream_);
        if (doy) launch_scatter_slots(g_.best_y, doy, d_row_perm_, d_inst_, d_mask_, m, B, stream_);
        if (!check(cudaMemcpyAsync(ctl.data(), g_.ctl, ctl.size() * sizeof(InstanceCtl), cudaMemcpyDeviceToHost, stream_), "download") ||
            !check(cudaStreamSynchronize(stream_), "harvest"))
            return false;
        for (int32_t b = 0; b < B; ++b) {
            if (!mask[b]) continue;
            const InstanceCtl& c = ctl[static_cast<size_t>(b)];
            const int64_t i = slot[b];
            if (status) status[i] = c.status;
            if (iterations) iterations[i] = c.iteration;
            if (stats) {
                double* st = stats + 8 * i;
                st[0] = c.best_pobj; st[1] = c.best_dobj; st[2] = c.best_pres; st[3] = c.best_dres;
                st[4] = c.best_gap; st[5] = static_cast<double>(c.step_trials); st[6] = c.omega;
                st[7] = static_cast<double>(c.restart_count);
            }
            slot[b] = -1;
        }
        return true;
    };

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream_);
    timing_reset();
    bool ok = refill();
    const int64_t trials_bound =
        (std::max<int64_t>(o.iteration_limit, 0) + std::max(o.polishing_iterations, 0) + 2) *
        std::max(o.maximum_step_trials, 1);
    const int64_t max_chunks = (trials_bound / std::max(1, slots - slack) + 64) * ((N + B - 1) / B + 1);
    int64_t chunks = 0;
    while (ok) {
        launch_slot_done(g_, B, d_done_, stream_);
        ok = check(cudaMemcpyAsync(done.data(), d_done_, done.size() * 4, cudaMemcpyDeviceToHost, stream_), "poll") &&
             check(cudaMemcpyAsync(h_active_, d_active_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_), "poll") &&
             check(cudaStreamSynchronize(stream_), "poll");
        if (!ok) break;
        if (chunks > 0) timing_collect(slots);
        ok = harvest() && refill();
        if (!ok) break;
        bool active = false;
        for (int32_t b = 0; b < B; ++b) active = active || slot[b] >= 0;
        if (!active && next >= N) break;
        if (++chunks > max_chunks) {
            error_ = "stream exceeded its chunk bound";
            ok = false;
            break;
        }
        ok = launch_chunk(slots);
    }
    cudaEventRecord(e1, stream_);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    device_seconds_ = 1e-3 * ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ok && !on_device) {
        if (out_x) ok = check(cudaMemcpyAsync(out_x, dox, static_cast<size_t>(N * n) * 8, cudaMemcpyDeviceToHost, stream_), "download");
        if (ok && out_y) ok = check(cudaMemcpyAsync(out_y, doy, static_cast<size_t>(N * m) * 8, cudaMemcpyDeviceToHost, stream_), "download");
        ok = ok && check(cudaStreamSynchronize(stream_), "download");
    }
    return ok;
}

}  // namespace pdlpgpu

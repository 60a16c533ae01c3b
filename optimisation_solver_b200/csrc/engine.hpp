// engine.hpp -- host side of the device PDLP engine.
#pragma once

#include "interleaved.cuh"
#include "kernels.cuh"
#include "layout.hpp"
#include "pdlpgpu.h"

#include <chrono>
#include <string>
#include <vector>

namespace pdlpgpu {

struct SolveSpec {
    std::vector<const pdlpgpu_lp*> lps;   // one per instance
    bool shared_matrix = false;           // every instance uses lps[0]'s matrix
    pdlpgpu_options opt{};
    pdlpgpu_ext_options ext{};
    std::vector<const pdlpgpu_warmstart*> warm;   // empty or one (nullable) per instance
    // Component tests: the LP is used as the working problem (no Ruiz pass),
    // and the caller may supply the preconditioner.
    bool working_given = false;
    const double* given_tau = nullptr;
    const double* given_sigma = nullptr;
};

// Device-side arrays of one batch. All live in one allocation.
class Engine {
public:
    explicit Engine(int device);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Host validation, layout and upload (prepare), then control state, the
    // setup kernels and the initial check (start). Returns false on a setup
    // failure (error()); invalid instances are recorded per instance.
    bool prepare(const SolveSpec& spec);
    bool start();
    bool setup(const SolveSpec& spec) { return prepare(spec) && start(); }
    // The iteration loop, to completion of every instance.
    bool run();
    // One result per instance of the spec (invalid ones included).
    void results(std::vector<pdlpgpu_result*>& out);

    const std::string& error() const { return error_; }
    double device_seconds() const { return device_seconds_; }
    int64_t launches() const { return launches_; }

    // --- sessions: one shared matrix, repeated batched solves --------------
    bool session_create(const pdlpgpu_lp& family, int32_t batch, const pdlpgpu_options& opt,
                        const pdlpgpu_ext_options& ext);
    bool session_load(bool on_device, const double* c, const double* rl, const double* ru,
                      const double* xl, const double* xu, const double* wx, const double* wy,
                      const double* ww);
    bool session_solve(int32_t* optimal);
    bool session_read(bool on_device, double* primal, double* dual, int32_t* status,
                      int64_t* iterations, double* stats);
    bool time_kernels(int reps, double* out);
    // Solves N instances through the session's slots, refilling each slot with
    // the next instance as soon as its instance finishes.
    bool session_stream(bool on_device, int64_t N, const double* const in[5], const double* wx,
                        const double* wy, const double* ww, double* out_x, double* out_y,
                        int32_t* status, int64_t* iterations, double* stats);
    int32_t count() const { return count_; }
    // Live durations over the last solve or stream, from CUDA events captured
    // in the iteration graph around the two kernels of four trial slots of
    // every chunk (first, second, middle, last): out[15] = {primal ms per
    // launch, dual ms per launch, samples, chunk ms, chunks, device seconds of
    // the loop, check-stage ms per chunk, then primal and dual ms at each of
    // the four positions}.
    void loop_timing(double* out) const;

    // --- component tests (single instance, internal order handled here) ---
    bool component_spmv(int transpose, int values, const double* in, double* out);
    bool component_ruiz(double* row_scale, double* col_scale, double* scaled_csr);
    bool component_precondition(double* tau, double* tau_inv, double* sigma, double* sigma_inv);
    bool component_trial(const double* tau, const double* tau_inv, const double* sigma,
                         const double* sigma_inv, const double* x, const double* y,
                         const double* ax, double step, double weight, double* x_out,
                         double* y_out, double* ax_out, double* reductions);
    bool component_evaluate(const double* x, const double* y, const double* rx, const double* ry,
                            double* metrics, double* verdicts);

private:
    template <class T> void enqueue_trial(const Work<T>& w);
    template <class T> void enqueue_check(const Work<T>& w);
    void enqueue_chunk(int slots, bool fp64_stage);
    // One chunk: the captured graph with or without the FP64 trial kernels,
    // as the last poll's count of FP64-stage instances asks.
    bool launch_chunk(int slots);
    // The check stage; with `il_sync` the iterates of the instances at a
    // check are moved out of the interleaved layout first and back after.
    void enqueue_check_stage(bool il_sync = false);
    int check_stage_launches(bool il_sync) const;
    int chunk_slots() const;
    // --- batch-interleaved layout (sessions)
    template <class T> bool il_build(Interleaved<T>& il, const Work<T>& w);
    void il_set_family(int32_t family);
    template <class T> IlMove<T> il_iterates(const Interleaved<T>& il, const Work<T>& w,
                                             bool to_planar, int select, const int32_t* mask) const;
    template <class T> IlMove<T> il_statics(const Interleaved<T>& il, const Work<T>& w, int select,
                                            const int32_t* mask) const;
    void il_move_iterates(bool to_planar, int select, const int32_t* mask);
    void il_move_statics(int select, const int32_t* mask);
    bool check(cudaError_t e, const char* what);
    // Host-to-device copy of consecutive host pieces into dst (stream order).
    struct HostPiece {
        const void* src;
        size_t bytes;
    };
    bool upload(void* dst, const std::vector<HostPiece>& pieces);
    bool upload(void* dst, const void* src, size_t bytes) { return upload(dst, {{src, bytes}}); }
    // Device-to-host copy, complete on return.
    bool download(void* dst, const void* src, size_t bytes);
    bool ensure_pinned();
    // Host phases of a solve, with PDLPGPU_TRACE=1 in the environment: the
    // seconds since the solve began at the end of each phase, printed to
    // stderr once the results are assembled.
    void mark(const char* phase);
    std::vector<std::pair<const char*, double>> trace_;
    bool build_graph(int slots, bool fp64_stage);
    bool ensure_graph();
    bool power_iteration();
    bool setup_kernels();
    bool init_control();
    template <class V> void to_internal_cols(const V* src, std::vector<V>& dst, int instance) const;
    template <class V> void to_internal_rows(const V* src, std::vector<V>& dst, int instance) const;

    int device_ = 0;
    int sms_ = 148;
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;     // chunk with the working precision's trial kernels
    cudaGraphExec_t graph64_ = nullptr;   // mixed: plus the FP64-stage trial kernels
    int graph_slots_ = 0;
    char* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    std::string error_;
    std::chrono::steady_clock::time_point t0_;

    // spec-derived
    SolveSpec spec_;
    bool mixed_ = false;
    Tuning tuning_;
    int32_t count_ = 0;                  // device instances
    std::vector<int32_t> device_of_;     // spec instance -> device instance or -1
    std::vector<std::string> invalid_;   // per spec instance: message if invalid
    std::vector<MatrixLayout> layouts_;  // per device instance (one when shared)
    std::vector<InstanceInfo> info_;
    int64_t rows_total_ = 0, cols_total_ = 0;
    int64_t a_slots_ = 0, at_slots_ = 0;
    int32_t a_slices_ = 0, at_slices_ = 0;
    std::vector<CtaWork> a_ctas_, at_ctas_;
    std::vector<VecWork> vec_;
    int first_a_ctas_ = 0, first_at_ctas_ = 0, first_vec_ = 0;
    HostCsr csr0_;                       // canonical A of instance 0 (component tests)

    // device
    Global g_{};
    Work<double> w64_{};
    Work<float> w32_{};
    DeviceOptions dopt_{};
    double* a_s64_ = nullptr;
    double* at_s64_ = nullptr;
    float* a_s32_ = nullptr;
    float* at_s32_ = nullptr;
    int32_t* d_active_ = nullptr;     // [2]: unfinished instances, those in the FP64 stage
    int32_t* h_active_ = nullptr;     // pinned copy
    // two pinned staging buffers of large uploads and their last copies
    char* pinned_[2] = {nullptr, nullptr};
    cudaEvent_t pinned_done_[2] = {nullptr, nullptr};
    double device_seconds_ = 0.0;
    int64_t launches_ = 0;
    bool ran_ = false;
    bool setup_ok_ = false;
    // session state
    std::vector<void*> extra_;              // device allocations beyond the arena
    int32_t* d_row_perm_ = nullptr;
    int32_t* d_col_perm_ = nullptr;
    double* fam_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // c, rl, ru, xl, xu (internal)
    double* warm_x_ = nullptr;
    double* warm_y_ = nullptr;
    double* warm_w_ = nullptr;
    bool session_warm_ = false;
    bool session_has_ww_ = false;
    double session_eta_max_ = 0.99;
    int64_t* d_inst_ = nullptr;       // stream: instance in each slot
    int32_t* d_mask_ = nullptr;       // stream: slots being refilled / harvested
    int32_t* d_done_ = nullptr;       // stream: finished flags
    int32_t* d_zero_perm_ = nullptr;  // {0}: identity permutation of length 1
    pdlpgpu_lp family_{};
    // batch-interleaved layout of the trial kernels (sessions)
    bool il_ = false;
    // Fused trials (k_fused): CTAs per cluster, 0 when the chunks launch two
    // kernels per trial slot. Chosen by choose_fused() for one-LP solves and
    // small batches.
    int fused_cluster_ = 0;
    FusedShape fused_shape32_{}, fused_shape64_{};   // shared memory of the FP32 / FP64 fused launches
    void choose_fused();
    Interleaved<float> il32_{};
    Interleaved<double> il64_{};
    int32_t il_family_ = (1 << kIlVecs) - 1;   // vectors every instance takes from the family
    int32_t graph_family_ = -1;                // il_family_ captured in graph_
    // live timing events of the chunk: [0] start, [1] end of the trial slots,
    // [2] end; then for each sampled slot position p (first, second, middle,
    // last): [3 + 3p] trial start, [4 + 3p] between the halves, [5 + 3p] end
    static constexpr int kTimedSlots = 4;
    cudaEvent_t tev_[3 + 3 * kTimedSlots] = {};
    // Orders the session's stream after the caller's work on the legacy
    // default stream before device-pointer inputs are read.
    bool wait_for_caller();
    cudaEvent_t caller_done_ = nullptr;
    double t_primal_[kTimedSlots] = {}, t_dual_[kTimedSlots] = {};
    double t_chunk_ = 0.0, t_check_ = 0.0;
    int64_t t_samples_ = 0, t_chunks_ = 0;
    void timing_reset();
    void timing_collect(int slots);
    void record_timing(int k);
    int timed_position(int k, int slots) const;
};

const char* message_text(int32_t id);

}  // namespace pdlpgpu

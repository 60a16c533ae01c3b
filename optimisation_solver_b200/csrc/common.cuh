// common.cuh -- structures shared by the host engine and the device kernels.
//
// Device layout of a batch of B >= 1 LPs (one LP is a batch of one):
//
//   * Rows of every instance are renumbered by decreasing length and columns by
//     decreasing degree, so that rows of similar length sit together. All
//     per-row vectors (y, A x, bounds, sigma, ...) live in that internal order,
//     instance after instance ("row space", R = sum m_b entries); likewise the
//     per-column vectors ("column space", N = sum n_b).
//   * A is stored twice in a sliced-ELL layout with per-slice lane groups
//     (called SELL-G here): the A side (one line per row, gathers from the
//     column space) and the A^T side (one line per column, gathers from the row
//     space). A slice is 32 lanes covering 32/G lines of G lanes each; lane g of
//     a line owns its entries g, g+G, g+2G, ... Step s of a slice is one
//     coalesced 32-element load; steps are grouped by the vector width V so
//     each lane loads V consecutive entries (128-bit loads at V=4 for FP32).
//     Column indices are local to the instance, so one A can serve every
//     instance of a shared-matrix batch.
//   * A CTA works on a contiguous range of slices of exactly one instance, so
//     per-instance reductions never need atomics: every CTA writes its own
//     partial, and the last CTA of the instance (an arrival counter) combines
//     them in a fixed order. Runs are therefore bitwise reproducible.
#pragma once

#include <cstddef>
#include <cstdint>

namespace pdlpgpu {

constexpr int kWarps = 8;              // warps per CTA in the SpMV-shaped kernels
constexpr int kThreads = kWarps * 32;
constexpr int kVecChunk = 2048;        // elements per CTA in the elementwise kernels

struct SliceDesc {
    int32_t data_off;   // slice data offset in units of 32 elements
    int32_t line0;      // first line of the slice, local to the instance
    int32_t steps;      // padded step count (multiple of the vector width)
    int32_t meta;       // bits 0-7: log2(G); bits 8-15: lines in the slice
};

struct CtaWork {
    int32_t instance;
    int32_t slice_begin;
    int32_t slice_end;
    int32_t pad;
};

struct VecWork {        // elementwise CTA: [begin, end) of one instance, rows or columns
    int32_t instance;
    int32_t is_row;
    int32_t begin;      // local index
    int32_t end;
};

struct InstanceInfo {
    int32_t m, n;
    int64_t row_off, col_off;          // offsets into the row / column spaces
    int64_t a_data_base;               // element offset of the instance's A-side slice data
    int64_t at_data_base;              // ... A^T side
    int32_t a_cta_begin, a_cta_end;    // CTA ranges in the SpMV maps
    int32_t at_cta_begin, at_cta_end;
    int32_t vec_cta_begin, vec_cta_end;  // CTA range in the elementwise map
    int32_t a_slice_base, at_slice_base; // slice index bases (slices of one instance are contiguous)
    int64_t a_len_base, at_len_base;     // index base of the line lengths (row_off/col_off, or 0 when shared)
};

// Per-instance scalar state of the solve; one writer at a time (the last CTA
// of the instance in the kernel that owns the decision). The first 64 bytes
// hold what every trial kernel reads at entry, so it is fetched with three
// 16-byte loads.
struct alignas(64) InstanceCtl {
    // --- hot block (64 bytes)
    double trial_eta, trial_omega;   // step and weight of the next trial
    double avg_frac;                 // fraction owed by the pending update
    int32_t phase;          // kPhaseMain / kPhasePolish / kPhaseDone
    int32_t stage;          // kStageTrial / kStageCheck
    int32_t pending_avg;    // average update owed for the current iterate
    int32_t fp64_stage;     // mixed solves: 1 once the FP64 stage has started
    int32_t ibuf;           // interleaved layout: buffer holding the committed iterate
    int32_t parity;         // current iterate lives in buffer [parity]
    int32_t check_kind;     // kCheckInitial / kCheckMain / kCheckPolish
    int32_t trials_this_iter;
    int32_t hot_pad[2];
    // --- control flow
    int32_t status;         // final status once phase == done
    int32_t message;        // message id
    int32_t restart_count;
    int32_t ray_kind;       // 1 dual (Farkas) ray, 2 primal ray
    int32_t diagnostics;    // stamp final step/weight into the result
    int32_t limit_status;
    // apply flags set by the check control, consumed by apply/refresh
    int32_t best_src;       // 0 none, 1 current, 2 average
    int32_t restart_src;    // 0 none, 1 current, 2 average (average copies avg into x)
    int32_t need_refresh;   // recompute A x for the current iterate
    int32_t to_polish;      // load best point into the iterate, in working coordinates
    int32_t save_ray;       // copy the ray scratch to the ray buffers
    int32_t have_avg_at_check;
    int32_t stall_checks;
    int32_t il_sync;        // interleaved layout: the iterate was copied out for a check
    int32_t to_fp64;        // mixed: the check moves the instance to the FP64 stage
    // --- counters
    int64_t iteration;       // main phase: committed iterations (state.iteration)
    int64_t step_trials;     // main phase trials
    int64_t since_restart;
    int64_t polish_iteration;
    int64_t polish_trials;
    int64_t polish_done_iterations;  // result.iterations of the polisher
    int64_t fp64_iterations;
    int64_t deadline_ns;     // 0 = none
    int64_t start_ns;
    int64_t polish_deadline_ns;
    // --- step control (main controller, polishing controller, trial step)
    double eta, omega, eta_max;
    double ctl_eta, ctl_omega;
    // --- averaging
    double avg_weight;       // total weight W
    // --- restart state
    double restart_baseline;
    double prev_candidate;
    double best_kkt_at_stall;
    // --- metrics of the best point
    double best_pobj, best_dobj, best_pres, best_dres, best_gap, best_kkt;
    int32_t best_finite, best_valid;
    // --- problem normalisers (original problem)
    double pnorm, dnorm;
    double objective_offset;
    // --- last trial reductions and ray verdicts (diagnostics and component tests)
    double dbg[12];
};

static_assert(offsetof(InstanceCtl, hot_pad) + 8 == 64, "hot block of InstanceCtl is 64 bytes");
static_assert(offsetof(InstanceCtl, ibuf) == 40, "trial kernels read the hot block by offset");

enum : int32_t { kPhaseMain = 0, kPhasePolish = 1, kPhaseDone = 2 };
enum : int32_t { kStageTrial = 0, kStageCheck = 1 };
enum : int32_t {
    kCheckInitial = 0,
    kCheckMain = 1,
    kCheckPolish = 2,
    kCheckTransition = 3,
    kCheckEvaluate = 4   // component test: metrics and ray verdicts of the current point only
};

enum : int32_t {
    kMsgNone = 0,
    kMsgInitialOptimal,
    kMsgNonFinite,
    kMsgLinesearch,
    kMsgInfeasible,
    kMsgUnbounded,
    kMsgOptimal,
    kMsgPolishOptimal,
    kMsgIterationLimit,
    kMsgTimeLimit,
    kMsgCount
};

// Options the device control needs, copied once per solve.
struct DeviceOptions {
    int64_t iteration_limit;
    int32_t check_frequency;
    int32_t max_trials;
    int32_t adaptive;
    int32_t averaging;
    int32_t restarts;
    int32_t detect_infeasibility;
    int32_t polishing;
    int32_t polishing_iterations;
    int32_t min_restart;
    int32_t max_restart;
    int32_t mixed;             // iterations in FP32 first
    int32_t fp32_stall_checks;
    double fp32_switch_kkt;    // mixed: stalls count once the best KKT score is at most this
    double primal_tol, dual_tol, gap_tol;
    double min_step_scale;
    double w_min, w_max, smoothing;
    double initial_step_safety;
    double sufficient, necessary, artificial;
    double infeasibility_tol;
    double time_limit;
    // The linesearch's step factors by iteration index k: step_pow[2k] =
    // (k + 2)^-0.3 and step_pow[2k + 1] = (k + 2)^-0.6, computed on the
    // device with the same pow (step_controller.cpp:30-68 needs them at
    // every trial); indices past step_pow_entries compute them directly.
    const double* step_pow;
    int64_t step_pow_entries;
    // 1: restarts compare normalised duality gaps instead of KKT errors.
    int32_t ndg_restarts;
};

// Partial sums per elementwise CTA of a check (slot meaning depends on side).
constexpr int kPrepSlots = 10;
// Partial sums per SpMV CTA of a check.
constexpr int kCheckSlots = 6;

__host__ __device__ inline int slice_glog(int32_t meta) { return meta & 0xff; }
__host__ __device__ inline int slice_lines(int32_t meta) { return (meta >> 8) & 0xff; }

}  // namespace pdlpgpu

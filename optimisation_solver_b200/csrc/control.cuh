// control.cuh -- per-instance scalar decisions of the PDLP loop, executed on
// the device by one thread (the last CTA of an instance in the kernel that
// owns the decision). Each routine restates the reference's host logic:
//
//   evaluate_step     StepController::evaluateTrial   step_controller.cpp:30-68
//   set_weight        StepController::setPrimalWeight :70-78
//   update_weight     StepController::updatePrimalWeight :80-98
//   restart_choose    RestartController::choose       restart_controller.cpp:8-63
//   is_optimal        TerminationChecker::isOptimal   termination.cpp:327-333
//   trial_control     the linesearch loop and commit  pdlp_solver.cpp:287-352
//   end_main_loop     loop exit and polishing entry   pdlp_solver.cpp:479-547
//   the polishing loop                                feasibility_polishing.cpp:31-145
#pragma once

#include "common.cuh"

#include <cmath>

namespace pdlpgpu {

__device__ __forceinline__ int64_t now_ns() {
    int64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// std::clamp: NaN passes through.
__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}
// std::min / std::max argument order.
template <class T> __device__ __forceinline__ T smin(T a, T b) { return b < a ? b : a; }
template <class T> __device__ __forceinline__ T smax(T a, T b) { return a < b ? b : a; }

// `factors`, when given, holds step_pow[2k] and step_pow[2k + 1] of this
// iteration index, loaded by the caller ahead of the decision.
__device__ inline bool evaluate_step(double& eta, double omega, double eta_max,
                                     const DeviceOptions& o, double pmove, double dmove,
                                     double inter, int64_t iteration, const double* factors = nullptr) {
    const double movement = omega * pmove + dmove / omega;
    const double coupling = fabs(inter);
    double limit = INFINITY;
    if (coupling > 0.0 && movement > 0.0) limit = movement / (2.0 * coupling);
    const double index = static_cast<double>(iteration) + 2.0;
    double p3, p6;
    if (factors) {
        p3 = factors[0];
        p6 = factors[1];
    } else if (iteration >= 0 && iteration < o.step_pow_entries) {
        p3 = o.step_pow[2 * iteration];
        p6 = o.step_pow[2 * iteration + 1];
    } else {
        p3 = pow(index, -0.3);
        p6 = pow(index, -0.6);
    }
    const double shrink = 1.0 - p3;
    const double grow = 1.0 + p6;
    const bool accepted = eta <= limit;
    double next = smin(shrink * limit, grow * eta);
    next = clampd(next, o.min_step_scale * eta_max, 1e12);
    if (!isfinite(next) || next <= 0.0) next = eta;
    eta = next;
    return accepted;
}

__device__ inline void set_weight(double& omega, const DeviceOptions& o, double w) {
    if (w > 0.0 && isfinite(w)) omega = clampd(w, o.w_min, o.w_max);
}

__device__ inline void update_weight(double& omega, const DeviceOptions& o, double pdist,
                                     double ddist) {
    if (pdist <= 1e-16 || ddist <= 1e-16 || !isfinite(pdist) || !isfinite(ddist)) return;
    const double target = clampd(ddist / pdist, 1e-12, 1e12);
    const double sm = clampd(o.smoothing, 0.0, 1.0);
    set_weight(omega, o, exp(sm * log(target) + (1.0 - sm) * log(omega)));
}

struct Metrics {
    double pobj, dobj, pres, dres, gap, kkt;
    bool finite, valid;
};

__device__ inline Metrics make_metrics(const InstanceCtl& c, double viol2, double support,
                                       double rinf2, double obj, double infimum, double cinf2) {
    Metrics m;
    m.pres = sqrt(viol2) / c.pnorm;
    m.dres = sqrt(cinf2 + rinf2) / c.dnorm;
    m.pobj = c.objective_offset + obj;
    m.dobj = c.objective_offset + infimum - support;
    m.finite = isfinite(m.pobj) && isfinite(m.dobj) && isfinite(m.pres) && isfinite(m.dres);
    if (!m.finite) {
        m.valid = false;
        m.gap = INFINITY;
        m.kkt = INFINITY;
        return m;
    }
    m.valid = true;
    m.gap = fabs(m.pobj - m.dobj) / (1.0 + fabs(m.pobj) + fabs(m.dobj));
    m.kkt = smax(smax(m.pres, m.dres), m.gap);
    return m;
}

__device__ inline bool is_optimal_best(const InstanceCtl& c, const DeviceOptions& o) {
    return c.best_finite && c.best_valid && c.best_pres <= o.primal_tol &&
           c.best_dres <= o.dual_tol && c.best_gap <= o.gap_tol;
}

__device__ inline void store_best(InstanceCtl& c, const Metrics& m) {
    c.best_pobj = m.pobj; c.best_dobj = m.dobj; c.best_pres = m.pres;
    c.best_dres = m.dres; c.best_gap = m.gap; c.best_kkt = m.kkt;
    c.best_finite = m.finite; c.best_valid = m.valid;
}

__device__ inline void finish(InstanceCtl& c, int32_t status, int32_t message, bool diagnostics) {
    c.phase = kPhaseDone;
    c.status = status;
    c.message = message;
    c.diagnostics = diagnostics ? 1 : 0;
    c.stage = kStageTrial;
}

// Polishing is over (feasibility_polishing.cpp returns): the caller keeps the
// better point, which is already in the best buffers (pdlp_solver.cpp:518-547).
__device__ inline void end_polish(InstanceCtl& c, const DeviceOptions& o) {
    if (is_optimal_best(c, o)) {
        c.iteration += c.polish_done_iterations;
        c.step_trials += c.polish_trials;
        finish(c, 0 /* optimal */, kMsgPolishOptimal, true);
    } else {
        finish(c, c.limit_status, c.limit_status == 4 ? kMsgTimeLimit : kMsgIterationLimit, true);
    }
}

// The main loop has exhausted its iteration or time budget
// (pdlp_solver.cpp:479-547). Either finish, or set up polishing: its start
// point is the best point mapped to working coordinates, its step is half the
// current one, and it gets a fresh step controller sharing only omega
// (feasibility_polishing.cpp:31-43).
__device__ inline void end_main_loop(InstanceCtl& c, const DeviceOptions& o, int32_t limit_status,
                                     int32_t n_cols) {
    c.limit_status = limit_status;
    if (o.polishing && o.polishing_iterations > 0 && n_cols > 0) {
        double remaining = 0.0;
        if (o.time_limit > 0.0) {
            remaining = o.time_limit - 1e-9 * static_cast<double>(now_ns() - c.start_ns);
            if (remaining <= 0.0) {
                finish(c, limit_status, limit_status == 4 ? kMsgTimeLimit : kMsgIterationLimit, true);
                return;
            }
        }
        c.phase = kPhasePolish;
        c.to_polish = 1;
        c.need_refresh = 1;
        c.stage = kStageCheck;
        c.check_kind = kCheckTransition;
        c.ctl_eta = clampd(o.initial_step_safety * c.eta_max, o.min_step_scale * c.eta_max, c.eta_max);
        c.ctl_omega = 1.0;
        set_weight(c.ctl_omega, o, c.omega);
        c.trial_eta = c.eta * 0.5;
        c.trial_omega = c.omega;
        c.polish_iteration = 0;
        c.polish_done_iterations = 0;
        c.polish_trials = 0;
        c.avg_weight = 0.0;
        c.pending_avg = 0;
        c.trials_this_iter = 0;
        c.polish_deadline_ns =
            remaining > 0.0 ? now_ns() + static_cast<int64_t>(remaining * 1e9) : 0;
        return;
    }
    finish(c, limit_status, limit_status == 4 ? kMsgTimeLimit : kMsgIterationLimit, true);
}

// Top of the main loop (pdlp_solver.cpp:277-285): the iteration bound, then
// the time limit; otherwise the next iteration's trials start.
__device__ inline void loop_top_main(InstanceCtl& c, const DeviceOptions& o, int32_t n_cols) {
    if (c.iteration >= o.iteration_limit) {
        end_main_loop(c, o, 3 /* iteration_limit */, n_cols);
        return;
    }
    if (o.time_limit > 0.0 && c.deadline_ns > 0 && now_ns() >= c.deadline_ns) {
        end_main_loop(c, o, 4 /* time_limit */, n_cols);
        return;
    }
    c.stage = kStageTrial;
}

// k % q (q > 0, validated at setup) in 32-bit arithmetic while k fits: the
// same value at a fraction of a 64-bit remainder's cost.
__device__ __forceinline__ int64_t count_mod(int64_t k, int32_t q) {
    if (k >= 0 && k <= 0x7fffffff) return static_cast<int32_t>(k) % q;
    return k % q;
}

__device__ inline void average_add(InstanceCtl& c, double weight) {   // iterate_average.cpp:40-82
    if (!(weight > 0.0)) return;
    const double total = c.avg_weight + weight;
    c.avg_frac = weight / total;
    c.avg_weight = total;
    c.pending_avg = 1;
}

// A control block copied by one warp as 16-byte words (either side may be
// shared or global memory).
__device__ __forceinline__ void copy_ctl_warp(InstanceCtl* dst, const InstanceCtl* src) {
    static_assert(sizeof(InstanceCtl) % 16 == 0 && sizeof(InstanceCtl) / 16 <= 32,
                  "one 16-byte word per lane");
    const int lane = threadIdx.x & 31;
    if (lane < static_cast<int>(sizeof(InstanceCtl) / 16))
        reinterpret_cast<int4*>(dst)[lane] = reinterpret_cast<const int4*>(src)[lane];
}

// After the two halves of one trial: finiteness test, linesearch decision,
// commit, averaging and the check boundary.
// `factors`: the linesearch's step factors of the trial's iteration index
// (evaluate_step), or null to read them from the options' table.
inline __device__ __noinline__ void trial_control(InstanceCtl& c, const DeviceOptions& o, double pmove,
                                     double dmove, double inter, int32_t n_cols,
                                     const double* factors = nullptr) {
    c.pending_avg = 0;
    c.dbg[0] = pmove;
    c.dbg[1] = dmove;
    c.dbg[2] = inter;
    const bool polishing = c.phase == kPhasePolish;
    if (polishing) ++c.polish_trials; else ++c.step_trials;
    const bool finite = isfinite(pmove) && isfinite(dmove) && isfinite(inter);
    if (!finite) {
        if (polishing) end_polish(c, o);
        else finish(c, 5 /* numerical_failure */, kMsgNonFinite, true);
        return;
    }
    bool accept;
    if (!polishing) {
        accept = !o.adaptive ||
                 evaluate_step(c.eta, c.omega, c.eta_max, o, pmove, dmove, inter, c.iteration, factors);
        c.trial_eta = c.eta;
        c.trial_omega = c.omega;
    } else if (!o.adaptive) {
        accept = true;
    } else {
        accept = evaluate_step(c.ctl_eta, c.ctl_omega, c.eta_max, o, pmove, dmove, inter,
                               c.polish_iteration, factors);
        c.trial_eta = c.ctl_eta;
    }
    if (!accept) {
        ++c.trials_this_iter;
        if (c.trials_this_iter >= o.max_trials) {
            if (polishing) end_polish(c, o);
            else finish(c, 5, kMsgLinesearch, true);
        }
        return;
    }
    c.parity ^= 1;
    c.trials_this_iter = 0;
    if (c.fp64_stage && o.mixed) ++c.fp64_iterations;
    if (!polishing) {
        ++c.iteration;
        ++c.since_restart;
        if (o.averaging) average_add(c, c.eta);
        if (count_mod(c.iteration, o.check_frequency) == 0) {
            c.stage = kStageCheck;
            c.check_kind = kCheckMain;
        } else {
            loop_top_main(c, o, n_cols);
        }
    } else {
        ++c.polish_iteration;
        ++c.polish_done_iterations;
        if (o.averaging) average_add(c, c.trial_eta);
        const bool last = c.polish_done_iterations == o.polishing_iterations;
        if (count_mod(c.polish_done_iterations, o.check_frequency) == 0 || last) {
            c.stage = kStageCheck;
            c.check_kind = kCheckPolish;
        }
    }
}

// The instance runs trial kernels of working precision T now.
template <class T>
__device__ __forceinline__ bool precision_matches(const InstanceCtl& c) {
    return (c.fp64_stage != 0) == (sizeof(T) == 8);
}

template <class T>
__device__ __forceinline__ bool trial_active(const InstanceCtl& c) {
    return c.phase != kPhaseDone && c.stage == kStageTrial && precision_matches<T>(c);
}

// Smallest dual step of the trial (a zero step would stall the prox).
template <class T> __device__ __forceinline__ T min_dual_step();
template <> __device__ __forceinline__ double min_dual_step<double>() { return 1e-300; }
template <> __device__ __forceinline__ float min_dual_step<float>() { return 1e-37f; }

// RestartController::choose (restart_controller.cpp:8-63). Returns 0 none,
// 1 current, 2 average; candidate score through `score`.
__device__ inline int restart_choose(InstanceCtl& c, const DeviceOptions& o, double cur_kkt,
                                     double avg_kkt, double* score) {
    *score = INFINITY;
    if (!o.restarts || c.since_restart < o.min_restart) return 0;
    const bool af = isfinite(avg_kkt), cf = isfinite(cur_kkt);
    if (!af && !cf) return 0;
    int cand = 2;
    double s = avg_kkt;
    if (!af || (cf && cur_kkt < avg_kkt)) {
        cand = 1;
        s = cur_kkt;
    }
    *score = s;
    const double prev = c.prev_candidate;
    c.prev_candidate = s;
    const double base = c.restart_baseline;
    const bool bf = isfinite(base);
    if (bf && s <= o.sufficient * base) return cand;
    if (bf && s <= o.necessary * base && isfinite(prev) && s > prev) return cand;
    int64_t art = static_cast<int64_t>(o.artificial * static_cast<double>(c.iteration));
    if (art < 1) art = 1;
    if (c.since_restart >= art || c.since_restart >= o.max_restart) return cand;
    return 0;
}

}  // namespace pdlpgpu

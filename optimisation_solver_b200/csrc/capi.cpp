// capi.cpp -- extern "C" entry points of libpdlpgpu (include/pdlpgpu.h and
// include/pdlpgpu_components.h). Every call catches everything: nothing
// throws across the C boundary (the reference's solve never throws either,
// pdlp_engine/src/pdlp_solver.cpp:116-134).
#include "engine.hpp"
#include "pdlpgpu.h"
#include "pdlpgpu_components.h"
#include "pdlpgpu_session.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& e) { g_last_error = e; }

pdlpgpu_ext_options ext_or_default(const pdlpgpu_ext_options* ext) {
    pdlpgpu_ext_options e;
    pdlpgpu_default_ext_options(&e);
    if (ext != nullptr) e = *ext;
    return e;
}

pdlpgpu_options opt_or_default(const pdlpgpu_options* o) {
    pdlpgpu_options d;
    pdlpgpu_default_options(&d);
    return o != nullptr ? *o : d;
}

pdlpgpu_result* failure_result(const pdlpgpu_lp* lp, const std::string& msg) {
    auto* r = static_cast<pdlpgpu_result*>(std::calloc(1, sizeof(pdlpgpu_result)));
    r->status = PDLPGPU_NUMERICAL_FAILURE;
    std::snprintf(r->status_message, sizeof(r->status_message), "%s", msg.c_str());
    r->num_rows = lp ? lp->num_rows : 0;
    r->num_cols = lp ? lp->num_cols : 0;
    r->primal_objective = std::nan("");
    r->dual_objective = -INFINITY;
    r->primal_residual = r->dual_residual = r->relative_gap = INFINITY;
    r->final_primal_weight = 1.0;
    return r;
}

// Runs a batch and fills results[0..count). Returns the number of OPTIMAL.
int32_t run_batch(const pdlpgpu_lp* const* lps, int32_t count, bool shared,
                  const pdlpgpu_options* options, const pdlpgpu_ext_options* ext,
                  const pdlpgpu_warmstart* const* warm, pdlpgpu_result** results) {
    pdlpgpu::SolveSpec spec;
    spec.lps.assign(lps, lps + count);
    spec.shared_matrix = shared;
    spec.opt = opt_or_default(options);
    spec.ext = ext_or_default(ext);
    if (warm != nullptr) spec.warm.assign(warm, warm + count);
    pdlpgpu::Engine engine(spec.ext.device);
    const bool ok = engine.setup(spec) && engine.run();
    if (!ok) set_error(engine.error());
    std::vector<pdlpgpu_result*> out;
    engine.results(out);
    int32_t optimal = 0;
    for (int32_t i = 0; i < count; ++i) {
        results[i] = out[static_cast<size_t>(i)];
        if (results[i]->status == PDLPGPU_OPTIMAL) ++optimal;
    }
    return ok ? optimal : (optimal > 0 ? optimal : -1);
}

}  // namespace

extern "C" {

void pdlpgpu_default_options(pdlpgpu_options* o) {
    std::memset(o, 0, sizeof(*o));
    o->iteration_limit = 200000;
    o->time_limit_seconds = 0.0;
    o->primal_tolerance = 1e-6;
    o->dual_tolerance = 1e-6;
    o->gap_tolerance = 1e-6;
    o->termination_check_frequency = 100;
    o->power_iteration_count = 100;
    o->thread_count = 0;
    o->parallel_nonzero_threshold = 20000;
    o->initial_step_safety = 0.90;
    o->minimum_step_scale = 1e-6;
    o->maximum_primal_weight = 1e6;
    o->minimum_primal_weight = 1e-6;
    o->use_ruiz_scaling = 1;
    o->ruiz_iterations = 10;
    o->detect_infeasibility = 1;
    o->infeasibility_tolerance = 1e-8;
    o->use_diagonal_preconditioning = 1;
    o->use_adaptive_linesearch = 1;
    o->maximum_step_trials = 60;
    o->use_averaging = 1;
    o->use_restarts = 1;
    o->use_feasibility_polishing = 1;
    o->minimum_restart_iterations = 64;
    o->maximum_restart_iterations = 100000;
    o->restart_sufficient_decay = 0.20;
    o->restart_necessary_decay = 0.80;
    o->restart_artificial_fraction = 0.36;
    o->initial_primal_weight = 1.0;
    o->primal_weight_smoothing = 0.50;
    o->polishing_iterations = 5000;
}

void pdlpgpu_default_ext_options(pdlpgpu_ext_options* e) { std::memset(e, 0, sizeof(*e)); }

int32_t pdlpgpu_solve_ex(const pdlpgpu_lp* lp, const pdlpgpu_options* options,
                         const pdlpgpu_ext_options* ext, const pdlpgpu_warmstart* warm,
                         pdlpgpu_result** result) {
    if (result == nullptr) return PDLPGPU_INVALID_PROBLEM;
    try {
        if (lp == nullptr) {
            *result = failure_result(nullptr, "CompiledLp is null");
            (*result)->status = PDLPGPU_INVALID_PROBLEM;
            return PDLPGPU_INVALID_PROBLEM;
        }
        const pdlpgpu_warmstart* w[1] = {warm};
        run_batch(&lp, 1, false, options, ext, warm ? w : nullptr, result);
        return (*result)->status;
    } catch (const std::exception& e) {
        set_error(e.what());
        *result = failure_result(lp, e.what());
        return (*result)->status;
    } catch (...) {
        *result = failure_result(lp, "unknown error");
        return (*result)->status;
    }
}

int32_t pdlpgpu_solve(const pdlpgpu_lp* lp, const pdlpgpu_options* options,
                      const pdlpgpu_warmstart* warm, pdlpgpu_result** result) {
    return pdlpgpu_solve_ex(lp, options, nullptr, warm, result);
}

int32_t pdlpgpu_solve_batch(const pdlpgpu_lp* const* lps, int32_t count,
                            const pdlpgpu_options* options, const pdlpgpu_ext_options* ext,
                            const pdlpgpu_warmstart* const* warm, pdlpgpu_result** results) {
    if (lps == nullptr || results == nullptr || count < 0) return -1;
    try {
        return run_batch(lps, count, false, options, ext, warm, results);
    } catch (const std::exception& e) {
        set_error(e.what());
        for (int32_t i = 0; i < count; ++i) results[i] = failure_result(lps[i], e.what());
        return -1;
    } catch (...) {
        for (int32_t i = 0; i < count; ++i) results[i] = failure_result(lps[i], "unknown error");
        return -1;
    }
}

int32_t pdlpgpu_batch_time_kernels(const pdlpgpu_lp* const* lps, int32_t count,
                                   const pdlpgpu_options* options, const pdlpgpu_ext_options* ext,
                                   int32_t reps, double* out) {
    if (lps == nullptr || out == nullptr || count <= 0 || reps <= 0) return -1;
    try {
        pdlpgpu::SolveSpec spec;
        spec.lps.assign(lps, lps + count);
        spec.opt = opt_or_default(options);
        spec.ext = ext_or_default(ext);
        pdlpgpu::Engine engine(spec.ext.device);
        if (!engine.setup(spec) || !engine.time_kernels(reps, out)) {
            set_error(engine.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& e) {
        set_error(e.what());
        return -1;
    }
}

void pdlpgpu_result_free(pdlpgpu_result* r) {
    if (r == nullptr) return;
    std::free(r->primal);
    std::free(r->row_dual);
    std::free(r->dual_ray);
    std::free(r->primal_ray);
    std::free(r);
}

const char* pdlpgpu_status_string(int32_t status) {
    switch (status) {
        case PDLPGPU_OPTIMAL: return "optimal";
        case PDLPGPU_INFEASIBLE: return "infeasible";
        case PDLPGPU_UNBOUNDED: return "unbounded";
        case PDLPGPU_ITERATION_LIMIT: return "iteration_limit";
        case PDLPGPU_TIME_LIMIT: return "time_limit";
        case PDLPGPU_NUMERICAL_FAILURE: return "numerical_failure";
        case PDLPGPU_INVALID_PROBLEM: return "invalid_problem";
        default: return "unknown";
    }
}

const char* pdlpgpu_last_error(void) { return g_last_error.c_str(); }

// Lets the other translation units report through pdlpgpu_last_error.
void pdlpgpu_internal_set_error(const char* message) { set_error(message ? message : ""); }

int32_t pdlpgpu_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ---------------------------------------------------------------------------
// Components
// ---------------------------------------------------------------------------
namespace {

bool component_engine(pdlpgpu::Engine& e, const pdlpgpu_lp* lp, int32_t precision,
                      bool working, double infeasibility_tolerance = 1e-8) {
    pdlpgpu::SolveSpec spec;
    spec.lps.push_back(lp);
    pdlpgpu_default_options(&spec.opt);
    spec.opt.infeasibility_tolerance = infeasibility_tolerance;
    pdlpgpu_default_ext_options(&spec.ext);
    spec.ext.precision = precision ? PDLPGPU_PRECISION_MIXED : PDLPGPU_PRECISION_FP64;
    spec.working_given = working;
    if (!e.prepare(spec)) {
        set_error(e.error());
        return false;
    }
    return true;
}

}  // namespace

int32_t pdlpgpu_spmv(const pdlpgpu_lp* lp, int32_t transpose, int32_t precision,
                     const double* in, double* out) {
    try {
        pdlpgpu::Engine e(0);
        if (!component_engine(e, lp, precision, true)) return -1;
        if (!e.component_spmv(transpose, precision ? 2 : 0, in, out)) {
            set_error(e.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_ruiz(const pdlpgpu_lp* lp, int32_t iterations, double* row_scale,
                     double* col_scale, double* scaled_values) {
    try {
        pdlpgpu::Engine e(0);
        pdlpgpu::SolveSpec spec;
        spec.lps.push_back(lp);
        pdlpgpu_default_options(&spec.opt);
        spec.opt.ruiz_iterations = iterations;
        pdlpgpu_default_ext_options(&spec.ext);
        if (!e.prepare(spec)) {
            set_error(e.error());
            return -1;
        }
        std::vector<double> rs(static_cast<size_t>(lp->num_rows)), cs(static_cast<size_t>(lp->num_cols));
        if (!e.component_ruiz(rs.data(), cs.data(), scaled_values)) {
            set_error(e.error());
            return -1;
        }
        if (row_scale) std::copy(rs.begin(), rs.end(), row_scale);
        if (col_scale) std::copy(cs.begin(), cs.end(), col_scale);
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_precondition(const pdlpgpu_lp* lp, double* tau, double* tau_inverse,
                             double* sigma, double* sigma_inverse) {
    try {
        pdlpgpu::Engine e(0);
        if (!component_engine(e, lp, 0, true)) return -1;
        if (!e.component_precondition(tau, tau_inverse, sigma, sigma_inverse)) {
            set_error(e.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_trial(const pdlpgpu_lp* lp, int32_t precision, const double* tau,
                      const double* tau_inverse, const double* sigma,
                      const double* sigma_inverse, const double* x, const double* y,
                      const double* ax, double step, double weight, double* x_out,
                      double* y_out, double* ax_out, double* reductions) {
    try {
        pdlpgpu::Engine e(0);
        if (!component_engine(e, lp, precision, true)) return -1;
        if (!e.component_trial(tau, tau_inverse, sigma, sigma_inverse, x, y, ax, step, weight,
                               x_out, y_out, ax_out, reductions)) {
            set_error(e.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_evaluate(const pdlpgpu_lp* lp, double infeasibility_tolerance,
                         const double* x, const double* y, const double* rx,
                         const double* ry, double* metrics, double* verdicts) {
    try {
        pdlpgpu::Engine e(0);
        if (!component_engine(e, lp, 0, true, infeasibility_tolerance)) return -1;
        if (!e.component_evaluate(x, y, rx, ry, metrics, verdicts)) {
            set_error(e.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_layout_stats(const pdlpgpu_lp* lp, const pdlpgpu_ext_options* ext,
                             int64_t* stats) {
    try {
        pdlpgpu::HostCsr a;
        const std::string err = pdlpgpu::canonicalize(*lp, a);
        if (!err.empty()) {
            set_error(err);
            return -1;
        }
        pdlpgpu::Tuning t = pdlpgpu::choose_tuning(a, ext && ext->precision == PDLPGPU_PRECISION_MIXED);
        if (ext && ext->lane_elements > 0) t.lane_elements = ext->lane_elements;
        if (ext && (ext->vector_width == 1 || ext->vector_width == 2 || ext->vector_width == 4))
            t.vector_width = ext->vector_width;
        const pdlpgpu::MatrixLayout L = pdlpgpu::build_layout(a, t);
        stats[0] = static_cast<int64_t>(L.a.slices.size());
        stats[1] = L.a.slots();
        stats[2] = L.a.entries;
        stats[3] = static_cast<int64_t>(L.at.slices.size());
        stats[4] = L.at.slots();
        stats[5] = L.at.entries;
        stats[6] = t.lane_elements;
        stats[7] = t.vector_width;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_layout_multiply(const pdlpgpu_lp* lp, const pdlpgpu_ext_options* ext,
                                const double* x, double* out) {
    try {
        pdlpgpu::HostCsr a;
        const std::string err = pdlpgpu::canonicalize(*lp, a);
        if (!err.empty()) {
            set_error(err);
            return -1;
        }
        pdlpgpu::Tuning t = pdlpgpu::choose_tuning(a, false);
        if (ext && ext->lane_elements > 0) t.lane_elements = ext->lane_elements;
        if (ext && (ext->vector_width == 1 || ext->vector_width == 2 || ext->vector_width == 4))
            t.vector_width = ext->vector_width;
        const pdlpgpu::MatrixLayout L = pdlpgpu::build_layout(a, t);
        const int V = t.vector_width;
        std::vector<double> xin(static_cast<size_t>(L.n));
        for (int32_t c = 0; c < L.n; ++c) xin[c] = x[L.col_perm[c]];
        for (const pdlpgpu::SliceDesc& sd : L.a.slices) {
            const int glog = pdlpgpu::slice_glog(sd.meta), nl = pdlpgpu::slice_lines(sd.meta);
            const int G = 1 << glog;
            const int64_t base = static_cast<int64_t>(sd.data_off) * 32;
            for (int r = 0; r < nl; ++r) {
                const int32_t line = sd.line0 + r;
                double lane_sum[32] = {0.0};
                for (int g = 0; g < G; ++g) {
                    const int lane = r * G + g;
                    for (int s = 0; s < sd.steps; ++s) {
                        const int k = (s << glog) + g;
                        if (k >= L.a.line_len[line]) continue;
                        const int64_t pos = base + (s / V) * 32 * V + lane * V + (s % V);
                        lane_sum[g] += L.a.val[pos] * xin[L.a.idx[pos]];
                    }
                }
                for (int o = G >> 1; o > 0; o >>= 1)
                    for (int g = 0; g < o; ++g) lane_sum[g] += lane_sum[g + o];
                out[L.row_perm[line]] = lane_sum[0];
            }
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}


// ---------------------------------------------------------------------------
// Sessions
// ---------------------------------------------------------------------------
}  // extern "C"

struct pdlpgpu_session {
    explicit pdlpgpu_session(int device) : engine(device) {}
    pdlpgpu::Engine engine;
};

extern "C" {

int32_t pdlpgpu_session_create(const pdlpgpu_lp* family, int32_t batch,
                               const pdlpgpu_options* options,
                               const pdlpgpu_ext_options* ext, pdlpgpu_session** session) {
    if (family == nullptr || session == nullptr || batch <= 0) {
        set_error("invalid session arguments");
        return -1;
    }
    try {
        const pdlpgpu_ext_options e = ext_or_default(ext);
        auto* s = new pdlpgpu_session(e.device);
        if (!s->engine.session_create(*family, batch, opt_or_default(options), e)) {
            set_error(s->engine.error());
            delete s;
            *session = nullptr;
            return -1;
        }
        *session = s;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        *session = nullptr;
        return -1;
    }
}

void pdlpgpu_session_destroy(pdlpgpu_session* session) { delete session; }

int32_t pdlpgpu_session_load(pdlpgpu_session* s, int32_t on_device, const double* objective,
                             const double* row_lower, const double* row_upper,
                             const double* var_lower, const double* var_upper,
                             const double* warm_primal, const double* warm_dual,
                             const double* warm_weight) {
    if (s == nullptr) return -1;
    try {
        if (!s->engine.session_load(on_device != 0, objective, row_lower, row_upper, var_lower,
                                    var_upper, warm_primal, warm_dual, warm_weight)) {
            set_error(s->engine.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_session_solve(pdlpgpu_session* s) {
    if (s == nullptr) return -1;
    try {
        int32_t optimal = 0;
        if (!s->engine.session_solve(&optimal)) {
            set_error(s->engine.error());
            return -1;
        }
        return optimal;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_session_read(pdlpgpu_session* s, int32_t on_device, double* primal, double* dual,
                             int32_t* status, int64_t* iterations, double* stats) {
    if (s == nullptr) return -1;
    try {
        if (!s->engine.session_read(on_device != 0, primal, dual, status, iterations, stats)) {
            set_error(s->engine.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_session_stream(pdlpgpu_session* s, int32_t on_device, int64_t count,
                               const double* objective, const double* row_lower,
                               const double* row_upper, const double* var_lower,
                               const double* var_upper, const double* warm_primal,
                               const double* warm_dual, const double* warm_weight,
                               double* primal, double* dual, int32_t* status, int64_t* iterations,
                               double* stats) {
    if (s == nullptr || count < 0) return -1;
    try {
        const double* in[5] = {objective, row_lower, row_upper, var_lower, var_upper};
        if (!s->engine.session_stream(on_device != 0, count, in, warm_primal, warm_dual, warm_weight,
                                      primal, dual, status, iterations, stats)) {
            set_error(s->engine.error());
            return -1;
        }
        int32_t optimal = 0;
        if (status != nullptr)
            for (int64_t i = 0; i < count; ++i) optimal += status[i] == PDLPGPU_OPTIMAL ? 1 : 0;
        return optimal;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t pdlpgpu_session_last_timing(pdlpgpu_session* s, double* device_seconds, int64_t* launches) {
    if (s == nullptr) return -1;
    if (device_seconds) *device_seconds = s->engine.device_seconds();
    if (launches) *launches = s->engine.launches();
    return 0;
}

int32_t pdlpgpu_session_loop_timing(pdlpgpu_session* s, double* out) {
    if (s == nullptr || out == nullptr) return -1;
    s->engine.loop_timing(out);
    return 0;
}

int32_t pdlpgpu_session_time_kernels(pdlpgpu_session* s, int32_t reps, double* out) {
    if (s == nullptr || reps <= 0) return -1;
    try {
        if (!s->engine.time_kernels(reps, out)) {
            set_error(s->engine.error());
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

}  // extern "C"

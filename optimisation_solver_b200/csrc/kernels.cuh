// kernels.cuh -- argument blocks and launch entry points of the device kernels.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>

namespace pdlpgpu {

// One side of A in the SELL-G layout.
struct Side {
    const SliceDesc* slices;
    const int32_t* idx;
    const double* val_orig;      // original coefficients (FP64), used by the checks
    const double* val_s64;       // Ruiz-scaled coefficients (FP64)
    const float* val_s32;        // Ruiz-scaled coefficients (FP32), mixed precision only
    const int32_t* line_len;
    const CtaWork* ctas;
    int32_t num_ctas;
};

// Arrays of one working precision (the scaled problem the iterations run on).
template <class T>
struct Work {
    T* X[2];
    T* Y[2];
    T* AX[2];
    T* avg_x;
    T* avg_y;
    T* rx;
    T* ry;
    T* c;
    T* xl;
    T* xu;
    T* tau;
    T* itau;
    T* rl;
    T* ru;
    T* sigma;
    T* isigma;
};

// Everything that does not depend on the working precision.
struct Global {
    InstanceCtl* ctl;
    const InstanceInfo* info;
    Side a, at;
    const VecWork* vec;
    int32_t num_vec;
    int32_t shared_matrix;
    // original problem (FP64) and the Ruiz scale vectors
    double* rs;
    double* cs;
    const double* c_orig;
    const double* xl_orig;
    const double* xu_orig;
    const double* rl_orig;
    const double* ru_orig;
    // check scratch and outputs (original coordinates)
    double* x_o;
    double* xa_o;
    double* p_proj;
    double* y_o;
    double* ya_o;
    double* dy_o;
    double* best_x;
    double* best_y;
    double* dray;
    double* pray;
    // warm start (original coordinates), may be null
    const double* warm_x;
    const double* warm_y;
    // setup scratch
    double* row_tmp;
    double* col_tmp;
    // per-CTA partials and per-instance arrival counters
    double* part_primal;
    double* part_dual;
    double* part_prep;
    double* part_check;
    int32_t* count_dual;
    int32_t* count_check;
    // 1: timing mode -- every instance runs its trial kernels, no decision is
    // taken and no state changes (the trial buffers are scratch).
    int32_t measure;
    // 1: mixed-precision solve (FP32 iterations, FP64 stage on stall)
    int32_t mixed;
    // Streams: when set, setup kernels act only on slots with slot_mask[b] != 0.
    const int32_t* slot_mask;
    // Normalised-gap restarts (DeviceOptions::ndg_restarts): a main check's
    // reduced costs c + A'y [column space] and row activities A x [row
    // space] of the current (0) and average (1) iterates, original
    // coordinates; and the restart point of each working precision.
    double* ndg_g[2];
    double* ndg_a[2];
    const float* rx32;
    const float* ry32;
    const double* rx64;
    const double* ry64;
};

// --- launches (kernels.cu). `vw` is the vector width (1, 2 or 4). ---------

template <class T>
void launch_primal(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw,
                   cudaStream_t s);
template <class T>
void launch_dual(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw,
                 cudaStream_t s);
// The shape of a fused launch's shared memory, over its instances.
struct FusedShape {
    int32_t slices_p, slices_d;     // most slices of an instance per side
    int32_t entries_p, entries_d;   // most CTA-map entries of an instance per side
    int32_t stage_bytes;            // most bytes of a CTA's staged slices (0: nothing staged)
    int32_t lines;                  // staged with copies: most rows + columns of an instance (else 0)
    int32_t multi;                  // some CTA-map entry has other than one slice
    int32_t elem;                   // bytes of the launch's working precision
};
// Dynamic shared memory of a fused CTA: one warp sum per primal slice, two
// per dual slice, one word per CTA-map entry; then, with copies, x and y of
// both parities; then the staged slices.
__host__ __device__ inline size_t fused_copies_offset(const FusedShape& f) {
    const size_t b = sizeof(double) * (static_cast<size_t>(f.slices_p) + 2 * static_cast<size_t>(f.slices_d)) +
                     sizeof(int32_t) * (static_cast<size_t>(f.entries_p) + static_cast<size_t>(f.entries_d));
    return (b + 15) & ~static_cast<size_t>(15);
}
__host__ __device__ inline size_t fused_stage_offset(const FusedShape& f) {
    return fused_copies_offset(f) + 2 * static_cast<size_t>(f.elem) * static_cast<size_t>(f.lines);
}
__host__ __device__ inline size_t fused_smem_bytes(const FusedShape& f) {
    return fused_stage_offset(f) + static_cast<size_t>(f.stage_bytes);
}
// A staged slice in shared memory: the index and value of each of its 32 x
// `steps` entries, then `consts` line constants per lane (element size
// `elem`).
constexpr int kFusedPrimalConsts = 5;   // objective, lower, upper, tau, 1/tau
constexpr int kFusedDualConsts = 4;     // sigma, 1/sigma, lower, upper
// With copies, the lines' own iterates follow the constants.
constexpr int kFusedPrimalOwn = 1;      // the average
constexpr int kFusedDualOwn = 3;        // Ax of both parities, the average
__host__ __device__ constexpr int fused_slice_bytes(int steps, int consts, int elem) {
    return 32 * steps * (4 + elem) + 32 * consts * elem;
}
// The trials of a check interval of `count` small instances in one launch:
// one cluster of `cluster` CTAs (512 threads each) per instance, at most
// `max_trials` trials each, stopping at a check or the end (kernels.cu,
// k_fused). Same results as launch_primal + launch_dual per trial.
template <class T>
cudaError_t launch_fused(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw, int count,
                         int cluster, int max_trials, const FusedShape& shape, cudaStream_t s);
// Clusters of that shape resident at once (0: the launch is not possible).
template <class T>
int fused_max_clusters(int vw, int cluster, const FusedShape& shape);
constexpr int kFusedCtaThreads = 512;
// Largest dynamic shared memory the engine gives a fused CTA (its static
// shared memory, the control block and the options, fit beside it).
constexpr size_t kFusedMaxSmemHost = 220 * 1024;
template <class T>
void launch_check_prep(const Global& g, const Work<T>& w, const DeviceOptions& o, cudaStream_t s);
void launch_check_spmv(const Global& g, const DeviceOptions& o, int vw, cudaStream_t s);
// With normalised-gap restarts (o.ndg_restarts): the decision of each
// instance at a check, after launch_check_spmv (one CTA per instance).
void launch_check_ndg(const Global& g, const DeviceOptions& o, int32_t count, cudaStream_t s);
template <class T>
void launch_check_apply(const Global& g, const Work<T>& w, const DeviceOptions& o, cudaStream_t s);
template <class T>
void launch_refresh(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw,
                    cudaStream_t s);
// active[0]: unfinished instances; active[1]: those in the FP64 stage of a
// mixed solve (both must be zeroed first).
void launch_finalize(const Global& g, int32_t count, int32_t* active, cudaStream_t s);
void launch_switch_fp64(const Global& g, const Work<float>& w32, const Work<double>& w64,
                        cudaStream_t s);

// Setup. `a_ctas`/`at_ctas` limit the launch to the first CTAs of the maps
// (instance 0 of a shared-matrix batch).
void launch_ruiz_max(const Global& g, int vw, int a_ctas, int at_ctas, cudaStream_t s);
void launch_ruiz_update(const Global& g, int vec_ctas, cudaStream_t s);
void launch_scale_values(const Global& g, double* a_s64, double* at_s64, float* a_s32,
                         float* at_s32, int vw, int a_ctas, int at_ctas, cudaStream_t s);
template <class T>
void launch_precondition(const Global& g, const Work<T>& w, int enabled, int vw, int a_ctas,
                         int at_ctas, cudaStream_t s);
template <class T>
void launch_setup_vectors(const Global& g, const Work<T>& w, cudaStream_t s);
// p[0..n) = v.
template <class T>
void launch_fill(T* p, int64_t n, T v, cudaStream_t s);
void launch_broadcast_scales(const Global& g, const InstanceInfo& first, int32_t count,
                             int64_t rows, int64_t cols, cudaStream_t s);
template <class T>
void launch_broadcast_precond(const Work<T>& w, const InstanceInfo& first, int32_t count,
                              int64_t rows, int64_t cols, cudaStream_t s);

void launch_power_dot(const Global& g, const double* x, const double* z, cudaStream_t s);
// table[2k] = (k + 2)^-0.3, table[2k + 1] = (k + 2)^-0.6 for k < entries.
void launch_step_pow(double* table, int64_t entries, cudaStream_t s);
void launch_power_step(const Global& g, int32_t count, int init, int it, int budget, cudaStream_t s);
void launch_power_scale(const Global& g, double* x, const double* z, cudaStream_t s);
void launch_power_finish(const Global& g, int32_t count, double safety, double min_scale,
                         cudaStream_t s);
void launch_stamp_clock(const Global& g, int32_t count, int64_t elapsed_ns, int64_t limit_ns,
                        cudaStream_t s);

// Sessions (one shared matrix; instance b's vectors at b*m / b*n).
// mode 0: dst[b][k] = src[b][perm[k]]   (original -> internal)
// mode 1: dst[b][perm[k]] = src[b][k]   (internal -> original)
// mode 2: dst[b][k] = src[k]           (broadcast one internal vector)
void launch_permute(const double* src, double* dst, const int32_t* perm, int64_t len,
                    int32_t count, int mode, cudaStream_t s);
void launch_norm_parts(const Global& g, cudaStream_t s);
// Streams: per slot b with mask[b] != 0, dst[b][k] = src[inst[b]][perm[k]]
// (src = null: fam[k]); scatter: out[inst[b]][perm[k]] = src[b][k].
void launch_gather_slots(const double* src, const double* fam, double* dst, const int32_t* perm,
                         const int64_t* inst, const int32_t* mask, int64_t len, int32_t count,
                         cudaStream_t s);
void launch_scatter_slots(const double* src, double* out, const int32_t* perm, const int64_t* inst,
                          const int32_t* mask, int64_t len, int32_t count, cudaStream_t s);
void launch_retire(const Global& g, int32_t count, cudaStream_t s);
void launch_slot_done(const Global& g, int32_t count, int32_t* done, cudaStream_t s);
void launch_init_ctl(const Global& g, const DeviceOptions& o, int32_t count, int32_t mixed,
                     int32_t warm, const double* warm_weight, double eta_max,
                     double initial_weight, double objective_offset, cudaStream_t s);

// Plain products over the layout: out = A v (transpose = 0) or A^T v, lines
// written in internal order. `values` selects orig (0), scaled FP64 (1), FP32 (2).
template <class T>
void launch_spmv(const Global& g, int transpose, int values, const T* v, T* out, int vw,
                 cudaStream_t s);

}  // namespace pdlpgpu

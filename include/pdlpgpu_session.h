/*
 * pdlpgpu_session.h -- repeated batched solves of one LP family on the device.
 *
 * No counterpart in the reference, which solves one LP per PdlpSolver::solve
 * call (pdlp_engine/src/pdlp_solver.cpp:116-548) and rebuilds everything each
 * time. A session fixes the constraint matrix of a family (one shared A, as
 * in a parameterised family where only costs, bounds and right-hand sides
 * change) and a batch size; its device layout, Ruiz scaling and
 * preconditioner are built once. Each solve then loads the per-instance
 * vectors -- from host arrays, or from device pointers already resident in
 * HBM -- and runs all instances to completion in one batched device loop.
 * Every instance keeps the reference's per-LP semantics (statuses,
 * tolerances, restarts, certificates).
 */
#ifndef PDLPGPU_SESSION_H
#define PDLPGPU_SESSION_H

#include "pdlpgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdlpgpu_session pdlpgpu_session;

/* `family` supplies the matrix and the default vectors for every instance.
 * Returns 0, or -1 with pdlpgpu_last_error() set. */
int32_t pdlpgpu_session_create(const pdlpgpu_lp* family, int32_t batch,
                               const pdlpgpu_options* options,
                               const pdlpgpu_ext_options* ext, pdlpgpu_session** session);

void pdlpgpu_session_destroy(pdlpgpu_session* session);

/* Per-instance vectors, row-major [batch][n] or [batch][m], original order.
 * NULL keeps the family's vector for every instance. `on_device` = 1 means the
 * pointers are device memory on the session's GPU (nothing crosses PCIe);
 * the session reads and writes such buffers only after all work enqueued so
 * far on the legacy default stream (CUDA's stream 0, where PyTorch enqueues
 * by default), so data produced there needs no synchronisation; data
 * produced on any other stream must be complete before the call. The same
 * holds for the device buffers of pdlpgpu_session_read and _stream.
 * warm_primal / warm_dual / warm_weight enable a warm start for every
 * instance (original coordinates, PDLP dual sign; weight <= 0 = default);
 * the better of warm and cold start by KKT score is used per instance. */
int32_t pdlpgpu_session_load(pdlpgpu_session* session, int32_t on_device,
                             const double* objective, const double* row_lower,
                             const double* row_upper, const double* var_lower,
                             const double* var_upper, const double* warm_primal,
                             const double* warm_dual, const double* warm_weight);

/* Runs every instance to completion. Returns the number that ended OPTIMAL,
 * or -1 on failure. */
int32_t pdlpgpu_session_solve(pdlpgpu_session* session);

/* Results of the last solve. primal [batch][n], dual [batch][m] (original
 * order, device pointers when on_device = 1); per-instance status and
 * iterations on the host; any pointer may be NULL. stats[batch][8] =
 * {primal objective, dual objective, primal residual, dual residual,
 * relative gap, step trials, final primal weight, restarts}. Returns 0 on
 * success. */
int32_t pdlpgpu_session_read(pdlpgpu_session* session, int32_t on_device, double* primal,
                             double* dual, int32_t* status, int64_t* iterations,
                             double* stats);

/* Solves `count` instances through the session's `batch` slots, refilling a
 * slot with the next queued instance as soon as its instance finishes, so a
 * few slow instances never hold the whole batch. Inputs as for
 * pdlpgpu_session_load but with `count` rows ([count][n] / [count][m];
 * warm_weight [count]); outputs primal [count][n], dual [count][m] (device
 * pointers when on_device = 1, else host), status and iterations [count]
 * and stats [count][8] (host, as pdlpgpu_session_read). Returns the number
 * of OPTIMAL instances, or -1 on failure. */
int32_t pdlpgpu_session_stream(pdlpgpu_session* session, int32_t on_device, int64_t count,
                               const double* objective, const double* row_lower,
                               const double* row_upper, const double* var_lower,
                               const double* var_upper, const double* warm_primal,
                               const double* warm_dual, const double* warm_weight,
                               double* primal, double* dual, int32_t* status,
                               int64_t* iterations, double* stats);

/* Device seconds of the last solve's iteration loop and the number of this
 * library's kernel launches in it. */
int32_t pdlpgpu_session_last_timing(pdlpgpu_session* session, double* device_seconds,
                                    int64_t* launches);

/* Live timing of the last solve or stream: CUDA events recorded inside the
 * captured iteration loop around the two kernels of four trial slots of every
 * chunk (its first, second, middle and last slot). out[15] = {primal ms per
 * launch, dual ms per launch, samples, ms per chunk, chunks, device seconds of
 * the loop, ms per chunk in the check stage, then primal and dual ms per
 * launch at each of the four slots}. */
int32_t pdlpgpu_session_loop_timing(pdlpgpu_session* session, double* out);

/* Times the two PDHG trial kernels with CUDA events on the session's stream,
 * `reps` launches each, with every instance forced active and no state
 * change. out[6] = {primal ms per launch, dual ms per launch, primal
 * algorithmic bytes per launch, dual algorithmic bytes per launch, padded
 * slots of the A^T side, padded slots of the A side}. */
int32_t pdlpgpu_session_time_kernels(pdlpgpu_session* session, int32_t reps, double* out);

#ifdef __cplusplus
}
#endif

#endif

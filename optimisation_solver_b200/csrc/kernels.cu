// kernels.cu -- the device kernels of the PDLP engine (sm_100a).
//
// Hot path, per linesearch trial (pdlp_engine/src/pdhg_kernel.cpp:47-277):
//   k_primal  over the A^T side: g = c + A'y, x' = clip(x - (eta/omega) tau g),
//             sum dx^2/tau; applies the iterate-average update owed by the last
//             commit (iterate_average.cpp:40-82) while x is in registers.
//   k_dual    over the A side: A x', extrapolation 2Ax' - Ax, dual prox
//             y' = max(v - s u, 0) + min(v - s l, 0), sum dy^2/sigma and
//             dy'(A dx); owed average update of y; then, in the last CTA of each
//             instance, the linesearch decision and commit (trial_control).
// Every check_frequency iterations (termination.cpp:66-325,
// infeasibility.cpp:51-192, pdlp_solver.cpp:354-476), in FP64 on the original
// problem:
//   k_check_prep   elementwise: original-coordinate copies of the current and
//                  averaged iterates and of the ray directions, and every
//                  reduction that needs no matrix product
//   k_check_spmv   both matrix passes at once, each gathering up to three
//                  vectors; the last CTA of an instance decides (best point,
//                  certificates, termination, restart)
//   k_check_apply  best-point copies, restarts, polishing entry, ray copies
//   k_refresh      A x after an iterate was replaced
//   k_finalize     clears the per-check flags
// Setup: Ruiz max-abs passes, scaled coefficients, Pock-Chambolle sums.
//
// Gathers go through the read-only path; matrix streams use 128-bit loads
// when the vector width allows. No atomics touch numerical data: the only
// atomic is the per-instance arrival counter.
#include "control.cuh"
#include "kernels.cuh"
#include "ndg.cuh"

#include <algorithm>
#include <cstdio>

namespace pdlpgpu {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Loads of V consecutive elements (V in {1, 2, 4}); the caller guarantees
// V-element alignment.
// ---------------------------------------------------------------------------
template <int V> __device__ __forceinline__ void ld(const int32_t* p, int32_t (&o)[V]);
template <> __device__ __forceinline__ void ld<1>(const int32_t* p, int32_t (&o)[1]) { o[0] = __ldg(p); }
template <> __device__ __forceinline__ void ld<2>(const int32_t* p, int32_t (&o)[2]) {
    const int2 v = __ldg(reinterpret_cast<const int2*>(p)); o[0] = v.x; o[1] = v.y;
}
template <> __device__ __forceinline__ void ld<4>(const int32_t* p, int32_t (&o)[4]) {
    const int4 v = __ldg(reinterpret_cast<const int4*>(p)); o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <int V> __device__ __forceinline__ void ld(const float* p, float (&o)[V]);
template <> __device__ __forceinline__ void ld<1>(const float* p, float (&o)[1]) { o[0] = __ldg(p); }
template <> __device__ __forceinline__ void ld<2>(const float* p, float (&o)[2]) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p)); o[0] = v.x; o[1] = v.y;
}
template <> __device__ __forceinline__ void ld<4>(const float* p, float (&o)[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p)); o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <int V> __device__ __forceinline__ void ld(const double* p, double (&o)[V]);
template <> __device__ __forceinline__ void ld<1>(const double* p, double (&o)[1]) { o[0] = __ldg(p); }
template <> __device__ __forceinline__ void ld<2>(const double* p, double (&o)[2]) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p)); o[0] = v.x; o[1] = v.y;
}
template <> __device__ __forceinline__ void ld<4>(const double* p, double (&o)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// Lane position inside a slice.
struct LanePos {
    int glog;     // log2 of the lane group
    int g;        // lane inside the group
    int line;     // local line index
    bool valid;   // the lane's line exists
};

__device__ __forceinline__ LanePos lane_pos(const SliceDesc& sd, int lane) {
    LanePos p;
    p.glog = slice_glog(sd.meta);
    const int r = lane >> p.glog;
    p.g = lane & ((1 << p.glog) - 1);
    p.line = sd.line0 + r;
    p.valid = r < slice_lines(sd.meta);
    return p;
}

// Sum of NQ products over the lane's entries of one line, then combined over
// the G lanes of the line with an xor butterfly (every lane ends with the same
// bits, so the result is deterministic). Up to kDepth vector loads of index
// and value are issued before their gathers, so a lane keeps several
// independent memory requests in flight instead of one load-gather chain.
// kDeep doubles the depth for FP32 vector loads (measured: the dual kernel
// gains, the primal kernel, whose lanes also stream five vectors, loses).
template <int V, int NQ, bool kDeep = false, class TA, class TV, class F>
__device__ __forceinline__ void line_sums(int64_t base, int steps, const LanePos& lp, int lane,
                                          int len, const int32_t* __restrict__ idx,
                                          const TV* __restrict__ val, TA (&acc)[NQ], F fetch) {
    // About four entries in flight per lane, eight for deep FP32 vector
    // loads (deeper FP64 or scalar pipelines spill at 64 registers).
    constexpr int kDepth = (kDeep && V >= 2 && sizeof(TV) == 4) ? 8 / V : (V >= 4 ? 1 : 4 / V);
    constexpr int kStep = kDepth * V;
    // Software pipeline: the index and value loads of the next group are in
    // flight while the current group's gathers are.
    auto load = [&](int s0, int32_t (&id)[kDepth][V], TV (&v)[kDepth][V]) {
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
            const int s = s0 + u * V;
            if (s < steps) {
                const int64_t p = base + static_cast<int64_t>(s) * 32 + lane * V;
                ld<V>(idx + p, id[u]);
                ld<V>(val + p, v[u]);
            } else {
#pragma unroll
                for (int q = 0; q < V; ++q) {
                    id[u][q] = 0;
                    v[u][q] = TV(0);
                }
            }
        }
    };
    int32_t id[kDepth][V];
    TV v[kDepth][V];
    load(0, id, v);
    for (int s0 = 0; s0 < steps; s0 += kStep) {
        int32_t nid[kDepth][V];
        TV nv[kDepth][V];
        load(s0 + kStep, nid, nv);
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
#pragma unroll
            for (int q = 0; q < V; ++q) {
                const int k = ((s0 + u * V + q) << lp.glog) + lp.g;
                if (k < len) fetch(acc, static_cast<TA>(v[u][q]), id[u][q]);
            }
        }
#pragma unroll
        for (int u = 0; u < kDepth; ++u)
#pragma unroll
            for (int q = 0; q < V; ++q) {
                id[u][q] = nid[u][q];
                v[u][q] = nv[u][q];
            }
    }
    for (int o = (1 << lp.glog) >> 1; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] += __shfl_xor_sync(kFull, acc[q], o);
    }
}

// Block-wide deterministic sum of NQ doubles; the result is valid in thread 0.
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ]) {
    __shared__ double red[NQ][kWarps * 4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(kFull, v[q], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) red[q][warp] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double t = 0.0;
            for (int w = 0; w < warps; ++w) t += red[q][w];
            v[q] = t;
        }
    }
}

// Warp-0 deterministic sum over a range of per-CTA partials (stride `slots`).
__device__ __forceinline__ double warp_range_sum(const double* part, int begin, int end,
                                                 int slots, int slot) {
    const int lane = threadIdx.x & 31;
    double t = 0.0;
    for (int k = begin + lane; k < end; k += 32) t += part[static_cast<int64_t>(k) * slots + slot];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
    return t;
}

// Warp-0 deterministic sums of three ranges of per-CTA partials at once:
// every lane issues its loads of all three before the first add, so the
// three reductions cost one round trip instead of three. Each result equals
// warp_range_sum's for the same range (same per-lane order, same butterfly).
template <bool kL2Only = false>
__device__ __forceinline__ void warp_range_sums3(const double* p0, int b0, int e0, int s0, int q0,
                                                 const double* p1, int b1, int e1, int s1, int q1,
                                                 const double* p2, int b2, int e2, int s2, int q2,
                                                 double (&out)[3]) {
    const int lane = threadIdx.x & 31;
    double t[3] = {0.0, 0.0, 0.0};
    constexpr int kAhead = 4;   // partials per lane and range loaded at once
    for (int k = 0;; k += 32 * kAhead) {
        if (b0 + k >= e0 && b1 + k >= e1 && b2 + k >= e2) break;
        double v[3][kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const int o = k + 32 * u + lane;
            auto get = [](const double* p) { return kL2Only ? __ldcg(p) : *p; };
            v[0][u] = b0 + o < e0 ? get(p0 + static_cast<int64_t>(b0 + o) * s0 + q0) : 0.0;
            v[1][u] = b1 + o < e1 ? get(p1 + static_cast<int64_t>(b1 + o) * s1 + q1) : 0.0;
            v[2][u] = b2 + o < e2 ? get(p2 + static_cast<int64_t>(b2 + o) * s2 + q2) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const int o = k + 32 * u + lane;
            if (b0 + o < e0) t[0] += v[0][u];
            if (b1 + o < e1) t[1] += v[1][u];
            if (b2 + o < e2) t[2] += v[2][u];
        }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        for (int o = 16; o > 0; o >>= 1) t[q] += __shfl_xor_sync(kFull, t[q], o);
        out[q] = t[q];
    }
}

// Arrival counter: returns true in every thread of the CTA that arrives last
// among `expected` CTAs of the instance (and resets the counter for the next
// launch, which a kernel boundary orders). Partials written before the call
// are visible to that CTA. One thread arrives for the CTA with an
// acquire-release atomic at GPU scope: the barrier orders the other threads'
// writes before it, its release publishes them, and in the last CTA its
// acquire makes every earlier arrival's writes visible -- one round trip
// where a full fence and an atomic took two.
__device__ __forceinline__ bool arrive_last(int32_t* counter, int expected) {
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        int prev;
        asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(prev) : "l"(counter) : "memory");
        last = prev == expected - 1;
        if (last) *counter = 0;
    }
    __syncthreads();
    return last != 0;
}


// Non-binding L2 prefetch of [p, p + bytes), shrunk inward to 16-byte
// boundaries (so it never reaches outside the range) and cut into pieces of at
// most 32 KiB spread over the CTA's threads starting at thread `first`.
__device__ __forceinline__ void prefetch_range(const void* p, int64_t bytes, int first) {
    if (bytes <= 0) return;
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + static_cast<uintptr_t>(bytes)) & ~uintptr_t(15);
    if (e <= a) return;
    constexpr uintptr_t kPiece = 32768;
    const uintptr_t pieces = (e - a + kPiece - 1) / kPiece;
    for (uintptr_t k = (threadIdx.x + blockDim.x - static_cast<unsigned>(first) % blockDim.x) % blockDim.x;
         k < pieces; k += blockDim.x) {
        const uintptr_t b = a + k * kPiece;
        const uint32_t n = static_cast<uint32_t>(e - b < kPiece ? e - b : kPiece);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"(n) : "memory");
    }
}

// The streams a SELL CTA reads once: its slices' index and value data and the
// per-line vectors of its contiguous line range, prefetched into L2 when the
// CTA starts, so its later slices find them there.
template <class T, int NV>
__device__ __forceinline__ void prefetch_cta(const Side& side, const CtaWork& cw, int64_t data_base,
                                             const T* vals, const T* const (&vecs)[NV], int nvec) {
    if (cw.slice_end <= cw.slice_begin) return;
    const SliceDesc first = side.slices[cw.slice_begin], last = side.slices[cw.slice_end - 1];
    const int64_t e0 = data_base + static_cast<int64_t>(first.data_off) * 32;
    const int64_t e1 = data_base + (static_cast<int64_t>(last.data_off) + last.steps) * 32;
    prefetch_range(side.idx + e0, (e1 - e0) * 4, 0);
    prefetch_range(vals + e0, (e1 - e0) * static_cast<int64_t>(sizeof(T)), 64);
    const int l0 = first.line0, l1 = last.line0 + slice_lines(last.meta);
    for (int v = 0; v < nvec; ++v)
        prefetch_range(vecs[v] + l0, static_cast<int64_t>(l1 - l0) * static_cast<int64_t>(sizeof(T)), 128 + 16 * v);
}

__device__ __forceinline__ bool check_have_avg(const InstanceCtl& c, const DeviceOptions& o) {
    if (c.check_kind == kCheckInitial) return c.have_avg_at_check != 0;
    return o.averaging && c.avg_weight != 0.0;
}

template <class T> __device__ __forceinline__ const T* matrix_values(const Side& s);
template <> __device__ __forceinline__ const double* matrix_values<double>(const Side& s) { return s.val_s64; }
template <> __device__ __forceinline__ const float* matrix_values<float>(const Side& s) { return s.val_s32; }


// ---------------------------------------------------------------------------
// Primal half (pdhg_kernel.cpp:47-104)
// ---------------------------------------------------------------------------
template <class T, int V>
__global__ void __launch_bounds__(kThreads, 4) k_primal(Global g, Work<T> w) {
    const CtaWork cw = g.at.ctas[blockIdx.x];
    const InstanceCtl& c = g.ctl[cw.instance];
    if (!g.measure && !trial_active<T>(c)) return;
    const InstanceInfo inf = g.info[cw.instance];
    const int p = c.parity;
    const T mult = static_cast<T>(c.trial_eta / c.trial_omega);
    const bool pending = !g.measure && c.pending_avg != 0;
    const T frac = static_cast<T>(c.avg_frac);

    const T* __restrict__ y = w.Y[p] + inf.row_off;
    const T* __restrict__ x = w.X[p] + inf.col_off;
    T* __restrict__ xt = w.X[p ^ 1] + inf.col_off;
    const T* __restrict__ cv = w.c + inf.col_off;
    const T* __restrict__ lo = w.xl + inf.col_off;
    const T* __restrict__ hi = w.xu + inf.col_off;
    const T* __restrict__ tau = w.tau + inf.col_off;
    const T* __restrict__ itau = w.itau + inf.col_off;
    T* __restrict__ avg = w.avg_x + inf.col_off;
    const T* vals = matrix_values<T>(g.at);
    {
        const T* const vecs[7] = {x, cv, lo, hi, tau, itau, avg};
        prefetch_cta<T, 7>(g.at, cw, inf.at_data_base, vals, vecs, pending ? 7 : 6);
    }

    double moved[1] = {0.0};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = g.at.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const bool owner = lp.valid && lp.g == 0;
        const int j = lp.line;
        const int len = lp.valid ? g.at.line_len[inf.at_len_base + j] : 0;
        // The epilogue's operands do not depend on the product: load them
        // first so their latency overlaps the gathers.
        T cj = T(0), prev = T(0), loj = T(0), hij = T(0), tj = T(0), itj = T(0), aj = T(0);
        if (owner) {
            cj = cv[j];
            prev = x[j];
            loj = lo[j];
            hij = hi[j];
            tj = tau[j];
            itj = itau[j];
            if (pending) aj = avg[j];
        }
        T sum[1] = {T(0)};
        line_sums<V, 1>(inf.at_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp,
                        lane, len, g.at.idx, vals, sum,
                        [&](T (&a)[1], T v, int i) { a[0] += v * y[i]; });
        if (owner) {
            const T gradient = cj + sum[0];
            const T upd = smax(loj, smin(prev - mult * tj * gradient, hij));
            xt[j] = upd;
            const double d = static_cast<double>(upd - prev);
            moved[0] += d * d * static_cast<double>(itj);
            if (pending) avg[j] = aj + frac * (prev - aj);
        }
    }
    block_sum<1>(moved);
    if (threadIdx.x == 0) g.part_primal[blockIdx.x] = moved[0];
}

// ---------------------------------------------------------------------------
// Dual half (pdhg_kernel.cpp:109-187) and the trial decision
// ---------------------------------------------------------------------------
template <class T, int V>
__global__ void __launch_bounds__(kThreads, 4) k_dual(Global g, Work<T> w, DeviceOptions o) {
    const CtaWork cw = g.a.ctas[blockIdx.x];
    InstanceCtl& c = g.ctl[cw.instance];
    if (!g.measure && !trial_active<T>(c)) return;
    const InstanceInfo inf = g.info[cw.instance];
    const int p = c.parity;
    const T dm = static_cast<T>(c.trial_eta * c.trial_omega);
    const bool pending = !g.measure && c.pending_avg != 0;
    const T frac = static_cast<T>(c.avg_frac);

    const T* __restrict__ xt = w.X[p ^ 1] + inf.col_off;
    const T* __restrict__ y = w.Y[p] + inf.row_off;
    T* __restrict__ yt = w.Y[p ^ 1] + inf.row_off;
    const T* __restrict__ ax = w.AX[p] + inf.row_off;
    T* __restrict__ axt = w.AX[p ^ 1] + inf.row_off;
    const T* __restrict__ lo = w.rl + inf.row_off;
    const T* __restrict__ hi = w.ru + inf.row_off;
    const T* __restrict__ sig = w.sigma + inf.row_off;
    const T* __restrict__ isig = w.isigma + inf.row_off;
    T* __restrict__ avg = w.avg_y + inf.row_off;
    const T* vals = matrix_values<T>(g.a);
    {
        const T* const vecs[7] = {ax, y, lo, hi, sig, isig, avg};
        prefetch_cta<T, 7>(g.a, cw, inf.a_data_base, vals, vecs, pending ? 7 : 6);
    }

    double red[2] = {0.0, 0.0};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = g.a.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const bool owner = lp.valid && lp.g == 0;
        const int i = lp.line;
        const int len = lp.valid ? g.a.line_len[inf.a_len_base + i] : 0;
        T axi = T(0), sgi = T(0), prev = T(0), loi = T(0), hii = T(0), isi = T(0), ai = T(0);
        if (owner) {
            axi = ax[i];
            sgi = sig[i];
            prev = y[i];
            loi = lo[i];
            hii = hi[i];
            isi = isig[i];
            if (pending) ai = avg[i];
        }
        T sum[1] = {T(0)};
        line_sums<V, 1, true>(inf.a_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp,
                              lane, len, g.a.idx, vals, sum,
                              [&](T (&a)[1], T v, int j) { a[0] += v * xt[j]; });
        if (owner) {
            const T next = sum[0];
            const T dact = next - axi;
            const T ext = next + dact;
            const T step = smax(dm * sgi, min_dual_step<T>());
            const T v = prev + step * ext;
            const T upd = smax(v - step * hii, T(0)) + smin(v - step * loi, T(0));
            yt[i] = upd;
            axt[i] = next;
            const double d = static_cast<double>(upd - prev);
            red[0] += d * d * static_cast<double>(isi);
            red[1] += d * static_cast<double>(dact);
            if (pending) avg[i] = ai + frac * (prev - ai);
        }
    }
    block_sum<2>(red);
    if (threadIdx.x == 0) {
        g.part_dual[2 * blockIdx.x] = red[0];
        g.part_dual[2 * blockIdx.x + 1] = red[1];
    }
    if (g.measure) return;
    // Whichever CTA turns out last decides: each brings the instance's
    // control block into its L1 while the arrival is in flight, so the
    // decision's reads of it do not each wait on L2.
    if (threadIdx.x < sizeof(InstanceCtl) / 128)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(reinterpret_cast<const char*>(&c) + 128 * threadIdx.x));
    if (!arrive_last(g.count_dual + cw.instance, inf.a_cta_end - inf.a_cta_begin)) return;
    // Options by reference from shared memory (a reference to the kernel
    // parameter would copy it to local memory in every thread).
    __shared__ DeviceOptions so;
    if (threadIdx.x == 0) so = o;
    __syncthreads();
    if (threadIdx.x < 32) {
        // The decision runs on a shared-memory copy of the control block:
        // after a store to a global line, the thread's next load of that line
        // would be served by L2, and the decision reads back much of what it
        // writes.
        __shared__ alignas(16) InstanceCtl sc;
        copy_ctl_warp(&sc, &c);
        double sums[3];
        warp_range_sums3(g.part_primal, inf.at_cta_begin, inf.at_cta_end, 1, 0,
                         g.part_dual, inf.a_cta_begin, inf.a_cta_end, 2, 0,
                         g.part_dual, inf.a_cta_begin, inf.a_cta_end, 2, 1, sums);
        __syncwarp();
        if (threadIdx.x == 0) trial_control(sc, so, sums[0], sums[1], sums[2], inf.n);
        __syncwarp();
        copy_ctl_warp(&c, &sc);
    }
}

// ---------------------------------------------------------------------------
// Fused trials of small LPs: one thread-block cluster per instance runs the
// trials of a check interval in one launch. Warp q of CTA rank r serves the
// instance's slices r * kFusedWarps + q, stepping by the cluster's warp count;
// per trial:
//   primal half of every slice (k_primal's arithmetic, its warp sum per slice)
//   cluster barrier
//   dual half of every slice (k_dual's arithmetic)
//   cluster barrier
//   rank 0: each CTA-map entry's slice sums added in slice order (k_primal's
//   and k_dual's block sums: one slice per warp, warps in order), then the
//   entries' three sums in k_dual's fixed order and trial_control
//   cluster barrier
// so an instance's results are the two-kernel path's bit for bit, without a
// launch, an arrival counter or a trip through the decision's dependent loads
// per half. Vectors another CTA writes inside the launch (the iterates, the
// partials, the control block) are read through L2 (ld.cg); the barrier's
// release and acquire order them. Every CTA of a cluster reads the same
// control block after the same barrier, so all of them leave the loop
// together.
// ---------------------------------------------------------------------------
constexpr int kFusedGroups = 2;   // 512 threads: up to 128 registers each
constexpr int kFusedThreads = kFusedGroups * kThreads;
constexpr int kFusedWarps = kFusedThreads / 32;

// Every thread of every CTA of the cluster; the warp is reconverged first
// (the decision runs in one thread of rank 0's first warp just before).
__device__ __forceinline__ void cluster_sync_all() {
    __syncwarp();
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_size() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

// block_sum over one 256-thread group (its warps added in warp order, as
// block_sum adds a CTA's); the result is valid in the group's thread 0.
// Named barrier 1 + group; a second barrier frees `red` for the next call.
// The lanes' values of one warp added by the butterfly of block_sum's first
// stage (every lane gets the sum).
template <int NQ>
__device__ __forceinline__ void warp_sum(double (&v)[NQ]) {
#pragma unroll
    for (int q = 0; q < NQ; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(kFull, v[q], o);
}

// The trial's snapshot of the control block, three 16-byte words.
struct alignas(16) FusedCtl {
    double mult_primal, mult_dual, frac;
    int active, parity, pending, pad;
};
static_assert(sizeof(FusedCtl) == 48, "the snapshot travels as three 16-byte words");

template <class T, int V>
__device__ __forceinline__ double fused_primal(const Global& g, const Work<T>& w, const CtaWork& cw,
                                               const InstanceInfo& inf, const FusedCtl& f, int lt) {
    const int p = f.parity;
    const T mult = static_cast<T>(f.mult_primal);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* y = w.Y[p] + inf.row_off;
    const T* x = w.X[p] + inf.col_off;
    T* xt = w.X[p ^ 1] + inf.col_off;
    const T* cv = w.c + inf.col_off;
    const T* lo = w.xl + inf.col_off;
    const T* hi = w.xu + inf.col_off;
    const T* tau = w.tau + inf.col_off;
    const T* itau = w.itau + inf.col_off;
    T* avg = w.avg_x + inf.col_off;
    const T* vals = matrix_values<T>(g.at);
    double moved = 0.0;
    const int warp = lt >> 5, lane = lt & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = g.at.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const bool owner = lp.valid && lp.g == 0;
        const int j = lp.line;
        const int len = lp.valid ? g.at.line_len[inf.at_len_base + j] : 0;
        T cj = T(0), prev = T(0), loj = T(0), hij = T(0), tj = T(0), itj = T(0), aj = T(0);
        if (owner) {
            cj = cv[j];
            prev = __ldcg(x + j);
            loj = lo[j];
            hij = hi[j];
            tj = tau[j];
            itj = itau[j];
            if (pending) aj = __ldcg(avg + j);
        }
        T sum[1] = {T(0)};
        line_sums<V, 1>(inf.at_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp, lane, len,
                        g.at.idx, vals, sum, [&](T (&a)[1], T v, int i) { a[0] += v * __ldcg(y + i); });
        if (owner) {
            const T gradient = cj + sum[0];
            const T upd = smax(loj, smin(prev - mult * tj * gradient, hij));
            xt[j] = upd;
            const double d = static_cast<double>(upd - prev);
            moved += d * d * static_cast<double>(itj);
            if (pending) avg[j] = aj + frac * (prev - aj);
        }
    }
    return moved;
}

template <class T, int V>
__device__ __forceinline__ void fused_dual(const Global& g, const Work<T>& w, const CtaWork& cw,
                                           const InstanceInfo& inf, const FusedCtl& f, int lt,
                                           double (&red)[2]) {
    const int p = f.parity;
    const T dm = static_cast<T>(f.mult_dual);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* xt = w.X[p ^ 1] + inf.col_off;
    const T* y = w.Y[p] + inf.row_off;
    T* yt = w.Y[p ^ 1] + inf.row_off;
    const T* ax = w.AX[p] + inf.row_off;
    T* axt = w.AX[p ^ 1] + inf.row_off;
    const T* lo = w.rl + inf.row_off;
    const T* hi = w.ru + inf.row_off;
    const T* sig = w.sigma + inf.row_off;
    const T* isig = w.isigma + inf.row_off;
    T* avg = w.avg_y + inf.row_off;
    const T* vals = matrix_values<T>(g.a);
    const int warp = lt >> 5, lane = lt & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = g.a.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const bool owner = lp.valid && lp.g == 0;
        const int i = lp.line;
        const int len = lp.valid ? g.a.line_len[inf.a_len_base + i] : 0;
        T axi = T(0), sgi = T(0), prev = T(0), loi = T(0), hii = T(0), isi = T(0), ai = T(0);
        if (owner) {
            axi = __ldcg(ax + i);
            sgi = sig[i];
            prev = __ldcg(y + i);
            loi = lo[i];
            hii = hi[i];
            isi = isig[i];
            if (pending) ai = __ldcg(avg + i);
        }
        T sum[1] = {T(0)};
        line_sums<V, 1, true>(inf.a_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp, lane, len,
                              g.a.idx, vals, sum, [&](T (&a)[1], T v, int j) { a[0] += v * __ldcg(xt + j); });
        if (owner) {
            const T next = sum[0];
            const T dact = next - axi;
            const T ext = next + dact;
            const T step = smax(dm * sgi, min_dual_step<T>());
            const T v = prev + step * ext;
            const T upd = smax(v - step * hii, T(0)) + smin(v - step * loi, T(0));
            yt[i] = upd;
            axt[i] = next;
            const double d = static_cast<double>(upd - prev);
            red[0] += d * d * static_cast<double>(isi);
            red[1] += d * static_cast<double>(dact);
            if (pending) avg[i] = ai + frac * (prev - ai);
        }
    }
}

// Distributed shared memory: the address of `local` in rank 0's shared
// memory, and loads and stores there.
__device__ __forceinline__ uint32_t rank0_addr(const void* local) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local));
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(0));
    return r;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, double v) {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
// The next trial's snapshot of an instance's control block.
__device__ __forceinline__ void fused_snapshot(const InstanceCtl& c, FusedCtl& f, bool fp64) {
    f.active = c.phase != kPhaseDone && c.stage == kStageTrial && (c.fp64_stage != 0) == fp64;
    f.parity = c.parity;
    f.pending = c.pending_avg;
    f.mult_primal = c.trial_eta / c.trial_omega;
    f.mult_dual = c.trial_eta * c.trial_omega;
    f.frac = c.avg_frac;
}

static_assert(kFusedThreads == kFusedCtaThreads, "the engine sizes clusters by this CTA size");
// Step factors a fused launch keeps in shared memory (trials past them read
// the options' table).
constexpr int kFusedFactors = 160;

// Distributed shared memory of rank `r`: the address of `local` there, and
// stores of the snapshot's fields.
__device__ __forceinline__ uint32_t rank_addr(const void* local, uint32_t r) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local));
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(a), "r"(r));
    return out;
}
__device__ __forceinline__ void st_cluster_i32(uint32_t addr, int v) {
    asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// Lane r in [1, C) of rank 0's first warp copies the snapshot (written by lane
// 0 before) into CTA r's `f`; the cluster barrier that follows publishes it.
__device__ __forceinline__ void fused_publish(const FusedCtl& f, uint32_t C, int lane) {
    __syncwarp();
    if (lane >= 1 && static_cast<uint32_t>(lane) < C) {
        const uint32_t a = rank_addr(&f, static_cast<uint32_t>(lane));
        const int4* w = reinterpret_cast<const int4*>(&f);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int4 v = w[q];
            asm volatile("st.shared::cluster.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a + 16u * q), "r"(v.x),
                         "r"(v.y), "r"(v.z), "r"(v.w)
                         : "memory");
        }
    }
}

// One warp's slice of one side, staged in shared memory for the launch: the
// cluster barriers between the halves acquire at cluster scope, after which
// the SM's L1 holds nothing of global memory, so the slice's entries and its
// lines' constants would otherwise come from L2 in every trial.
template <class T>
struct FusedLane {
    const int32_t* idx;   // [32 * steps], the layout of the slice data
    const T* val;
    const T* k;           // line constants [consts][32]
    T* v;                 // the lines' own iterates [vecs][32] (launches with copies)
    LanePos lp;
    int steps, len;
    bool has, owner;
};

// Carves the warp's region of one side: the slice's entries, its lines'
// constants and, with copies, the lines' own iterates (`nvecs` vectors).
template <class T>
__device__ __forceinline__ void fused_stage(const Side& side, const T* vals, int64_t data_base, int len_base,
                                            int s, bool has, unsigned char* dst, const T* const* consts,
                                            int nconsts, const T* const* vecs, int nvecs, int lane,
                                            FusedLane<T>& L) {
    L.has = has;
    L.owner = false;
    L.steps = 0;
    L.len = 0;
    if (!has) return;
    const SliceDesc sd = side.slices[s];
    L.lp = lane_pos(sd, lane);
    L.owner = L.lp.valid && L.lp.g == 0;
    L.steps = sd.steps;
    L.len = L.lp.valid ? side.line_len[len_base + L.lp.line] : 0;
    int32_t* idx = reinterpret_cast<int32_t*>(dst);
    T* val = reinterpret_cast<T*>(dst + 4 * 32 * sd.steps);
    T* k = val + 32 * sd.steps;
    const int64_t base = data_base + static_cast<int64_t>(sd.data_off) * 32;
    for (int q = lane; q < 32 * sd.steps; q += 32) {
        idx[q] = side.idx[base + q];
        val[q] = vals[base + q];
    }
    for (int c = 0; c < nconsts; ++c) k[c * 32 + lane] = L.owner ? consts[c][L.lp.line] : T(0);
    T* v = k + 32 * nconsts;
    for (int c = 0; c < nvecs; ++c) v[c * 32 + lane] = L.owner ? vecs[c][L.lp.line] : T(0);
    __syncwarp();
    L.idx = idx;
    L.val = val;
    L.k = k;
    L.v = v;
}

// line_sums over a staged slice: the same products added in the same order
// (steps 0, 1, ... of the lane, then the lane group's butterfly), with eight
// gathers in flight since the entries come from shared memory; `get(i)`
// gathers element i of the other side's vector.
template <int V, class T, class Get>
__device__ __forceinline__ void staged_sums(const FusedLane<T>& L, int lane, Get get, T (&acc)[1]) {
    constexpr int kAhead = 8;
    for (int s0 = 0; s0 < L.steps; s0 += kAhead) {
        T gv[kAhead], wv[kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const int st = s0 + u;
            gv[u] = T(0);
            wv[u] = T(0);
            if (st < L.steps && (st << L.lp.glog) + L.lp.g < L.len) {
                const int q = (st / V) * (32 * V) + lane * V + st % V;
                wv[u] = L.val[q];
                gv[u] = get(L.idx[q]);
            }
        }
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const int st = s0 + u;
            if (st < L.steps && (st << L.lp.glog) + L.lp.g < L.len) acc[0] += wv[u] * gv[u];
        }
    }
    for (int o = (1 << L.lp.glog) >> 1; o > 0; o >>= 1) acc[0] += __shfl_xor_sync(kFull, acc[0], o);
}

// fused_primal over the warp's staged slice.
template <class T, int V>
__device__ __forceinline__ double fused_primal_staged(const Work<T>& w, const InstanceInfo& inf, const FusedCtl& f,
                                                      const FusedLane<T>& L, int lane) {
    const int p = f.parity;
    const T mult = static_cast<T>(f.mult_primal);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* y = w.Y[p] + inf.row_off;
    const T* x = w.X[p] + inf.col_off;
    T* xt = w.X[p ^ 1] + inf.col_off;
    T* avg = w.avg_x + inf.col_off;
    const int j = L.lp.line;
    T prev = T(0), aj = T(0);
    if (L.owner) {
        prev = __ldcg(x + j);
        if (pending) aj = __ldcg(avg + j);
    }
    T sum[1] = {T(0)};
    staged_sums<V>(L, lane, [&](int i) { return __ldcg(y + i); }, sum);
    double moved = 0.0;
    if (L.owner) {
        const T cj = L.k[lane], loj = L.k[32 + lane], hij = L.k[64 + lane];
        const T tj = L.k[96 + lane], itj = L.k[128 + lane];
        const T gradient = cj + sum[0];
        const T upd = smax(loj, smin(prev - mult * tj * gradient, hij));
        xt[j] = upd;
        const double d = static_cast<double>(upd - prev);
        moved += d * d * static_cast<double>(itj);
        if (pending) avg[j] = aj + frac * (prev - aj);
    }
    return moved;
}

// fused_dual over the warp's staged slice.
template <class T, int V>
__device__ __forceinline__ void fused_dual_staged(const Work<T>& w, const InstanceInfo& inf, const FusedCtl& f,
                                                  const FusedLane<T>& L, int lane, double (&red)[2]) {
    const int p = f.parity;
    const T dm = static_cast<T>(f.mult_dual);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* xt = w.X[p ^ 1] + inf.col_off;
    const T* y = w.Y[p] + inf.row_off;
    T* yt = w.Y[p ^ 1] + inf.row_off;
    const T* ax = w.AX[p] + inf.row_off;
    T* axt = w.AX[p ^ 1] + inf.row_off;
    T* avg = w.avg_y + inf.row_off;
    const int i = L.lp.line;
    T axi = T(0), prev = T(0), ai = T(0);
    if (L.owner) {
        axi = __ldcg(ax + i);
        prev = __ldcg(y + i);
        if (pending) ai = __ldcg(avg + i);
    }
    T sum[1] = {T(0)};
    staged_sums<V>(L, lane, [&](int j) { return __ldcg(xt + j); }, sum);
    if (L.owner) {
        const T sgi = L.k[lane], isi = L.k[32 + lane], loi = L.k[64 + lane], hii = L.k[96 + lane];
        const T next = sum[0];
        const T dact = next - axi;
        const T ext = next + dact;
        const T step = smax(dm * sgi, min_dual_step<T>());
        const T v = prev + step * ext;
        const T upd = smax(v - step * hii, T(0)) + smin(v - step * loi, T(0));
        yt[i] = upd;
        axt[i] = next;
        const double d = static_cast<double>(upd - prev);
        red[0] += d * d * static_cast<double>(isi);
        red[1] += d * static_cast<double>(dact);
        if (pending) avg[i] = ai + frac * (prev - ai);
    }
}

// Launches with copies: every CTA holds the instance's whole x and y (both
// parities) in its shared memory, so the gathers are local; the owner lane of
// a line writes its new value into every CTA's copy (the lanes of a slice own
// consecutive lines, so each remote store is one contiguous run), and keeps
// the line's average (and Ax) in its own region. No trial touches global
// memory.
template <class T>
struct FusedCopies {
    T* x[2];   // [n] each, this CTA's copy
    T* y[2];   // [m] each
};

// The value v of element `e` of a copied vector, stored into all C copies.
template <class T>
__device__ __forceinline__ void store_copies(const T* elem, T v, uint32_t C);
template <>
__device__ __forceinline__ void store_copies<double>(const double* elem, double v, uint32_t C) {
    for (uint32_t r = 0; r < C; ++r) st_cluster(rank_addr(elem, r), v);
}
template <>
__device__ __forceinline__ void store_copies<float>(const float* elem, float v, uint32_t C) {
    for (uint32_t r = 0; r < C; ++r)
        asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(rank_addr(elem, r)), "f"(v) : "memory");
}

// fused_primal with copies; own region: the line's average.
template <class T, int V>
__device__ __forceinline__ double fused_primal_copies(const FusedCtl& f, const FusedLane<T>& L,
                                                      const FusedCopies<T>& cc, uint32_t C, int lane) {
    const int p = f.parity;
    const T mult = static_cast<T>(f.mult_primal);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* y = cc.y[p];
    const int j = L.lp.line;
    T prev = T(0), aj = T(0);
    if (L.owner) {
        prev = cc.x[p][j];
        if (pending) aj = L.v[lane];
    }
    T sum[1] = {T(0)};
    staged_sums<V>(L, lane, [&](int i) { return y[i]; }, sum);
    double moved = 0.0;
    if (L.owner) {
        const T cj = L.k[lane], loj = L.k[32 + lane], hij = L.k[64 + lane];
        const T tj = L.k[96 + lane], itj = L.k[128 + lane];
        const T gradient = cj + sum[0];
        const T upd = smax(loj, smin(prev - mult * tj * gradient, hij));
        store_copies<T>(cc.x[p ^ 1] + j, upd, C);
        const double d = static_cast<double>(upd - prev);
        moved += d * d * static_cast<double>(itj);
        if (pending) L.v[lane] = aj + frac * (prev - aj);
    }
    return moved;
}

// fused_dual with copies; own region: Ax of both parities, the average.
template <class T, int V>
__device__ __forceinline__ void fused_dual_copies(const FusedCtl& f, const FusedLane<T>& L,
                                                  const FusedCopies<T>& cc, uint32_t C, int lane,
                                                  double (&red)[2]) {
    const int p = f.parity;
    const T dm = static_cast<T>(f.mult_dual);
    const bool pending = f.pending != 0;
    const T frac = static_cast<T>(f.frac);
    const T* xt = cc.x[p ^ 1];
    const int i = L.lp.line;
    T axi = T(0), prev = T(0), ai = T(0);
    if (L.owner) {
        axi = L.v[p * 32 + lane];
        prev = cc.y[p][i];
        if (pending) ai = L.v[64 + lane];
    }
    T sum[1] = {T(0)};
    staged_sums<V>(L, lane, [&](int jj) { return xt[jj]; }, sum);
    if (L.owner) {
        const T sgi = L.k[lane], isi = L.k[32 + lane], loi = L.k[64 + lane], hii = L.k[96 + lane];
        const T next = sum[0];
        const T dact = next - axi;
        const T ext = next + dact;
        const T step = smax(dm * sgi, min_dual_step<T>());
        const T v = prev + step * ext;
        const T upd = smax(v - step * hii, T(0)) + smin(v - step * loi, T(0));
        store_copies<T>(cc.y[p ^ 1] + i, upd, C);
        L.v[(p ^ 1) * 32 + lane] = next;
        const double d = static_cast<double>(upd - prev);
        red[0] += d * d * static_cast<double>(isi);
        red[1] += d * static_cast<double>(dact);
        if (pending) L.v[64 + lane] = ai + frac * (prev - ai);
    }
}

// One thread per CTA-map entry of rank 0 replaces the entry's slice sums
// (`nq` values per slice) by their in-order total, stored at the entry's
// first slice. Table word: first slice << 4 | slice count.
__device__ __forceinline__ void fused_entry_totals(const int32_t* tab, int entries, double* part, int nq) {
    for (int e = static_cast<int>(threadIdx.x); e < entries; e += kFusedThreads) {
        const int first = tab[e] >> 4, cnt = tab[e] & 15;
        if (cnt == 0) continue;
        for (int q = 0; q < nq; ++q) {
            double t = 0.0;
            for (int k = 0; k < cnt; ++k) t += part[(first + k) * nq + q];
            part[first * nq + q] = t;
        }
    }
}

__device__ __forceinline__ double fused_entry(const int32_t* tab, int e, const double* part, int nq, int q) {
    return (tab[e] & 15) ? part[(tab[e] >> 4) * nq + q] : 0.0;
}

template <class T, int V>
__global__ void __launch_bounds__(kFusedThreads, 1) k_fused(Global g, Work<T> w, DeviceOptions o,
                                                           int max_trials, FusedShape fs) {
    // Rank 0 keeps the instance's control block in its shared memory for the
    // whole launch (the decision's reads and writes stay on chip), writes
    // each trial's snapshot into every CTA's `f`, and receives every slice's
    // warp sums in `part_p` / `part_d` through distributed shared memory. The
    // block goes back to global memory when the launch ends.
    __shared__ DeviceOptions so;
    __shared__ FusedCtl f;
    __shared__ alignas(16) InstanceCtl sctl;
    // Rank 0: step_pow entries of iteration indices fac0 .. fac0 + nfac - 1.
    __shared__ double sfac[2 * kFusedFactors];
    __shared__ int64_t fac0;
    __shared__ int nfac;
    extern __shared__ __align__(16) unsigned char fused_smem[];
    double* const part_p = reinterpret_cast<double*>(fused_smem);
    double* const part_d = part_p + fs.slices_p;
    int32_t* const tab_p = reinterpret_cast<int32_t*>(part_d + 2 * fs.slices_d);
    int32_t* const tab_d = tab_p + fs.entries_p;
    unsigned char* const stage = fused_smem + fused_stage_offset(fs);
    T* const copies = reinterpret_cast<T*>(fused_smem + fused_copies_offset(fs));
    const uint32_t C = cluster_size(), rank = cluster_rank();
    const int b = static_cast<int>(blockIdx.x / C);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    InstanceCtl* cp = g.ctl + b;
    const InstanceInfo inf = g.info[b];
    // The instance's slices are contiguous in its CTA map (append_cta_map).
    const int ps0 = g.at.ctas[inf.at_cta_begin].slice_begin, ps1 = g.at.ctas[inf.at_cta_end - 1].slice_end;
    const int ds0 = g.a.ctas[inf.a_cta_begin].slice_begin, ds1 = g.a.ctas[inf.a_cta_end - 1].slice_end;
    const int ne_p = inf.at_cta_end - inf.at_cta_begin, ne_d = inf.a_cta_end - inf.a_cta_begin;
    // One warp per slice: slice s goes to warp s mod (cluster warps).
    const int stride = static_cast<int>(C) * kFusedWarps;
    const int slot = static_cast<int>(rank) * kFusedWarps + warp;
    constexpr bool kFp64 = sizeof(T) == 8;
    const T* vals_p = matrix_values<T>(g.at);
    const T* vals_d = matrix_values<T>(g.a);
    if (threadIdx.x == 0) so = o;
    if (rank == 0) {
        static_assert(sizeof(InstanceCtl) % 16 == 0, "the control block copies as 16-byte words");
        if (threadIdx.x < sizeof(InstanceCtl) / 16)
            reinterpret_cast<int4*>(&sctl)[threadIdx.x] = reinterpret_cast<const int4*>(cp)[threadIdx.x];
        for (int e = threadIdx.x; e < ne_p; e += kFusedThreads) {
            const CtaWork cw = g.at.ctas[inf.at_cta_begin + e];
            tab_p[e] = ((cw.slice_begin - ps0) << 4) | (cw.slice_end - cw.slice_begin);
        }
        for (int e = threadIdx.x; e < ne_d; e += kFusedThreads) {
            const CtaWork cw = g.a.ctas[inf.a_cta_begin + e];
            tab_d[e] = ((cw.slice_begin - ds0) << 4) | (cw.slice_end - cw.slice_begin);
        }
        // The linesearch's step factors of the launch's iteration indices
        // (one phase per launch: a phase ends at a check, which ends it).
        {
            const InstanceCtl& c0 = *cp;
            const int64_t k0 = c0.phase == kPhasePolish ? c0.polish_iteration : c0.iteration;
            const int64_t avail = k0 >= 0 && k0 < o.step_pow_entries ? o.step_pow_entries - k0 : 0;
            const int n = static_cast<int>(avail < kFusedFactors ? avail : kFusedFactors);
            for (int q = threadIdx.x; q < 2 * n; q += kFusedThreads) sfac[q] = o.step_pow[2 * k0 + q];
            if (threadIdx.x == 0) {
                fac0 = k0;
                nfac = n;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) fused_snapshot(sctl, f, kFp64);
    }
    // Staged launches give every warp at most one slice per side; with
    // copies, the x and y of both parities are in every CTA.
    const bool staged = fs.stage_bytes > 0 && fs.elem == static_cast<int>(sizeof(T));
    const bool with_copies = staged && fs.lines > 0;
    FusedLane<T> LP{}, LD{};
    FusedCopies<T> cc{};
    T* const xg[2] = {w.X[0] + inf.col_off, w.X[1] + inf.col_off};
    T* const yg[2] = {w.Y[0] + inf.row_off, w.Y[1] + inf.row_off};
    // The lines' own iterates with copies: primal the average; dual Ax of
    // both parities, the average.
    const T* const own_p[1] = {w.avg_x + inf.col_off};
    const T* const own_d[3] = {w.AX[0] + inf.row_off, w.AX[1] + inf.row_off, w.avg_y + inf.row_off};
    const int words_p = kFusedPrimalConsts + (with_copies ? kFusedPrimalOwn : 0);
    const int words_d = kFusedDualConsts + (with_copies ? kFusedDualOwn : 0);
    if (with_copies) {
        cc.x[0] = copies;
        cc.x[1] = copies + inf.n;
        cc.y[0] = copies + 2 * inf.n;
        cc.y[1] = copies + 2 * inf.n + inf.m;
        for (int q = threadIdx.x; q < inf.n; q += kFusedThreads) {
            cc.x[0][q] = xg[0][q];
            cc.x[1][q] = xg[1][q];
        }
        for (int q = threadIdx.x; q < inf.m; q += kFusedThreads) {
            cc.y[0][q] = yg[0][q];
            cc.y[1][q] = yg[1][q];
        }
    }
    if (staged) {
        // The warps' shares of the stage, in warp order (lane q of every
        // warp computes warp q's bytes).
        const int sp = ps0 + static_cast<int>(rank) * kFusedWarps + lane;
        const int sd = ds0 + static_cast<int>(rank) * kFusedWarps + lane;
        int need = 0;
        if (lane < kFusedWarps) {
            if (sp < ps1) need += fused_slice_bytes(g.at.slices[sp].steps, words_p, sizeof(T));
            if (sd < ds1) need += fused_slice_bytes(g.a.slices[sd].steps, words_d, sizeof(T));
        }
        int incl = need;
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += t;
        }
        const int off = __shfl_sync(kFull, incl - need, warp);
        const int s_p = ps0 + slot, s_d = ds0 + slot;
        const T* const cp_consts[kFusedPrimalConsts] = {w.c + inf.col_off, w.xl + inf.col_off, w.xu + inf.col_off,
                                                        w.tau + inf.col_off, w.itau + inf.col_off};
        const T* const cd_consts[kFusedDualConsts] = {w.sigma + inf.row_off, w.isigma + inf.row_off,
                                                      w.rl + inf.row_off, w.ru + inf.row_off};
        fused_stage<T>(g.at, vals_p, inf.at_data_base, inf.at_len_base, s_p, s_p < ps1, stage + off, cp_consts,
                       kFusedPrimalConsts, own_p, with_copies ? kFusedPrimalOwn : 0, lane, LP);
        const int off_d = off + (s_p < ps1 ? fused_slice_bytes(LP.steps, words_p, sizeof(T)) : 0);
        fused_stage<T>(g.a, vals_d, inf.a_data_base, inf.a_len_base, s_d, s_d < ds1, stage + off_d, cd_consts,
                       kFusedDualConsts, own_d, with_copies ? kFusedDualOwn : 0, lane, LD);
    }
    const uint32_t pp_addr = rank0_addr(part_p);
    const uint32_t pd_addr = rank0_addr(part_d);
    // Remote shared memory is written only once every CTA of the cluster
    // runs: the first snapshot goes out after a barrier.
    cluster_sync_all();
    if (rank == 0 && threadIdx.x < 32) fused_publish(f, C, lane);
    cluster_sync_all();
    for (int t = 0; t < max_trials; ++t) {
        if (!f.active) break;
        if (with_copies) {
            if (LP.has) {
                double v[1] = {fused_primal_copies<T, V>(f, LP, cc, C, lane)};
                warp_sum<1>(v);
                if (lane == 0) st_cluster(pp_addr + 8u * static_cast<uint32_t>(slot), v[0]);
            }
        } else if (staged) {
            if (LP.has) {
                double v[1] = {fused_primal_staged<T, V>(w, inf, f, LP, lane)};
                warp_sum<1>(v);
                if (lane == 0) st_cluster(pp_addr + 8u * static_cast<uint32_t>(ps0 + slot - ps0), v[0]);
            }
        } else {
            for (int s = ps0 + slot; s < ps1; s += stride) {
                const CtaWork one{b, s, s + 1, 0};
                double v[1] = {fused_primal<T, V>(g, w, one, inf, f, lane)};
                warp_sum<1>(v);
                if (lane == 0) st_cluster(pp_addr + 8u * static_cast<uint32_t>(s - ps0), v[0]);
            }
        }
        cluster_sync_all();
        if (with_copies) {
            if (LD.has) {
                double r2[2] = {0.0, 0.0};
                fused_dual_copies<T, V>(f, LD, cc, C, lane, r2);
                warp_sum<2>(r2);
                if (lane == 0) {
                    const uint32_t q = 16u * static_cast<uint32_t>(slot);
                    st_cluster(pd_addr + q, r2[0]);
                    st_cluster(pd_addr + q + 8u, r2[1]);
                }
            }
        } else if (staged) {
            if (LD.has) {
                double r2[2] = {0.0, 0.0};
                fused_dual_staged<T, V>(w, inf, f, LD, lane, r2);
                warp_sum<2>(r2);
                if (lane == 0) {
                    const uint32_t q = 16u * static_cast<uint32_t>(slot);
                    st_cluster(pd_addr + q, r2[0]);
                    st_cluster(pd_addr + q + 8u, r2[1]);
                }
            }
        } else {
            for (int s = ds0 + slot; s < ds1; s += stride) {
                const CtaWork one{b, s, s + 1, 0};
                double r2[2] = {0.0, 0.0};
                fused_dual<T, V>(g, w, one, inf, f, lane, r2);
                warp_sum<2>(r2);
                if (lane == 0) {
                    const uint32_t q = 16u * static_cast<uint32_t>(s - ds0);
                    st_cluster(pd_addr + q, r2[0]);
                    st_cluster(pd_addr + q + 8u, r2[1]);
                }
            }
        }
        cluster_sync_all();
        if (rank == 0) {
            if (fs.multi) {
                // (With one slice per entry an entry's total, 0 + its slice's
                // sum, is that sum: a sum of lane values that start at +0 is
                // never -0.)
                fused_entry_totals(tab_p, ne_p, part_p, 1);
                fused_entry_totals(tab_d, ne_d, part_d, 2);
                __syncthreads();
            }
            if (threadIdx.x < 32) {
                // k_dual's fixed-order sums over the entries' totals
                // (warp_range_sums3: entries lane, lane + 32, ... in order,
                // then the butterfly).
                double sums[3] = {0.0, 0.0, 0.0};
                for (int e = lane; e < ne_p; e += 32) sums[0] += fused_entry(tab_p, e, part_p, 1, 0);
                for (int e = lane; e < ne_d; e += 32) {
                    sums[1] += fused_entry(tab_d, e, part_d, 2, 0);
                    sums[2] += fused_entry(tab_d, e, part_d, 2, 1);
                }
                warp_sum<3>(sums);
                if (threadIdx.x == 0) {
                    const int64_t k = sctl.phase == kPhasePolish ? sctl.polish_iteration : sctl.iteration;
                    const double* fk = k >= fac0 && k - fac0 < nfac ? sfac + 2 * (k - fac0) : nullptr;
                    trial_control(sctl, so, sums[0], sums[1], sums[2], inf.n, fk);
                    fused_snapshot(sctl, f, kFp64);
                }
                fused_publish(f, C, lane);
            }
        }
        cluster_sync_all();
    }
    // Every CTA left the loop at the same trial (the same snapshot after the
    // same barrier); the barrier keeps every CTA's shared memory alive until
    // the last remote store into it has landed.
    cluster_sync_all();
    if (with_copies) {
        // Every copy is the same: rank 0 writes x and y back, the owner lanes
        // their lines' own iterates.
        if (rank == 0) {
            for (int q = threadIdx.x; q < inf.n; q += kFusedThreads) {
                xg[0][q] = cc.x[0][q];
                xg[1][q] = cc.x[1][q];
            }
            for (int q = threadIdx.x; q < inf.m; q += kFusedThreads) {
                yg[0][q] = cc.y[0][q];
                yg[1][q] = cc.y[1][q];
            }
        }
        if (LP.has && LP.owner) w.avg_x[inf.col_off + LP.lp.line] = LP.v[lane];
        if (LD.has && LD.owner) {
            const int i = inf.row_off + LD.lp.line;
            w.AX[0][i] = LD.v[lane];
            w.AX[1][i] = LD.v[32 + lane];
            w.avg_y[i] = LD.v[64 + lane];
        }
    }
    if (rank == 0) {
        if (threadIdx.x < sizeof(InstanceCtl) / 16)
            reinterpret_cast<int4*>(cp)[threadIdx.x] = reinterpret_cast<const int4*>(&sctl)[threadIdx.x];
    }
}

// ---------------------------------------------------------------------------
// Check, elementwise part (termination.cpp rowPass/columnPass terms without a
// product, infeasibility.cpp normalisation and cone projections,
// pdlp_solver.cpp:373-389 and :455-459)
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) k_check_prep(Global g, Work<T> w, DeviceOptions o) {
    const VecWork vw = g.vec[blockIdx.x];
    const InstanceCtl& c = g.ctl[vw.instance];
    if (c.stage != kStageCheck || c.check_kind == kCheckTransition || !precision_matches<T>(c)) return;
    const InstanceInfo inf = g.info[vw.instance];
    const int p = c.parity;
    const bool pending = c.pending_avg != 0;
    const T frac = static_cast<T>(c.avg_frac);
    const bool have_avg = check_have_avg(c, o);
    const bool rays =
        (c.check_kind == kCheckMain || c.check_kind == kCheckEvaluate) && o.detect_infeasibility;

    double acc[kPrepSlots];
#pragma unroll
    for (int q = 0; q < kPrepSlots; ++q) acc[q] = 0.0;

    if (!vw.is_row) {
        const int64_t off = inf.col_off;
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const int64_t k = off + j;
            const T x = w.X[p][k];
            T a = w.avg_x[k];
            if (pending) {
                a = a + frac * (x - a);
                w.avg_x[k] = a;
            }
            const double cs = g.cs[k];
            const double xo = cs * static_cast<double>(x);
            g.x_o[k] = xo;
            const double co = g.c_orig[k];
            acc[0] += co * xo;
            if (have_avg) {
                const double xao = cs * static_cast<double>(a);
                g.xa_o[k] = xao;
                acc[1] += co * xao;
            }
            if (rays) {
                const double d = cs * (static_cast<double>(x) - static_cast<double>(w.rx[k]));
                acc[2] += d * d;
                double q = d;
                if (isfinite(g.xu_orig[k])) q = smin(q, 0.0);
                if (isfinite(g.xl_orig[k])) q = smax(q, 0.0);
                const double drift = d - q;
                acc[3] += drift * drift;
                acc[4] += co * q;
                g.p_proj[k] = q;
            }
            if (c.check_kind == kCheckMain) {
                const double r = static_cast<double>(w.rx[k]);
                const double dc = static_cast<double>(x) - r;
                acc[5] += dc * dc;
                const double da = static_cast<double>(a) - r;
                acc[6] += da * da;
            }
        }
    } else {
        const int64_t off = inf.row_off;
        for (int i = vw.begin + threadIdx.x; i < vw.end; i += blockDim.x) {
            const int64_t k = off + i;
            const T y = w.Y[p][k];
            T a = w.avg_y[k];
            if (pending) {
                a = a + frac * (y - a);
                w.avg_y[k] = a;
            }
            const double rs = g.rs[k];
            const double lo = g.rl_orig[k], hi = g.ru_orig[k];
            const bool lo_f = isfinite(lo), hi_f = isfinite(hi);
            const double yo = rs * static_cast<double>(y);
            g.y_o[k] = yo;
            {
                double q = yo;
                if (!hi_f) q = smin(q, 0.0);
                if (!lo_f) q = smax(q, 0.0);
                const double drift = yo - q;
                acc[1] += drift * drift;
                if (q > 0.0) acc[0] += q * hi;
                else if (q < 0.0) acc[0] += q * lo;
            }
            if (have_avg) {
                const double yao = rs * static_cast<double>(a);
                g.ya_o[k] = yao;
                double q = yao;
                if (!hi_f) q = smin(q, 0.0);
                if (!lo_f) q = smax(q, 0.0);
                const double drift = yao - q;
                acc[3] += drift * drift;
                if (q > 0.0) acc[2] += q * hi;
                else if (q < 0.0) acc[2] += q * lo;
            }
            if (rays) {
                const double d = rs * (static_cast<double>(y) - static_cast<double>(w.ry[k]));
                g.dy_o[k] = d;
                acc[4] += d * d;
                double q = d;
                if (!hi_f) q = smin(q, 0.0);
                if (!lo_f) q = smax(q, 0.0);
                const double drift = d - q;
                acc[5] += drift * drift;
                if (q > 0.0) acc[6] += q * hi;
                else if (q < 0.0) acc[6] += q * lo;
            }
            if (c.check_kind == kCheckMain) {
                const double r = static_cast<double>(w.ry[k]);
                const double dc = static_cast<double>(y) - r;
                acc[7] += dc * dc;
                const double da = static_cast<double>(a) - r;
                acc[8] += da * da;
            }
        }
    }
    block_sum<kPrepSlots>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kPrepSlots; ++q)
            g.part_prep[static_cast<int64_t>(blockIdx.x) * kPrepSlots + q] = acc[q];
    }
}

// ---------------------------------------------------------------------------
// Check, matrix passes and decision
// ---------------------------------------------------------------------------
// The decision of one check from its sums (pdlp_solver.cpp:239-476,
// feasibility_polishing.cpp:107-141). C/R: column- and row-side elementwise
// sums (kPrepSlots each), A3: row-pass sums, T6: column-pass sums.
// `ndg`: with normalised-gap restarts at a main check, the gaps of the
// current and average iterates (else null).
__device__ __noinline__ void check_decide(const DeviceOptions& o, InstanceCtl& c, int32_t n_cols,
                                          const double* C, const double* R, const double* A3,
                                          const double* T6, const double* ndg) {

    c.pending_avg = 0;
    const bool have_avg = check_have_avg(c, o);
    const Metrics cur = make_metrics(c, A3[0], R[0], R[1], C[0], T6[1], T6[0]);
    const Metrics avg = have_avg ? make_metrics(c, A3[1], R[2], R[3], C[1], T6[3], T6[2]) : cur;

    if (c.check_kind == kCheckEvaluate) {
        store_best(c, cur);
        for (int q = 3; q < 12; ++q) c.dbg[q] = 0.0;
        const double dn = sqrt(R[4]);
        if (o.detect_infeasibility && dn > 1e-300 && isfinite(dn)) {
            const double inv = 1.0 / dn;
            const double value = (T6[5] - R[6]) * inv;
            c.dbg[4] = value;
            c.dbg[5] = 1.0;
            if (isfinite(value) && value > 0.0) {
                c.dbg[5] = sqrt(T6[4] + R[5]) * inv / value;
                c.dbg[3] = c.dbg[5] <= o.infeasibility_tol ? 1.0 : 0.0;
            }
        }
        const double pn = sqrt(C[2]);
        if (o.detect_infeasibility && pn > 1e-300 && isfinite(pn)) {
            const double inv = 1.0 / pn;
            const double rate = C[4] * inv;
            c.dbg[7] = rate;
            c.dbg[8] = 1.0;
            if (isfinite(rate) && rate < 0.0) {
                c.dbg[8] = sqrt(C[3] + A3[2]) * inv / (-rate);
                c.dbg[6] = c.dbg[8] <= o.infeasibility_tol ? 1.0 : 0.0;
            }
        }
        c.stage = kStageTrial;
        c.phase = kPhaseDone;
        return;
    }

    if (c.check_kind == kCheckInitial) {
        // pdlp_solver.cpp:239-264 (a warm start competes with the cold point,
        // which sits in the average buffers).
        c.restart_src = 1;
        Metrics start = cur;
        c.best_src = 1;
        if (have_avg && avg.kkt < cur.kkt) {
            start = avg;
            c.best_src = 2;
            c.restart_src = 2;
            c.need_refresh = 1;
        }
        store_best(c, start);
        // A normalised gap needs a radius, which the starting point does not
        // have yet: only the artificial test can trigger the first restart.
        c.restart_baseline = o.ndg_restarts ? INFINITY : start.kkt;
        c.avg_weight = 0.0;
        c.have_avg_at_check = 0;
        if (is_optimal_best(c, o)) {
            finish(c, 0, kMsgInitialOptimal, false);
            return;
        }
        loop_top_main(c, o, n_cols);
        return;
    }

    if (c.check_kind == kCheckPolish) {   // feasibility_polishing.cpp:107-141
        if (c.polish_deadline_ns > 0 && now_ns() >= c.polish_deadline_ns) {
            end_polish(c, o);
            return;
        }
        if (cur.kkt < c.best_kkt) {
            c.best_src = 1;
            store_best(c, cur);
        }
        if (have_avg && avg.kkt < c.best_kkt) {
            c.best_src = 2;
            store_best(c, avg);
        }
        if (is_optimal_best(c, o) || c.polish_done_iterations == o.polishing_iterations) {
            end_polish(c, o);
            return;
        }
        c.stage = kStageTrial;
        return;
    }

    // Main check (pdlp_solver.cpp:354-476).
    if (cur.kkt < c.best_kkt) {
        c.best_src = 1;
        store_best(c, cur);
    }
    if (have_avg && avg.kkt < c.best_kkt) {
        c.best_src = 2;
        store_best(c, avg);
    }
    if (o.detect_infeasibility) {
        // Dual ray: value = inf_box (A'd)'x - support(d), both linear in d, so
        // the sums over the raw direction are scaled by 1/||d|| afterwards.
        const double dn = sqrt(R[4]);
        if (dn > 1e-300 && isfinite(dn)) {
            const double inv = 1.0 / dn;
            const double value = (T6[5] - R[6]) * inv;
            if (isfinite(value) && value > 0.0) {
                const double viol = sqrt(T6[4] + R[5]) * inv;
                if (viol / value <= o.infeasibility_tol) {
                    finish(c, 1, kMsgInfeasible, true);
                    c.save_ray = 1;
                    c.ray_kind = 1;
                    return;
                }
            }
        }
        const double pn = sqrt(C[2]);
        if (pn > 1e-300 && isfinite(pn)) {
            const double inv = 1.0 / pn;
            const double rate = C[4] * inv;
            if (isfinite(rate) && rate < 0.0) {
                const double viol = sqrt(C[3] + A3[2]) * inv;
                if (viol / (-rate) <= o.infeasibility_tol) {
                    finish(c, 2, kMsgUnbounded, true);
                    c.save_ray = 2;
                    c.ray_kind = 2;
                    return;
                }
            }
        }
    }
    if (is_optimal_best(c, o)) {
        finish(c, 0, kMsgOptimal, true);
        return;
    }
    double score;
    const int choice = ndg ? restart_choose(c, o, ndg[0], ndg[1], &score)
                           : restart_choose(c, o, cur.kkt, avg.kkt, &score);
    if (choice != 0) {
        const bool from_avg = choice == 2 && have_avg;
        update_weight(c.omega, o, sqrt(from_avg ? C[6] : C[5]), sqrt(from_avg ? R[8] : R[7]));
        c.trial_omega = c.omega;
        c.restart_src = from_avg ? 2 : 1;
        if (from_avg) c.need_refresh = 1;
        c.restart_baseline = score;
        c.avg_weight = 0.0;
        c.prev_candidate = INFINITY;
        c.since_restart = 0;
        ++c.restart_count;
    }
    if (o.mixed && !c.fp64_stage) {
        // Mixed precision: FP32 iterations go on while the best KKT score
        // keeps falling or is still far (above fp32_switch_kkt) from the
        // tolerance; after fp32_stall_checks checks without a 10% drop the
        // instance continues in FP64 from its last FP32 restart point (the
        // restart point this check may just have set), with a fresh average.
        if (!(c.best_kkt_at_stall > 0.0) || c.best_kkt < 0.9 * c.best_kkt_at_stall ||
            !(c.best_kkt <= o.fp32_switch_kkt)) {
            c.best_kkt_at_stall = c.best_kkt;
            c.stall_checks = 0;
        } else if (++c.stall_checks >= o.fp32_stall_checks) {
            c.to_fp64 = 1;
            c.need_refresh = 1;
            c.avg_weight = 0.0;
            c.since_restart = 0;
            c.prev_candidate = INFINITY;
            c.stall_checks = 0;
        }
    }
    loop_top_main(c, o, n_cols);
}

__device__ __noinline__ void check_control(const Global& g, const DeviceOptions& o, InstanceCtl& c,
                              const InstanceInfo& inf, const double* ndg) {
    // Column-side and row-side elementwise partials.
    double C[kPrepSlots], R[kPrepSlots], A3[3], T6[kCheckSlots];
    for (int q = 0; q < kPrepSlots; ++q) { C[q] = 0.0; R[q] = 0.0; }
    const int lane = threadIdx.x & 31;
    for (int q = 0; q < kPrepSlots; ++q) {
        double tc = 0.0, tr = 0.0;
        for (int k = inf.vec_cta_begin + lane; k < inf.vec_cta_end; k += 32) {
            const double v = g.part_prep[static_cast<int64_t>(k) * kPrepSlots + q];
            if (g.vec[k].is_row) tr += v; else tc += v;
        }
        for (int s = 16; s > 0; s >>= 1) {
            tc += __shfl_xor_sync(kFull, tc, s);
            tr += __shfl_xor_sync(kFull, tr, s);
        }
        C[q] = tc;
        R[q] = tr;
    }
    for (int q = 0; q < 3; ++q)
        A3[q] = warp_range_sum(g.part_check, inf.a_cta_begin, inf.a_cta_end, kCheckSlots, q);
    const int at0 = g.a.num_ctas + inf.at_cta_begin, at1 = g.a.num_ctas + inf.at_cta_end;
    for (int q = 0; q < kCheckSlots; ++q) T6[q] = warp_range_sum(g.part_check, at0, at1, kCheckSlots, q);
    if (lane != 0) return;
    check_decide(o, c, inf.n, C, R, A3, T6, ndg);
}

// The candidate coordinates of a main check in the scaled space of the
// iterations (x = x_o / cs, y = y_o / rs, c + A'y scaled by cs, A x by rs,
// bounds scaled like the iterates), from what the check stored in original
// coordinates; the restart point comes from the working arrays.
struct CheckNdgCoord {
    const Global* g;
    int64_t col0, row0, n;
    int which;    // 0 current, 1 average
    bool fp32;    // restart point in the FP32 working arrays
    __device__ NdgCoord operator()(int64_t k) const {
        NdgCoord q;
        if (k < n) {
            const int64_t j = col0 + k;
            const double cs = g->cs[j], ics = 1.0 / cs;
            q.v = (which ? g->xa_o[j] : g->x_o[j]) * ics;
            q.d = cs * g->ndg_g[which][j];
            q.lo = g->xl_orig[j] * ics;
            q.hi = g->xu_orig[j] * ics;
            q.r = fp32 ? static_cast<double>(g->rx32[j]) : g->rx64[j];
        } else {
            const int64_t i = row0 + (k - n);
            const double rs = g->rs[i];
            q.v = (which ? g->ya_o[i] : g->y_o[i]) * (1.0 / rs);
            q.d = rs * g->ndg_a[which][i];
            q.lo = g->rl_orig[i] * rs;
            q.hi = g->ru_orig[i] * rs;
            q.r = fp32 ? static_cast<double>(g->ry32[i]) : g->ry64[i];
        }
        return q;
    }
};

// Normalised gaps of the current and the average iterate (the same value
// twice without an average), computed by the whole CTA; out[0..1] in shared
// memory, valid after the CTA's next barrier.
__device__ __noinline__ void check_ndg(const Global& g, const DeviceOptions& o, const InstanceCtl& c,
                                       const InstanceInfo& inf, double* out) {
    __shared__ double scratch[16 * 32];
    const bool fp32 = o.mixed && !c.fp64_stage;
    CheckNdgCoord q{&g, inf.col_off, inf.row_off, inf.n, 0, fp32};
    const double cur = block_normalized_gap(inf.n, inf.m, c.omega, q, scratch, nullptr);
    double avg = cur;
    if (check_have_avg(c, o)) {
        q.which = 1;
        avg = block_normalized_gap(inf.n, inf.m, c.omega, q, scratch, nullptr);
    }
    if (threadIdx.x == 0) {
        out[0] = cur;
        out[1] = avg;
    }
}

template <int V>
__global__ void __launch_bounds__(kThreads) k_check_spmv(Global g, DeviceOptions o) {
    const bool a_side = blockIdx.x < static_cast<unsigned>(g.a.num_ctas);
    const int cta = a_side ? blockIdx.x : blockIdx.x - g.a.num_ctas;
    const CtaWork cw = (a_side ? g.a.ctas : g.at.ctas)[cta];
    InstanceCtl& c = g.ctl[cw.instance];
    if (c.stage != kStageCheck || c.check_kind == kCheckTransition) return;
    const InstanceInfo inf = g.info[cw.instance];
    const bool have_avg = check_have_avg(c, o);
    const bool rays =
        (c.check_kind == kCheckMain || c.check_kind == kCheckEvaluate) && o.detect_infeasibility;
    const bool ndg = o.ndg_restarts && o.restarts && c.check_kind == kCheckMain;

    double acc[kCheckSlots];
#pragma unroll
    for (int q = 0; q < kCheckSlots; ++q) acc[q] = 0.0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (a_side) {   // rowPass (termination.cpp:66-135) for current/average, A*d for the primal ray
        const double* xo = g.x_o + inf.col_off;
        const double* xa = g.xa_o + inf.col_off;
        const double* pp = g.p_proj + inf.col_off;
        for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
            const SliceDesc sd = g.a.slices[s];
            const LanePos lp = lane_pos(sd, lane);
            const int len = lp.valid ? g.a.line_len[inf.a_len_base + lp.line] : 0;
            double sum[3] = {0.0, 0.0, 0.0};
            line_sums<V, 3>(inf.a_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps,
                            lp, lane, len, g.a.idx, g.a.val_orig, sum,
                            [&](double (&a)[3], double v, int j) {
                                a[0] += v * xo[j];
                                if (have_avg) a[1] += v * xa[j];
                                if (rays) a[2] += v * pp[j];
                            });
            if (lp.valid && lp.g == 0) {
                const int64_t k = inf.row_off + lp.line;
                if (ndg) {
                    g.ndg_a[0][k] = sum[0];
                    if (have_avg) g.ndg_a[1][k] = sum[1];
                }
                const double lo = g.rl_orig[k], hi = g.ru_orig[k];
                const double e0 = sum[0] - smax(lo, smin(sum[0], hi));
                acc[0] += e0 * e0;
                if (have_avg) {
                    const double e1 = sum[1] - smax(lo, smin(sum[1], hi));
                    acc[1] += e1 * e1;
                }
                if (rays) {
                    double q = sum[2];
                    if (isfinite(hi)) q = smin(q, 0.0);
                    if (isfinite(lo)) q = smax(q, 0.0);
                    const double drift = sum[2] - q;
                    acc[2] += drift * drift;
                }
            }
        }
    } else {        // columnPass (termination.cpp:140-209), A'd for the dual ray
        const double* yo = g.y_o + inf.row_off;
        const double* ya = g.ya_o + inf.row_off;
        const double* dy = g.dy_o + inf.row_off;
        for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
            const SliceDesc sd = g.at.slices[s];
            const LanePos lp = lane_pos(sd, lane);
            const int len = lp.valid ? g.at.line_len[inf.at_len_base + lp.line] : 0;
            double sum[3] = {0.0, 0.0, 0.0};
            line_sums<V, 3>(inf.at_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps,
                            lp, lane, len, g.at.idx, g.at.val_orig, sum,
                            [&](double (&a)[3], double v, int i) {
                                a[0] += v * yo[i];
                                if (have_avg) a[1] += v * ya[i];
                                if (rays) a[2] += v * dy[i];
                            });
            if (lp.valid && lp.g == 0) {
                const int64_t k = inf.col_off + lp.line;
                const double co = g.c_orig[k];
                const double lo = g.xl_orig[k], hi = g.xu_orig[k];
                const bool lo_f = isfinite(lo), hi_f = isfinite(hi);
                for (int which = 0; which < 2; ++which) {
                    if (which == 1 && !have_avg) break;
                    const double reduced = co + sum[which];
                    if (ndg) g.ndg_g[which][k] = reduced;
                    double q = reduced;
                    if (!lo_f) q = smin(q, 0.0);
                    if (!hi_f) q = smax(q, 0.0);
                    const double drift = reduced - q;
                    acc[2 * which] += drift * drift;
                    if (q > 0.0) acc[2 * which + 1] += q * lo;
                    else if (q < 0.0) acc[2 * which + 1] += q * hi;
                }
                if (rays) {
                    const double r = sum[2];
                    double q = r;
                    if (!lo_f) q = smin(q, 0.0);
                    if (!hi_f) q = smax(q, 0.0);
                    const double drift = r - q;
                    acc[4] += drift * drift;
                    if (q > 0.0) acc[5] += q * lo;
                    else if (q < 0.0) acc[5] += q * hi;
                }
            }
        }
    }
    block_sum<kCheckSlots>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kCheckSlots; ++q)
            g.part_check[static_cast<int64_t>(blockIdx.x) * kCheckSlots + q] = acc[q];
    }
    const int expected = (inf.a_cta_end - inf.a_cta_begin) + (inf.at_cta_end - inf.at_cta_begin);
    if (!arrive_last(g.count_check + cw.instance, expected)) return;
    // With normalised-gap restarts, k_check_ndg takes the decision.
    if (o.ndg_restarts) return;
    __shared__ DeviceOptions so;   // see k_dual
    if (threadIdx.x == 0) so = o;
    __syncthreads();
    if (threadIdx.x < 32) check_control(g, so, c, inf, nullptr);
}

// The check decision with normalised-gap restarts: one CTA per instance,
// after k_check_spmv. At a main check the CTA first computes the two
// candidates' normalised gaps from the products k_check_spmv stored.
__global__ void __launch_bounds__(kThreads) k_check_ndg(Global g, DeviceOptions o) {
    const int b = blockIdx.x;
    InstanceCtl& c = g.ctl[b];
    if (c.stage != kStageCheck || c.check_kind == kCheckTransition) return;
    const InstanceInfo inf = g.info[b];
    __shared__ DeviceOptions so;   // see k_dual
    __shared__ double gaps[2];
    if (threadIdx.x == 0) so = o;
    __syncthreads();
    const bool main = o.restarts && c.check_kind == kCheckMain;
    if (main) check_ndg(g, so, c, inf, gaps);
    __syncthreads();
    if (threadIdx.x < 32) check_control(g, so, c, inf, main ? gaps : nullptr);
}

// ---------------------------------------------------------------------------
// Check, application of the decisions
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads) k_check_apply(Global g, Work<T> w) {
    const VecWork vw = g.vec[blockIdx.x];
    const InstanceCtl& c = g.ctl[vw.instance];
    if (!(c.best_src || c.restart_src || c.to_polish || c.save_ray)) return;
    if (!precision_matches<T>(c)) return;
    const InstanceInfo inf = g.info[vw.instance];
    const int p = c.parity;
    if (!vw.is_row) {
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const int64_t k = inf.col_off + j;
            if (c.best_src == 1) g.best_x[k] = g.x_o[k];
            else if (c.best_src == 2) g.best_x[k] = g.xa_o[k];
            if (c.save_ray == 2)
                g.pray[k] = g.cs[k] * (static_cast<double>(w.X[p][k]) - static_cast<double>(w.rx[k]));
            if (c.restart_src) {
                if (c.restart_src == 2) w.X[p][k] = w.avg_x[k];
                w.rx[k] = w.X[p][k];
            }
            if (c.to_polish) {   // toScaled (scaling.cpp:39-53)
                w.X[p][k] = static_cast<T>(g.best_x[k] / g.cs[k]);
            }
        }
    } else {
        for (int i = vw.begin + threadIdx.x; i < vw.end; i += blockDim.x) {
            const int64_t k = inf.row_off + i;
            if (c.best_src == 1) g.best_y[k] = g.y_o[k];
            else if (c.best_src == 2) g.best_y[k] = g.ya_o[k];
            if (c.save_ray == 1) g.dray[k] = g.dy_o[k];
            if (c.restart_src) {
                if (c.restart_src == 2) w.Y[p][k] = w.avg_y[k];
                w.ry[k] = w.Y[p][k];
            }
            if (c.to_polish) {
                w.Y[p][k] = static_cast<T>(g.best_y[k] / g.rs[k]);
            }
        }
    }
}

// A x for the current iterate of instances whose iterate was replaced
// (CpuPdhgKernel::refreshActivity, pdhg_kernel.cpp:40-42).
template <class T, int V>
__global__ void __launch_bounds__(kThreads) k_refresh(Global g, Work<T> w) {
    const CtaWork cw = g.a.ctas[blockIdx.x];
    const InstanceCtl& c = g.ctl[cw.instance];
    // An instance moving to the FP64 stage gets its FP64 product here.
    if (!c.need_refresh || !(precision_matches<T>(c) || (sizeof(T) == 8 && c.to_fp64))) return;
    const InstanceInfo inf = g.info[cw.instance];
    const int p = c.parity;
    const T* __restrict__ x = w.X[p] + inf.col_off;
    T* __restrict__ ax = w.AX[p] + inf.row_off;
    const T* vals = matrix_values<T>(g.a);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = g.a.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const int len = lp.valid ? g.a.line_len[inf.a_len_base + lp.line] : 0;
        T sum[1] = {T(0)};
        line_sums<V, 1>(inf.a_data_base + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp,
                        lane, len, g.a.idx, vals, sum,
                        [&](T (&a)[1], T v, int j) { a[0] += v * x[j]; });
        if (lp.valid && lp.g == 0) ax[lp.line] = sum[0];
    }
}

// Clears the per-check flags, completes a move to the FP64 stage, and counts
// the unfinished instances (active[0]) and those among them in the FP64
// stage of a mixed solve (active[1]).
__global__ void k_finalize(Global g, int32_t count, int32_t* active) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    InstanceCtl& c = g.ctl[b];
    if (c.to_fp64) {
        c.fp64_stage = 1;
        c.to_fp64 = 0;
    }
    if (c.phase != kPhaseDone && active != nullptr) {
        atomicAdd(active, 1);
        if (c.fp64_stage && g.mixed) atomicAdd(active + 1, 1);
    }
    if (c.stage == kStageCheck && c.check_kind == kCheckTransition) c.stage = kStageTrial;
    c.best_src = 0;
    c.restart_src = 0;
    c.need_refresh = 0;
    c.to_polish = 0;
    c.save_ray = 0;
    c.il_sync = 0;
}

// Mixed precision: the FP64 stage starts from the last FP32 restart point.
__global__ void k_switch_fp64(Global g, Work<float> w32, Work<double> w64) {
    const VecWork vw = g.vec[blockIdx.x];
    const InstanceCtl& c = g.ctl[vw.instance];
    if (!c.to_fp64) return;
    const InstanceInfo inf = g.info[vw.instance];
    const int p = c.parity;
    if (!vw.is_row) {
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const int64_t k = inf.col_off + j;
            const double v = static_cast<double>(w32.rx[k]);
            w64.X[p][k] = v;
            w64.rx[k] = v;
        }
    } else {
        for (int i = vw.begin + threadIdx.x; i < vw.end; i += blockDim.x) {
            const int64_t k = inf.row_off + i;
            const double v = static_cast<double>(w32.ry[k]);
            w64.Y[p][k] = v;
            w64.ry[k] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Setup: Ruiz equilibration (scaling.cpp:55-107). Row maxima over the A side
// and column maxima over the A^T side read the same scale state, as the
// reference's single sweep does; max is exact, so the scale vectors equal the
// reference's bit for bit.
// ---------------------------------------------------------------------------
template <int V>
__global__ void __launch_bounds__(kThreads) k_ruiz_max(Global g, int a_ctas) {
    const bool a_side = blockIdx.x < static_cast<unsigned>(a_ctas);
    const Side side = a_side ? g.a : g.at;
    const CtaWork cw = side.ctas[a_side ? blockIdx.x : blockIdx.x - a_ctas];
    const InstanceInfo inf = g.info[cw.instance];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* line_scale = a_side ? g.rs + inf.row_off : g.cs + inf.col_off;
    const double* other = a_side ? g.cs + inf.col_off : g.rs + inf.row_off;
    double* out = a_side ? g.row_tmp + inf.row_off : g.col_tmp + inf.col_off;
    const int64_t dbase = a_side ? inf.a_data_base : inf.at_data_base;
    const int64_t lbase = a_side ? inf.a_len_base : inf.at_len_base;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = side.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const int len = lp.valid ? side.line_len[lbase + lp.line] : 0;
        const double f = lp.valid ? line_scale[lp.line] : 0.0;
        double mx = 0.0;
        const int64_t base = dbase + static_cast<int64_t>(sd.data_off) * 32;
        for (int st = 0; st < sd.steps; st += V) {
            const int64_t pidx = base + static_cast<int64_t>(st) * 32 + lane * V;
            int32_t id[V];
            double v[V];
            ld<V>(side.idx + pidx, id);
            ld<V>(side.val_orig + pidx, v);
#pragma unroll
            for (int q = 0; q < V; ++q) {
                const int k = ((st + q) << lp.glog) + lp.g;
                if (k < len) {
                    // |a_ij| * r_i * c_j, multiplied in the reference's order
                    const double m = a_side ? fabs(v[q]) * f * other[id[q]]
                                            : fabs(v[q]) * other[id[q]] * f;
                    mx = smax(mx, m);
                }
            }
        }
        for (int o = (1 << lp.glog) >> 1; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
        if (lp.valid && lp.g == 0) out[lp.line] = mx;
    }
}

__global__ void k_ruiz_update(Global g) {
    const VecWork vw = g.vec[blockIdx.x];
    const InstanceInfo inf = g.info[vw.instance];
    double* scale = vw.is_row ? g.rs + inf.row_off : g.cs + inf.col_off;
    const double* mx = vw.is_row ? g.row_tmp + inf.row_off : g.col_tmp + inf.col_off;
    for (int k = vw.begin + threadIdx.x; k < vw.end; k += blockDim.x) {
        const double m = mx[k];
        if (m > 1e-30) scale[k] /= sqrt(m);
    }
}

// Scaled coefficients (SparseMatrix::scaled, sparse_matrix.cpp:243-274).
template <int V>
__global__ void __launch_bounds__(kThreads) k_scale_values(Global g, double* a_s64, double* at_s64,
                                                        float* a_s32, float* at_s32, int a_ctas) {
    const bool a_side = blockIdx.x < static_cast<unsigned>(a_ctas);
    const Side side = a_side ? g.a : g.at;
    const CtaWork cw = side.ctas[a_side ? blockIdx.x : blockIdx.x - a_ctas];
    const InstanceInfo inf = g.info[cw.instance];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* line_scale = a_side ? g.rs + inf.row_off : g.cs + inf.col_off;
    const double* other = a_side ? g.cs + inf.col_off : g.rs + inf.row_off;
    double* out64 = a_side ? a_s64 : at_s64;
    float* out32 = a_side ? a_s32 : at_s32;
    const int64_t dbase = a_side ? inf.a_data_base : inf.at_data_base;
    const int64_t lbase = a_side ? inf.a_len_base : inf.at_len_base;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = side.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const int len = lp.valid ? side.line_len[lbase + lp.line] : 0;
        const double f = lp.valid ? line_scale[lp.line] : 0.0;
        const int64_t base = dbase + static_cast<int64_t>(sd.data_off) * 32;
        for (int st = 0; st < sd.steps; ++st) {
            const int64_t pidx = base + static_cast<int64_t>(st - st % V) * 32 + lane * V + st % V;
            const int k = (st << lp.glog) + lp.g;
            double r = 0.0;
            if (k < len) r = side.val_orig[pidx] * (f * other[side.idx[pidx]]);
            out64[pidx] = r;
            if (out32) out32[pidx] = static_cast<float>(r);
        }
    }
}

// Pock-Chambolle (preconditioner.cpp:31-80): row and column L1 sums of the
// scaled matrix, each over its own side.
template <class T, int V>
__global__ void __launch_bounds__(kThreads) k_precondition(Global g, Work<T> w, int a_ctas) {
    const bool a_side = blockIdx.x < static_cast<unsigned>(a_ctas);
    const Side side = a_side ? g.a : g.at;
    const CtaWork cw = side.ctas[a_side ? blockIdx.x : blockIdx.x - a_ctas];
    const InstanceInfo inf = g.info[cw.instance];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t dbase = a_side ? inf.a_data_base : inf.at_data_base;
    const int64_t lbase = a_side ? inf.a_len_base : inf.at_len_base;
    T* sc = a_side ? w.sigma + inf.row_off : w.tau + inf.col_off;
    T* isc = a_side ? w.isigma + inf.row_off : w.itau + inf.col_off;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = side.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const int len = lp.valid ? side.line_len[lbase + lp.line] : 0;
        double sum[1] = {0.0};
        line_sums<V, 1>(dbase + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp, lane, len,
                        side.idx, side.val_s64, sum,
                        [&](double (&a)[1], double v, int) { a[0] += fabs(v); });
        if (lp.valid && lp.g == 0) {
            const double scale = sum[0] > 1e-12 ? 1.0 / sum[0] : 1.0;
            sc[lp.line] = static_cast<T>(scale);
            isc[lp.line] = static_cast<T>(1.0 / scale);
        }
    }
}

__device__ __forceinline__ double scale_bound(double b, double f) { return isfinite(b) ? b * f : b; }

__device__ __forceinline__ double initial_value(double lo, double hi) {   // pdlp_solver.cpp:30-41
    if (lo <= 0.0 && 0.0 <= hi) return 0.0;
    if (isfinite(lo)) return lo;
    if (isfinite(hi)) return hi;
    return 0.0;
}

// Scaled objective and bounds (scaling.cpp:109-135), the starting point
// (pdlp_solver.cpp:168-176) or a warm start, and its cold alternative.
template <class T>
__global__ void k_setup_vectors(Global g, Work<T> w) {
    const VecWork vw = g.vec[blockIdx.x];
    if (g.slot_mask != nullptr && g.slot_mask[vw.instance] == 0) return;
    const InstanceInfo inf = g.info[vw.instance];
    const bool warm = g.warm_x != nullptr || g.warm_y != nullptr;
    if (!vw.is_row) {
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const int64_t k = inf.col_off + j;
            const double f = g.cs[k];
            const double lo = scale_bound(g.xl_orig[k], 1.0 / f);
            const double hi = scale_bound(g.xu_orig[k], 1.0 / f);
            w.c[k] = static_cast<T>(g.c_orig[k] * f);
            w.xl[k] = static_cast<T>(lo);
            w.xu[k] = static_cast<T>(hi);
            const double cold = initial_value(lo, hi);
            double x0 = cold;
            if (g.warm_x != nullptr) {
                const double v = g.warm_x[k] / f;
                x0 = isfinite(v) ? smax(lo, smin(v, hi)) : cold;
            }
            w.X[0][k] = static_cast<T>(x0);
            w.X[1][k] = static_cast<T>(x0);
            w.rx[k] = static_cast<T>(x0);
            w.avg_x[k] = static_cast<T>(warm ? cold : 0.0);
        }
    } else {
        for (int i = vw.begin + threadIdx.x; i < vw.end; i += blockDim.x) {
            const int64_t k = inf.row_off + i;
            const double f = g.rs[k];
            w.rl[k] = static_cast<T>(scale_bound(g.rl_orig[k], f));
            w.ru[k] = static_cast<T>(scale_bound(g.ru_orig[k], f));
            double y0 = 0.0;
            if (g.warm_y != nullptr) {
                const double v = g.warm_y[k] / f;
                y0 = isfinite(v) ? v : 0.0;
            }
            w.Y[0][k] = static_cast<T>(y0);
            w.Y[1][k] = static_cast<T>(y0);
            w.ry[k] = static_cast<T>(y0);
            w.avg_y[k] = static_cast<T>(0.0);
            w.AX[0][k] = T(0);
            w.AX[1][k] = T(0);
        }
    }
}

// Shared-matrix batches: scales and preconditioner depend on A only, so the
// vectors of instance 0 are copied to every other instance.
__global__ void k_broadcast_scales(double* rs, double* cs, int64_t rows, int64_t cols, int32_t count) {
    const int64_t total = (rows + cols) * (count - 1);
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = 1 + t / (rows + cols), e = t % (rows + cols);
        if (e < rows) rs[b * rows + e] = rs[e];
        else cs[b * cols + (e - rows)] = cs[e - rows];
    }
}

template <class T>
__global__ void k_broadcast_precond(T* sigma, T* isigma, T* tau, T* itau, int64_t rows, int64_t cols,
                                    int32_t count) {
    const int64_t total = (rows + cols) * (count - 1);
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = 1 + t / (rows + cols), e = t % (rows + cols);
        if (e < rows) {
            sigma[b * rows + e] = sigma[e];
            isigma[b * rows + e] = isigma[e];
        } else {
            tau[b * cols + (e - rows)] = tau[e - rows];
            itau[b * cols + (e - rows)] = itau[e - rows];
        }
    }
}

// Plain product over one side, lines in internal order.
template <class T, int V>
__global__ void __launch_bounds__(kThreads) k_spmv(Global g, int transpose, const T* vals,
                                                   const T* v, T* out) {
    const Side side = transpose ? g.at : g.a;
    const CtaWork cw = side.ctas[blockIdx.x];
    const InstanceInfo inf = g.info[cw.instance];
    const T* src = v + (transpose ? inf.row_off : inf.col_off);
    T* dst = out + (transpose ? inf.col_off : inf.row_off);
    const int64_t dbase = transpose ? inf.at_data_base : inf.a_data_base;
    const int64_t lbase = transpose ? inf.at_len_base : inf.a_len_base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = cw.slice_begin + warp; s < cw.slice_end; s += kWarps) {
        const SliceDesc sd = side.slices[s];
        const LanePos lp = lane_pos(sd, lane);
        const int len = lp.valid ? side.line_len[lbase + lp.line] : 0;
        T sum[1] = {T(0)};
        line_sums<V, 1>(dbase + static_cast<int64_t>(sd.data_off) * 32, sd.steps, lp, lane, len,
                        side.idx, vals, sum, [&](T (&a)[1], T x, int j) { a[0] += x * src[j]; });
        if (lp.valid && lp.g == 0) dst[lp.line] = sum[0];
    }
}


// The linesearch's step factors by iteration index (DeviceOptions::step_pow).
__global__ void k_step_pow(double* table, int64_t entries) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < entries;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double index = static_cast<double>(k) + 2.0;
        table[2 * k] = pow(index, -0.3);
        table[2 * k + 1] = pow(index, -0.6);
    }
}

// ---------------------------------------------------------------------------
// Power iteration on A'A (preconditioner.cpp:82-140), used only when the
// diagonal preconditioner is off. Per-instance state lives in ctl.dbg:
// [4] estimate, [5] previous, [6] scale 1/||z||, [7] state (0 running,
// 1 converged, 2 stopped on a zero vector, 3 budget exhausted), [8] unit flag.
// ---------------------------------------------------------------------------
__global__ void k_power_dot(Global g, const double* x, const double* z) {
    const VecWork vw = g.vec[blockIdx.x];
    const InstanceInfo inf = g.info[vw.instance];
    double acc[2] = {0.0, 0.0};
    if (!vw.is_row && g.ctl[vw.instance].dbg[7] == 0.0) {
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const double a = x[inf.col_off + j], b = z[inf.col_off + j];
            acc[0] += a * b;
            acc[1] += b * b;
        }
    }
    block_sum<2>(acc);
    if (threadIdx.x == 0) {
        g.part_prep[static_cast<int64_t>(blockIdx.x) * kPrepSlots] = acc[0];
        g.part_prep[static_cast<int64_t>(blockIdx.x) * kPrepSlots + 1] = acc[1];
    }
}

__global__ void k_power_step(Global g, int32_t count, int init, int it, int budget) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    InstanceCtl& c = g.ctl[b];
    if (c.dbg[7] != 0.0) return;
    const InstanceInfo inf = g.info[b];
    double xz = 0.0, zz = 0.0;
    for (int k = inf.vec_cta_begin; k < inf.vec_cta_end; ++k) {
        if (g.vec[k].is_row) continue;
        xz += g.part_prep[static_cast<int64_t>(k) * kPrepSlots];
        zz += g.part_prep[static_cast<int64_t>(k) * kPrepSlots + 1];
    }
    const double norm = sqrt(zz);
    if (init) {
        c.dbg[8] = norm == 0.0 ? 1.0 : 0.0;
        c.dbg[6] = norm > 0.0 ? 1.0 / norm : 0.0;
        return;
    }
    const double est = sqrt(smax(xz, 0.0));
    c.dbg[4] = est;
    if (norm == 0.0) {
        c.dbg[7] = 2.0;
        return;
    }
    c.dbg[6] = 1.0 / norm;
    c.dbg[8] = 0.0;
    if (it > 0 && est > 0.0 && fabs(est - c.dbg[5]) <= 1e-8 * est) {
        c.dbg[7] = 1.0;
        return;
    }
    c.dbg[5] = est;
    if (it == budget - 1) c.dbg[7] = 3.0;
}

__global__ void k_power_scale(Global g, double* x, const double* z) {
    const VecWork vw = g.vec[blockIdx.x];
    if (vw.is_row) return;
    const InstanceCtl& c = g.ctl[vw.instance];
    if (c.dbg[7] != 0.0) return;
    const InstanceInfo inf = g.info[vw.instance];
    const double s = c.dbg[6];
    const bool unit = c.dbg[8] != 0.0;
    const double u = inf.n > 0 ? 1.0 / sqrt(static_cast<double>(inf.n)) : 0.0;
    for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x)
        x[inf.col_off + j] = unit ? u : z[inf.col_off + j] * s;
}

// pdlp_solver.cpp:188-202 and the StepController constructor (step_controller.cpp:17-28).
__global__ void k_power_finish(Global g, int32_t count, double safety, double min_scale) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    InstanceCtl& c = g.ctl[b];
    const double est = c.dbg[4];
    const bool converged = c.dbg[7] == 1.0 || c.dbg[7] == 2.0;
    const double safe = est > 0.0 ? 0.99 / (est * (converged ? 1.02 : 1.25)) : 1.0;
    c.eta_max = safe;
    c.eta = clampd(safety * safe, min_scale * safe, safe);
    c.trial_eta = c.eta;
    for (int q = 3; q < 12; ++q) c.dbg[q] = 0.0;
}

// The solve clock: the reference's clock starts when solve() is entered, so
// the host's setup time is carried in.
__global__ void k_stamp_clock(Global g, int32_t count, int64_t elapsed_ns, int64_t limit_ns) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    if (g.slot_mask != nullptr && g.slot_mask[b] == 0) return;
    InstanceCtl& c = g.ctl[b];
    c.start_ns = now_ns() - elapsed_ns;
    c.deadline_ns = limit_ns > 0 ? c.start_ns + limit_ns : 0;
}


// ---------------------------------------------------------------------------
// Sessions: order changes between the caller's layout and the internal one,
// the TerminationChecker normalisers (termination.cpp:58-62) and the initial
// control state, all on the device.
// ---------------------------------------------------------------------------
__global__ void k_permute(const double* __restrict__ src, double* __restrict__ dst,
                          const int32_t* __restrict__ perm, int64_t len, int32_t count, int mode) {
    const int64_t total = len * count;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / len, k = t - b * len;
        if (mode == 0) dst[t] = src[b * len + perm[k]];
        else if (mode == 1) dst[b * len + perm[k]] = src[t];
        else dst[t] = src[k];
    }
}

__global__ void __launch_bounds__(kThreads) k_norm_parts(Global g) {
    const VecWork vw = g.vec[blockIdx.x];
    if (g.slot_mask != nullptr && g.slot_mask[vw.instance] == 0) return;
    const InstanceInfo inf = g.info[vw.instance];
    double acc[1] = {0.0};
    if (!vw.is_row) {
        for (int j = vw.begin + threadIdx.x; j < vw.end; j += blockDim.x) {
            const double v = g.c_orig[inf.col_off + j];
            acc[0] += v * v;
        }
    } else {
        for (int i = vw.begin + threadIdx.x; i < vw.end; i += blockDim.x) {
            const double l = g.rl_orig[inf.row_off + i], u = g.ru_orig[inf.row_off + i];
            if (isfinite(l)) acc[0] += l * l;
            if (isfinite(u) && u != l) acc[0] += u * u;
        }
    }
    block_sum<1>(acc);
    if (threadIdx.x == 0) g.part_prep[static_cast<int64_t>(blockIdx.x) * kPrepSlots] = acc[0];
}

// The host's init_control, per instance on the device.
__global__ void k_init_ctl(Global g, DeviceOptions o, int32_t count, int32_t mixed, int32_t warm,
                           const double* warm_weight, double eta_max, double initial_weight,
                           double objective_offset) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    if (g.slot_mask != nullptr && g.slot_mask[b] == 0) return;
    const InstanceInfo inf = g.info[b];
    double rows = 0.0, cols = 0.0;
    for (int k = inf.vec_cta_begin; k < inf.vec_cta_end; ++k) {
        const double v = g.part_prep[static_cast<int64_t>(k) * kPrepSlots];
        if (g.vec[k].is_row) rows += v; else cols += v;
    }
    InstanceCtl c;
    memset(&c, 0, sizeof(c));
    c.phase = kPhaseMain;
    c.stage = kStageCheck;
    c.check_kind = kCheckInitial;
    c.need_refresh = 1;
    c.fp64_stage = mixed ? 0 : 1;
    c.status = -1;
    c.limit_status = 3;
    c.have_avg_at_check = warm;
    c.eta_max = eta_max;
    c.eta = clampd(o.initial_step_safety * eta_max, o.min_step_scale * eta_max, eta_max);
    c.omega = 1.0;
    set_weight(c.omega, o, initial_weight);
    if (warm_weight != nullptr && warm_weight[b] > 0.0) set_weight(c.omega, o, warm_weight[b]);
    c.trial_eta = c.ctl_eta = c.eta;
    c.trial_omega = c.ctl_omega = c.omega;
    c.best_pobj = nan("");
    c.best_dobj = -INFINITY;
    c.best_pres = c.best_dres = c.best_gap = c.best_kkt = INFINITY;
    c.restart_baseline = INFINITY;
    c.prev_candidate = INFINITY;
    c.pnorm = 1.0 + sqrt(rows);
    c.dnorm = 1.0 + sqrt(cols);
    c.objective_offset = objective_offset;
    g.ctl[b] = c;
}


// ---------------------------------------------------------------------------
// Streams: refill finished slots with the next instances of a queue.
// ---------------------------------------------------------------------------
__global__ void k_gather_slots(const double* __restrict__ src, const double* __restrict__ fam,
                               double* __restrict__ dst, const int32_t* __restrict__ perm,
                               const int64_t* __restrict__ inst, const int32_t* __restrict__ mask,
                               int64_t len, int32_t count) {
    const int64_t total = len * count;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / len, k = t - b * len;
        if (mask[b] == 0) continue;
        dst[t] = src != nullptr ? src[inst[b] * len + perm[k]] : fam[k];
    }
}

__global__ void k_scatter_slots(const double* __restrict__ src, double* __restrict__ out,
                                const int32_t* __restrict__ perm, const int64_t* __restrict__ inst,
                                const int32_t* __restrict__ mask, int64_t len, int32_t count) {
    const int64_t total = len * count;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / len, k = t - b * len;
        if (mask[b] == 0) continue;
        out[inst[b] * len + perm[k]] = src[t];
    }
}

// Marks every slot finished (no work) before a stream fills them.
__global__ void k_retire(Global g, int32_t count) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    InstanceCtl& c = g.ctl[b];
    c.phase = kPhaseDone;
    c.stage = kStageTrial;
    c.best_src = c.restart_src = c.need_refresh = c.to_polish = c.save_ray = 0;
}

__global__ void k_slot_done(Global g, int32_t count, int32_t* done) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < count) done[b] = g.ctl[b].phase == kPhaseDone ? 1 : 0;
}

inline unsigned blocks_for(int64_t n, int per) { return static_cast<unsigned>((n + per - 1) / per); }

}  // namespace

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
template <class T>
void launch_primal(const Global& g, const Work<T>& w, const DeviceOptions&, int vw, cudaStream_t s) {
    if (g.at.num_ctas == 0) return;
    switch (vw) {
        case 4: k_primal<T, 4><<<g.at.num_ctas, kThreads, 0, s>>>(g, w); break;
        case 2: k_primal<T, 2><<<g.at.num_ctas, kThreads, 0, s>>>(g, w); break;
        default: k_primal<T, 1><<<g.at.num_ctas, kThreads, 0, s>>>(g, w); break;
    }
}

namespace {
template <class T, int V>
cudaError_t fused_v(const Global& g, const Work<T>& w, const DeviceOptions& o, int count, int cluster,
                    int max_trials, const FusedShape& shape, cudaStream_t s) {
    const size_t smem = fused_smem_bytes(shape);
    const cudaError_t e =
        cudaFuncSetAttribute(k_fused<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(count * cluster));
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // Clusters of 16 CTAs are beyond the portable size of 8.
    cudaFuncSetAttribute(k_fused<T, V>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return cudaLaunchKernelEx(&cfg, k_fused<T, V>, g, w, o, max_trials, shape);
}

template <class T, int V>
int fused_clusters_v(int cluster, size_t smem) {
    if (cudaFuncSetAttribute(k_fused<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(cluster));
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cluster > 8 &&
        cudaFuncSetAttribute(k_fused<T, V>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_fused<T, V>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
}  // namespace

template <class T>
cudaError_t launch_fused(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw, int count,
                         int cluster, int max_trials, const FusedShape& shape, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    switch (vw) {
        case 4: return fused_v<T, 4>(g, w, o, count, cluster, max_trials, shape, s);
        case 2: return fused_v<T, 2>(g, w, o, count, cluster, max_trials, shape, s);
        default: return fused_v<T, 1>(g, w, o, count, cluster, max_trials, shape, s);
    }
}

template <class T>
int fused_max_clusters(int vw, int cluster, const FusedShape& shape) {
    const size_t smem = fused_smem_bytes(shape);
    switch (vw) {
        case 4: return fused_clusters_v<T, 4>(cluster, smem);
        case 2: return fused_clusters_v<T, 2>(cluster, smem);
        default: return fused_clusters_v<T, 1>(cluster, smem);
    }
}

template <class T>
void launch_dual(const Global& g, const Work<T>& w, const DeviceOptions& o, int vw, cudaStream_t s) {
    if (g.a.num_ctas == 0) return;
    switch (vw) {
        case 4: k_dual<T, 4><<<g.a.num_ctas, kThreads, 0, s>>>(g, w, o); break;
        case 2: k_dual<T, 2><<<g.a.num_ctas, kThreads, 0, s>>>(g, w, o); break;
        default: k_dual<T, 1><<<g.a.num_ctas, kThreads, 0, s>>>(g, w, o); break;
    }
}

template <class T>
void launch_check_prep(const Global& g, const Work<T>& w, const DeviceOptions& o, cudaStream_t s) {
    if (g.num_vec) k_check_prep<T><<<g.num_vec, kThreads, 0, s>>>(g, w, o);
}

void launch_check_spmv(const Global& g, const DeviceOptions& o, int vw, cudaStream_t s) {
    const int n = g.a.num_ctas + g.at.num_ctas;
    if (n == 0) return;
    switch (vw) {
        case 4: k_check_spmv<4><<<n, kThreads, 0, s>>>(g, o); break;
        case 2: k_check_spmv<2><<<n, kThreads, 0, s>>>(g, o); break;
        default: k_check_spmv<1><<<n, kThreads, 0, s>>>(g, o); break;
    }
}

void launch_check_ndg(const Global& g, const DeviceOptions& o, int32_t count, cudaStream_t s) {
    if (o.ndg_restarts && count > 0) k_check_ndg<<<count, kThreads, 0, s>>>(g, o);
}

template <class T>
void launch_check_apply(const Global& g, const Work<T>& w, const DeviceOptions&, cudaStream_t s) {
    if (g.num_vec) k_check_apply<T><<<g.num_vec, kThreads, 0, s>>>(g, w);
}

template <class T>
void launch_refresh(const Global& g, const Work<T>& w, const DeviceOptions&, int vw, cudaStream_t s) {
    if (g.a.num_ctas == 0) return;
    switch (vw) {
        case 4: k_refresh<T, 4><<<g.a.num_ctas, kThreads, 0, s>>>(g, w); break;
        case 2: k_refresh<T, 2><<<g.a.num_ctas, kThreads, 0, s>>>(g, w); break;
        default: k_refresh<T, 1><<<g.a.num_ctas, kThreads, 0, s>>>(g, w); break;
    }
}

void launch_finalize(const Global& g, int32_t count, int32_t* active, cudaStream_t s) {
    if (count) k_finalize<<<blocks_for(count, 256), 256, 0, s>>>(g, count, active);
}

void launch_switch_fp64(const Global& g, const Work<float>& w32, const Work<double>& w64,
                        cudaStream_t s) {
    if (g.num_vec) k_switch_fp64<<<g.num_vec, kThreads, 0, s>>>(g, w32, w64);
}

void launch_ruiz_max(const Global& g, int vw, int a_ctas, int at_ctas, cudaStream_t s) {
    if (a_ctas + at_ctas == 0) return;
    switch (vw) {
        case 4: k_ruiz_max<4><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_ctas); break;
        case 2: k_ruiz_max<2><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_ctas); break;
        default: k_ruiz_max<1><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_ctas); break;
    }
}

void launch_ruiz_update(const Global& g, int vec_ctas, cudaStream_t s) {
    if (vec_ctas) k_ruiz_update<<<vec_ctas, kThreads, 0, s>>>(g);
}

void launch_scale_values(const Global& g, double* a_s64, double* at_s64, float* a_s32,
                         float* at_s32, int vw, int a_ctas, int at_ctas, cudaStream_t s) {
    if (a_ctas + at_ctas == 0) return;
    switch (vw) {
        case 4: k_scale_values<4><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_s64, at_s64, a_s32, at_s32, a_ctas); break;
        case 2: k_scale_values<2><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_s64, at_s64, a_s32, at_s32, a_ctas); break;
        default: k_scale_values<1><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, a_s64, at_s64, a_s32, at_s32, a_ctas); break;
    }
}

template <class T>
void launch_precondition(const Global& g, const Work<T>& w, int enabled, int vw, int a_ctas,
                         int at_ctas, cudaStream_t s) {
    if (!enabled || a_ctas + at_ctas == 0) return;
    switch (vw) {
        case 4: k_precondition<T, 4><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, w, a_ctas); break;
        case 2: k_precondition<T, 2><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, w, a_ctas); break;
        default: k_precondition<T, 1><<<a_ctas + at_ctas, kThreads, 0, s>>>(g, w, a_ctas); break;
    }
}

template <class T>
void launch_setup_vectors(const Global& g, const Work<T>& w, cudaStream_t s) {
    if (g.num_vec) k_setup_vectors<T><<<g.num_vec, kThreads, 0, s>>>(g, w);
}

template <class T>
__global__ void k_fill(T* __restrict__ p, int64_t n, T v) {
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        p[k] = v;
}

template <class T>
void launch_fill(T* p, int64_t n, T v, cudaStream_t s) {
    if (n > 0) k_fill<T><<<static_cast<int>(std::min<int64_t>(blocks_for(n, 256), 148 * 16)), 256, 0, s>>>(p, n, v);
}

void launch_broadcast_scales(const Global& g, const InstanceInfo& first, int32_t count,
                             int64_t rows, int64_t cols, cudaStream_t s) {
    (void)first;
    if (count > 1) k_broadcast_scales<<<592, 256, 0, s>>>(g.rs, g.cs, rows, cols, count);
}

template <class T>
void launch_broadcast_precond(const Work<T>& w, const InstanceInfo&, int32_t count, int64_t rows,
                              int64_t cols, cudaStream_t s) {
    if (count > 1)
        k_broadcast_precond<T><<<592, 256, 0, s>>>(w.sigma, w.isigma, w.tau, w.itau, rows, cols, count);
}

template <class T>
void launch_spmv(const Global& g, int transpose, int values, const T* v, T* out, int vw,
                 cudaStream_t s) {
    const Side& side = transpose ? g.at : g.a;
    if (side.num_ctas == 0) return;
    const T* vals;
    if constexpr (sizeof(T) == 8) {
        vals = values == 0 ? side.val_orig : side.val_s64;
    } else {
        vals = side.val_s32;
    }
    switch (vw) {
        case 4: k_spmv<T, 4><<<side.num_ctas, kThreads, 0, s>>>(g, transpose, vals, v, out); break;
        case 2: k_spmv<T, 2><<<side.num_ctas, kThreads, 0, s>>>(g, transpose, vals, v, out); break;
        default: k_spmv<T, 1><<<side.num_ctas, kThreads, 0, s>>>(g, transpose, vals, v, out); break;
    }
}

void launch_step_pow(double* table, int64_t entries, cudaStream_t s) {
    if (entries > 0) k_step_pow<<<blocks_for(entries, 256), 256, 0, s>>>(table, entries);
}

void launch_power_dot(const Global& g, const double* x, const double* z, cudaStream_t s) {
    if (g.num_vec) k_power_dot<<<g.num_vec, kThreads, 0, s>>>(g, x, z);
}
void launch_power_step(const Global& g, int32_t count, int init, int it, int budget, cudaStream_t s) {
    if (count) k_power_step<<<blocks_for(count, 128), 128, 0, s>>>(g, count, init, it, budget);
}
void launch_power_scale(const Global& g, double* x, const double* z, cudaStream_t s) {
    if (g.num_vec) k_power_scale<<<g.num_vec, kThreads, 0, s>>>(g, x, z);
}
void launch_power_finish(const Global& g, int32_t count, double safety, double min_scale, cudaStream_t s) {
    if (count) k_power_finish<<<blocks_for(count, 128), 128, 0, s>>>(g, count, safety, min_scale);
}
void launch_stamp_clock(const Global& g, int32_t count, int64_t elapsed_ns, int64_t limit_ns, cudaStream_t s) {
    if (count) k_stamp_clock<<<blocks_for(count, 128), 128, 0, s>>>(g, count, elapsed_ns, limit_ns);
}

void launch_permute(const double* src, double* dst, const int32_t* perm, int64_t len,
                    int32_t count, int mode, cudaStream_t s) {
    const int64_t total = len * count;
    if (total == 0) return;
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    k_permute<<<blocks, 256, 0, s>>>(src, dst, perm, len, count, mode);
}
void launch_norm_parts(const Global& g, cudaStream_t s) {
    if (g.num_vec) k_norm_parts<<<g.num_vec, kThreads, 0, s>>>(g);
}
void launch_init_ctl(const Global& g, const DeviceOptions& o, int32_t count, int32_t mixed,
                     int32_t warm, const double* warm_weight, double eta_max,
                     double initial_weight, double objective_offset, cudaStream_t s) {
    if (count)
        k_init_ctl<<<blocks_for(count, 128), 128, 0, s>>>(g, o, count, mixed, warm, warm_weight,
                                                          eta_max, initial_weight, objective_offset);
}

void launch_gather_slots(const double* src, const double* fam, double* dst, const int32_t* perm,
                         const int64_t* inst, const int32_t* mask, int64_t len, int32_t count,
                         cudaStream_t s) {
    const int64_t total = len * count;
    if (total == 0) return;
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    k_gather_slots<<<blocks, 256, 0, s>>>(src, fam, dst, perm, inst, mask, len, count);
}
void launch_scatter_slots(const double* src, double* out, const int32_t* perm, const int64_t* inst,
                          const int32_t* mask, int64_t len, int32_t count, cudaStream_t s) {
    const int64_t total = len * count;
    if (total == 0) return;
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    k_scatter_slots<<<blocks, 256, 0, s>>>(src, out, perm, inst, mask, len, count);
}
void launch_retire(const Global& g, int32_t count, cudaStream_t s) {
    if (count) k_retire<<<blocks_for(count, 128), 128, 0, s>>>(g, count);
}
void launch_slot_done(const Global& g, int32_t count, int32_t* done, cudaStream_t s) {
    if (count) k_slot_done<<<blocks_for(count, 128), 128, 0, s>>>(g, count, done);
}

#define PDLPGPU_INSTANTIATE(T)                                                                      \
    template void launch_primal<T>(const Global&, const Work<T>&, const DeviceOptions&, int, cudaStream_t); \
    template cudaError_t launch_fused<T>(const Global&, const Work<T>&, const DeviceOptions&, int, int, int, \
                                         int, const FusedShape&, cudaStream_t);                      \
    template int fused_max_clusters<T>(int, int, const FusedShape&);                                 \
    template void launch_dual<T>(const Global&, const Work<T>&, const DeviceOptions&, int, cudaStream_t);   \
    template void launch_check_prep<T>(const Global&, const Work<T>&, const DeviceOptions&, cudaStream_t);  \
    template void launch_check_apply<T>(const Global&, const Work<T>&, const DeviceOptions&, cudaStream_t); \
    template void launch_refresh<T>(const Global&, const Work<T>&, const DeviceOptions&, int, cudaStream_t); \
    template void launch_precondition<T>(const Global&, const Work<T>&, int, int, int, int, cudaStream_t);  \
    template void launch_setup_vectors<T>(const Global&, const Work<T>&, cudaStream_t);                    \
    template void launch_fill<T>(T*, int64_t, T, cudaStream_t);                                              \
    template void launch_broadcast_precond<T>(const Work<T>&, const InstanceInfo&, int32_t, int64_t, int64_t, cudaStream_t); \
    template void launch_spmv<T>(const Global&, int, int, const T*, T*, int, cudaStream_t);

PDLPGPU_INSTANTIATE(double)
PDLPGPU_INSTANTIATE(float)

}  // namespace pdlpgpu

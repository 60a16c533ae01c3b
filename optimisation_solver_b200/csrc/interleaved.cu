// interleaved.cu -- PDHG trial kernels over the batch-interleaved layout of a
// shared-matrix session, and the transposes between it and the per-instance
// layout the checks use.
//
// Per trial (pdlp_engine/src/pdhg_kernel.cpp:47-187), lane l of a warp holds
// instances group * G + l * V + v (V = 1, 2 or 4 per lane, G = 32 V) and the
// warp walks one line:
//   k_il_primal  column j: g = c + A'y, x' = clip(x - (eta/omega) tau g),
//                sum dx^2/tau; the owed iterate-average update of x
//                (iterate_average.cpp:40-82)
//   k_il_dual    row i: A x', extrapolation 2Ax' - Ax, dual prox, sum
//                dy^2/sigma and dy'(A dx); the owed average update of y; then,
//                in the last CTA of each group, the linesearch decision and
//                commit of its G instances (trial_control, one thread each).
// Sums are per lane: each CTA adds its warps' values in warp order and
// writes one partial per lane; the deciding CTA adds the partials in CTA
// order, so a run is bitwise reproducible and needs no atomics on data.
#include "control.cuh"
#include "interleaved.cuh"

#include <algorithm>
#include <utility>

namespace pdlpgpu {
namespace {

constexpr int kIlWarps = 8;
constexpr int kIlThreads = kIlWarps * 32;

// True in every thread of the CTA that arrives last of `expected` CTAs
// (and resets the counter; the next use is in a later kernel). Everything
// written before is visible to it. One thread arrives for the CTA with an
// acquire-release atomic at GPU scope: the barrier orders the other
// threads' writes before it, its release publishes them, and in the last CTA
// its acquire makes every earlier arrival's writes visible -- one round trip
// where a full fence and an atomic took two.
__device__ __forceinline__ bool arrive_last_cta(int32_t* counter, int expected) {
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

// Programmatic dependent launch: the trial kernels are launched so that the
// next one may start while this one finishes. A kernel waits for its
// predecessor (wait) before it touches anything the predecessor writes --
// the control blocks, the iterates, the partial sums -- and lets its own
// successor start (trigger) only after that wait, so a successor never runs
// ahead of a still-running decision two kernels back.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Non-binding bulk prefetch of `bytes` (a multiple of 16, from a 16-byte
// aligned address) into L2: DRAM bytes in flight that cost no registers.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetches the group's slice of `kinds` [line][bp] streams for lines
// [l0, l1): one G-element row (128-512 bytes, 16-byte aligned because bp and
// the group offset are multiples of G = 32 V) per line and stream.
template <class T, int kMax>
__device__ __forceinline__ void prefetch_rows(const T* const (&streams)[kMax], int kinds, int64_t bp,
                                              int64_t group_off, unsigned row_bytes, int l0, int l1) {
    const int total = (l1 - l0) * kinds;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int l = l0 + q / kinds, k = q - (q / kinds) * kinds;
        prefetch_l2(streams[k] + static_cast<int64_t>(l) * bp + group_off, row_bytes);
    }
}

// V consecutive elements (one 4/8/16-byte access).
template <class T, int V>
struct Pack;
template <> struct Pack<float, 1> { using type = float; };
template <> struct Pack<float, 2> { using type = float2; };
template <> struct Pack<float, 4> { using type = float4; };
template <> struct Pack<double, 1> { using type = double; };
template <> struct Pack<double, 2> { using type = double2; };

template <class T, int V>
__device__ __forceinline__ void ldv(const T* p, T (&o)[V]) {
    if constexpr (V == 1) {
        o[0] = *p;
    } else if constexpr (V == 2) {
        const auto v = *reinterpret_cast<const typename Pack<T, 2>::type*>(p);
        o[0] = v.x; o[1] = v.y;
    } else {
        const auto v = *reinterpret_cast<const typename Pack<T, 4>::type*>(p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
}

template <class T, int V>
__device__ __forceinline__ void stv(T* p, const T (&o)[V]) {
    if constexpr (V == 1) {
        *p = o[0];
    } else if constexpr (V == 2) {
        typename Pack<T, 2>::type v;
        v.x = o[0]; v.y = o[1];
        *reinterpret_cast<typename Pack<T, 2>::type*>(p) = v;
    } else {
        typename Pack<T, 4>::type v;
        v.x = o[0]; v.y = o[1]; v.z = o[2]; v.w = o[3];
        *reinterpret_cast<typename Pack<T, 4>::type*>(p) = v;
    }
}

// Use-once streams (evict-first in L2), so that the trial point, which the
// dual gathers next and the following primal reads, stays resident.
template <class T, int V>
__device__ __forceinline__ void ldv_cs(const T* p, T (&o)[V]) {
    if constexpr (V == 1) {
        o[0] = __ldcs(p);
    } else if constexpr (V == 2) {
        const auto v = __ldcs(reinterpret_cast<const typename Pack<T, 2>::type*>(p));
        o[0] = v.x; o[1] = v.y;
    } else {
        const auto v = __ldcs(reinterpret_cast<const typename Pack<T, 4>::type*>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
}

template <class T, int V>
__device__ __forceinline__ void stv_cs(T* p, const T (&o)[V]) {
    if constexpr (V == 1) {
        __stcs(p, o[0]);
    } else if constexpr (V == 2) {
        typename Pack<T, 2>::type v;
        v.x = o[0]; v.y = o[1];
        __stcs(reinterpret_cast<typename Pack<T, 2>::type*>(p), v);
    } else {
        typename Pack<T, 4>::type v;
        v.x = o[0]; v.y = o[1]; v.z = o[2]; v.w = o[3];
        __stcs(reinterpret_cast<typename Pack<T, 4>::type*>(p), v);
    }
}

// Stores the active elements only (all of them with one access when every
// instance of the lane is active): an idle instance's buffer may hold its
// committed point.
template <class T, int V>
__device__ __forceinline__ void stv_masked(T* p, const T (&o)[V], uint32_t mask) {
    if (mask == (1u << V) - 1) {
        stv<T, V>(p, o);
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
            if ((mask >> v) & 1) p[v] = o[v];
    }
}

// The V instances of a lane: instance group * G + lane * V + v.
template <class T, int V>
struct Lanes {
    uint32_t active;    // bit v: the instance runs this trial
    uint32_t pending;   // average update owed
    uint32_t fix;       // committed point in buffer W (it idled or was rejected)
    T frac[V];
    T step[V];          // eta / omega (primal) or eta * omega (dual)
};

// The hot block of an instance's control (the fields at its head, laid out
// by InstanceCtl) in three independent 16-byte loads.
struct HotCtl {
    double eta, omega, frac;
    int32_t phase, stage, pending, fp64, ibuf;
};

__device__ __forceinline__ HotCtl load_hot(const InstanceCtl* c) {
    const int4* p = reinterpret_cast<const int4*>(c);
    const int4 a = p[0], b = p[1], d = p[2];
    HotCtl h;
    h.eta = __hiloint2double(a.y, a.x);
    h.omega = __hiloint2double(a.w, a.z);
    h.frac = __hiloint2double(b.y, b.x);
    h.phase = b.z;
    h.stage = b.w;
    h.pending = d.x;
    h.fp64 = d.y;
    h.ibuf = d.z;
    return h;
}

// The lane's instances' state. Every warp of a CTA serves the same
// instances, so warp 0 alone reads their control blocks (one L2 request per
// block per CTA instead of one per warp: hundreds of CTAs read the same few
// hundred blocks at kernel entry) and shares them through `hot` (G entries
// of shared memory). Contains a CTA-wide barrier.
template <class T, int V>
__device__ __forceinline__ Lanes<T, V> lane_state(const Interleaved<T>& il, const InstanceCtl* ctl,
                                                  int first, int measure, int R, bool primal,
                                                  HotCtl* hot) {
    Lanes<T, V> s{0u, 0u, 0u, {}, {}};
    const int lane = threadIdx.x & 31;
    if ((threadIdx.x >> 5) == 0) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int b = first + v < il.count ? first + v : il.count - 1;
            hot[lane * V + v] = load_hot(ctl + b);
        }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const HotCtl h = hot[lane * V + v];
        s.frac[v] = T(0);
        s.step[v] = T(0);
        const bool exists = first + v < il.count;
        const bool act = exists && (measure || (h.phase != kPhaseDone && h.stage == kStageTrial &&
                                                (h.fp64 != 0) == (sizeof(T) == 8)));
        if (!act) continue;
        s.active |= 1u << v;
        s.step[v] = static_cast<T>(primal ? h.eta / h.omega : h.eta * h.omega);
        if (measure) continue;
        if (h.pending) s.pending |= 1u << v;
        s.frac[v] = static_cast<T>(h.frac);
        if (h.ibuf != R) s.fix |= 1u << v;
    }
    return s;
}

// Committed values of the lane's V instances at offset e: buffer R, or W for
// the instances whose point is there.
template <class T, int V>
__device__ __forceinline__ void load_committed(const T* R, const T* W, int64_t e, uint32_t fix,
                                               T (&o)[V]) {
    ldv<T, V>(R + e, o);
    if (fix) {
        T alt[V];
        ldv<T, V>(W + e, alt);
#pragma unroll
        for (int v = 0; v < V; ++v)
            if ((fix >> v) & 1) o[v] = alt[v];
    }
}

// Problem vector k at line `line` for the lane: family vectors are [line].
template <class T, int V>
__device__ __forceinline__ void load_vec(const Interleaved<T>& il, int k, bool fam, int64_t line,
                                         int64_t e, T (&o)[V]) {
    if (fam) {
        const T x = __ldg(il.vec[k] + line);
#pragma unroll
        for (int v = 0; v < V; ++v) o[v] = x;
    } else {
        ldv<T, V>(il.vec[k] + e, o);
    }
}

// ---------------------------------------------------------------------------
// Per-group sums
// ---------------------------------------------------------------------------
// CTA partial of NQ per-instance sums: thread (warp w, lane l) holds the sums
// of instances l * V + v; warps are added in order. Valid in threads t < G
// (instance t of the group).
template <int NQ, int V>
__device__ __forceinline__ void cta_sums(const double (&acc)[NQ][V], double (&out)[NQ]) {
    constexpr int G = 32 * V;
    __shared__ double red[NQ][kIlWarps][G];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) red[q][warp][lane * V + v] = acc[q][v];
    __syncthreads();
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double s = 0.0;
        if (t < G) {
#pragma unroll
            for (int w = 0; w < kIlWarps; ++w) s += red[q][w][t];
        }
        out[q] = s;
    }
}

// Sum of `n` (at most kIlBatch) rows of a partials array for instance t, in
// row order; every load is issued before the first add.
template <int NQ, int G>
__device__ __forceinline__ void sum_rows(const double* part, int k0, int n, int t, double (&s)[NQ]) {
    double v[kIlBatch][NQ];
#pragma unroll
    for (int k = 0; k < kIlBatch; ++k)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            v[k][q] = k < n ? part[(static_cast<int64_t>(k0 + k) * NQ + q) * G + t] : 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) s[q] = 0.0;
#pragma unroll
    for (int k = 0; k < kIlBatch; ++k)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (k < n) s[q] += v[k][q];
}

// First level of a group sum: the CTA writes its partial; the last CTA of
// its batch of kIlBatch CTAs writes the batch sum. Returns true in the CTA
// that completed the batch.
template <int NQ, int G>
__device__ __forceinline__ bool batch_sums(const double (&cta)[NQ], double* part, double* part2,
                                           int32_t* cnt, int ctas, int cta_index) {
    const int t = threadIdx.x;
    if (t < G) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) part[(static_cast<int64_t>(cta_index) * NQ + q) * G + t] = cta[q];
    }
    const int batch = cta_index / kIlBatch;
    const int b0 = batch * kIlBatch;
    const int b1 = b0 + kIlBatch < ctas ? b0 + kIlBatch : ctas;
    if (!arrive_last_cta(cnt + batch, b1 - b0)) return false;
    if (t < G) {
        double s[NQ];
        sum_rows<NQ, G>(part, b0, b1 - b0, t, s);
#pragma unroll
        for (int q = 0; q < NQ; ++q) part2[(static_cast<int64_t>(batch) * NQ + q) * G + t] = s[q];
    }
    return true;
}

// Sum of the first `n` rows of a batch-sum array for instance t, in order.
template <int NQ, int G>
__device__ __forceinline__ void sum_batches(const double* part2, int n, int t, double (&tot)[NQ]) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) tot[q] = 0.0;
    for (int k0 = 0; k0 < n; k0 += kIlBatch) {
        double s[NQ];
        sum_rows<NQ, G>(part2, k0, n - k0 < kIlBatch ? n - k0 : kIlBatch, t, s);
        // The chunk sums are added in order; each chunk is itself an in-order
        // sum, so the total is fixed by n alone.
#pragma unroll
        for (int q = 0; q < NQ; ++q) tot[q] += s[q];
    }
}

// ---------------------------------------------------------------------------
// Shared-memory staging of a tile's matrix entries (double-buffered: the
// entries of the next tile are copied while the current one is processed)
// ---------------------------------------------------------------------------
template <class T>
struct Stage {
    int32_t ptr[kIlTileLines + 1];   // entry offsets relative to the tile
    int32_t idx[kIlTileEntries];
    T val[kIlTileEntries];
};

template <int kBytes>
__device__ __forceinline__ void copy_async(void* dst, const void* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(kBytes));
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_group 0;\n" ::); }

template <class T>
__device__ __forceinline__ void stage_tile_async(const IlTile& t, const int64_t* __restrict__ ptr,
                                                 const int32_t* __restrict__ idx,
                                                 const T* __restrict__ val, Stage<T>& st) {
    for (int q = threadIdx.x; q < t.entries; q += blockDim.x) {
        copy_async<4>(st.idx + q, idx + t.e0 + q);
        copy_async<sizeof(T)>(st.val + q, val + t.e0 + q);
    }
    for (int q = threadIdx.x; q <= t.lines; q += blockDim.x)
        st.ptr[q] = static_cast<int32_t>(__ldg(ptr + t.line0 + q) - t.e0);
    copy_async_commit();
}

// sum_k val[k] * src[idx[k] * bp + ...] for the lane's V instances, entries
// in order; kU gathers in flight. Instances with `fix` gather their committed
// values from `alt` (rare).
template <int kU, class T, int V>
__device__ __forceinline__ void gather_sum(const int32_t* idx, const T* val, int n,
                                           const T* __restrict__ src, const T* __restrict__ alt,
                                           uint32_t fix, int64_t bp, T (&sum)[V]) {
#pragma unroll
    for (int v = 0; v < V; ++v) sum[v] = T(0);
    int k = 0;
    for (; k + kU <= n; k += kU) {
        int32_t i[kU];
        T w[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            i[u] = idx[k + u];
            w[u] = val[k + u];
        }
        T g[kU][V];
#pragma unroll
        for (int u = 0; u < kU; ++u) load_committed<T, V>(src, alt, i[u] * bp, fix, g[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u)
#pragma unroll
            for (int v = 0; v < V; ++v) sum[v] += w[u] * g[u][v];
    }
    for (; k < n; ++k) {
        T g[V];
        load_committed<T, V>(src, alt, idx[k] * bp, fix, g);
        const T w = val[k];
#pragma unroll
        for (int v = 0; v < V; ++v) sum[v] += w * g[v];
    }
}

// Lines per warp pass: about four lane-vectors of each kind in flight per
// warp within 128 registers.
template <class T, int V>
constexpr int kPrimalU = (sizeof(T) == 4 ? 4 : 2) / V > 0 ? (sizeof(T) == 4 ? 4 : 2) / V : 1;
template <class T, int V>
constexpr int kDualU = (sizeof(T) == 4 && V == 1) ? 2 : 1;
// Gathers in flight per lane in the dual's entry loop.
template <int V>
constexpr int kDualGather = V >= 4 ? 4 : 8;

// ---------------------------------------------------------------------------
// Primal half
// ---------------------------------------------------------------------------
template <class T, int V>
struct PrimalCtx {
    const Interleaved<T>* il;
    Lanes<T, V> ls;
    const T* XR;
    const T* XW_read;
    T* xr;
    T* xw;
    const T* YR;
    const T* YW;
    T* avg;
    int64_t col0;      // first instance of the lane
    bool fc, fl, fu;
};

// Bounds of a line: one value per lane-instance, or one for all (kFam: both
// bounds are the family's).
template <class T, int V, bool kFam>
struct Bounds {
    static constexpr int N = kFam ? 1 : V;
    T lo[N], hi[N];
    __device__ __forceinline__ T l(int v) const { return lo[kFam ? 0 : v]; }
    __device__ __forceinline__ T h(int v) const { return hi[kFam ? 0 : v]; }
};

template <class T, int V, bool kFam>
__device__ __forceinline__ void load_bounds(const Interleaved<T>& il, int klo, int khi, bool flo,
                                            bool fhi, int64_t line, int64_t e, Bounds<T, V, kFam>& B) {
    if constexpr (kFam) {
        B.lo[0] = __ldg(il.vec[klo] + line);
        B.hi[0] = __ldg(il.vec[khi] + line);
    } else {
        load_vec<T, V>(il, klo, flo, line, e, B.lo);
        load_vec<T, V>(il, khi, fhi, line, e, B.hi);
    }
}

template <class T, int V, bool kFam>
struct PrimalLine {
    T c[V], prev[V], a[V];
    Bounds<T, V, kFam> b;
    T tj, itj;
};

template <class T, int V, bool kFam>
__device__ __forceinline__ void primal_load(const PrimalCtx<T, V>& x, int j, PrimalLine<T, V, kFam>& L) {
    const Interleaved<T>& il = *x.il;
    const int64_t e = j * static_cast<int64_t>(il.bp) + x.col0;
    L.tj = __ldg(il.tau + j);
    L.itj = __ldg(il.itau + j);
    load_committed<T, V>(x.XR, x.XW_read, e, x.ls.fix, L.prev);
    if (x.fc) load_vec<T, V>(il, kIlC, true, j, e, L.c);
    else ldv_cs<T, V>(il.vec[kIlC] + e, L.c);
    load_bounds<T, V, kFam>(il, kIlXl, kIlXu, x.fl, x.fu, j, e, L.b);
    if (x.ls.pending) ldv_cs<T, V>(x.avg + e, L.a);
}

template <class T, int V, bool kFam>
__device__ __forceinline__ void primal_store(const PrimalCtx<T, V>& x, int j, const PrimalLine<T, V, kFam>& L,
                                             const T (&sum)[V], double (&moved)[V]) {
    const Interleaved<T>& il = *x.il;
    const int64_t e = j * static_cast<int64_t>(il.bp) + x.col0;
    T upd[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const T gradient = L.c[v] + sum[v];
        upd[v] = smax(L.b.l(v), smin(L.prev[v] - x.ls.step[v] * L.tj * gradient, L.b.h(v)));
        const double d = static_cast<double>(upd[v] - L.prev[v]);
        if ((x.ls.active >> v) & 1) moved[v] += d * d * static_cast<double>(L.itj);
    }
    stv_masked<T, V>(x.xw + e, upd, x.ls.active);
    if (x.ls.pending) {
        T a[V];
#pragma unroll
        for (int v = 0; v < V; ++v)
            a[v] = ((x.ls.pending >> v) & 1) ? L.a[v] + x.ls.frac[v] * (L.prev[v] - L.a[v]) : L.a[v];
        stv_cs<T, V>(x.avg + e, a);
    }
    if (x.ls.fix) {
#pragma unroll
        for (int v = 0; v < V; ++v)
            if ((x.ls.fix >> v) & 1) x.xr[e + v] = L.prev[v];
    }
}

// The lines of one tile: each warp takes lines l, l + 8, ... kU at a time,
// issuing every line's loads and gathers before its arithmetic.
template <int kU, bool kStaged, bool kFam, class T, int V>
__device__ __forceinline__ void primal_tile(const PrimalCtx<T, V>& x, const IlTile& t,
                                            const Stage<T>& st, double (&moved)[V]) {
    const Interleaved<T>& il = *x.il;
    const int warp = threadIdx.x >> 5;
    const int64_t bp = il.bp;
    for (int l0 = warp; l0 < t.lines; l0 += kU * kIlWarps) {
        PrimalLine<T, V, kFam> L[kU];
        T sum[kU][V];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int l = l0 + u * kIlWarps;
            if (l < t.lines) primal_load(x, t.line0 + l, L[u]);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int l = l0 + u * kIlWarps;
            if (l >= t.lines) continue;
            if (kStaged) {
                gather_sum<2, T, V>(st.idx + st.ptr[l], st.val + st.ptr[l], st.ptr[l + 1] - st.ptr[l],
                                    x.YR + x.col0, x.YW + x.col0, x.ls.fix, bp, sum[u]);
            } else {
                const int64_t k0 = __ldg(il.at_ptr + t.line0 + l), k1 = __ldg(il.at_ptr + t.line0 + l + 1);
                gather_sum<2, T, V>(il.at_idx + k0, il.at_val + k0, static_cast<int>(k1 - k0),
                                    x.YR + x.col0, x.YW + x.col0, x.ls.fix, bp, sum[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int l = l0 + u * kIlWarps;
            if (l < t.lines) primal_store(x, t.line0 + l, L[u], sum[u], moved);
        }
    }
}

template <class T, int V, bool kFam>
__global__ void __launch_bounds__(kIlThreads, 3) k_il_primal(Interleaved<T> il, InstanceCtl* ctl,
                                                             int measure, int slot) {
    constexpr int G = 32 * V;
    __shared__ Stage<T> st[2];
    __shared__ HotCtl hot[G];
    const int group = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int R = slot & 1, W = R ^ 1;
    PrimalCtx<T, V> x;
    x.il = &il;
    x.col0 = static_cast<int64_t>(group) * G + lane * V;
    // The matrix does not change: its first tile is staged before the wait.
    const int t0 = il.at_cta[blockIdx.x], t1 = il.at_cta[blockIdx.x + 1];
    if (t0 < t1) {
        const IlTile first = il.at_tiles[t0];
        if (first.staged) stage_tile_async(first, il.at_ptr, il.at_idx, il.at_val, st[0]);
    }
    // The streams this CTA reads -- the committed x (buffer R, written by the
    // previous primal kernel), the iterate average and the objective -- were
    // final before this kernel started (the previous dual kernel waited for
    // the previous primal kernel to complete), so their first two tiles are
    // prefetched into L2 before the wait; each tile prefetches the one after.
    const T* const pstreams[3] = {il.X[R], il.avg_x, il.vec[kIlC]};
    const int pkinds = ((il.family >> kIlC) & 1) ? 2 : 3;
    const int64_t goff = static_cast<int64_t>(group) * G;
    const unsigned rbytes = static_cast<unsigned>(G * sizeof(T));
    for (int ti = t0; ti < t1 && ti < t0 + 2; ++ti) {
        const IlTile pt = il.at_tiles[ti];
        prefetch_rows<T, 3>(pstreams, pkinds, il.bp, goff, rbytes, pt.line0, pt.line0 + pt.lines);
    }
    pdl_wait();
    pdl_trigger();
    x.ls = lane_state<T, V>(il, ctl, static_cast<int>(x.col0), measure, R, true, hot);
    if (!__syncthreads_or(x.ls.active != 0)) {
        copy_async_wait();
        return;
    }
    x.XR = il.X[R];
    x.XW_read = il.X[W];
    x.xr = il.X[R];
    x.xw = il.X[W];
    x.YR = il.Y[R];
    x.YW = il.Y[W];
    x.avg = il.avg_x;
    x.fc = (il.family >> kIlC) & 1;
    x.fl = (il.family >> kIlXl) & 1;
    x.fu = (il.family >> kIlXu) & 1;

    double moved[1][V];
#pragma unroll
    for (int v = 0; v < V; ++v) moved[0][v] = 0.0;
    for (int ti = t0; ti < t1; ++ti) {
        const IlTile t = il.at_tiles[ti];
        copy_async_wait();
        __syncthreads();
        if (ti + 1 < t1) {
            const IlTile nt = il.at_tiles[ti + 1];
            if (nt.staged) stage_tile_async(nt, il.at_ptr, il.at_idx, il.at_val, st[(ti + 1 - t0) & 1]);
        }
        if (ti + 2 < t1) {
            const IlTile pt = il.at_tiles[ti + 2];
            prefetch_rows<T, 3>(pstreams, pkinds, il.bp, goff, rbytes, pt.line0, pt.line0 + pt.lines);
        }
        if (t.staged) primal_tile<kPrimalU<T, V>, true, kFam>(x, t, st[(ti - t0) & 1], moved[0]);
        else primal_tile<1, false, kFam>(x, t, st[0], moved[0]);
        __syncthreads();
    }
    double cta[1];
    cta_sums<1, V>(moved, cta);
    // The partial only: the dual kernel's CTAs add the batches.
    if (threadIdx.x < G)
        il.part_primal[(static_cast<int64_t>(group) * il.col_ctas + blockIdx.x) * G + threadIdx.x] = cta[0];
}

// ---------------------------------------------------------------------------
// Dual half and the trial decision
// ---------------------------------------------------------------------------
template <class T, int V>
struct DualCtx {
    const Interleaved<T>* il;
    Lanes<T, V> ls;
    const T* xt;       // trial x of the lane's instances
    const T* YR;
    const T* YW;
    const T* AXR;
    const T* AXW;
    T* yr;
    T* yw;
    T* axr;
    T* axw;
    T* avg;
    int64_t col0;
    bool fl, fu;
};

template <class T, int V, bool kFam>
struct DualLine {
    T ax[V], prev[V], a[V];
    Bounds<T, V, kFam> b;
    T sg, isg;
};

template <class T, int V, bool kFam>
__device__ __forceinline__ void dual_load(const DualCtx<T, V>& x, int i, DualLine<T, V, kFam>& L) {
    const Interleaved<T>& il = *x.il;
    const int64_t e = i * static_cast<int64_t>(il.bp) + x.col0;
    L.sg = __ldg(il.sigma + i);
    L.isg = __ldg(il.isigma + i);
    load_committed<T, V>(x.AXR, x.AXW, e, x.ls.fix, L.ax);
    load_committed<T, V>(x.YR, x.YW, e, x.ls.fix, L.prev);
    load_bounds<T, V, kFam>(il, kIlRl, kIlRu, x.fl, x.fu, i, e, L.b);
    if (x.ls.pending) ldv<T, V>(x.avg + e, L.a);
}

template <class T, int V, bool kFam>
__device__ __forceinline__ void dual_store(const DualCtx<T, V>& x, int i, const DualLine<T, V, kFam>& L,
                                           const T (&next)[V], double (&red)[2][V]) {
    const Interleaved<T>& il = *x.il;
    const int64_t e = i * static_cast<int64_t>(il.bp) + x.col0;
    T upd[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const T dact = next[v] - L.ax[v];
        const T ext = next[v] + dact;
        const T step = smax(x.ls.step[v] * L.sg, min_dual_step<T>());
        const T w = L.prev[v] + step * ext;
        upd[v] = smax(w - step * L.b.h(v), T(0)) + smin(w - step * L.b.l(v), T(0));
        const double d = static_cast<double>(upd[v] - L.prev[v]);
        if ((x.ls.active >> v) & 1) {
            red[0][v] += d * d * static_cast<double>(L.isg);
            red[1][v] += d * static_cast<double>(dact);
        }
    }
    stv_masked<T, V>(x.yw + e, upd, x.ls.active);
    stv_masked<T, V>(x.axw + e, next, x.ls.active);
    if (x.ls.pending) {
        T a[V];
#pragma unroll
        for (int v = 0; v < V; ++v)
            a[v] = ((x.ls.pending >> v) & 1) ? L.a[v] + x.ls.frac[v] * (L.prev[v] - L.a[v]) : L.a[v];
        stv<T, V>(x.avg + e, a);
    }
    if (x.ls.fix) {
#pragma unroll
        for (int v = 0; v < V; ++v)
            if ((x.ls.fix >> v) & 1) {
                x.yr[e + v] = L.prev[v];
                x.axr[e + v] = L.ax[v];
            }
    }
}

// Shared memory of the dual: one staged row tile, its segment table and the
// per-segment partial sums of the lane's V instances.
template <class T, int V>
struct DualStage {
    int32_t ptr[kIlTileLines + 1];
    int32_t lseg[kIlTileLines + 1];      // line l: segments lseg[l] .. lseg[l + 1] - 1
    int32_t segb[kIlTileSegs + 1];       // segment q: entries segb[q] .. segb[q + 1] - 1
    int32_t idx[kIlTileEntries];
    T val[kIlTileEntries];
    T part[kIlTileSegs][32 * V];
};

template <class T, int V>
__device__ __forceinline__ void stage_row_tile(const Interleaved<T>& il, const IlTile& t,
                                               DualStage<T, V>& st) {
    for (int q = threadIdx.x; q < t.entries; q += blockDim.x) {
        copy_async<4>(st.idx + q, il.a_idx + t.e0 + q);
        copy_async<sizeof(T)>(st.val + q, il.a_val + t.e0 + q);
    }
    copy_async_commit();
    const int32_t s0 = __ldg(il.a_lseg + t.line0);
    const int32_t segs = __ldg(il.a_lseg + t.line0 + t.lines) - s0;
    for (int q = threadIdx.x; q <= t.lines; q += blockDim.x) {
        st.ptr[q] = static_cast<int32_t>(__ldg(il.a_ptr + t.line0 + q) - t.e0);
        st.lseg[q] = __ldg(il.a_lseg + t.line0 + q) - s0;
    }
    for (int q = threadIdx.x; q <= segs; q += blockDim.x)
        st.segb[q] = static_cast<int32_t>(__ldg(il.a_segstart + s0 + q) - t.e0);
}

// A staged row tile in two passes: every warp gathers whole segments (all of
// a segment's entries in flight at once) into shared memory; then each row
// adds its segments in order and takes its dual step.
template <bool kFam, class T, int V>
__device__ __forceinline__ void dual_tile_segmented(const DualCtx<T, V>& x, const IlTile& t,
                                                    DualStage<T, V>& st, double (&red)[2][V]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t bp = x.il->bp;
    const int segs = st.lseg[t.lines];
    for (int q = warp; q < segs; q += kIlWarps) {
        const int b0 = st.segb[q];
        T sum[V];
        gather_sum<kIlSegEntries, T, V>(st.idx + b0, st.val + b0, st.segb[q + 1] - b0, x.xt, x.xt, 0u,
                                        bp, sum);
#pragma unroll
        for (int v = 0; v < V; ++v) st.part[q][lane * V + v] = sum[v];
    }
    __syncthreads();
    for (int l = warp; l < t.lines; l += kIlWarps) {
        DualLine<T, V, kFam> L;
        dual_load(x, t.line0 + l, L);
        T next[V];
#pragma unroll
        for (int v = 0; v < V; ++v) next[v] = T(0);
        for (int q = st.lseg[l]; q < st.lseg[l + 1]; ++q)
#pragma unroll
            for (int v = 0; v < V; ++v) next[v] += st.part[q][lane * V + v];
        dual_store(x, t.line0 + l, L, next, red);
    }
}

// A row too long to stage: warp 0 reads its entries from global memory.
template <bool kFam, class T, int V>
__device__ __forceinline__ void dual_line_global(const DualCtx<T, V>& x, const IlTile& t,
                                                 double (&red)[2][V]) {
    const Interleaved<T>& il = *x.il;
    if ((threadIdx.x >> 5) != 0) return;
    DualLine<T, V, kFam> L;
    dual_load(x, t.line0, L);
    const int64_t k0 = __ldg(il.a_ptr + t.line0), k1 = __ldg(il.a_ptr + t.line0 + 1);
    T sum[V];
    gather_sum<kDualGather<V>, T, V>(il.a_idx + k0, il.a_val + k0, static_cast<int>(k1 - k0), x.xt, x.xt,
                                     0u, il.bp, sum);
    dual_store(x, t.line0, L, sum, red);
}

template <class T, int V, bool kFam>
__global__ void __launch_bounds__(kIlThreads, 3) k_il_dual(Interleaved<T> il, InstanceCtl* ctl,
                                                           DeviceOptions o, int measure, int slot) {
    constexpr int G = 32 * V;
    static_assert(kIlThreads >= 2 * G, "the decision adds its two sums in two halves of the CTA");
    // The lane states are read before the first tile is staged (the barrier
    // in lane_state orders them), so they share the stage's memory.
    __shared__ union Smem {
        DualStage<T, V> st;
        HotCtl hot[G];
    } sm;
    DualStage<T, V>& st = sm.st;
    const int group = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int R = slot & 1, W = R ^ 1;
    DualCtx<T, V> x;
    x.il = &il;
    x.col0 = static_cast<int64_t>(group) * G + lane * V;
    // The control blocks were last written by the decision of the previous
    // dual kernel, which is complete (see pdl_wait): read before the wait.
    x.ls = lane_state<T, V>(il, ctl, static_cast<int>(x.col0), measure, R, false, sm.hot);
    if (!__syncthreads_or(x.ls.active != 0)) return;
    const int t0 = il.a_cta[blockIdx.x], t1 = il.a_cta[blockIdx.x + 1];
    if (t0 < t1 && il.a_tiles[t0].staged) stage_row_tile(il, il.a_tiles[t0], st);
    // No L2 prefetch of the rows' streams here: issued while the primal
    // kernel finishes, it competed with the primal's tail (flow stream, 256
    // slots: 5.41 ms per chunk with it, 5.28 without).
    pdl_wait();
    pdl_trigger();
    x.xt = il.X[W] + x.col0;
    x.YR = il.Y[R];
    x.YW = il.Y[W];
    x.AXR = il.AX[R];
    x.AXW = il.AX[W];
    x.yr = il.Y[R];
    x.yw = il.Y[W];
    x.axr = il.AX[R];
    x.axw = il.AX[W];
    x.avg = il.avg_y;
    x.fl = (il.family >> kIlRl) & 1;
    x.fu = (il.family >> kIlRu) & 1;

    double red[2][V];
#pragma unroll
    for (int v = 0; v < V; ++v) red[0][v] = red[1][v] = 0.0;
    for (int ti = t0; ti < t1; ++ti) {
        const IlTile t = il.a_tiles[ti];
        if (t.staged) {
            if (ti != t0) stage_row_tile(il, t, st);
            copy_async_wait();
            __syncthreads();
            dual_tile_segmented<kFam>(x, t, st, red);
        } else {
            dual_line_global<kFam>(x, t, red);
        }
        __syncthreads();
    }
    double cta[2];
    cta_sums<2, V>(red, cta);
    if (measure) return;
    const int64_t gp = static_cast<int64_t>(group);
    const int t = threadIdx.x;
    // The primal kernel's batch sums, spread over this kernel's CTAs.
    if (t < G) {
        const double* pp = il.part_primal + gp * il.col_ctas * G;
        double* pp2 = il.part2_primal + gp * il.col_batches * G;
        for (int k = blockIdx.x; k < il.col_batches; k += il.row_ctas) {
            const int b0 = k * kIlBatch;
            const int n = il.col_ctas - b0 < kIlBatch ? il.col_ctas - b0 : kIlBatch;
            double sp[1];
            sum_rows<1, G>(pp, b0, n, t, sp);
            pp2[static_cast<int64_t>(k) * G + t] = sp[0];
        }
    }
    int32_t* cnt = il.cnt_dual + gp * (il.row_batches + 1);
    if (!batch_sums<2, G>(cta, il.part_dual + gp * il.row_ctas * 2 * G, il.part2_dual + gp * il.row_batches * 2 * G,
                          cnt, il.row_ctas, blockIdx.x))
        return;
    if (!arrive_last_cta(cnt + il.row_batches, il.row_batches)) return;
    // The options by reference from shared memory: a reference to the kernel
    // parameter would make every thread of every CTA copy it to local memory.
    __shared__ DeviceOptions so;
    __shared__ double primal_sum[G];
    if (t == 0) so = o;
    // The instance's hot block and the group's two sums are fetched at
    // once: threads [0, G) add the dual kernel's batch sums of instance t,
    // threads [G, 2G) the primal kernel's of instance t - G.
    const int b = static_cast<int>(gp * G) + t;
    const bool mine = t < G && b < il.count;
    HotCtl h{};
    if (mine) {
        // The decision reads fields from every 128-byte line of the block:
        // they come into L1 while the sums below are fetched.
        const char* cb = reinterpret_cast<const char*>(ctl + b);
#pragma unroll
        for (int q = 128; q < static_cast<int>(sizeof(InstanceCtl)); q += 128)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(cb + q));
        h = load_hot(ctl + b);
    }
    double dd[2] = {0.0, 0.0};
    if (t < G) {
        sum_batches<2, G>(il.part2_dual + gp * il.row_batches * 2 * G, il.row_batches, t, dd);
    } else if (t < 2 * G) {
        double pm[1];
        sum_batches<1, G>(il.part2_primal + gp * il.col_batches * G, il.col_batches, t - G, pm);
        primal_sum[t - G] = pm[0];
    }
    __syncthreads();
    // The linesearch decision of each instance of the group (one thread each).
    if (!mine) return;
    if (h.phase == kPhaseDone || h.stage != kStageTrial || (h.fp64 != 0) != (sizeof(T) == 8)) return;
    InstanceCtl& c = ctl[b];
    const int before = c.parity;
    trial_control(c, so, primal_sum[t], dd[0], dd[1], il.n);
    c.ibuf = c.parity != before ? W : R;
}

// ---------------------------------------------------------------------------
// Transposes between the layouts, one 32-line x 32-instance tile per CTA
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_il_move(IlMove<T> mv) {
    __shared__ T tile[32][33];
    __shared__ int32_t sel[32], par[32], ib[32];
    const int group = blockIdx.y;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (threadIdx.x < 32) {
        const int b = group * 32 + tx;
        int s = 0, p = 0, q = 0;
        if (b < mv.count) {
            const InstanceCtl& c = mv.ctl[b];
            switch (mv.select) {
                case kIlAll: s = 1; break;
                case kIlMasked: s = mv.mask[b] != 0; break;
                case kIlAtCheck: s = c.stage == kStageCheck && precision_matches<T>(c); break;
                default: s = c.il_sync != 0; break;
            }
            p = c.parity;
            q = c.ibuf;
        }
        sel[tx] = s;
        par[tx] = p;
        ib[tx] = q;
    }
    __syncthreads();
    int pi = 0;
    while (pi + 1 < mv.pairs && static_cast<int>(blockIdx.x) >= mv.pair[pi + 1].tile0) ++pi;
    const IlPair<T>& P = mv.pair[pi];
    const int l0 = (static_cast<int>(blockIdx.x) - P.tile0) * 32;
    const int64_t bp = mv.bp;
    if (mv.to_planar) {
        for (int r = ty; r < 32; r += 8) {
            const int line = l0 + r;
            T v = T(0);
            if (line < P.lines && sel[tx])
                v = P.il[P.by_ibuf ? ib[tx] : 0][line * bp + group * 32 + tx];
            tile[r][tx] = v;
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            const int64_t b = group * 32 + r;
            const int line = l0 + tx;
            if (sel[r] && line < P.lines)
                P.planar[P.by_parity ? par[r] : 0][b * P.lines + line] = tile[tx][r];
        }
    } else {
        for (int r = ty; r < 32; r += 8) {
            const int64_t b = group * 32 + r;
            const int line = l0 + tx;
            T v = T(0);
            if (sel[r] && line < P.lines) v = P.planar[P.by_parity ? par[r] : 0][b * P.lines + line];
            tile[tx][r] = v;
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            const int line = l0 + r;
            if (line < P.lines && sel[tx]) P.il[P.by_ibuf ? ib[tx] : 0][line * bp + group * 32 + tx] = tile[r][tx];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < 32 && sel[tx]) {
        InstanceCtl& c = mv.ctl[group * 32 + tx];
        if (mv.select == kIlAtCheck) c.il_sync = 1;
        if (mv.reset_ibuf) c.ibuf = 0;
    }
}

template <class T>
__global__ void k_il_scale(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ orig, T* __restrict__ val,
                           const double* __restrict__ ls, const double* __restrict__ os,
                           int32_t lines) {
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= lines) return;
    const double f = ls[line];
    for (int64_t k = ptr[line]; k < ptr[line + 1]; ++k)   // SparseMatrix::scaled, sparse_matrix.cpp:243-274
        val[k] = static_cast<T>(orig[k] * (f * os[idx[k]]));
}

__device__ __forceinline__ double il_scale_bound(double b, double f) { return isfinite(b) ? b * f : b; }

struct FamSrc {
    const double* v[kIlVecs];
};

template <class T>
__global__ void k_il_family(Interleaved<T> il, FamSrc src, const double* __restrict__ rs,
                            const double* __restrict__ cs) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < il.n) {   // scaling.cpp:109-135, as the per-instance setup scales them
        const double f = cs[t];
        il.fam[kIlC][t] = static_cast<T>(src.v[kIlC][t] * f);
        il.fam[kIlXl][t] = static_cast<T>(il_scale_bound(src.v[kIlXl][t], 1.0 / f));
        il.fam[kIlXu][t] = static_cast<T>(il_scale_bound(src.v[kIlXu][t], 1.0 / f));
    }
    if (t < il.m) {
        const double f = rs[t];
        il.fam[kIlRl][t] = static_cast<T>(il_scale_bound(src.v[kIlRl][t], f));
        il.fam[kIlRu][t] = static_cast<T>(il_scale_bound(src.v[kIlRu][t], f));
    }
}

}  // namespace

// Both trial kernels ask for one shared-memory carveout: the smallest that
// holds, for either kernel, as many CTAs as its registers allow. Left to
// itself the driver configures each kernel's SMs for its own needs (the dual
// needs more shared memory than the primal), and an SM switches
// configuration only once it is empty, so a kernel's CTAs could not take the
// place of the previous kernel's finished CTAs on a busy SM: the
// programmatic launch lost most of its overlap. The smallest common carveout
// leaves the rest of the SM's memory to L1, which the dual's decision reads
// its control blocks through (measured on the flow stream, 256 slots: chunk
// 5.83 ms with each kernel's own carveout, 5.52 with the largest, 5.35 with
// this one). Set on the current device at setup, before any launch is
// captured.
template <class T, int V>
void same_carveout() {
    const void* const kernels[4] = {
        reinterpret_cast<const void*>(k_il_primal<T, V, false>), reinterpret_cast<const void*>(k_il_primal<T, V, true>),
        reinterpret_cast<const void*>(k_il_dual<T, V, false>), reinterpret_cast<const void*>(k_il_dual<T, V, true>)};
    int dev = 0, smem_sm = 0, regs_sm = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    size_t need = 0;
    for (const void* k : kernels) {
        cudaFuncAttributes a{};
        if (cudaFuncGetAttributes(&a, k) != cudaSuccess || a.numRegs <= 0) continue;
        const int blocks = regs_sm / (a.numRegs * kIlThreads);
        need = std::max(need, static_cast<size_t>(blocks) * (a.sharedSizeBytes + static_cast<size_t>(reserved)));
    }
    // The driver takes the carveout as a preference and rounds it to the
    // nearest shared-memory size an SM supports, so the request names the
    // smallest supported size that holds `need` exactly.
    constexpr int kSizesKb[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
    int percent = 100;
    if (smem_sm > 0 && need > 0) {
        for (int kb : kSizesKb) {
            const size_t bytes = static_cast<size_t>(kb) * 1024;
            if (bytes >= need && bytes <= static_cast<size_t>(smem_sm)) {
                percent = static_cast<int>((100 * bytes + static_cast<size_t>(smem_sm) - 1) / static_cast<size_t>(smem_sm));
                break;
            }
        }
    }
    for (const void* k : kernels) cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
    cudaGetLastError();
}

template <class T, int V>
int blocks_per_sm(bool dual) {
    int r = 0;
    same_carveout<T, V>();
    if (dual) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_il_dual<T, V, false>, kIlThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_il_primal<T, V, false>, kIlThreads, 0);
    return r > 0 ? r : 1;
}

template <class T>
int il_blocks_per_sm(int vl, bool dual) {
    if constexpr (sizeof(T) == 4) {
        if (vl == 4) return blocks_per_sm<T, 4>(dual);
    }
    if (vl == 2) return blocks_per_sm<T, 2>(dual);
    return blocks_per_sm<T, 1>(dual);
}

namespace {

// A trial kernel launched with programmatic stream serialization (see
// pdl_wait): it may start while the previous kernel in the stream finishes.
template <class... P, class... A>
void launch_pdl(void (*kernel)(P...), dim3 grid, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kIlThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

constexpr int32_t kXBounds = (1 << kIlXl) | (1 << kIlXu);
constexpr int32_t kRBounds = (1 << kIlRl) | (1 << kIlRu);

template <class T, int V>
void primal_v(const Interleaved<T>& il, InstanceCtl* ctl, int measure, int slot, cudaStream_t s) {
    const dim3 grid(il.col_ctas, il.groups);
    if ((il.family & kXBounds) == kXBounds)
        launch_pdl(k_il_primal<T, V, true>, grid, s, il, ctl, measure, slot);
    else
        launch_pdl(k_il_primal<T, V, false>, grid, s, il, ctl, measure, slot);
}

template <class T, int V>
void dual_v(const Interleaved<T>& il, InstanceCtl* ctl, const DeviceOptions& o, int measure, int slot,
            cudaStream_t s) {
    const dim3 grid(il.row_ctas, il.groups);
    if ((il.family & kRBounds) == kRBounds)
        launch_pdl(k_il_dual<T, V, true>, grid, s, il, ctl, o, measure, slot);
    else
        launch_pdl(k_il_dual<T, V, false>, grid, s, il, ctl, o, measure, slot);
}

}  // namespace

template <class T>
void launch_il_primal(const Interleaved<T>& il, InstanceCtl* ctl, int measure, int slot,
                      cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {
        if (il.vl == 4) return primal_v<T, 4>(il, ctl, measure, slot, s);
    }
    if (il.vl == 2) primal_v<T, 2>(il, ctl, measure, slot, s);
    else primal_v<T, 1>(il, ctl, measure, slot, s);
}

template <class T>
void launch_il_dual(const Interleaved<T>& il, InstanceCtl* ctl, const DeviceOptions& o,
                    int measure, int slot, cudaStream_t s) {
    if constexpr (sizeof(T) == 4) {
        if (il.vl == 4) return dual_v<T, 4>(il, ctl, o, measure, slot, s);
    }
    if (il.vl == 2) dual_v<T, 2>(il, ctl, o, measure, slot, s);
    else dual_v<T, 1>(il, ctl, o, measure, slot, s);
}

template <class T>
void launch_il_move(const IlMove<T>& mv, int groups, cudaStream_t s) {
    if (mv.pairs == 0 || mv.tiles == 0) return;
    k_il_move<T><<<dim3(mv.tiles, groups), 256, 0, s>>>(mv);
}

template <class T>
void launch_il_scale(const int64_t* ptr, const int32_t* idx, const double* orig, T* val,
                     const double* line_scale, const double* other_scale, int32_t lines,
                     cudaStream_t s) {
    if (lines <= 0) return;
    k_il_scale<T><<<(lines + 255) / 256, 256, 0, s>>>(ptr, idx, orig, val, line_scale, other_scale, lines);
}

template <class T>
void launch_il_family(const Interleaved<T>& il, const double* const fam[kIlVecs],
                      const double* rs, const double* cs, cudaStream_t s) {
    FamSrc src;
    for (int k = 0; k < kIlVecs; ++k) src.v[k] = fam[k];
    const int len = il.n > il.m ? il.n : il.m;
    if (len <= 0) return;
    k_il_family<T><<<(len + 255) / 256, 256, 0, s>>>(il, src, rs, cs);
}

#define PDLPGPU_IL_INSTANTIATE(T)                                                                 \
    template int il_blocks_per_sm<T>(int, bool);                                                         \
    template void launch_il_primal<T>(const Interleaved<T>&, InstanceCtl*, int, int, cudaStream_t); \
    template void launch_il_dual<T>(const Interleaved<T>&, InstanceCtl*, const DeviceOptions&, int, \
                                    int, cudaStream_t);                                          \
    template void launch_il_move<T>(const IlMove<T>&, int, cudaStream_t);                         \
    template void launch_il_scale<T>(const int64_t*, const int32_t*, const double*, T*,           \
                                     const double*, const double*, int32_t, cudaStream_t);        \
    template void launch_il_family<T>(const Interleaved<T>&, const double* const*, const double*, \
                                      const double*, cudaStream_t);
PDLPGPU_IL_INSTANTIATE(float)
PDLPGPU_IL_INSTANTIATE(double)

}  // namespace pdlpgpu

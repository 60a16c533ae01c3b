// mlp.cu -- the learned warm start's network, trained and evaluated with
// this library's own sm_100a kernels:
//
//   gemm_tn      C[M][N] = A[M][K] * B[N][K]^T, BF16 operands, FP32
//                accumulation on the 5th-generation tensor cores: TMA
//                (cp.async.bulk.tensor, 128-byte swizzle) fills a 3-stage
//                shared-memory ring, one thread issues tcgen05.mma
//                (M=128, N=128, K=16) into a TMEM accumulator and commits
//                each stage back to the producer through mbarriers, and the
//                epilogue reads TMEM with tcgen05.ld. Two CTAs share an SM,
//                so one's epilogue overlaps the other's main loop; tiles run
//                in grouped order for L2 reuse. Optional split-K writes one
//                FP32 partial per K range.
//   epilogue     sum of the split-K partials in a fixed order, bias,
//                ReLU, BF16/FP32 outputs
//   transpose, loss, ReLU backward, bias gradients, Adam
//
// Every mbarrier wait gives up after two seconds of %globaltimer, records an
// error code and lets the CTA drain its copies, free its TMEM and return, so
// a fault in the pipeline cannot hang the device.
#include "pdlpgpu_mlp.h"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <random>
#include <string>
#include <vector>

extern "C" void pdlpgpu_internal_set_error(const char* message);

namespace pdlpgpu_mlp_impl {

using bf16 = __nv_bfloat16;

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 64;                       // 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 3;                    // two CTAs per SM (shared memory)
constexpr int GEMM_THREADS = 128;
constexpr int STAGE_A_BYTES = BM * BK * 2;   // 16 KiB
constexpr int STAGE_B_BYTES = BN * BK * 2;   // 16 KiB
constexpr int GEMM_SMEM = STAGES * (STAGE_A_BYTES + STAGE_B_BYTES) + 1024 /*align*/ + 256 /*barriers*/;
constexpr int64_t kWaitNs = 2000000000LL;

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ int64_t gtimer() {
    int64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and an error code) after kWaitNs without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int* err, int code) {
    if (mbar_test(bar, phase)) return true;
    const int64_t t0 = gtimer();
    while (true) {
        if (mbar_test(bar, phase)) return true;
        if (gtimer() - t0 > kWaitNs) {
            atomicExch(err, code);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3fff);         // start address
    d |= static_cast<uint64_t>(1) << 16;                      // leading byte offset (16 B; unused)
    d |= static_cast<uint64_t>(1024 >> 4) << 32;              // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;                      // descriptor version
    d |= static_cast<uint64_t>(2) << 61;                      // SWIZZLE_128B
    return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M=128, N=BN.
constexpr uint32_t kInstrDesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                (static_cast<uint32_t>(BN >> 3) << 17) |
                                (static_cast<uint32_t>(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kInstrDesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
        "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// GEMM: one CTA per (128 x 128 output tile, K range)
// ---------------------------------------------------------------------------
struct GemmArgs {
    int M, N, K;
    int kblocks_per_split;
    float* C;                // [splits][M][N]
    int64_t split_stride;
    int* err;
};

__global__ void __launch_bounds__(GEMM_THREADS, 2)
gemm_tn(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
        GemmArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sa = smem;
    uint8_t* sb = smem + STAGES * STAGE_A_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sb + STAGES * STAGE_B_BYTES);
    uint64_t* full = bars;                    // [STAGES]
    uint64_t* empty = bars + STAGES;          // [STAGES]
    uint64_t* done = bars + 2 * STAGES;       // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Grouped tile order: consecutive CTAs sweep kGroupM row tiles for each
    // column tile, so the CTAs in flight share their A and B panels in L2.
    constexpr int kGroupM = 16;
    const int pid = blockIdx.x + blockIdx.y * gridDim.x;
    const int per_group = kGroupM * gridDim.y;
    const int first_m = (pid / per_group) * kGroupM;
    const int group_m = min(static_cast<int>(gridDim.x) - first_m, kGroupM);
    const int m0 = (first_m + (pid % per_group) % group_m) * BM;
    const int n0 = ((pid % per_group) / group_m) * BN;
    const int total_kb = (a.K + BK - 1) / BK;
    const int kb0 = blockIdx.z * a.kblocks_per_split;
    const int kb1 = min(total_kb, kb0 + a.kblocks_per_split);
    const int nk = max(0, kb1 - kb0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // Warp-specialised pipeline. Lane 0 of warp 0 produces: it refills a
    // stage as soon as the MMAs that read it have completed (`empty`), never
    // waiting on the MMAs of other stages. Lane 0 of warp 1 consumes: it
    // waits for a stage's bytes (`full`), issues its four MMAs and commits
    // the stage back, so the tensor pipe always has the next stage queued.
    __shared__ int consumed_by_mma;
    if (threadIdx.x == 0) consumed_by_mma = 0;
    __syncthreads();
    int issued = 0;
    if (warp == 0 && lane == 0 && nk > 0) {
        const uint32_t tx = STAGE_A_BYTES + STAGE_B_BYTES;
        for (int i = 0; i < nk; ++i) {
            const int s = i % STAGES;
            if (i >= STAGES && !mbar_wait(smem_u32(&empty[s]), ((i / STAGES) - 1) & 1, a.err, 2)) break;
            const uint32_t fb = smem_u32(&full[s]);
            mbar_expect_tx(fb, tx);
            tma_load_2d(smem_u32(sa + s * STAGE_A_BYTES), &map_a, fb, (kb0 + i) * BK, m0);
            tma_load_2d(smem_u32(sb + s * STAGE_B_BYTES), &map_b, fb, (kb0 + i) * BK, n0);
            ++issued;
        }
    } else if (warp == 1 && lane == 0 && nk > 0) {
        int i = 0;
        for (; i < nk; ++i) {
            const int s = i % STAGES;
            if (!mbar_wait(smem_u32(&full[s]), (i / STAGES) & 1, a.err, 1)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_base = smem_u32(sa + s * STAGE_A_BYTES);
            const uint32_t b_base = smem_u32(sb + s * STAGE_B_BYTES);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                // K advances 16 BF16 = 32 bytes inside the 128-byte swizzle row.
                mma_bf16(tmem, smem_desc(a_base + kk * 32), smem_desc(b_base + kk * 32),
                         (i > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&empty[s]));
        }
        consumed_by_mma = i;
        // Arrives once every MMA issued above has completed.
        mma_commit(smem_u32(done));
    }
    __syncthreads();
    // After an error, copies the MMA warp never consumed may still be in
    // flight: the producer waits for them (bounded) before the stage memory
    // is reused below.
    if (warp == 0 && lane == 0)
        for (int i = consumed_by_mma; i < issued; ++i)
            mbar_wait(smem_u32(&full[i % STAGES]), (i / STAGES) & 1, a.err, 3);
    bool have = nk > 0;
    if (have) have = mbar_wait(smem_u32(done), 0, a.err, 4);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // Epilogue: warp w owns TMEM lanes [32w, 32w + 32) = output rows. Each
    // 32 x 32 block goes through shared memory (the drained stage buffers),
    // so every store instruction writes 32 consecutive floats of one row.
    float* tile = reinterpret_cast<float*>(sa) + warp * 32 * 33;
    const int row0 = m0 + warp * 32;
    float* cbase = a.C + blockIdx.z * a.split_stride;
    for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t r[32];
        tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, r);
#pragma unroll
        for (int j = 0; j < 32; ++j) tile[lane * 33 + j] = have ? __uint_as_float(r[j]) : 0.0f;
        __syncwarp();
        const int col = n0 + c0 + lane;
        for (int rr = 0; rr < 32; ++rr) {
            const int row = row0 + rr;
            if (row < a.M && col < a.N) cbase[static_cast<int64_t>(row) * a.N + col] = tile[rr * 33 + lane];
        }
        __syncwarp();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
    }
}

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------
// out = act(sum_z partial[z] + bias) -> optional FP32 and BF16 copies.
__global__ void epilogue(const float* partial, int splits, int64_t split_stride, int M, int N,
                         const float* bias, int relu, float* out_f32, bf16* out_bf16) {
    const int64_t total = static_cast<int64_t>(M) * N;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float v = 0.0f;
        for (int z = 0; z < splits; ++z) v += partial[z * split_stride + t];
        if (bias) v += bias[t % N];
        if (relu) v = v > 0.0f ? v : 0.0f;
        if (out_f32) out_f32[t] = v;
        if (out_bf16) out_bf16[t] = __float2bfloat16_rn(v);
    }
}

// dst[c][r] = src[r][c] for a rows x cols BF16 matrix.
__global__ void transpose_bf16(const bf16* src, bf16* dst, int rows, int cols) {
    __shared__ bf16 tile[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    for (int k = 0; k < 32; k += 8) {
        const int r = blockIdx.y * 32 + threadIdx.y + k;
        if (r < rows && c < cols) tile[threadIdx.y + k][threadIdx.x] = src[static_cast<int64_t>(r) * cols + c];
    }
    __syncthreads();
    const int r2 = blockIdx.y * 32 + threadIdx.x;
    for (int k = 0; k < 32; k += 8) {
        const int c2 = blockIdx.x * 32 + threadIdx.y + k;
        if (r2 < rows && c2 < cols) dst[static_cast<int64_t>(c2) * rows + r2] = tile[threadIdx.x][threadIdx.y + k];
    }
}

// d = 2 w_j (out - target) / batch, in FP32 and BF16; per-row loss partials.
__global__ void loss_grad(const float* out, const float* target, const float* w, int B, int N,
                          float* d_f32, bf16* d_bf16, float* row_loss) {
    const int b = blockIdx.x;
    float acc = 0.0f;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const int64_t t = static_cast<int64_t>(b) * N + j;
        const float e = out[t] - target[t];
        acc += w[j] * e * e;
        const float g = 2.0f * w[j] * e / static_cast<float>(B);
        d_f32[t] = g;
        d_bf16[t] = __float2bfloat16_rn(g);
    }
    __shared__ float red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) row_loss[b] = red[0] / static_cast<float>(B);
}

__global__ void sum_rows(const float* row_loss, int B, float* loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.0f;
        for (int b = 0; b < B; ++b) s += row_loss[b];
        *loss = s;
    }
}

// dZ = dH * (H > 0) -> FP32 and BF16.
__global__ void relu_backward(const float* dh, const bf16* h, int64_t total, float* dz_f32, bf16* dz_bf16) {
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float v = __bfloat162float(h[t]) > 0.0f ? dh[t] : 0.0f;
        dz_f32[t] = v;
        dz_bf16[t] = __float2bfloat16_rn(v);
    }
}

// db[j] = sum_b d[b][j] (rows summed in order).
__global__ void column_sums(const float* d, int B, int N, float* db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += d[static_cast<int64_t>(b) * N + j];
    db[j] = s;
}

// Adam (Kingma and Ba, 2015) with bias correction; refreshes the BF16 copy.
__global__ void adam(float* p, const float* g, float* m, float* v, bf16* p_bf16, int64_t n, float lr,
                     float b1, float b2, float eps, float c1, float c2) {
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float gr = g[t];
        const float mt = b1 * m[t] + (1.0f - b1) * gr;
        const float vt = b2 * v[t] + (1.0f - b2) * gr * gr;
        m[t] = mt;
        v[t] = vt;
        const float upd = lr * (mt / c1) / (sqrtf(vt / c2) + eps);
        const float pn = p[t] - upd;
        p[t] = pn;
        if (p_bf16) p_bf16[t] = __float2bfloat16_rn(pn);
    }
}

__global__ void to_bf16(const float* src, bf16* dst, int64_t n) {
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[t] = __float2bfloat16_rn(src[t]);
}

// --- codec between LP instances and the network -----------------------------
// Features: standardised instance parameters, BF16, zero-padded to `padded`.
__global__ void encode_features(const double* params, int B, int P, int padded, const float* mean,
                                const float* inv_std, bf16* out) {
    const int64_t total = static_cast<int64_t>(B) * padded;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / padded;
        const int k = static_cast<int>(t - b * padded);
        float v = 0.0f;
        if (k < P) v = (static_cast<float>(params[b * P + k]) - mean[k]) * inv_std[k];
        out[t] = __float2bfloat16_rn(v);
    }
}

// Targets: primal / scale, standardised dual, standardised log weight, zeros.
__global__ void encode_targets(const double* x, const double* y, const double* w, int B, int n, int m,
                               int O, const double* scale, const float* ymean, const float* yinv,
                               float wmean, float winv, float* out) {
    const int64_t total = static_cast<int64_t>(B) * O;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / O;
        const int j = static_cast<int>(t - b * O);
        float v = 0.0f;
        if (j < n) v = static_cast<float>(x[b * n + j] / scale[j]);
        else if (j < n + m) v = (static_cast<float>(y[b * m + (j - n)]) - ymean[j - n]) * yinv[j - n];
        else if (j == n + m) v = (logf(static_cast<float>(w[b])) - wmean) * winv;
        out[t] = v;
    }
}

// Warm start from network outputs: x = clamp(out, 0, 1) * scale, y and the
// weight de-standardised.
__global__ void decode_warmstart(const float* out, int B, int n, int m, int O, const double* scale,
                                 const float* ymean, const float* ystd, float wmean, float wstd,
                                 double* wx, double* wy, double* ww) {
    const int64_t total = static_cast<int64_t>(B) * (n + m + 1);
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = t / (n + m + 1);
        const int j = static_cast<int>(t - b * (n + m + 1));
        const float v = out[b * O + j];
        if (j < n) wx[b * n + j] = static_cast<double>(fminf(fmaxf(v, 0.0f), 1.0f)) * scale[j];
        else if (j < n + m) wy[b * m + (j - n)] = static_cast<double>(v * ystd[j - n] + ymean[j - n]);
        else ww[b] = static_cast<double>(expf(v * wstd + wmean));
    }
}

inline unsigned grid_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return static_cast<unsigned>(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mutex;

bool encoder(std::string& err) {
    std::lock_guard<std::mutex> lock(g_encode_mutex);
    if (g_encode) return true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || fn == nullptr) {
        err = "cuTensorMapEncodeTiled unavailable";
        return false;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return true;
}

// 2-D BF16 row-major [rows][cols] tensor map with a (BK x box_rows) box.
bool make_map(CUtensorMap& map, const void* base, int64_t rows, int64_t cols, int box_rows,
              std::string& err) {
    if (!encoder(err)) return false;
    if ((cols * 2) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) {
        err = "GEMM operand rows must be 16-byte multiples and 16-byte aligned";
        return false;
    }
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols * 2)};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = g_encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed";
        return false;
    }
    return true;
}

struct GemmLaunch {
    int splits = 1;
};

// C[splits][M][N] partials of A[M][K] * B[N][K]^T.
bool gemm(const bf16* A, const bf16* B, float* C, int M, int N, int K, int splits, int* err,
          cudaStream_t s, std::string& msg) {
    if (M <= 0 || N <= 0 || K <= 0) return true;
    if (K % 8 != 0) {
        msg = "GEMM K must be a multiple of 8";
        return false;
    }
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_set[dev & 63]) {
        if (cudaFuncSetAttribute(gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM) != cudaSuccess) {
            msg = "cudaFuncSetAttribute failed";
            return false;
        }
        attr_set[dev & 63] = true;
    }
    CUtensorMap ma, mb;
    if (!make_map(ma, A, M, K, BM, msg) || !make_map(mb, B, N, K, BN, msg)) return false;
    const int total_kb = (K + BK - 1) / BK;
    splits = std::max(1, std::min(splits, total_kb));
    const int per = (total_kb + splits - 1) / splits;
    splits = (total_kb + per - 1) / per;
    GemmArgs ga{M, N, K, per, C, static_cast<int64_t>(M) * N, err};
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, splits);
    gemm_tn<<<grid, GEMM_THREADS, GEMM_SMEM, s>>>(ma, mb, ga);
    return cudaGetLastError() == cudaSuccess;
}

int splits_for(int M, int N, int K) {
    const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
    const int kb = (K + BK - 1) / BK;
    int s = std::max(1, 148 / std::max(1, tiles));
    return std::min(s, std::max(1, kb / 4));
}

}  // namespace pdlpgpu_mlp_impl

using namespace pdlpgpu_mlp_impl;

struct pdlpgpu_mlp {
    int in = 0, hidden = 0, out = 0, batch = 0, device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t caller_done = nullptr;
    std::vector<void*> allocs;
    // parameters (FP32 master), BF16 copies, Adam moments, gradients
    float *W1 = nullptr, *b1 = nullptr, *W2 = nullptr, *b2 = nullptr, *W3 = nullptr, *b3 = nullptr;
    bf16 *W1h = nullptr, *W2h = nullptr, *W3h = nullptr;
    float *mW1, *vW1, *mb1, *vb1, *mW2, *vW2, *mb2, *vb2, *mW3, *vW3, *mb3, *vb3;
    float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3;
    // activations and scratch
    bf16 *H1 = nullptr, *H2 = nullptr;
    float *Out = nullptr, *dOut = nullptr, *dH = nullptr, *dZ = nullptr;
    bf16 *dOuth, *dZh;
    bf16 *T1, *T2;              // transposes
    float* partial = nullptr;   // split-K partials
    int64_t partial_elems = 0;
    float* row_loss = nullptr;
    float* loss_dev = nullptr;
    int* err = nullptr;
    int64_t step = 0;
    int64_t launches = 0;
    std::string msg;

    ~pdlpgpu_mlp() {
        for (void* p : allocs) cudaFree(p);
        if (caller_done) cudaEventDestroy(caller_done);
        if (stream) cudaStreamDestroy(stream);
    }

    // The caller's device arguments (features, targets, parameters) are
    // usually written just before the call on the legacy default stream --
    // by pdlpgpu_encode_features, or by PyTorch, which enqueues there by
    // default -- and the model's own stream does not synchronise with it
    // implicitly (it is non-blocking): it waits for all work enqueued there
    // so far before it reads them.
    bool wait_for_caller() {
        if (!caller_done && cudaEventCreateWithFlags(&caller_done, cudaEventDisableTiming) != cudaSuccess)
            return false;
        return cudaEventRecord(caller_done, cudaStreamLegacy) == cudaSuccess &&
               cudaStreamWaitEvent(stream, caller_done, 0) == cudaSuccess;
    }

    template <class T>
    bool alloc(T*& p, int64_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, static_cast<size_t>(std::max<int64_t>(n, 1)) * sizeof(T)) != cudaSuccess) {
            msg = "cudaMalloc failed";
            return false;
        }
        cudaMemsetAsync(q, 0, static_cast<size_t>(std::max<int64_t>(n, 1)) * sizeof(T), stream);
        allocs.push_back(q);
        p = static_cast<T*>(q);
        return true;
    }

    bool run_gemm(const bf16* A, const bf16* B, int M, int N, int K, int splits) {
        ++launches;
        return gemm(A, B, partial, M, N, K, splits, err, stream, msg);
    }

    void finish(int M, int N, int splits, const float* bias, int relu, float* of, bf16* ob) {
        epilogue<<<grid_for(static_cast<int64_t>(M) * N), 256, 0, stream>>>(
            partial, splits, static_cast<int64_t>(M) * N, M, N, bias, relu, of, ob);
        ++launches;
    }

    void transpose(const bf16* src, bf16* dst, int rows, int cols) {
        dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
        transpose_bf16<<<grid, block, 0, stream>>>(src, dst, rows, cols);
        ++launches;
    }

    int effective_splits(int M, int N, int K) const {
        const int total_kb = (K + BK - 1) / BK;
        int s = std::max(1, std::min(splits_for(M, N, K), total_kb));
        const int per = (total_kb + s - 1) / s;
        return (total_kb + per - 1) / per;
    }

    bool forward(const bf16* X) {
        const int B = batch;
        int s = effective_splits(B, hidden, in);
        if (!run_gemm(X, W1h, B, hidden, in, s)) return false;
        finish(B, hidden, s, b1, 1, nullptr, H1);
        s = effective_splits(B, hidden, hidden);
        if (!run_gemm(H1, W2h, B, hidden, hidden, s)) return false;
        finish(B, hidden, s, b2, 1, nullptr, H2);
        s = effective_splits(B, out, hidden);
        if (!run_gemm(H2, W3h, B, out, hidden, s)) return false;
        finish(B, out, s, b3, 0, Out, nullptr);
        return true;
    }

    bool backward(const bf16* X, const float* target, const float* w) {
        const int B = batch;
        loss_grad<<<B, 256, 0, stream>>>(Out, target, w, B, out, dOut, dOuth, row_loss);
        sum_rows<<<1, 32, 0, stream>>>(row_loss, B, loss_dev);
        column_sums<<<(out + 255) / 256, 256, 0, stream>>>(dOut, B, out, gb3);
        launches += 3;
        // dW3 = dOut^T H2
        transpose(dOuth, T1, B, out);        // [out][B]
        transpose(H2, T2, B, hidden);        // [hidden][B]
        if (!run_gemm(T1, T2, out, hidden, B, 1)) return false;
        finish(out, hidden, 1, nullptr, 0, gW3, nullptr);
        // dH2 = dOut W3 = dOut (W3^T)^T
        transpose(W3h, T1, out, hidden);     // [hidden][out]
        int s = effective_splits(B, hidden, out);
        if (!run_gemm(dOuth, T1, B, hidden, out, s)) return false;
        finish(B, hidden, s, nullptr, 0, dH, nullptr);
        relu_backward<<<grid_for(static_cast<int64_t>(B) * hidden), 256, 0, stream>>>(
            dH, H2, static_cast<int64_t>(B) * hidden, dZ, dZh);
        column_sums<<<(hidden + 255) / 256, 256, 0, stream>>>(dZ, B, hidden, gb2);
        launches += 2;
        // dW2 = dZ2^T H1
        transpose(dZh, T1, B, hidden);
        transpose(H1, T2, B, hidden);
        if (!run_gemm(T1, T2, hidden, hidden, B, 1)) return false;
        finish(hidden, hidden, 1, nullptr, 0, gW2, nullptr);
        // dH1 = dZ2 W2
        transpose(W2h, T1, hidden, hidden);
        s = effective_splits(B, hidden, hidden);
        if (!run_gemm(dZh, T1, B, hidden, hidden, s)) return false;
        finish(B, hidden, s, nullptr, 0, dH, nullptr);
        relu_backward<<<grid_for(static_cast<int64_t>(B) * hidden), 256, 0, stream>>>(
            dH, H1, static_cast<int64_t>(B) * hidden, dZ, dZh);
        column_sums<<<(hidden + 255) / 256, 256, 0, stream>>>(dZ, B, hidden, gb1);
        launches += 2;
        // dW1 = dZ1^T X
        transpose(dZh, T1, B, hidden);
        transpose(X, T2, B, in);             // [in][B]
        if (!run_gemm(T1, T2, hidden, in, B, 1)) return false;
        finish(hidden, in, 1, nullptr, 0, gW1, nullptr);
        return true;
    }

    void adam_all(float lr) {
        ++step;
        const float b1c = 0.9f, b2c = 0.999f, eps = 1e-8f;
        const float c1 = 1.0f - std::pow(b1c, static_cast<float>(step));
        const float c2 = 1.0f - std::pow(b2c, static_cast<float>(step));
        struct P { float* p; float* g; float* m; float* v; bf16* h; int64_t n; };
        const P ps[6] = {{W1, gW1, mW1, vW1, W1h, int64_t(hidden) * in},
                         {b1, gb1, mb1, vb1, nullptr, hidden},
                         {W2, gW2, mW2, vW2, W2h, int64_t(hidden) * hidden},
                         {b2, gb2, mb2, vb2, nullptr, hidden},
                         {W3, gW3, mW3, vW3, W3h, int64_t(out) * hidden},
                         {b3, gb3, mb3, vb3, nullptr, out}};
        for (const P& q : ps) {
            adam<<<grid_for(q.n), 256, 0, stream>>>(q.p, q.g, q.m, q.v, q.h, q.n, lr, b1c, b2c, eps, c1, c2);
            ++launches;
        }
    }

    void refresh_bf16() {
        to_bf16<<<grid_for(int64_t(hidden) * in), 256, 0, stream>>>(W1, W1h, int64_t(hidden) * in);
        to_bf16<<<grid_for(int64_t(hidden) * hidden), 256, 0, stream>>>(W2, W2h, int64_t(hidden) * hidden);
        to_bf16<<<grid_for(int64_t(out) * hidden), 256, 0, stream>>>(W3, W3h, int64_t(out) * hidden);
    }

    bool check_err(const char* what) {
        int h = 0;
        if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            msg = std::string(what) + ": " + cudaGetErrorString(cudaGetLastError());
            return false;
        }
        if (h != 0) {
            msg = std::string(what) + ": tensor-core pipeline wait timed out (code " + std::to_string(h) + ")";
            cudaMemsetAsync(err, 0, sizeof(int), stream);
            return false;
        }
        return true;
    }
};

namespace {
int fail(const std::string& m) {
    pdlpgpu_internal_set_error(m.c_str());
    return -1;
}
}  // namespace

extern "C" {

int32_t pdlpgpu_mlp_create(int32_t in, int32_t hidden, int32_t out, int32_t batch, uint64_t seed,
                           int32_t device, pdlpgpu_mlp** result) {
    if (in <= 0 || in % 8 != 0 || hidden <= 0 || hidden % 64 != 0 || out <= 0 || out % 64 != 0 ||
        batch <= 0 || batch % 8 != 0)
        return fail("mlp: in must be a multiple of 8, hidden and out of 64, batch of 8");
    auto* m = new pdlpgpu_mlp();
    m->in = in; m->hidden = hidden; m->out = out; m->batch = batch; m->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete m;
        return fail("mlp: cannot use the device");
    }
    const int64_t H = hidden, I = in, O = out, B = batch;
    bool ok = m->alloc(m->W1, H * I) && m->alloc(m->b1, H) && m->alloc(m->W2, H * H) &&
              m->alloc(m->b2, H) && m->alloc(m->W3, O * H) && m->alloc(m->b3, O) &&
              m->alloc(m->W1h, H * I) && m->alloc(m->W2h, H * H) && m->alloc(m->W3h, O * H);
    for (auto* q : {&m->mW1, &m->vW1, &m->gW1}) ok = ok && m->alloc(*q, H * I);
    for (auto* q : {&m->mW2, &m->vW2, &m->gW2}) ok = ok && m->alloc(*q, H * H);
    for (auto* q : {&m->mW3, &m->vW3, &m->gW3}) ok = ok && m->alloc(*q, O * H);
    for (auto* q : {&m->mb1, &m->vb1, &m->gb1, &m->mb2, &m->vb2, &m->gb2}) ok = ok && m->alloc(*q, H);
    for (auto* q : {&m->mb3, &m->vb3, &m->gb3}) ok = ok && m->alloc(*q, O);
    const int64_t big = std::max(std::max(B * O, O * H), std::max(H * I, B * I));
    ok = ok && m->alloc(m->H1, B * H) && m->alloc(m->H2, B * H) && m->alloc(m->Out, B * O) &&
         m->alloc(m->dOut, B * O) && m->alloc(m->dOuth, B * O) && m->alloc(m->dH, B * H) &&
         m->alloc(m->dZ, B * H) && m->alloc(m->dZh, B * H) && m->alloc(m->T1, big) &&
         m->alloc(m->T2, big) && m->alloc(m->row_loss, B) && m->alloc(m->loss_dev, 1) &&
         m->alloc(m->err, 1);
    // Split-K partials: the largest split GEMMs are [B x H] with K = in or out.
    m->partial_elems = std::max<int64_t>(std::max(O * H, H * I), std::max(B * O, 160 * B * H));
    ok = ok && m->alloc(m->partial, m->partial_elems);
    if (!ok) {
        const std::string msg = m->msg;
        delete m;
        return fail("mlp: " + msg);
    }
    // He initialisation (normal, std sqrt(2/fan_in)), seeded.
    std::mt19937_64 rng(seed);
    auto init = [&](float* dst, int64_t rows, int64_t fan_in) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / static_cast<float>(fan_in)));
        std::vector<float> h(static_cast<size_t>(rows * fan_in));
        for (float& v : h) v = nd(rng);
        cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream);
        cudaStreamSynchronize(m->stream);
    };
    init(m->W1, H, I);
    init(m->W2, H, H);
    init(m->W3, O, H);
    m->refresh_bf16();
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) {
        delete m;
        return fail("mlp: initialisation failed");
    }
    *result = m;
    return 0;
}

void pdlpgpu_mlp_destroy(pdlpgpu_mlp* m) { delete m; }

int32_t pdlpgpu_mlp_forward(pdlpgpu_mlp* m, const uint16_t* inputs, float* outputs) {
    if (!m) return -1;
    cudaSetDevice(m->device);
    m->launches = 0;
    if (!m->wait_for_caller()) return fail("mlp forward: stream wait failed");
    if (!m->forward(reinterpret_cast<const bf16*>(inputs))) return fail("mlp forward: " + m->msg);
    if (cudaMemcpyAsync(outputs, m->Out, sizeof(float) * m->batch * m->out, cudaMemcpyDeviceToDevice,
                        m->stream) != cudaSuccess)
        return fail("mlp forward: copy failed");
    if (!m->check_err("mlp forward")) return fail(m->msg);
    return 0;
}

int32_t pdlpgpu_mlp_gradients(pdlpgpu_mlp* m, const uint16_t* inputs, const float* targets,
                              const float* w, float* dW1, float* db1, float* dW2, float* db2,
                              float* dW3, float* db3, float* loss) {
    if (!m) return -1;
    cudaSetDevice(m->device);
    m->launches = 0;
    if (!m->wait_for_caller()) return fail("mlp gradients: stream wait failed");
    const bf16* X = reinterpret_cast<const bf16*>(inputs);
    if (!m->forward(X) || !m->backward(X, targets, w)) return fail("mlp gradients: " + m->msg);
    const int64_t H = m->hidden, I = m->in, O = m->out;
    auto cp = [&](float* dst, const float* src, int64_t n) {
        if (dst) cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
    };
    cp(dW1, m->gW1, H * I); cp(db1, m->gb1, H); cp(dW2, m->gW2, H * H); cp(db2, m->gb2, H);
    cp(dW3, m->gW3, O * H); cp(db3, m->gb3, O);
    if (loss) cudaMemcpyAsync(loss, m->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (!m->check_err("mlp gradients")) return fail(m->msg);
    return 0;
}

int32_t pdlpgpu_mlp_train_step(pdlpgpu_mlp* m, const uint16_t* inputs, const float* targets,
                               const float* w, float lr, float* loss) {
    if (!m) return -1;
    cudaSetDevice(m->device);
    m->launches = 0;
    if (!m->wait_for_caller()) return fail("mlp train: stream wait failed");
    const bf16* X = reinterpret_cast<const bf16*>(inputs);
    if (!m->forward(X) || !m->backward(X, targets, w)) return fail("mlp train: " + m->msg);
    m->adam_all(lr);
    if (loss) cudaMemcpyAsync(loss, m->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (!m->check_err("mlp train")) return fail(m->msg);
    return 0;
}

int32_t pdlpgpu_mlp_get_params(pdlpgpu_mlp* m, float* W1, float* b1, float* W2, float* b2,
                               float* W3, float* b3) {
    if (!m) return -1;
    cudaSetDevice(m->device);
    if (!m->wait_for_caller()) return fail("mlp get_params: stream wait failed");
    const int64_t H = m->hidden, I = m->in, O = m->out;
    auto cp = [&](float* dst, const float* src, int64_t n) {
        if (dst) cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
    };
    cp(W1, m->W1, H * I); cp(b1, m->b1, H); cp(W2, m->W2, H * H); cp(b2, m->b2, H);
    cp(W3, m->W3, O * H); cp(b3, m->b3, O);
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? 0 : fail("mlp get_params failed");
}

int32_t pdlpgpu_mlp_set_params(pdlpgpu_mlp* m, const float* W1, const float* b1, const float* W2,
                               const float* b2, const float* W3, const float* b3) {
    if (!m) return -1;
    cudaSetDevice(m->device);
    if (!m->wait_for_caller()) return fail("mlp set_params: stream wait failed");
    const int64_t H = m->hidden, I = m->in, O = m->out;
    auto cp = [&](float* dst, const float* src, int64_t n) {
        if (src) cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
    };
    cp(m->W1, W1, H * I); cp(m->b1, b1, H); cp(m->W2, W2, H * H); cp(m->b2, b2, H);
    cp(m->W3, W3, O * H); cp(m->b3, b3, O);
    m->refresh_bf16();
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? 0 : fail("mlp set_params failed");
}

int64_t pdlpgpu_mlp_launches(pdlpgpu_mlp* m) { return m ? m->launches : 0; }

int32_t pdlpgpu_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                          float* C, int32_t splits) {
    int* err = nullptr;
    float* partial = nullptr;
    std::string msg;
    if (M <= 0 || N <= 0 || K <= 0) return fail("gemm: sizes must be positive");
    const int total_kb = (K + BK - 1) / BK;
    splits = std::max(1, std::min(splits, total_kb));
    const int per = (total_kb + splits - 1) / splits;
    const int s_eff = (total_kb + per - 1) / per;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return fail("gemm: cudaMalloc failed");
    cudaMemset(err, 0, sizeof(int));
    if (s_eff > 1 && cudaMalloc(&partial, sizeof(float) * static_cast<size_t>(s_eff) * M * N) != cudaSuccess) {
        cudaFree(err);
        return fail("gemm: cudaMalloc failed");
    }
    float* target = s_eff > 1 ? partial : C;
    bool ok = gemm(reinterpret_cast<const bf16*>(A), reinterpret_cast<const bf16*>(B), target, M, N, K,
                   s_eff, err, nullptr, msg);
    if (ok && s_eff > 1)
        epilogue<<<grid_for(static_cast<int64_t>(M) * N), 256>>>(partial, s_eff, static_cast<int64_t>(M) * N,
                                                                  M, N, nullptr, 0, C, nullptr);
    int h = 0;
    if (cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
    if (h != 0) {
        ok = false;
        msg = "tensor-core pipeline wait timed out (code " + std::to_string(h) + ")";
    }
    cudaFree(err);
    if (partial) cudaFree(partial);
    return ok ? 0 : fail("gemm: " + (msg.empty() ? std::string(cudaGetErrorString(cudaGetLastError())) : msg));
}


int32_t pdlpgpu_gemm_time(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                          float* C, int32_t splits, int32_t reps, double* ms_per_call) {
    if (M <= 0 || N <= 0 || K <= 0 || reps <= 0 || ms_per_call == nullptr)
        return fail("gemm_time: sizes and repetitions must be positive");
    const int total_kb = (K + BK - 1) / BK;
    splits = std::max(1, std::min(splits, total_kb));
    const int per = (total_kb + splits - 1) / splits;
    const int s_eff = (total_kb + per - 1) / per;
    int* err = nullptr;
    float* partial = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return fail("gemm_time: cudaMalloc failed");
    cudaMemset(err, 0, sizeof(int));
    if (s_eff > 1 && cudaMalloc(&partial, sizeof(float) * static_cast<size_t>(s_eff) * M * N) != cudaSuccess) {
        cudaFree(err);
        return fail("gemm_time: cudaMalloc failed");
    }
    float* target = s_eff > 1 ? partial : C;
    std::string msg;
    auto once = [&]() {
        bool ok = gemm(reinterpret_cast<const bf16*>(A), reinterpret_cast<const bf16*>(B), target, M, N, K,
                       s_eff, err, nullptr, msg);
        if (ok && s_eff > 1)
            epilogue<<<grid_for(static_cast<int64_t>(M) * N), 256>>>(partial, s_eff, static_cast<int64_t>(M) * N,
                                                                      M, N, nullptr, 0, C, nullptr);
        return ok;
    };
    bool ok = once();   // warm-up: tensor maps, instruction cache
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int r = 0; ok && r < reps; ++r) ok = once();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int h = 0;
    if (cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
    if (h != 0) {
        ok = false;
        msg = "tensor-core pipeline wait timed out (code " + std::to_string(h) + ")";
    }
    cudaFree(err);
    if (partial) cudaFree(partial);
    *ms_per_call = ms / reps;
    return ok ? 0 : fail("gemm_time: " + (msg.empty() ? std::string(cudaGetErrorString(cudaGetLastError())) : msg));
}

int32_t pdlpgpu_encode_features(const double* params, int32_t batch, int32_t count, int32_t padded,
                                const float* mean, const float* inv_std, uint16_t* out) {
    if (batch <= 0 || count <= 0 || padded < count) return fail("encode_features: bad sizes");
    encode_features<<<grid_for(static_cast<int64_t>(batch) * padded), 256>>>(
        params, batch, count, padded, mean, inv_std, reinterpret_cast<bf16*>(out));
    return cudaGetLastError() == cudaSuccess ? 0 : fail("encode_features: launch failed");
}

int32_t pdlpgpu_encode_targets(const double* primal, const double* dual, const double* weight,
                               int32_t batch, int32_t n, int32_t m, int32_t out_width,
                               const double* primal_scale, const float* dual_mean,
                               const float* dual_inv_std, float weight_mean, float weight_inv_std,
                               float* targets) {
    if (batch <= 0 || out_width < n + m + 1) return fail("encode_targets: bad sizes");
    encode_targets<<<grid_for(static_cast<int64_t>(batch) * out_width), 256>>>(
        primal, dual, weight, batch, n, m, out_width, primal_scale, dual_mean, dual_inv_std,
        weight_mean, weight_inv_std, targets);
    return cudaGetLastError() == cudaSuccess ? 0 : fail("encode_targets: launch failed");
}

int32_t pdlpgpu_decode_warmstart(const float* outputs, int32_t batch, int32_t n, int32_t m,
                                 int32_t out_width, const double* primal_scale,
                                 const float* dual_mean, const float* dual_std, float weight_mean,
                                 float weight_std, double* primal, double* dual, double* weight) {
    if (batch <= 0 || out_width < n + m + 1) return fail("decode_warmstart: bad sizes");
    decode_warmstart<<<grid_for(static_cast<int64_t>(batch) * (n + m + 1)), 256>>>(
        outputs, batch, n, m, out_width, primal_scale, dual_mean, dual_std, weight_mean, weight_std,
        primal, dual, weight);
    return cudaGetLastError() == cudaSuccess ? 0 : fail("decode_warmstart: launch failed");
}

}  // extern "C"

// noalloc.cu -- one fused PDHG trial that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a serving process that
// owns every byte of device memory through its own pool and a fixed budget,
// or a solve loop that must not take the device-wide synchronisation an
// allocation can cause. pdlpgpu_trial_noalloc serves them: the caller passes
// every input and output as device memory it already owns, and the only
// scratch the kernels need -- one partial sum per CTA -- lives in the
// file-scope array below, which the driver places in device memory when it
// loads this library (each GPU that loads it keeps those 192 KiB until the
// process exits). Nothing here calls cudaMalloc, cudaFree or an allocating
// library routine.
//
// The computation is pdlpgpu_trial's (the reference's CpuPdhgKernel::trial,
// pdlp_engine/src/pdhg_kernel.cpp:47-187) on plain CSR inputs: a warp per
// line, the primal half over the rows of A^T, the dual half over the rows
// of A, then one CTA adds the partial sums in a fixed order.
#include "pdlpgpu_components.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

extern "C" void pdlpgpu_internal_set_error(const char* message);

namespace {

constexpr int kNaThreads = 256;                     // 8 warps, one line per warp at a time
constexpr int kNaLinesPerCta = 1024;
constexpr int kNaMaxCtas = 8192;                    // per half
constexpr int64_t kNaMaxLines = int64_t(kNaLinesPerCta) * kNaMaxCtas;   // 8,388,608
constexpr unsigned kFull = 0xffffffffu;

// Slots [0, kNaMaxCtas): primal partials; then two per dual CTA.
static __device__ __align__(256) double g_noalloc_scratch[3 * kNaMaxCtas];

// Address of the array in each CUDA context it was looked up in. The key is
// the context's unique ID, not the device ordinal: after cudaDeviceReset, or
// under a caller's own driver context, the library's module is loaded again at
// another address, and a lookup made in an earlier context would be stale.
// Context IDs are never reused within a process, unlike context handles.
struct ScratchEntry {
    unsigned long long context_id;
    double* address;
};
std::mutex g_scratch_mutex;
std::vector<ScratchEntry> g_scratch_entries;
using CtxGetCurrent = int (*)(void**);                    // cuCtxGetCurrent(CUcontext*)
using CtxGetId = int (*)(void*, unsigned long long*);     // cuCtxGetId(CUcontext, id*)
CtxGetCurrent g_ctx_get_current = nullptr;
CtxGetId g_ctx_get_id = nullptr;

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

__device__ __forceinline__ double line_dot(const int64_t* start, const int32_t* index,
                                           const double* values, int64_t line, const double* v) {
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int64_t k = start[line] + lane; k < start[line + 1]; k += 32) acc += values[k] * v[index[k]];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    return acc;
}

__device__ __forceinline__ void cta_sum(double& a, double& b, double* out_a, double* out_b) {
    __shared__ double red[2][kNaThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int w = 0; w < kNaThreads / 32; ++w) {
            sa += red[0][w];
            sb += red[1][w];
        }
        *out_a = sa;
        if (out_b != nullptr) *out_b = sb;
    }
}

__global__ void __launch_bounds__(kNaThreads)
na_primal(int32_t cols, const int64_t* at_start, const int32_t* at_index, const double* at_values,
          const double* c, const double* xl, const double* xu, const double* tau,
          const double* itau, const double* x, const double* y, double mult, double* x_out,
          double* scratch) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t first = int64_t(blockIdx.x) * kNaLinesPerCta;
    const int64_t last = first + kNaLinesPerCta < cols ? first + kNaLinesPerCta : cols;
    double moved = 0.0;
    for (int64_t j = first + warp; j < last; j += kNaThreads / 32) {
        const double g = c[j] + line_dot(at_start, at_index, at_values, j, y);
        if (lane == 0) {
            const double prev = x[j];
            const double upd = dmax(xl[j], dmin(prev - mult * tau[j] * g, xu[j]));
            x_out[j] = upd;
            const double d = upd - prev;
            moved += d * d * itau[j];
        }
    }
    double unused = 0.0;
    cta_sum(moved, unused, scratch + blockIdx.x, nullptr);
}

__global__ void __launch_bounds__(kNaThreads)
na_dual(int32_t rows, const int64_t* a_start, const int32_t* a_index, const double* a_values,
        const double* rl, const double* ru, const double* sigma, const double* isigma,
        const double* y, const double* ax, const double* x_out, double dmult, double* y_out,
        double* ax_out, double* scratch) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t first = int64_t(blockIdx.x) * kNaLinesPerCta;
    const int64_t last = first + kNaLinesPerCta < rows ? first + kNaLinesPerCta : rows;
    double moved = 0.0, inter = 0.0;
    for (int64_t i = first + warp; i < last; i += kNaThreads / 32) {
        const double next = line_dot(a_start, a_index, a_values, i, x_out);
        if (lane == 0) {
            const double dact = next - ax[i];
            const double ext = next + dact;
            const double step = dmax(dmult * sigma[i], 1e-300);
            const double prev = y[i];
            const double v = prev + step * ext;
            const double upd = dmax(v - step * ru[i], 0.0) + dmin(v - step * rl[i], 0.0);
            y_out[i] = upd;
            ax_out[i] = next;
            const double d = upd - prev;
            moved += d * d * isigma[i];
            inter += d * dact;
        }
    }
    double* base = scratch + kNaMaxCtas + 2 * blockIdx.x;
    cta_sum(moved, inter, base, base + 1);
}

// Adds the partials this call wrote, in CTA order.
__global__ void na_reduce(int primal_ctas, int dual_ctas, const double* scratch, double* out) {
    if (threadIdx.x != 0) return;
    double p = 0.0, d = 0.0, it = 0.0;
    for (int k = 0; k < primal_ctas; ++k) p += scratch[k];
    for (int k = 0; k < dual_ctas; ++k) {
        d += scratch[kNaMaxCtas + 2 * k];
        it += scratch[kNaMaxCtas + 2 * k + 1];
    }
    out[0] = p;
    out[1] = d;
    out[2] = it;
}

bool driver_entry(const char* name, void** fn, std::string& error) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || *fn == nullptr) {
        error = std::string(name) + " unavailable";
        return false;
    }
    return true;
}

// Device address of the scratch array in the current context. The first call
// in each context does the lookup (with that context current); later calls
// reuse it.
double* scratch_in_current_context(std::string& error) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_ctx_get_current == nullptr || g_ctx_get_id == nullptr) {
        void* current = nullptr;
        void* id = nullptr;
        if (!driver_entry("cuCtxGetCurrent", &current, error) ||
            !driver_entry("cuCtxGetId", &id, error))
            return nullptr;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrent>(current);
        g_ctx_get_id = reinterpret_cast<CtxGetId>(id);
    }
    void* context = nullptr;
    double* fresh = nullptr;
    if (g_ctx_get_current(&context) != 0) {
        error = "cuCtxGetCurrent failed";
        return nullptr;
    }
    if (context == nullptr) {
        // No context is current yet: the runtime makes the device's primary
        // context current while it resolves the symbol.
        const cudaError_t rc = cudaGetSymbolAddress(reinterpret_cast<void**>(&fresh), g_noalloc_scratch);
        if (rc != cudaSuccess) {
            error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc);
            return nullptr;
        }
        if (g_ctx_get_current(&context) != 0 || context == nullptr) {
            error = "no current CUDA context";
            return nullptr;
        }
    }
    unsigned long long id = 0;
    if (g_ctx_get_id(context, &id) != 0) {
        error = "cuCtxGetId failed";
        return nullptr;
    }
    for (const ScratchEntry& e : g_scratch_entries)
        if (e.context_id == id) return e.address;
    if (fresh == nullptr) {
        const cudaError_t rc = cudaGetSymbolAddress(reinterpret_cast<void**>(&fresh), g_noalloc_scratch);
        if (rc != cudaSuccess) {
            error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc);
            return nullptr;
        }
    }
    g_scratch_entries.push_back({id, fresh});
    return fresh;
}

int fail(const std::string& message) {
    pdlpgpu_internal_set_error(message.c_str());
    return -1;
}

}  // namespace

extern "C" int32_t pdlpgpu_trial_noalloc(
    int32_t rows, int32_t cols, const int64_t* a_row_start, const int32_t* a_col_index,
    const double* a_values, const int64_t* at_row_start, const int32_t* at_col_index,
    const double* at_values, const double* objective, const double* var_lower,
    const double* var_upper, const double* tau, const double* tau_inverse,
    const double* row_lower, const double* row_upper, const double* sigma,
    const double* sigma_inverse, const double* x, const double* y, const double* ax,
    double step, double weight, double* x_out, double* y_out, double* ax_out,
    double* reductions, void* stream) {
    if (rows < 0 || cols < 0) return fail("pdlpgpu_trial_noalloc: negative dimensions");
    if (rows > kNaMaxLines || cols > kNaMaxLines)
        return fail("pdlpgpu_trial_noalloc: at most 8388608 rows and 8388608 columns "
                    "(the static scratch holds 8192 partial sums per half)");
    if (!(weight > 0.0)) return fail("pdlpgpu_trial_noalloc: weight must be positive");
    // Every pointer a launch would dereference must be given: NULL is refused
    // here, before anything is enqueued, instead of faulting on the device.
    if (reductions == nullptr) return fail("pdlpgpu_trial_noalloc: reductions is NULL");
    if (cols > 0) {
        const void* column_side[] = {at_row_start, at_col_index, at_values, objective, var_lower,
                                     var_upper, tau, tau_inverse, x, x_out};
        for (const void* p : column_side)
            if (p == nullptr)
                return fail("pdlpgpu_trial_noalloc: a column-side pointer (A^T, objective, "
                            "variable bounds, tau, x, x_out) is NULL with cols > 0");
    }
    if (rows > 0) {
        const void* row_side[] = {a_row_start, a_col_index, a_values, row_lower, row_upper,
                                  sigma, sigma_inverse, y, ax, y_out, ax_out};
        for (const void* p : row_side)
            if (p == nullptr)
                return fail("pdlpgpu_trial_noalloc: a row-side pointer (A, row bounds, sigma, "
                            "y, ax, y_out, ax_out) is NULL with rows > 0");
    }
    std::string error;
    double* scratch = scratch_in_current_context(error);
    if (scratch == nullptr) return fail("pdlpgpu_trial_noalloc: " + error);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int pc = static_cast<int>((int64_t(cols) + kNaLinesPerCta - 1) / kNaLinesPerCta);
    const int dc = static_cast<int>((int64_t(rows) + kNaLinesPerCta - 1) / kNaLinesPerCta);
    if (pc > 0)
        na_primal<<<pc, kNaThreads, 0, s>>>(cols, at_row_start, at_col_index, at_values, objective,
                                            var_lower, var_upper, tau, tau_inverse, x, y,
                                            step / weight, x_out, scratch);
    if (dc > 0)
        na_dual<<<dc, kNaThreads, 0, s>>>(rows, a_row_start, a_col_index, a_values, row_lower,
                                          row_upper, sigma, sigma_inverse, y, ax, x_out,
                                          step * weight, y_out, ax_out, scratch);
    na_reduce<<<1, 32, 0, s>>>(pc, dc, scratch, reductions);
    const cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess) return fail(std::string("pdlpgpu_trial_noalloc: ") + cudaGetErrorString(rc));
    return 0;
}

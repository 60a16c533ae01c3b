// ndg.cu -- pdlpgpu_normalized_gap: the normalised duality gap of one
// primal-dual point (ndg.cuh), computed on the device by the CTA-wide routine
// the check stage uses, from vectors the caller gives. A component call for
// testing and diagnostics: it allocates, uploads, runs one CTA and downloads.
#include "ndg.cuh"
#include "pdlpgpu_components.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

extern "C" void pdlpgpu_internal_set_error(const char* message);

namespace {

// Coordinates straight from the given arrays: [0, n) primal, [n, n + m) dual.
struct ArrayCoord {
    const double* v;
    const double* d;
    const double* lo;
    const double* hi;
    const double* r;
    __device__ pdlpgpu::NdgCoord operator()(int64_t k) const {
        return pdlpgpu::NdgCoord{v[k], d[k], lo[k], hi[k], r[k]};
    }
};

__global__ void __launch_bounds__(256) k_normalized_gap(int64_t n, int64_t m, double w, ArrayCoord q,
                                                        double* out) {
    __shared__ double scratch[16 * 32];
    double radius = 0.0;
    const double gap = pdlpgpu::block_normalized_gap(n, m, w, q, scratch, &radius);
    if (threadIdx.x == 0) {
        out[0] = gap;
        out[1] = radius;
    }
}

}  // namespace

extern "C" int32_t pdlpgpu_normalized_gap(int32_t n, int32_t m, double weight, const double* x,
                                          const double* g, const double* x_lower, const double* x_upper,
                                          const double* x_ref, const double* y, const double* a,
                                          const double* r_lower, const double* r_upper,
                                          const double* y_ref, double* out) {
    if (n < 0 || m < 0 || out == nullptr || !(weight > 0.0) ||
        (n > 0 && (!x || !g || !x_lower || !x_upper || !x_ref)) ||
        (m > 0 && (!y || !a || !r_lower || !r_upper || !y_ref))) {
        pdlpgpu_internal_set_error("normalized_gap: invalid arguments");
        return -1;
    }
    const size_t total = static_cast<size_t>(n) + static_cast<size_t>(m);
    // Five concatenated arrays of n + m values, then the two outputs.
    std::vector<double> host(5 * total + 2, 0.0);
    const double* prim[5] = {x, g, x_lower, x_upper, x_ref};
    const double* dual[5] = {y, a, r_lower, r_upper, y_ref};
    for (int k = 0; k < 5; ++k) {
        for (int32_t j = 0; j < n; ++j) host[k * total + j] = prim[k][j];
        for (int32_t i = 0; i < m; ++i) host[k * total + n + i] = dual[k][i];
    }
    double* dev = nullptr;
    auto fail = [&](cudaError_t e) {
        pdlpgpu_internal_set_error((std::string("normalized_gap: ") + cudaGetErrorString(e)).c_str());
        if (dev) cudaFree(dev);
        return -1;
    };
    cudaError_t e = cudaMalloc(&dev, host.size() * sizeof(double));
    if (e != cudaSuccess) return fail(e);
    e = cudaMemcpy(dev, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(e);
    const ArrayCoord q{dev, dev + total, dev + 2 * total, dev + 3 * total, dev + 4 * total};
    k_normalized_gap<<<1, 256>>>(n, m, weight, q, dev + 5 * total);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(e);
    e = cudaMemcpy(out, dev + 5 * total, 2 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(e);
    cudaFree(dev);
    return 0;
}

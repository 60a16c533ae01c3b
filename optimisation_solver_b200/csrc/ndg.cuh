// ndg.cuh -- the normalised duality gap of a primal-dual point, computed by
// one CTA (the restart metric the reference names as its main outstanding
// item, pdlp_engine/README.md:226-233; the definition and the bisection are
// those of Applegate et al., "Practical large-scale linear programming using
// primal-dual hybrid gradient", NeurIPS 2021, section 3 and appendix).
//
// The saddle function of the PDHG iteration is
//     L(x, y) = c'x + y'Ax - h*(y),  x in X = [l_x, u_x],
// h* the support function of the row bounds [l_r, u_r] (finite on the dual
// domain Y: y_i <= 0 where u_i is infinite, y_i >= 0 where l_i is). With the
// weighted norm ||(dx, dy)||_w^2 = w ||dx||^2 + ||dy||^2 / w (w the primal
// weight) the normalised gap of z = (x, y) at radius r is
//     rho(r; z) = (1/r) max { L(x, yh) - L(xh, y) : zh in X x Y, ||zh - z||_w <= r }.
// With g = c + A'y and a = Ax the objective is
//     sum_j -g_j (xh_j - x_j) + sum_i [(yh_i - y_i) a_i - h*_i(yh_i) + h*_i(y_i)],
// separable and concave. For a multiplier lam > 0 of the ball constraint each
// coordinate's maximiser has a closed form (a clipped step for x, the branch
// of the kink at 0 for y), and the distance it reaches, dist(lam), does not
// increase with lam. The gap is the objective at the lam with dist(lam) = r,
// found by bracketing in log(lam); when the whole box lies inside the ball
// (dist stays below r as lam -> 0) it is the box maximum over r.
#pragma once

#include <cmath>
#include <cstdint>

namespace pdlpgpu {

// One coordinate of the candidate: value v (x_j or y_i), gradient d (g_j or
// a_i), bounds [lo, hi] (variable bounds or row bounds) and its restart
// point's value r.
struct NdgCoord {
    double v, d, lo, hi, r;
};

// Primal coordinate: step from v at multiplier lam (lam <= 0: the box limit);
// `inv` = 1 / (lam w), computed once per multiplier.
__device__ __forceinline__ double ndg_primal_step(const NdgCoord& q, double lam, double inv) {
    double s;
    if (lam > 0.0) {
        s = -q.d * inv;
    } else {
        s = q.d < 0.0 ? INFINITY : (q.d > 0.0 ? -INFINITY : 0.0);
    }
    const double lo = q.lo - q.v, hi = q.hi - q.v;
    return s < lo ? lo : (s > hi ? hi : s);
}

// Support function of [lo, hi] at v on the dual domain (0 at v = 0).
__device__ __forceinline__ double ndg_support(double v, double lo, double hi) {
    return v > 0.0 ? hi * v : (v < 0.0 ? lo * v : 0.0);
}

// Dual coordinate: maximiser of (yh - v) d - h*(yh) - lam / (2 w) (yh - v)^2;
// `wl` = w / lam.
__device__ __forceinline__ double ndg_dual_point(const NdgCoord& q, double lam, double wl) {
    const bool hi_f = isfinite(q.hi), lo_f = isfinite(q.lo);
    if (lam > 0.0) {
        const double up = q.v + wl * (q.d - q.hi);
        const double dn = q.v + wl * (q.d - q.lo);
        if (hi_f && up > 0.0) return up;
        if (lo_f && dn < 0.0) return dn;
        return 0.0;
    }
    // lam -> 0: the ray along the steeper ascent side, when it is unbounded.
    if (hi_f && q.d - q.hi > 0.0) return INFINITY;
    if (lo_f && q.d - q.lo < 0.0) return -INFINITY;
    return 0.0;
}

// Sum over the CTA of K values per thread, returned in every thread (fixed
// order: warps by shuffles, then warps in index order).
template <int K>
__device__ __forceinline__ void ndg_block_sum(double (&v)[K], double* scratch /* [K][32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k * 32 + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double t = 0.0;
        for (int q = 0; q < warps; ++q) t += scratch[k * 32 + q];
        v[k] = t;
    }
}

// The normalised gap rho(r; z) of the candidate whose n primal and m dual
// coordinates `coord(k)` returns (k < n primal, else dual), with r the
// candidate's distance to its restart point. Every thread of the CTA calls
// it with the same arguments and gets the value; `scratch` holds 16 x 32
// doubles of shared memory. +inf when r is zero or not finite.
template <class Coord>
__device__ double block_normalized_gap(int64_t n, int64_t m, double w, Coord coord, double* scratch,
                                       double* radius_out) {
    constexpr int K = 16;        // multipliers per pass
    constexpr int kPasses = 4;   // bracket narrowed K + 1 times per pass
    const int64_t total = n + m;
    // Pass 1: the radius, the distance at lam = 1 (clipped) and without the
    // box (unclipped, an upper bound of dist(lam) * lam).
    double s3[3] = {0.0, 0.0, 0.0};
    const double iw = 1.0 / w;
    for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
        const NdgCoord q = coord(k);
        if (k < n) {
            const double e = q.v - q.r;
            s3[0] += w * e * e;
            const double st = ndg_primal_step(q, 1.0, iw);
            s3[1] += w * st * st;
            s3[2] += q.d * q.d * iw;
        } else {
            const double e = q.v - q.r;
            s3[0] += e * e * iw;
            const double st = ndg_dual_point(q, 1.0, w) - q.v;
            s3[1] += st * st * iw;
            const double up = isfinite(q.hi) ? w * (q.d - q.hi) : 0.0;
            const double dn = isfinite(q.lo) ? w * (q.d - q.lo) : 0.0;
            const double u = fabs(up) > fabs(dn) ? up : dn;
            s3[2] += u * u * iw;
        }
    }
    {
        double v3[K];
#pragma unroll
        for (int k = 0; k < K; ++k) v3[k] = k < 3 ? s3[k] : 0.0;
        ndg_block_sum<K>(v3, scratch);
        s3[0] = v3[0];
        s3[1] = v3[1];
        s3[2] = v3[2];
    }
    const double r = sqrt(s3[0]);
    if (radius_out) *radius_out = r;
    if (!(r > 0.0) || !isfinite(r)) return INFINITY;
    const double d1 = sqrt(s3[1]), u1 = sqrt(s3[2]);
    // dist(lam) >= d1 / lam for lam >= 1 and <= d1 / lam for lam <= 1, and
    // dist(lam) <= u1 / lam always.
    double lo, hi;
    if (d1 >= r) {
        lo = d1 / r;
        hi = fmax(u1 / r, lo);
    } else {
        hi = d1 / r;
        lo = hi * 1e-12;
    }
    double lam = hi;
    if (hi > 0.0 && lo > 0.0) {
        // Is the box inside the ball? Then the gap is the box maximum.
        bool inside = false;
        if (d1 < r) {
            double v1[K];
#pragma unroll
            for (int k = 0; k < K; ++k) v1[k] = 0.0;
            const double inv = 1.0 / (lo * w), wl = w / lo;
            for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
                const NdgCoord q = coord(k);
                double st;
                if (k < n) {
                    st = ndg_primal_step(q, lo, inv);
                    v1[0] += w * st * st;
                } else {
                    st = ndg_dual_point(q, lo, wl) - q.v;
                    v1[0] += st * st * iw;
                }
            }
            ndg_block_sum<K>(v1, scratch);
            inside = !(v1[0] >= r * r);
        }
        if (inside) {
            lam = 0.0;
        } else {
            for (int pass = 0; pass < kPasses && hi > lo * (1.0 + 1e-12); ++pass) {
                const double ratio = log(hi / lo);
                // Per multiplier: lam, 1 / (lam w) and w / lam (no division in
                // the coordinate loop).
                __shared__ double lks[3][K];
                if (threadIdx.x < K) {
                    const double l = lo * exp(ratio * static_cast<double>(threadIdx.x + 1) /
                                              static_cast<double>(K + 1));
                    lks[0][threadIdx.x] = l;
                    lks[1][threadIdx.x] = 1.0 / (l * w);
                    lks[2][threadIdx.x] = w / l;
                }
                __syncthreads();
                double lk[K], v[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    lk[k] = lks[0][k];
                    v[k] = 0.0;
                }
                for (int64_t j = threadIdx.x; j < total; j += blockDim.x) {
                    const NdgCoord q = coord(j);
                    if (j < n) {
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const double st = ndg_primal_step(q, lk[k], lks[1][k]);
                            v[k] += w * st * st;
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const double st = ndg_dual_point(q, lk[k], lks[2][k]) - q.v;
                            v[k] += st * st * iw;
                        }
                    }
                }
                ndg_block_sum<K>(v, scratch);
                // dist is non-increasing in lam: the first multiplier that
                // reaches the ball closes the new bracket.
                double nlo = lo, nhi = hi;
                for (int k = 0; k < K; ++k) {
                    if (v[k] <= r * r) {
                        nhi = lk[k];
                        break;
                    }
                    nlo = lk[k];
                }
                lo = nlo;
                hi = nhi;
            }
            lam = hi;
        }
    }
    // The objective at the point of multiplier lam (inside the ball).
    double ov[K];
#pragma unroll
    for (int k = 0; k < K; ++k) ov[k] = 0.0;
    const double inv = lam > 0.0 ? 1.0 / (lam * w) : 0.0, wl = lam > 0.0 ? w / lam : 0.0;
    for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
        const NdgCoord q = coord(k);
        if (k < n) {
            const double st = ndg_primal_step(q, lam, inv);
            if (st != 0.0) ov[0] += -q.d * st;
        } else {
            const double yh = ndg_dual_point(q, lam, wl);
            ov[0] += (yh - q.v) * q.d - ndg_support(yh, q.lo, q.hi) + ndg_support(q.v, q.lo, q.hi);
        }
    }
    ndg_block_sum<K>(ov, scratch);
    return ov[0] / r;
}

}  // namespace pdlpgpu

// Hessian products for QP.
//  * CSR Q (the reference's full-storage form, lp.hpp:43-45): the row-block
//    SpMV of gb_spmv.cuh, one or two right-hand sides (x and the average).
//  * Diagonal-plus-low-rank Q = 2 (F F^T + diag D), F n x k row-major:
//      t = F^T x     (k_ftx_partial + k_ftx_final: fixed-order FP64 reduction)
//      qx_j = 2 (F_j . t + D_j x_j)   (k_dplr_expand: one warp per row)
//    which reads F twice per product instead of the n^2 dense Q.
#pragma once
#include "gb_pdhg.cuh"

namespace gb {

constexpr int kMaxRank = 128;
constexpr int kFtxGrid = 296;  // 2 CTAs per SM, fixed for a fixed summation order

template <class V>
struct Store2Epi {
    V* __restrict__ y0;
    V* __restrict__ y1;
    __device__ __forceinline__ bool begin(int) const { return true; }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int r, const V (&s)[2], const NoPre&) {
        y0[r] = s[0];
        y1[r] = s[1];
    }
};
// qx = Q x, qxa = Q xa (xa = inv * sumx)
template <class M, class V>
__global__ void __launch_bounds__(kThreads) k_spmv_q2(const __grid_constant__ CsrView<M> Q, const V* __restrict__ x,
                                                     const V* __restrict__ sumx, const SolveState* st,
                                                     V* __restrict__ qx, V* __restrict__ qxa) {
    extern __shared__ __align__(16) unsigned char smem[];
    const double inv = 1.0 / static_cast<double>(st->it_since + st->check_every);
    Store2Epi<V> epi{qx, qxa};
    spmv_run<2, M, V>(Q, blockIdx.x, GatherXAvg<V, 2>{x, sumx, nullptr, inv}, epi, smem);
}

// Partial F^T v for NV vectors: v0 = x, v1 = inv * sumx (when NV == 2).
template <class V, int NV>
__global__ void __launch_bounds__(kThreads) k_ftx_partial(int n, int k, const V* __restrict__ F,
                                                         const V* __restrict__ x, const V* __restrict__ sumx,
                                                         const SolveState* st, double* __restrict__ part) {
    __shared__ double sh[kWarps][NV * kMaxRank];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double inv = 0.0;
    if constexpr (NV > 1) inv = 1.0 / static_cast<double>(st->it_since + st->check_every);
    double acc[NV][kMaxRank / 32];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < kMaxRank / 32; ++q) acc[v][q] = 0.0;
    const int rows_per = div_up_dev(n, gridDim.x);
    const int r0 = blockIdx.x * rows_per, r1 = min(n, r0 + rows_per);
    for (int j = r0 + wid; j < r1; j += kWarps) {
        double xv[NV];
        xv[0] = double(x[j]);
        if (NV > 1) xv[NV > 1 ? 1 : 0] = double(avg_of(sumx, j, inv));
        const V* Fj = F + static_cast<size_t>(j) * k;
#pragma unroll
        for (int q = 0; q < kMaxRank / 32; ++q) {
            const int kk = lane + 32 * q;
            if (kk < k) {
                const double f = double(Fj[kk]);
#pragma unroll
                for (int v = 0; v < NV; ++v) acc[v][q] += f * xv[v];
            }
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int q = 0; q < kMaxRank / 32; ++q) {
            const int kk = lane + 32 * q;
            if (kk < k) sh[wid][v * kMaxRank + kk] = acc[v][q];
        }
    __syncthreads();
    for (int e = threadIdx.x; e < NV * k; e += kThreads) {
        const int v = e / k, kk = e % k;
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sh[w][v * kMaxRank + kk];
        part[static_cast<size_t>(blockIdx.x) * NV * k + e] = s;
    }
}

static __global__ void k_ftx_final(int np, int width, const double* __restrict__ part, double* __restrict__ t) {
    for (int e = threadIdx.x; e < width; e += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < np; ++b) s += part[static_cast<size_t>(b) * width + e];
        t[e] = s;
    }
}

// qx_j = 2 (F_j . t + D_j x_j); NV == 2 also writes qxa from t[k..2k) and xa.
template <class V, int NV>
__global__ void __launch_bounds__(kThreads) k_dplr_expand(int n, int k, const V* __restrict__ F,
                                                         const V* __restrict__ D, const double* __restrict__ t,
                                                         const V* __restrict__ x, const V* __restrict__ sumx,
                                                         const SolveState* st, V* __restrict__ qx,
                                                         V* __restrict__ qxa) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    double inv = 0.0;
    if constexpr (NV > 1) inv = 1.0 / static_cast<double>(st->it_since + st->check_every);
    for (int j = warp; j < n; j += nw) {
        const V* Fj = F + static_cast<size_t>(j) * k;
        double s[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = 0.0;
        for (int kk = lane; kk < k; kk += 32) {
            const double f = double(Fj[kk]);
#pragma unroll
            for (int v = 0; v < NV; ++v) s[v] += f * t[v * k + kk];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = warp_sum(s[v]);
        if (lane == 0) {
            const double d = double(D[j]);
            qx[j] = static_cast<V>(2.0 * (s[0] + d * double(x[j])));
            if (NV > 1) qxa[j] = static_cast<V>(2.0 * (s[NV > 1 ? 1 : 0] + d * double(avg_of(sumx, j, inv))));
        }
    }
}

}  // namespace gb

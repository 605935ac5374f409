// Hessian products for QP.
//  * CSR Q (the reference's full-storage form, lp.hpp:43-45): the row-block
//    SpMV of gb_spmv.cuh, one or two right-hand sides (x and the average).
//  * Diagonal-plus-low-rank Q = 2 (F F^T + diag D), F n x k row-major:
//      t = F^T x     (k_ftx_partial + k_ftx_final: fixed-order FP64 reduction)
//      qx_j = 2 (F_j . t + D_j x_j)   (k_dplr_expand: rows staged per warp)
//    which reads F twice per product instead of the n^2 dense Q.
#pragma once
#include "gb_pdhg.cuh"

namespace gb {

constexpr int kMaxRank = 128;
constexpr int kFtxGrid = 592;  // fixed (not the SM count), so the summation order is fixed

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

// Partial F^T v for NV vectors (v0 = x, v1 = inv * sumx when NV == 2) over a
// contiguous slice of rows per CTA.  The CTA's threads form G = kThreads / k
// groups of k: thread (g, c) takes column c of rows r0 + g, r0 + g + G, ...,
// so consecutive threads read consecutive entries of F (coalesced); the G
// group sums are then added in group order.  Output is term-major,
// part[e * gridDim.x + blockIdx.x] for e = v * k + c.
template <class V, int NV>
__global__ void __launch_bounds__(kThreads) k_ftx_partial(int n, int k, const V* __restrict__ F,
                                                         const V* __restrict__ x, const V* __restrict__ sumx,
                                                         const SolveState* st, double* __restrict__ part) {
    __shared__ double sh[NV][kThreads];
    pdl_enter();
    double inv = 0.0;
    if constexpr (NV > 1) inv = 1.0 / static_cast<double>(st->it_since + st->check_every);
    const int G = kThreads / k;  // k <= kMaxRank, so G >= 2
    const int g = threadIdx.x / k, c = threadIdx.x - g * k;
    const int rows_per = div_up_dev(n, gridDim.x);
    const int r0 = blockIdx.x * rows_per, r1 = min(n, r0 + rows_per);
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    if (g < G) {
        for (int r = r0 + g; r < r1; r += G) {
            const double f = double(F[static_cast<size_t>(r) * k + c]);
            acc[0] += f * double(x[r]);
            if constexpr (NV > 1) acc[1] += f * double(avg_of(sumx, r, inv));
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) sh[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int e = threadIdx.x; e < NV * k; e += kThreads) {
        const int v = e / k, cc = e - v * k;
        double t = 0.0;
        for (int gg = 0; gg < G; ++gg) t += sh[v][gg * k + cc];
        part[static_cast<size_t>(e) * gridDim.x + blockIdx.x] = t;
    }
}

// t[e] = sum over the np partials of entry e: one warp per entry, lanes over
// the partials (coalesced, term-major), then a fixed-order shuffle sum.
static __global__ void k_ftx_final(int np, const double* __restrict__ part, double* __restrict__ t) {
    pdl_enter();
    const int e = blockIdx.x, lane = threadIdx.x;
    const double* p = part + static_cast<size_t>(e) * np;
    double s = 0.0;
    for (int b = lane; b < np; b += 32) s += p[b];
    s = warp_sum(s);
    if (lane == 0) t[e] = s;
}

// qx_j = 2 (F_j . t + D_j x_j); NV == 2 also writes qxa from t[k..2k) and xa.
// Each warp stages kExpandRows consecutive rows of F (one contiguous range)
// in shared memory with coalesced loads, then each lane forms one row's dot
// product in column order.
constexpr int kExpandRows = 32;
constexpr int kExpandWarps = 4;
template <class V, int NV>
constexpr size_t expand_smem_bytes(int k) {
    return sizeof(double) * NV * kMaxRank + sizeof(V) * static_cast<size_t>(kExpandWarps) * kExpandRows * k;
}
inline int expand_grid(int n) { return div_up(div_up(n, kExpandRows), kExpandWarps); }

template <class V, int NV>
__global__ void __launch_bounds__(kExpandWarps * 32) k_dplr_expand(int n, int k, const V* __restrict__ F,
                                                                  const V* __restrict__ D,
                                                                  const double* __restrict__ t,
                                                                  const V* __restrict__ x,
                                                                  const V* __restrict__ sumx, const SolveState* st,
                                                                  V* __restrict__ qx, V* __restrict__ qxa) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* ts = reinterpret_cast<double*>(smem);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    V* fs = reinterpret_cast<V*>(smem + sizeof(double) * NV * kMaxRank) + static_cast<size_t>(wid) * kExpandRows * k;
    pdl_enter();
    for (int e = threadIdx.x; e < NV * k; e += blockDim.x) ts[e] = t[e];
    __syncthreads();
    double inv = 0.0;
    if constexpr (NV > 1) inv = 1.0 / static_cast<double>(st->it_since + st->check_every);
    const int nw = gridDim.x * kExpandWarps;
    for (int r0 = (blockIdx.x * kExpandWarps + wid) * kExpandRows; r0 < n; r0 += nw * kExpandRows) {
        const int rows = min(kExpandRows, n - r0);
        const V* src = F + static_cast<size_t>(r0) * k;
        for (int e = lane; e < rows * k; e += 32) fs[e] = src[e];
        __syncwarp();
        if (lane < rows) {
            const V* fr = fs + lane * k;
            double s0 = 0.0, s1 = 0.0;
            for (int c = 0; c < k; ++c) {
                const double f = double(fr[c]);
                s0 += f * ts[c];
                if constexpr (NV > 1) s1 += f * ts[k + c];
            }
            const int j = r0 + lane;
            const double d = double(D[j]);
            qx[j] = static_cast<V>(2.0 * (s0 + d * double(x[j])));
            if constexpr (NV > 1) qxa[j] = static_cast<V>(2.0 * (s1 + d * double(avg_of(sumx, j, inv))));
        }
        __syncwarp();
    }
}

}  // namespace gb

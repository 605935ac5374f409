// Device-side problem setup: stored transpose, Ruiz + Pock-Chambolle
// scaling, bound/objective rescaling, ||A'|| and ||Q'|| power iterations.
// Restates src/scaling.cpp:8-155 and src/lp.cpp:55-72 as GPU kernels so that
// a problem never round-trips through host memory after its upload.
#pragma once
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "gb_spmv.cuh"

namespace gb {

// ---------------------------------------------------------------- deterministic reductions
constexpr int kRedGrid = 592;  // 4 CTAs per SM, fixed so the summation order is fixed

// Pass 1: each CTA folds a grid-stride slice; pass 2 folds the partials.
template <class F>
__global__ void __launch_bounds__(kThreads) k_red1(long long n, F f, double* partials) {
    __shared__ double sh[kWarps];
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads)
        acc += f(i);
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}
// out = post(sum of partials)
template <class P>
__global__ void __launch_bounds__(kThreads) k_red2(int np, const double* partials, double* out, P post) {
    __shared__ double sh[kWarps];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kThreads) acc += partials[i];
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) post(v[0], out);
}
struct PostSqrt {
    __device__ void operator()(double s, double* out) const { *out = sqrt(s); }
};
struct PostSqrtPlus1 {
    __device__ void operator()(double s, double* out) const { *out = sqrt(s) + 1.0; }
};
struct PostIdent {
    __device__ void operator()(double s, double* out) const { *out = s; }
};

struct Sq {
    const double* v;
    __device__ double operator()(long long i) const { return v[i] * v[i]; }
};
struct FiniteBoundSq {  // scaling.cpp:15-24
    const double* lo;
    const double* hi;
    __device__ double operator()(long long i) const {
        const double a = isfinite(lo[i]) ? fabs(lo[i]) : 0.0;
        const double b = isfinite(hi[i]) ? fabs(hi[i]) : 0.0;
        const double v = (a < b) ? b : a;
        return v * v;
    }
};

template <class F, class P>
inline void reduce_to(cudaStream_t s, long long n, F f, double* partials, double* out, P post) {
    k_red1<F><<<kRedGrid, kThreads, 0, s>>>(n, f, partials);
    k_red2<P><<<1, kThreads, 0, s>>>(kRedGrid, partials, out, post);
}

// ---------------------------------------------------------------- plain SpMV (y = A x)
template <class V>
struct StoreEpi {
    V* __restrict__ y;
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int r, const V (&s)[1], const NoPre&) { y[r] = s[0]; }
};
template <class M, class V>
__global__ void __launch_bounds__(kThreads) k_spmv(const __grid_constant__ CsrView<M> A, const V* __restrict__ x,
                                                  V* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem[];
    StoreEpi<V> epi{y};
    spmv_run<1, M, V>(A, blockIdx.x, GatherOne<V>{x}, epi, smem);
}

// ---------------------------------------------------------------- transpose / scaling kernels
static __global__ void k_row_of(int rows, const int* __restrict__ ptr, int* __restrict__ row_of) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < rows; r += nw)
        for (int p = ptr[r] + lane; p < ptr[r + 1]; p += 32) row_of[p] = r;
}
static __global__ void k_iota(int n, int* v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}
static __global__ void k_count_cols(int nnz, const int* __restrict__ idx, int* __restrict__ cnt) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
        atomicAdd(cnt + idx[p], 1);
}
static __global__ void k_gather_transpose(int nnz, const int* __restrict__ perm, const int* __restrict__ row_of,
                                   const double* __restrict__ val, int* __restrict__ at_idx,
                                   double* __restrict__ at_val) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += gridDim.x * blockDim.x) {
        const int p = perm[q];
        at_idx[q] = row_of[p];
        if (at_val) at_val[q] = val[p];
    }
}

// Per-row max |a| (mode 0) or sum |a| (mode 1) of a CSR matrix whose value of
// entry q is val[perm ? perm[q] : q]; then the factor 1/sqrt (scaling.cpp:56-57).
static __global__ void k_row_norm_factor(int rows, const int* __restrict__ ptr, const int* __restrict__ perm,
                                  const double* __restrict__ val, int mode, double* __restrict__ fac) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < rows; r += nw) {
        double acc = 0.0;
        for (int q = ptr[r] + lane; q < ptr[r + 1]; q += 32) {
            const double a = fabs(val[perm ? perm[q] : q]);
            acc = mode == 0 ? ((acc < a) ? a : acc) : acc + a;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_down_sync(0xffffffffu, acc, o);
            acc = mode == 0 ? ((acc < t) ? t : acc) : acc + t;
        }
        if (lane == 0) fac[r] = acc > 0 ? 1.0 / sqrt(acc) : 1.0;
    }
}

// apply (scaling.cpp:27-33): val *= rs[row] * cs[col]
static __global__ void k_apply_scaling(int nnz, const int* __restrict__ row_of, const int* __restrict__ idx,
                                const double* __restrict__ rs, const double* __restrict__ cs, double* __restrict__ val) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
        val[p] *= rs[row_of[p]] * cs[idx[p]];
}
static __global__ void k_mul_into(int n, const double* __restrict__ f, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] *= f[i];
}
static __global__ void k_fill(int n, double a, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = a;
}

// scaling.cpp:78-88: c' = sign c C, l' = l / C, u' = u / C, lo' = lo R, hi' = hi R
static __global__ void k_scale_vectors(int n, int m, double sign, const double* c, const double* l, const double* u,
                                const double* lo, const double* hi, const double* R, const double* Cs, double* cs_,
                                double* ls, double* us, double* los, double* his) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        cs_[j] = sign * c[j] * Cs[j];
        ls[j] = l[j] / Cs[j];
        us[j] = u[j] / Cs[j];
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        los[i] = lo[i] * R[i];
        his[i] = hi[i] * R[i];
    }
}
// scaling.cpp:89-101 (bscale / cscale live on the device at sc[0], sc[1])
static __global__ void k_rescale(int n, int m, const double* sc, const double* R, const double* Cs, double* c, double* l,
                          double* u, double* lo, double* hi, double* Rres, double* Cres) {
    const double bscale = sc[0], cscale = sc[1];
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        c[j] /= cscale;
        l[j] /= bscale;
        u[j] /= bscale;
        Cres[j] = Cs[j] / cscale;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        lo[i] /= bscale;
        hi[i] /= bscale;
        Rres[i] = R[i] / bscale;
    }
}
// CSR Hessian: Q'_ij = Q_ij * sign * C_i * C_j * bscale / cscale (scaling.cpp:104-107)
static __global__ void k_scale_q(int nnz, const int* __restrict__ row_of, const int* __restrict__ idx, double sign,
                          const double* __restrict__ Cs, const double* sc, double* __restrict__ val) {
    const double bscale = sc[0], cscale = sc[1];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
        val[p] *= sign * Cs[row_of[p]] * Cs[idx[p]] * bscale / cscale;
}
// DPLR Hessian Q = 2 (F F^T + diag D) scaled the same way:
//   F'_jk = sqrt(bscale/cscale) C_j F_jk,  D'_j = (bscale/cscale) C_j^2 D_j.
static __global__ void k_scale_dplr(int n, int k, const double* __restrict__ Cs, const double* sc, double* __restrict__ F,
                             double* __restrict__ D) {
    const double s2 = sc[0] / sc[1], s1 = sqrt(s2);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * k;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = static_cast<int>(e / k);
        F[e] *= s1 * Cs[j];
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) D[j] *= s2 * Cs[j] * Cs[j];
}

// power-iteration step: if *nz > 0 (and not stopped): lambda = nz, v = z / nz; else stop.
static __global__ void k_power_step(int n, const double* __restrict__ z, double* __restrict__ v, double* pw) {
    // pw[0] = latest norm, pw[1] = lambda, pw[2] = stopped flag
    const double nz = pw[0];
    if (pw[2] != 0.0) return;
    if (nz == 0.0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) pw[2] = 1.0;
        return;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) v[j] = z[j] / nz;
    if (blockIdx.x == 0 && threadIdx.x == 0) pw[1] = nz;
}

// x0 = clamp(0, l, u), y0 = 0 (pdhg_impl.hpp:255-257)
static __global__ void k_start_point(int n, int m, const double* l, const double* u, double* x, double* y) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        double v = (0.0 < l[j]) ? l[j] : 0.0;
        x[j] = (u[j] < v) ? u[j] : v;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = 0.0;
}

template <class T>
__global__ void k_convert(long long n, const double* __restrict__ s, T* __restrict__ d) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = static_cast<T>(s[i]);
}

// x_orig = x' C bscale, y_orig = sign y' R cscale (pdhg_impl.hpp:310-314)
static __global__ void k_unscale(int n, int m, double sign, const double* x, const double* y, const double* Cs,
                          const double* R, const double* sc, double* xo, double* yo) {
    const double bscale = sc[0], cscale = sc[1];
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) xo[j] = x[j] * Cs[j] * bscale;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) yo[i] = sign * y[i] * R[i] * cscale;
}

}  // namespace gb

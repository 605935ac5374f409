// Device-side problem setup: stored transpose, Ruiz + Pock-Chambolle
// scaling, bound/objective rescaling, ||A'|| and ||Q'|| power iterations.
// Restates src/scaling.cpp:8-155 and src/lp.cpp:55-72 as GPU kernels so that
// a problem never round-trips through host memory after its upload.
#pragma once
#include "gb_sort.cuh"
#include "gb_spmv.cuh"

namespace gb {

// ---------------------------------------------------------------- deterministic reductions
constexpr int kRedGrid = 592;  // 4 CTAs per SM, fixed so the summation order is fixed

// One launch, two passes: each CTA folds a grid-stride slice into
// partials[cta]; the last CTA to arrive folds the partials in CTA order and
// writes out = post(sum), then re-arms the arrival counter.  The summation
// order is fixed by kRedGrid alone.
template <class F, class P>
__global__ void __launch_bounds__(kThreads) k_red(long long n, F f, double* partials, unsigned* arrivals,
                                                  double* out, P post) {
    __shared__ double sh[kWarps];
    __shared__ bool last;
    pdl_enter();
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads)
        acc += f(i);
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v[0];
        __threadfence();  // the partial is visible before the arrival is counted
        last = atomicAdd(arrivals, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0.0;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += kThreads) a += __ldcg(partials + i);
    double w[1] = {a};
    block_sum<1>(w, sh);
    if (threadIdx.x == 0) {
        post(w[0], out);
        *arrivals = 0u;
    }
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

// `partials` holds kRedGrid doubles; `arrivals` is zero between launches.
template <class F, class P>
inline void reduce_to(cudaStream_t s, long long n, F f, double* partials, unsigned* arrivals, double* out, P post) {
    launch_pdl(k_red<F, P>, kRedGrid, kThreads, 0, s, n, f, partials, arrivals, out, post);
}

// ---------------------------------------------------------------- plain SpMV (y = A x)
template <class V>
struct StoreEpi {
    V* __restrict__ y;
    __device__ __forceinline__ bool begin(int) const { return true; }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int r, const V (&s)[1], const NoPre&) { y[r] = s[0]; }
};
template <class M, class V>
__global__ void __launch_bounds__(kThreads) k_spmv(const __grid_constant__ CsrView<M> A, const V* __restrict__ x,
                                                  V* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_enter();
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
// Rows go to groups of 2^lg lanes (lg = 5: one row per warp).  The caller
// passes lg = 5 for the sums (mode 1), whose order it fixes, and a group
// matched to the average row length for the maxima (mode 0), which are the
// same in any order.  Every lane of a warp runs the same rounds, so the
// shuffles always see the whole warp.
static __global__ void k_row_norm_factor(int rows, const int* __restrict__ ptr, const int* __restrict__ perm,
                                  const double* __restrict__ val, int mode, double* __restrict__ fac, int lg) {
    pdl_enter();
    const int G = 1 << lg, rpw = 32 >> lg;  // lanes per row, rows per warp and round
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane32 = threadIdx.x & 31;
    const int lane = lane32 & (G - 1);
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r0 = warp * rpw; r0 < rows; r0 += nw * rpw) {
        const int r = r0 + (lane32 >> lg);
        double acc = 0.0;
        if (r < rows) {
            for (int q = ptr[r] + lane; q < ptr[r + 1]; q += G) {
                const double a = fabs(val[perm ? perm[q] : q]);
                acc = mode == 0 ? ((acc < a) ? a : acc) : acc + a;
            }
        }
        for (int o = G >> 1; o > 0; o >>= 1) {
            const double t = __shfl_down_sync(0xffffffffu, acc, o, G);
            acc = mode == 0 ? ((acc < t) ? t : acc) : acc + t;
        }
        if (r < rows && lane == 0) fac[r] = acc > 0 ? 1.0 / sqrt(acc) : 1.0;
    }
}

// apply (scaling.cpp:27-33): val *= rs[row] * cs[col]
// One Ruiz / Pock-Chambolle pass applied (scaling.cpp:27-33): a_ij *= rs_i cs_j,
// R *= rs, C *= cs, in one launch.
static __global__ void k_apply_scaling(int nnz, const int* __restrict__ row_of, const int* __restrict__ idx,
                                const double* __restrict__ rs, const double* __restrict__ cs, double* __restrict__ val,
                                int m, double* __restrict__ R, int n, double* __restrict__ C) {
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (int p = t; p < nnz; p += stride) val[p] *= rs[row_of[p]] * cs[idx[p]];
    for (int i = t; i < m; i += stride) R[i] *= rs[i];
    for (int j = t; j < n; j += stride) C[j] *= cs[j];
}
static __global__ void k_fill(int n, double a, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = a;
}

// Per-instance scalars of a batch live in rows of kScal doubles.
constexpr int kScal = 16;
enum ScalIdx : int {
    S_BSCALE = 0, S_CSCALE = 1, S_NORMA = 2, S_NORMQ = 3, S_BNORM = 4, S_CNORM = 5, S_W0 = 6,
    S_PW_NORM = 7, S_PW_LAMBDA = 8, S_PW_STOP = 9, S_CN = 10, S_BN = 11, S_SIGN = 12, S_OBJC = 13
};
__device__ __forceinline__ int inst_of(const int* map, int i) { return map ? map[i] : 0; }

// Segmented fixed-order reduction: CTA k folds f(i) over [off[k], off[k+1])
// and writes post(sum) to out[k * kScal].
template <class F, class P>
__global__ void __launch_bounds__(kThreads) k_seg_red(const int* off, F f, double* out, P post) {
    __shared__ double sh[kWarps];
    pdl_enter();
    const int k = blockIdx.x;
    double acc = 0.0;
    for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += kThreads) acc += f(i);
    double v[1] = {acc};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) post(v[0], out + static_cast<size_t>(k) * kScal);
}

// scaling.cpp:78-88: c' = sign c C, l' = l / C, u' = u / C, lo' = lo R, hi' = hi R
static __global__ void k_scale_vectors(int n, int m, const int* inst_col, const double* sc, const double* c,
                                       const double* l, const double* u, const double* lo, const double* hi,
                                       const double* R, const double* Cs, double* cs_, double* ls, double* us,
                                       double* los, double* his) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double sign = sc[static_cast<size_t>(inst_of(inst_col, j)) * kScal + S_SIGN];
        cs_[j] = sign * c[j] * Cs[j];
        ls[j] = l[j] / Cs[j];
        us[j] = u[j] / Cs[j];
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        los[i] = lo[i] * R[i];
        his[i] = hi[i] * R[i];
    }
}
// scaling.cpp:89-101 (per-instance bscale / cscale)
static __global__ void k_rescale(int n, int m, const int* inst_col, const int* inst_row, const double* sc,
                                 const double* R, const double* Cs, double* c, double* l, double* u, double* lo,
                                 double* hi, double* Rres, double* Cres) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double* s = sc + static_cast<size_t>(inst_of(inst_col, j)) * kScal;
        const double bscale = s[S_BSCALE], cscale = s[S_CSCALE];
        c[j] /= cscale;
        l[j] /= bscale;
        u[j] /= bscale;
        Cres[j] = Cs[j] / cscale;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double bscale = sc[static_cast<size_t>(inst_of(inst_row, i)) * kScal + S_BSCALE];
        lo[i] /= bscale;
        hi[i] /= bscale;
        Rres[i] = R[i] / bscale;
    }
}
// CSR Hessian (one instance): Q'_ij = Q_ij * sign * C_i * C_j * bscale / cscale (scaling.cpp:104-107)
static __global__ void k_scale_q(int nnz, const int* __restrict__ row_of, const int* __restrict__ idx,
                                 const double* __restrict__ Cs, const double* sc, double* __restrict__ val) {
    const double bscale = sc[S_BSCALE], cscale = sc[S_CSCALE], sign = sc[S_SIGN];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
        val[p] *= sign * Cs[row_of[p]] * Cs[idx[p]] * bscale / cscale;
}
// DPLR Hessian Q = 2 (F F^T + diag D) scaled the same way (one instance):
//   F'_jk = sqrt(bscale/cscale) C_j F_jk,  D'_j = (bscale/cscale) C_j^2 D_j.
static __global__ void k_scale_dplr(int n, int k, const double* __restrict__ Cs, const double* sc,
                                    double* __restrict__ F, double* __restrict__ D) {
    const double s2 = sc[S_BSCALE] / sc[S_CSCALE], s1 = sqrt(s2);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * k;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = static_cast<int>(e / k);
        F[e] *= s1 * Cs[j];
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) D[j] *= s2 * Cs[j] * Cs[j];
}

// Power iteration, per instance (scaling.cpp:137-152): v = z / ||z|| unless
// the instance's iteration stopped or ||z|| == 0 ...
// With `count` > 0 the same launch then records, per instance, lambda = ||z||
// ("if (nz == 0.0) break; lambda = nz").  The two parts touch the scalars
// independently: the flag part sets S_PW_STOP only for an instance whose norm
// is 0, whose columns the vector part leaves alone whichever value it reads.
static __global__ void k_power_vec(int n, const int* inst_col, double* sc, const double* z, double* v, int count) {
    pdl_enter();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double* s = sc + static_cast<size_t>(inst_of(inst_col, j)) * kScal;
        const double nz = s[S_PW_NORM];
        if (s[S_PW_STOP] == 0.0 && nz != 0.0) v[j] = z[j] / nz;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        double* s = sc + static_cast<size_t>(k) * kScal;
        if (s[S_PW_STOP] != 0.0) continue;
        if (s[S_PW_NORM] == 0.0) s[S_PW_STOP] = 1.0;
        else s[S_PW_LAMBDA] = s[S_PW_NORM];
    }
}
static __global__ void k_power_reset(int count, double* sc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double* s = sc + static_cast<size_t>(k) * kScal;
    s[S_PW_LAMBDA] = 0.0;
    s[S_PW_STOP] = 0.0;
}
// ||A'|| = sqrt(lambda) * 1.01, or 1 for an instance without nonzeros
// (scaling.cpp:132, 153-154); ||Q'|| = lambda * 1.01 (scaling.cpp:124).
static __global__ void k_finish_norms(int count, const int* nnz_off, double* sc, int q) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double* s = sc + static_cast<size_t>(k) * kScal;
    if (q) s[S_NORMQ] = s[S_PW_LAMBDA] * 1.01;
    else s[S_NORMA] = (nnz_off[k + 1] == nnz_off[k]) ? 1.0 : sqrt(s[S_PW_LAMBDA]) * 1.01;
}
// w0 = ||c'|| / ||b'||_finite (pdhg_impl.hpp:258-261)
static __global__ void k_w0(int count, double* sc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double* s = sc + static_cast<size_t>(k) * kScal;
    const double c = s[S_CN], b = s[S_BN];
    s[S_W0] = (c > 1e-10 && b > 1e-10) ? c / b : 1.0;
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

// Warm start (extension): the caller's point in original units, mapped by
// the inverse of k_unscale and projected onto the scaled bounds; a NaN entry
// keeps the default start k_start_point wrote.
static __global__ void k_warm_point(int n, int m, const int* inst_col, const int* inst_row, const double* l,
                                    const double* u, const double* Cs, const double* R, const double* sc,
                                    const double* xin, const double* yin, double* x, double* y) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double v = xin[j];
        if (isnan(v)) continue;
        const double xs = v / (Cs[j] * sc[static_cast<size_t>(inst_of(inst_col, j)) * kScal + S_BSCALE]);
        x[j] = fmin(fmax(xs, l[j]), u[j]);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double v = yin[i];
        if (isnan(v)) continue;
        const double* s = sc + static_cast<size_t>(inst_of(inst_row, i)) * kScal;
        y[i] = s[S_SIGN] * v / (R[i] * s[S_CSCALE]);
    }
}

// x_orig = x' C bscale, y_orig = sign y' R cscale (pdhg_impl.hpp:310-314)
static __global__ void k_unscale(int n, int m, const int* inst_col, const int* inst_row, const double* x,
                                 const double* y, const double* Cs, const double* R, const double* sc, double* xo,
                                 double* yo) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        xo[j] = x[j] * Cs[j] * sc[static_cast<size_t>(inst_of(inst_col, j)) * kScal + S_BSCALE];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double* s = sc + static_cast<size_t>(inst_of(inst_row, i)) * kScal;
        yo[i] = s[S_SIGN] * y[i] * R[i] * s[S_CSCALE];
    }
}

}  // namespace gb

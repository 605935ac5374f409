// Differentiable batched LP layer (gb_diff_*).  No counterpart in the
// reference: it differentiates the restarted PDHG of src/pdhg_impl.hpp.
//
// Forward (gb_diff_forward)
//   1. The batch engine solves every instance to opt->tol (gb_engine.cu).
//   2. A tail of K plain PDHG iterations (src/pdhg_impl.hpp:133-139 with the
//      final step sizes tau = eta / w, sigma = eta w, no restart check) runs
//      from the returned point.  Its state is checkpointed every R
//      iterations; the last iterate z_K = (x_K, y_K) is the layer's output and
//      is certified again in FP64.
// Backward (gb_diff_backward), FP64 on the scaled problem
//   3. Exact reverse mode through the K tail iterations: segment by segment
//      (last first) the R iterations are recomputed from their checkpoint,
//      keeping iterates and projection codes, then reversed step by step:
//        k_rev_cols  A^T pass: adjoint of the primal step (projection mask,
//                    extrapolation xbar = 2x+ - x), accumulates dL/dc
//        k_rev_da    dL/dA_ij -= sigma lq_i xbar_j + y_i lg_j
//        k_rev_rows  A pass: adjoint of the dual step (projection mask),
//                    accumulates dL/dlo, dL/dhi
//   4. Implicit completion.  The tail start z_0 is (to the solve tolerance) a
//      fixed point z = T(z; theta) of the PDHG map, so its own dependence on
//      theta adds (dT/dtheta)^T nu with nu = (I - J0^T)^{-1} mu_0, where mu_0 is
//      the adjoint left at z_0 and J0 the Jacobian of T there.  With the
//      projection masks of z_0 (free columns F, dual-active rows D) that
//      fixed point reduces exactly to
//          B^T p = mu_x[F],   B q = mu_y[D],   B = A'[D, F],
//      i.e. one symmetric indefinite system [[0, B^T], [B, 0]] (q; p) =
//      (mu_x; mu_y), solved per instance by MINRES (Paige & Saunders, SIAM J.
//      Numer. Anal. 12, 1975) on the same SpMV kernels.  Then dc' += q,
//      d(lo|hi)' += p, dA' -= p xbar^T + y q^T.  For a nondegenerate vertex B
//      is the optimal basis matrix and this is the basis sensitivity; plain
//      unrolling would need O(cond(B)^2) iterations to get there.  With the
//      completion switched off (gb_diff_set_implicit(d, 0, .)) the result is
//      the gradient of the K-step map with z_0 held fixed.
//   5. Gradients go back through the scaling of src/scaling.cpp:75-101 with
//      the scaling factors held constant.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <cstring>
#include <memory>

#include "gb_problem.cuh"
#include "gb_sort.cuh"

namespace gb {
namespace {

using i8 = int8_t;

// ---------------------------------------------------------------- forward tail
// x+ = clamp(x - tau (c - A^T y), l, u), xbar = 2 x+ - x (backend_cpu.cpp:67-80);
// code 1 = strictly inside the box (derivative 1), 0 / 2 = clamped low / high.
struct TailColEpi {
    const double* __restrict__ x;
    const double* __restrict__ c;
    const double* __restrict__ l;
    const double* __restrict__ u;
    const double* __restrict__ tau;
    double* __restrict__ xn;
    double* __restrict__ xb;
    i8* __restrict__ code;
    double t;
    __device__ __forceinline__ bool begin(int inst) {
        t = tau[inst];
        return true;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int j, const double (&s)[1], const NoPre&) {
        const double xj = x[j], lj = l[j], uj = u[j];
        const double z = xj - t * (c[j] - s[0]);
        const double xp = z < lj ? lj : (z > uj ? uj : z);
        xn[j] = xp;
        xb[j] = 2.0 * xp - xj;
        code[j] = (z > lj && z < uj) ? i8(1) : (z <= lj ? i8(0) : i8(2));
    }
};

// q = y - sigma A xbar, y+ = q + clamp(-q, sigma lo, sigma hi) (backend_cpu.cpp:81-92);
// code 0 = -q inside [sigma lo, sigma hi] (y+ = 0), 1 / 2 = clamped to lo / hi.
struct TailRowEpi {
    const double* __restrict__ y;
    const double* __restrict__ lo;
    const double* __restrict__ hi;
    const double* __restrict__ sig;
    double* __restrict__ yn;
    i8* __restrict__ code;
    double s_;
    __device__ __forceinline__ bool begin(int inst) {
        s_ = sig[inst];
        return true;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int i, const double (&s)[1], const NoPre&) {
        const double q = y[i] - s_ * s[0];
        const double t = -q, a = s_ * lo[i], b = s_ * hi[i];
        if (t < a) {
            yn[i] = q + a;
            code[i] = 1;
        } else if (t > b) {
            yn[i] = q + b;
            code[i] = 2;
        } else {
            yn[i] = q + t;
            code[i] = 0;
        }
    }
};

__global__ void __launch_bounds__(kThreads) k_tail_cols(const __grid_constant__ CsrView<double> AT,
                                                        const double* __restrict__ y, TailColEpi e) {
    extern __shared__ __align__(16) unsigned char smem[];
    TailColEpi epi = e;
    pdl_enter();
    spmv_run<1, double, double>(AT, blockIdx.x, GatherOne<double>{y}, epi, smem);
}
__global__ void __launch_bounds__(kThreads) k_tail_rows(const __grid_constant__ CsrView<double> A,
                                                        const double* __restrict__ xb, TailRowEpi e) {
    extern __shared__ __align__(16) unsigned char smem[];
    TailRowEpi epi = e;
    pdl_enter();
    spmv_run<1, double, double>(A, blockIdx.x, GatherOne<double>{xb}, epi, smem);
}

// ---------------------------------------------------------------- reverse pass
// Adjoint of one iteration, given lx, ly (adjoints of x+, y+) and
// lq = [code_y != 0] ly:
//   lxbar = -sigma A^T lq;  lz = [code_x == 1] (lx + 2 lxbar);
//   lx <- lz - lxbar;  lg = -tau lz (= dL/dc contribution);  ly <- lq - A lg.
struct RevColEpi {
    const i8* __restrict__ code;
    const double* __restrict__ tau;
    const double* __restrict__ sig;
    double* __restrict__ lx;
    double* __restrict__ lg;
    double* __restrict__ gc;
    double t, s_;
    __device__ __forceinline__ bool begin(int inst) {
        t = tau[inst];
        s_ = sig[inst];
        return true;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int j, const double (&s)[1], const NoPre&) {
        const double lxb = -s_ * s[0];
        const double ltot = lx[j] + 2.0 * lxb;
        const double lz = code[j] == 1 ? ltot : 0.0;
        lx[j] = lz - lxb;
        const double g = -t * lz;
        lg[j] = g;
        gc[j] += g;
    }
};

// ly = lq - (A lg)_i; when the previous step of the segment exists its lq and
// bound gradients are formed right away (same row, same thread).
struct RevRowEpi {
    const i8* __restrict__ code_prev;
    const double* __restrict__ sig;
    double* __restrict__ lq;
    double* __restrict__ ly;
    double* __restrict__ glo;
    double* __restrict__ ghi;
    double s_;
    __device__ __forceinline__ bool begin(int inst) {
        s_ = sig[inst];
        return true;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int i, const double (&s)[1], const NoPre&) {
        const double l = lq[i] - s[0];
        ly[i] = l;
        if (code_prev) {
            const int c = code_prev[i];
            lq[i] = c ? l : 0.0;
            if (c == 1) glo[i] += s_ * l;
            else if (c == 2) ghi[i] += s_ * l;
        }
    }
};

__global__ void __launch_bounds__(kThreads) k_rev_cols(const __grid_constant__ CsrView<double> AT,
                                                       const double* __restrict__ lq, RevColEpi e) {
    extern __shared__ __align__(16) unsigned char smem[];
    RevColEpi epi = e;
    pdl_enter();
    spmv_run<1, double, double>(AT, blockIdx.x, GatherOne<double>{lq}, epi, smem);
}
__global__ void __launch_bounds__(kThreads) k_rev_rows(const __grid_constant__ CsrView<double> A,
                                                       const double* __restrict__ lg, RevRowEpi e) {
    extern __shared__ __align__(16) unsigned char smem[];
    RevRowEpi epi = e;
    pdl_enter();
    spmv_run<1, double, double>(A, blockIdx.x, GatherOne<double>{lg}, epi, smem);
}

// lq = [code != 0] ly and the bound gradients of the step whose dual codes are `code`.
__global__ void k_rev_start(int m, const int* __restrict__ inst_row, const i8* __restrict__ code,
                            const double* __restrict__ sig, const double* __restrict__ ly, double* __restrict__ lq,
                            double* __restrict__ glo, double* __restrict__ ghi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int c = code[i];
        const double l = ly[i];
        lq[i] = c ? l : 0.0;
        const double s = sig[inst_of(inst_row, i)];
        if (c == 1) glo[i] += s * l;
        else if (c == 2) ghi[i] += s * l;
    }
}

// dL/dA'_e of one iteration: g = c - A^T y and q = y - sigma A xbar both read A.
__global__ void k_rev_da(int nnz, const int* __restrict__ row_of, const int* __restrict__ idx,
                         const int* __restrict__ inst_row, const double* __restrict__ sig,
                         const double* __restrict__ lq, const double* __restrict__ xb, const double* __restrict__ y,
                         const double* __restrict__ lg, double* __restrict__ ga) {
    pdl_enter();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
        const int i = row_of[e], j = idx[e];
        const double s = sig[inst_of(inst_row, i)];
        ga[e] -= s * lq[i] * xb[j] + y[i] * lg[j];
    }
}

// ---------------------------------------------------------------- implicit completion (MINRES)
struct alignas(16) MrState {
    double beta1, beta, cs, sn, dbar, epsln, phibar, tol;
    long long it, max_it;
    int done, converged, free_cols, active_rows;
};

// MINRES vectors live in the compact index space of the reduced system:
// x-part entry c is free column fidx[c], y-part entry r dual-active row
// didx[r]; instance k owns x-part [col_off[k], col_off[k+1]) and y-part
// [row_off[k], row_off[k+1]).
struct MrVecs {
    const int* col_off;
    const int* row_off;
    const int* fidx;
    const int* didx;
    double *vx, *vy, *vpx, *vpy, *px, *py, *d1x, *d1y, *d2x, *d2y, *sx, *sy;
    MrState* st;
};

// Right-hand side (mu_x on free columns; mu_y on dual-active rows), v_1 = b / beta_1.
// Instances with sel[k] == 0 (sel != nullptr) keep their state and solution.
__global__ void __launch_bounds__(kThreads) k_mr_init(const __grid_constant__ MrVecs a, const double* __restrict__ mux,
                                                      const double* __restrict__ muy, long long max_it, double tol,
                                                      const int* __restrict__ sel) {
    __shared__ double red[kWarps * 3];
    __shared__ double inv;
    const int k = blockIdx.x;
    if (sel != nullptr && sel[k] == 0) return;
    const int c0 = a.col_off[k], c1 = a.col_off[k + 1], r0 = a.row_off[k], r1 = a.row_off[k + 1];
    double v[1] = {0.0};
    for (int c = c0 + threadIdx.x; c < c1; c += kThreads) {
        const double b = mux[a.fidx[c]];
        a.vx[c] = b;
        a.vpx[c] = a.px[c] = a.d1x[c] = a.d2x[c] = a.sx[c] = 0.0;
        v[0] += b * b;
    }
    for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
        const double b = muy[a.didx[r]];
        a.vy[r] = b;
        a.vpy[r] = a.py[r] = a.d1y[r] = a.d2y[r] = a.sy[r] = 0.0;
        v[0] += b * b;
    }
    block_sum<1>(v, red);
    if (threadIdx.x == 0) {
        MrState s;
        memset(&s, 0, sizeof(s));
        s.beta1 = sqrt(v[0]);
        s.beta = s.beta1;
        s.cs = -1.0;
        s.phibar = s.beta1;
        s.tol = tol;
        s.free_cols = c1 - c0;
        s.active_rows = r1 - r0;
        // In exact arithmetic MINRES ends within dim = |F| + |D| steps; finite
        // precision Lanczos needs a few times that on consistent systems, and an
        // inconsistent one (a wrong active set) never converges.
        s.max_it = min(max_it, 4LL * (s.free_cols + s.active_rows) + 100);
        s.converged = s.beta1 == 0.0;
        s.done = s.converged || max_it <= 0;
        a.st[k] = s;
        inv = s.beta1 > 0.0 ? 1.0 / s.beta1 : 0.0;
    }
    __syncthreads();
    const double iv = inv;
    for (int j = c0 + threadIdx.x; j < c1; j += kThreads) a.vx[j] *= iv;
    for (int i = r0 + threadIdx.x; i < r1; i += kThreads) a.vy[i] *= iv;
}

// p = K v with K = [[0, B^T], [B, 0]] in the compact index space: the B pass
// (rows D) gives the y-part, the B^T pass (rows F) the x-part.
struct MrEpi {
    double* __restrict__ out;
    const MrState* __restrict__ st;
    __device__ __forceinline__ bool begin(int inst) const { return st[inst].done == 0; }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int r, const double (&s)[1], const NoPre&) { out[r] = s[0]; }
};
struct MrOpArgs {
    CsrView<double> A, AT;
    MrVecs v;
};
__global__ void __launch_bounds__(kThreads) k_mr_op(const __grid_constant__ MrOpArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (static_cast<int>(blockIdx.x) < a.A.nb) {
        MrEpi e{a.v.py, a.v.st};
        spmv_run<1, double, double>(a.A, blockIdx.x, GatherOne<double>{a.v.vx}, e, smem);
    } else {
        MrEpi e{a.v.px, a.v.st};
        spmv_run<1, double, double>(a.AT, blockIdx.x - a.A.nb, GatherOne<double>{a.v.vy}, e, smem);
    }
}

// One MINRES step of instance k by its CTA (fixed-order reductions): Lanczos
// (alpha, beta), the two Givens rotations, direction and solution update.
// p = K v is in px / py on entry.
// Sum of one value per thread over an NT-thread CTA into thread 0's v[0], in
// the order of block_sum (each warp's shuffle sum, then the warps in order).
template <int NT>
__device__ __forceinline__ void mr_cta_sum(double (&v)[1], double* red) {
    const double t = warp_sum(v[0]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double u = 0.0;
        for (int w = 0; w < NT / 32; ++w) u += red[w];
        v[0] = u;
    }
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ void mr_update_step(const MrVecs& a, int k, MrState* sp, double* red, double* bc) {
    const int c0 = a.col_off[k], c1 = a.col_off[k + 1], r0 = a.row_off[k], r1 = a.row_off[k + 1];
    double v[1] = {0.0};
    for (int j = c0 + threadIdx.x; j < c1; j += NT) v[0] += a.vx[j] * a.px[j];
    for (int i = r0 + threadIdx.x; i < r1; i += NT) v[0] += a.vy[i] * a.py[i];
    mr_cta_sum<NT>(v, red);
    if (threadIdx.x == 0) bc[0] = v[0];
    __syncthreads();
    const double alpha = bc[0], beta = sp->beta;
    v[0] = 0.0;
    for (int j = c0 + threadIdx.x; j < c1; j += NT) {
        const double p = a.px[j] - alpha * a.vx[j] - beta * a.vpx[j];
        a.px[j] = p;
        v[0] += p * p;
    }
    for (int i = r0 + threadIdx.x; i < r1; i += NT) {
        const double p = a.py[i] - alpha * a.vy[i] - beta * a.vpy[i];
        a.py[i] = p;
        v[0] += p * p;
    }
    mr_cta_sum<NT>(v, red);
    if (threadIdx.x == 0) {
        MrState s = *sp;
        const double bn = sqrt(v[0]);
        const double oldeps = s.epsln;
        const double delta = s.cs * s.dbar + s.sn * alpha;
        const double gbar = s.sn * s.dbar - s.cs * alpha;
        s.epsln = s.sn * bn;
        s.dbar = -s.cs * bn;
        double gamma = sqrt(gbar * gbar + bn * bn);
        if (!(gamma > 1e-300)) gamma = 1e-300;
        s.cs = gbar / gamma;
        s.sn = bn / gamma;
        const double phi = s.cs * s.phibar;
        s.phibar = s.sn * s.phibar;
        s.beta = bn;
        s.it += 1;
        s.converged = (s.phibar <= s.tol * s.beta1) || !(bn > 1e-300);
        s.done = s.converged || s.it >= s.max_it || !isfinite(s.phibar);
        *sp = s;
        bc[1] = phi;
        bc[2] = 1.0 / gamma;
        bc[3] = oldeps;
        bc[4] = delta;
        bc[5] = bn > 1e-300 ? 1.0 / bn : 0.0;
    }
    __syncthreads();
    const double phi = bc[1], ig = bc[2], oldeps = bc[3], delta = bc[4], ib = bc[5];
    for (int j = c0 + threadIdx.x; j < c1; j += NT) {
        const double w = (a.vx[j] - oldeps * a.d2x[j] - delta * a.d1x[j]) * ig;
        a.d2x[j] = a.d1x[j];
        a.d1x[j] = w;
        a.sx[j] += phi * w;
        a.vpx[j] = a.vx[j];
        a.vx[j] = a.px[j] * ib;
    }
    for (int i = r0 + threadIdx.x; i < r1; i += NT) {
        const double w = (a.vy[i] - oldeps * a.d2y[i] - delta * a.d1y[i]) * ig;
        a.d2y[i] = a.d1y[i];
        a.d1y[i] = w;
        a.sy[i] += phi * w;
        a.vpy[i] = a.vy[i];
        a.vy[i] = a.py[i] * ib;
    }
}

// One MINRES step per instance (one CTA per instance), after k_mr_op.
__global__ void __launch_bounds__(kThreads) k_mr_update(const __grid_constant__ MrVecs a) {
    __shared__ double red[kWarps];
    __shared__ double bc[6];
    const int k = blockIdx.x;
    MrState* sp = a.st + k;
    if (sp->done) return;
    mr_update_step<kThreads>(a, k, sp, red, bc);
}

// Every MINRES step of one instance in one CTA, for reduced systems small
// enough that one CTA forms p = K v in a few microseconds: the B pass (rows D
// of the instance, giving the y-part) and the B^T pass (rows F, the x-part),
// kMrLanes lanes per row summed by shuffles in a fixed order, then
// mr_update_step; until the instance's state is done, which its step bound
// guarantees.  Instances are independent, so CTAs never wait on one another.
constexpr int kMrLanes = 2;
constexpr int kMrSolveThreads = 512;  // a step's passes and sweeps over ~1,000 entries in one or two rounds
constexpr long long kMrOneLaunchNnz = 1 << 16;  // B and B^T nonzeros of the widest instance
bool mr_one_launch_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("GANIT_B200_MR_ONE_LAUNCH");
        return v == nullptr || std::string(v) != "0";
    }();
    return on;
}
__device__ __forceinline__ void mr_rows(const CsrView<double>& B, int r0, int r1, const double* v, double* out) {
    const int lane = threadIdx.x % kMrLanes, grp = threadIdx.x / kMrLanes;
    constexpr int ngrp = kMrSolveThreads / kMrLanes;
    for (int base = r0; base < r1; base += ngrp) {  // the same number of rounds for every thread
        const int r = base + grp;
        double t = 0.0;
        if (r < r1) {
            const int p1 = B.ptr[r + 1];
#pragma unroll 4
            for (int q = B.ptr[r] + lane; q < p1; q += kMrLanes) t += B.val[q] * v[B.idx[q]];
        }
#pragma unroll
        for (int o = kMrLanes / 2; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o, kMrLanes);
        if (r < r1 && lane == 0) out[r] = t;
    }
}
__global__ void __launch_bounds__(kMrSolveThreads) k_mr_solve(const __grid_constant__ MrOpArgs a) {
    __shared__ double red[kMrSolveThreads / 32];
    __shared__ double bc[6];
    const int k = blockIdx.x;
    MrState* sp = a.v.st + k;
    const int f0 = a.v.col_off[k], f1 = a.v.col_off[k + 1], d0 = a.v.row_off[k], d1 = a.v.row_off[k + 1];
    while (*reinterpret_cast<volatile const int*>(&sp->done) == 0) {  // uniform: read after a barrier
        mr_rows(a.A, d0, d1, a.v.vx, a.v.py);
        mr_rows(a.AT, f0, f1, a.v.vy, a.v.px);
        __syncthreads();
        mr_update_step<kMrSolveThreads>(a.v, k, sp, red, bc);
        __syncthreads();  // v and the state are written before the next step reads them
    }
}

// Per instance: (free columns, dual-active rows) of the codes, one CTA each.
__global__ void __launch_bounds__(kThreads) k_code_counts(const int* __restrict__ col_off,
                                                          const int* __restrict__ row_off, const i8* __restrict__ cx,
                                                          const i8* __restrict__ cy, int2* __restrict__ out) {
    const int k = blockIdx.x;
    int f = 0, d = 0;
    for (int j = col_off[k] + threadIdx.x; j < col_off[k + 1]; j += kThreads) f += cx[j] == 1;
    for (int i = row_off[k] + threadIdx.x; i < row_off[k + 1]; i += kThreads) d += cy[i] != 0;
    __shared__ int sf[kWarps], sd[kWarps];
    for (int o = 16; o > 0; o >>= 1) {
        f += __shfl_down_sync(0xffffffffu, f, o);
        d += __shfl_down_sync(0xffffffffu, d, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sf[threadIdx.x >> 5] = f;
        sd[threadIdx.x >> 5] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tf = 0, td = 0;
        for (int w = 0; w < kWarps; ++w) {
            tf += sf[w];
            td += sd[w];
        }
        out[k] = make_int2(tf, td);
    }
}

// ---- the reduced system B = A'[D, F] in compact form, built per MINRES solve
// (F: free columns, cx == 1; D: dual-active rows, cy != 0) of the instances
// a solve selects (sel == nullptr: all), so that a solve for a few instances
// launches their blocks alone.  Flags with one trailing 0, so that the
// exclusive scan's last entry is the count.
__global__ void k_mr_flags(int n, int m, const i8* __restrict__ cx, const i8* __restrict__ cy, const int* inst_col,
                           const int* inst_row, const int* __restrict__ sel, int* __restrict__ ff,
                           int* __restrict__ df) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= n; j += stride)
        ff[j] = (j < n && cx[j] == 1 && (sel == nullptr || sel[inst_of(inst_col, j)])) ? 1 : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += stride)
        df[i] = (i < m && cy[i] != 0 && (sel == nullptr || sel[inst_of(inst_row, i)])) ? 1 : 0;
}

// From the scanned flags: full -> compact maps (-1 outside F / D), compact ->
// full lists, and each instance's compact offsets.
__global__ void k_mr_maps(int n, int m, int count, const int* __restrict__ col_off, const int* __restrict__ row_off,
                          const int* __restrict__ ff, const int* __restrict__ fs, const int* __restrict__ df,
                          const int* __restrict__ ds, int* __restrict__ cmap, int* __restrict__ rmap,
                          int* __restrict__ fidx, int* __restrict__ didx, int* __restrict__ f_off,
                          int* __restrict__ d_off) {
    const int stride = gridDim.x * blockDim.x;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int j = t; j < n; j += stride) {
        cmap[j] = ff[j] ? fs[j] : -1;
        if (ff[j]) fidx[fs[j]] = j;
    }
    for (int i = t; i < m; i += stride) {
        rmap[i] = df[i] ? ds[i] : -1;
        if (df[i]) didx[ds[i]] = i;
    }
    for (int k = t; k <= count; k += stride) {
        f_off[k] = fs[col_off[k]];
        d_off[k] = ds[row_off[k]];
    }
}

// Entries of compact row r (full row rows[r] of ptr/idx) whose column maps
// into the compact space: one warp per row.
__global__ void k_mr_row_counts(int nr, const int* __restrict__ rows, const int* __restrict__ ptr,
                                const int* __restrict__ idx, const int* __restrict__ map, int* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nr; r += nw) {
        const int i = rows[r];
        int c = 0;
        for (int p = ptr[i] + lane; p < ptr[i + 1]; p += 32) c += map[idx[p]] >= 0;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[r] = c;
    }
}

// The same entries, in source order, into out_ptr's slots, columns mapped:
// each warp keeps its row's order with a ballot prefix.
__global__ void k_mr_row_fill(int nr, const int* __restrict__ rows, const int* __restrict__ ptr,
                              const int* __restrict__ idx, const double* __restrict__ val,
                              const int* __restrict__ map, const int* __restrict__ out_ptr, int* __restrict__ out_idx,
                              double* __restrict__ out_val) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nr; r += nw) {
        const int i = rows[r];
        int q = out_ptr[r];
        for (int p0 = ptr[i]; p0 < ptr[i + 1]; p0 += 32) {
            const int p = p0 + lane;
            const int c = p < ptr[i + 1] ? map[idx[p]] : -1;
            const unsigned keep = __ballot_sync(0xffffffffu, c >= 0);
            if (c >= 0) {
                const int at = q + __popc(keep & ((1u << lane) - 1u));
                out_idx[at] = c;
                out_val[at] = val[p];
            }
            q += __popc(keep);
        }
    }
}

// Compact solution -> full index space (zero outside F / D), for the
// instances selected (sel == nullptr: all).
__global__ void k_mr_scatter(int n, int m, const int* inst_col, const int* inst_row, const int* __restrict__ sel,
                             const int* __restrict__ cmap, const int* __restrict__ rmap,
                             const double* __restrict__ sx, const double* __restrict__ sy, double* __restrict__ ox,
                             double* __restrict__ oy) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        if (sel == nullptr || sel[inst_of(inst_col, j)]) ox[j] = cmap[j] >= 0 ? sx[cmap[j]] : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        if (sel == nullptr || sel[inst_of(inst_row, i)]) oy[i] = rmap[i] >= 0 ? sy[rmap[i]] : 0.0;
}

// Condition of the MINRES loop graph: repeat while some instance has not finished.
__global__ void __launch_bounds__(kThreads) k_mr_cond(const MrState* __restrict__ st, int count,
                                                      unsigned long long cond) {
    int any = 0;
    for (int k = threadIdx.x; k < count; k += kThreads) any |= st[k].done == 0;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(cond), any ? 1u : 0u);
}

// Parameter gradient of T at z_0 against nu: dc' += q, d(lo|hi)' += p, dA' -= p xbar0^T + y0 q^T.
__global__ void k_implicit_grads(int n, int m, int nnz, const int* __restrict__ row_of, const int* __restrict__ idx,
                                 const i8* __restrict__ cy, const double* __restrict__ q, const double* __restrict__ p,
                                 const double* __restrict__ xb0, const double* __restrict__ y0, double* __restrict__ gc,
                                 double* __restrict__ glo, double* __restrict__ ghi, double* __restrict__ ga) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) gc[j] += q[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const int c = cy[i];
        if (c == 1) glo[i] += p[i];
        else if (c == 2) ghi[i] += p[i];
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
        const int i = row_of[e], j = idx[e];
        ga[e] -= p[i] * xb0[j] + y0[i] * q[j];
    }
}

// ---------------------------------------------------------------- solution polishing
// Reduced KKT system of the active set read off one PDHG step (codes):
//   B^T y_D = c'_F,  B x_F = bnd_D - A'[D, N] x_N,
// x_N at the bound its code names, bnd the row bound its code names.
__global__ void k_polish_rhs_cols(int n, const i8* __restrict__ cx, const double* __restrict__ c,
                                  const double* __restrict__ l, const double* __restrict__ u, double* __restrict__ rhs_x,
                                  double* __restrict__ xn) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int k = cx[j];
        rhs_x[j] = k == 1 ? c[j] : 0.0;
        xn[j] = k == 1 ? 0.0 : (k == 0 ? l[j] : u[j]);
    }
}
struct PolishRowEpi {
    const i8* __restrict__ cy;
    const double* __restrict__ lo;
    const double* __restrict__ hi;
    double* __restrict__ rhs_y;
    __device__ __forceinline__ bool begin(int) const { return true; }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int i, const double (&s)[1], const NoPre&) {
        const int k = cy[i];
        rhs_y[i] = k == 0 ? 0.0 : (k == 1 ? lo[i] : hi[i]) - s[0];
    }
};
__global__ void __launch_bounds__(kThreads) k_polish_rhs_rows(const __grid_constant__ CsrView<double> A,
                                                              const double* __restrict__ xn, PolishRowEpi e) {
    extern __shared__ __align__(16) unsigned char smem[];
    PolishRowEpi epi = e;
    spmv_run<1, double, double>(A, blockIdx.x, GatherOne<double>{xn}, epi, smem);
}
// Polished point of the instances in `use` (others keep (x, y)); x_F is
// clamped into its box so that a wrong active set shows in the FP64 KKT.
__global__ void k_polish_point(int n, int m, const int* inst_col, const int* inst_row, const int* __restrict__ use,
                               const i8* __restrict__ cx, const i8* __restrict__ cy, const double* __restrict__ sol_x,
                               const double* __restrict__ sol_y, const double* __restrict__ l,
                               const double* __restrict__ u, double* __restrict__ x, double* __restrict__ y) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        if (!use[inst_of(inst_col, j)]) continue;
        const int k = cx[j];
        const double lj = l[j], uj = u[j];
        if (k == 1) {
            const double v = sol_x[j];
            x[j] = v < lj ? lj : (v > uj ? uj : v);
        } else {
            x[j] = k == 0 ? lj : uj;
        }
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        if (use[inst_of(inst_row, i)]) y[i] = cy[i] != 0 ? sol_y[i] : 0.0;
}
// (x, y) <- (xs, ys) on the instances in `restore`.
__global__ void k_restore(int n, int m, const int* inst_col, const int* inst_row, const int* __restrict__ restore,
                          const double* __restrict__ xs, const double* __restrict__ ys, double* __restrict__ x,
                          double* __restrict__ y) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        if (restore[inst_of(inst_col, j)]) x[j] = xs[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        if (restore[inst_of(inst_row, i)]) y[i] = ys[i];
}

// ---------------------------------------------------------------- scaling of adjoints and gradients
// x = x' C bscale, y = sign y' R cscale  =>  dL/dx' = dL/dx C bscale, dL/dy' = sign dL/dy R cscale.
__global__ void k_adjoint_in(int n, int m, const int* inst_col, const int* inst_row, const double* __restrict__ sc,
                             const double* __restrict__ Cs, const double* __restrict__ R, const double* __restrict__ gx,
                             const double* __restrict__ gy, double* __restrict__ lx, double* __restrict__ ly) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        lx[j] = gx[j] * Cs[j] * sc[static_cast<size_t>(inst_of(inst_col, j)) * kScal + S_BSCALE];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double* s = sc + static_cast<size_t>(inst_of(inst_row, i)) * kScal;
        ly[i] = s[S_SIGN] * gy[i] * R[i] * s[S_CSCALE];
    }
}
// c' = sign c C / cscale, lo' = lo R / bscale, hi' = hi R / bscale, A' = R A C.
__global__ void k_grads_out(int n, int m, int nnz, const int* inst_col, const int* inst_row,
                            const int* __restrict__ row_of, const int* __restrict__ idx, const double* __restrict__ sc,
                            const double* __restrict__ Cs, const double* __restrict__ R, const double* __restrict__ gc,
                            const double* __restrict__ glo, const double* __restrict__ ghi,
                            const double* __restrict__ ga, double* __restrict__ oc, double* __restrict__ olo,
                            double* __restrict__ ohi, double* __restrict__ oa) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double* s = sc + static_cast<size_t>(inst_of(inst_col, j)) * kScal;
        oc[j] = s[S_SIGN] * gc[j] * Cs[j] / s[S_CSCALE];
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double b = sc[static_cast<size_t>(inst_of(inst_row, i)) * kScal + S_BSCALE];
        olo[i] = glo[i] * R[i] / b;
        ohi[i] = ghi[i] * R[i] / b;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) oa[e] = ga[e] * R[row_of[e]] * Cs[idx[e]];
}


constexpr int kMrChunk = 64;  // MINRES steps between tests of the per-instance flags

}  // namespace

// ---------------------------------------------------------------- host object
struct Diff {
    FreeBatchEnd free_batch;        // first member, destroyed last: closes the teardown's free batch
    std::unique_ptr<Problem> P;
    int K = 200, R = 20, nseg = 10;
    long long mr_max = 20000;
    double mr_tol = 1e-10;
    bool polish = true;
    std::vector<double> tau_h, sig_h;
    DevBuf<double> tau, sig;
    DevBuf<double> ck_x, ck_y;      // nseg checkpoints (x, y)
    DevBuf<double> sx, sy, sxb;     // iterates of one segment: (R+1) n, (R+1) m, R n
    DevBuf<i8> scx, scy;            // projection codes of one segment: R n, R m
    int seg_valid = -1;             // segment whose iterates the buffers hold
    DevBuf<double> lx, ly, lq, lg, gc, glo, ghi, ga;
    DevBuf<double> mr[12];          // MINRES vectors, compact index space (x-parts n, y-parts m long)
    DevBuf<double> mr_sol_x, mr_sol_y;  // its solution in the full index space
    // the reduced system of the last solve: flags and scans (n + 1, m + 1),
    // maps, lists, per-instance compact offsets, B and B^T in CSR with schedules
    DevBuf<int> mr_ff, mr_fs, mr_df, mr_ds, mr_cmap, mr_rmap, mr_fidx, mr_didx, mr_foff, mr_doff, mr_scan;
    DevBuf<int> b_ptr, b_idx, bt_ptr, bt_idx;
    DevBuf<double> b_val, bt_val;
    DevSchedule b_s, bt_s;
    std::vector<int> mr_foff_h, mr_doff_h, b_ptr_h, bt_ptr_h;
    DevBuf<MrState> mst;
    MrState* mst_host = nullptr;
    DevBuf<int> flags;              // per-instance selection (polish use / restore)
    int* flags_host = nullptr;
    DevBuf<int2> counts;            // per instance: free columns, dual-active rows of the polishing codes
    int2* counts_host = nullptr;
    DevBuf<double> io_n, io_m, io_m2, io_z;
    DevBuf<double> kx, ky;          // vertices certified in an early polishing round (scaled)
    std::unique_ptr<LevelGraph> mr_graph;  // the MINRES loop (built on first use; fixed buffers)
    std::vector<gb_diff_info> info;
    bool forward_done = false;
    bool backward_done = false;
    long long launches = 0;

    ~Diff() {
        if (P) cudaSetDevice(P->device);
        begin_free_batch();
        free_batch.open = true;
        host_free(mst_host);
        host_free(flags_host);
        host_free(counts_host);
    }

    size_t n() const { return static_cast<size_t>(P->n); }
    size_t m() const { return static_cast<size_t>(P->m); }
    size_t nnz() const { return static_cast<size_t>(P->A.nnz); }
    double* x_at(int k) { return sx.get() + k * n(); }
    double* y_at(int k) { return sy.get() + k * m(); }
    double* xb_at(int k) { return sxb.get() + k * n(); }
    i8* cx_at(int k) { return scx.get() + k * n(); }
    i8* cy_at(int k) { return scy.get() + k * m(); }

    MrVecs mr_vecs() {
        MrVecs v;
        v.col_off = mr_foff.get();
        v.row_off = mr_doff.get();
        v.fidx = mr_fidx.get();
        v.didx = mr_didx.get();
        v.vx = mr[0].get(); v.vy = mr[1].get(); v.vpx = mr[2].get(); v.vpy = mr[3].get();
        v.px = mr[4].get(); v.py = mr[5].get(); v.d1x = mr[6].get(); v.d1y = mr[7].get();
        v.d2x = mr[8].get(); v.d2y = mr[9].get(); v.sx = mr[10].get(); v.sy = mr[11].get();
        v.st = mst.get();
        return v;
    }

    // `steps` iterations from (sx[0], sy[0]) keeping iterates and codes.
    void run_segment(int steps) {
        Problem& p = *P;
        cudaStream_t s = p.stream;
        const size_t smem = spmv_smem_bytes<1, double>();
        const CsrView<double> A = p.A.view<double>(), AT = p.AT.view<double>();
        for (int k = 0; k < steps; ++k) {
            if (AT.nb) {
                TailColEpi e{x_at(k), p.c.get(), p.l.get(), p.u.get(), tau.get(), x_at(k + 1), xb_at(k), cx_at(k), 0.0};
                launch_pdl(k_tail_cols, AT.nb, kThreads, smem, s, AT, static_cast<const double*>(y_at(k)), e);
            }
            if (A.nb) {
                TailRowEpi e{y_at(k), p.lo.get(), p.hi.get(), sig.get(), y_at(k + 1), cy_at(k), 0.0};
                launch_pdl(k_tail_rows, A.nb, kThreads, smem, s, A, static_cast<const double*>(xb_at(k)), e);
            }
            launches += 2;
        }
    }
    void recompute(int seg) {
        cudaStream_t s = P->stream;
        GB_CUDA(cudaMemcpyAsync(x_at(0), ck_x.get() + seg * n(), n() * sizeof(double), cudaMemcpyDeviceToDevice, s));
        GB_CUDA(cudaMemcpyAsync(y_at(0), ck_y.get() + seg * m(), m() * sizeof(double), cudaMemcpyDeviceToDevice, s));
        run_segment(R);
        seg_valid = seg;
    }

    // The reduced system of the codes of step 0 of the resident segment: F
    // (free columns) and D (dual-active rows) of every instance, B = A'[D, F]
    // and B^T = A'^T[F, D] in CSR over compact indices (entries in source
    // order), and their row-block schedules, segmented by instance; only the
    // instances `sel` selects (nullptr: all) get rows and columns.
    void build_reduced(const int* sel) {
        Problem& p = *P;
        cudaStream_t s = p.stream;
        const int n = p.n, m = p.m, K = p.count;
        const int gv = elem_grid(std::max(n, m) + 1, p.sms);
        k_mr_flags<<<gv, kThreads, 0, s>>>(n, m, cx_at(0), cy_at(0), p.icol(), p.irow(), sel, mr_ff.get(),
                                           mr_df.get());
        exclusive_scan(mr_ff.get(), mr_fs.get(), n + 1, mr_scan.get(), s);
        exclusive_scan(mr_df.get(), mr_ds.get(), m + 1, mr_scan.get(), s);
        k_mr_maps<<<gv, kThreads, 0, s>>>(n, m, K, p.d_col_off.get(), p.d_row_off.get(), mr_ff.get(), mr_fs.get(),
                                          mr_df.get(), mr_ds.get(), mr_cmap.get(), mr_rmap.get(), mr_fidx.get(),
                                          mr_didx.get(), mr_foff.get(), mr_doff.get());
        mr_foff_h.resize(K + 1);
        mr_doff_h.resize(K + 1);
        GB_CUDA(cudaMemcpyAsync(mr_foff_h.data(), mr_foff.get(), sizeof(int) * (K + 1), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaMemcpyAsync(mr_doff_h.data(), mr_doff.get(), sizeof(int) * (K + 1), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        const int nf = mr_foff_h[K], nd = mr_doff_h[K];
        const int gw = elem_grid(static_cast<long long>(std::max(std::max(nf, nd), 1)) * 32, p.sms);
        GB_CUDA(cudaMemsetAsync(b_ptr.get() + nd, 0, sizeof(int), s));
        GB_CUDA(cudaMemsetAsync(bt_ptr.get() + nf, 0, sizeof(int), s));
        if (nd) k_mr_row_counts<<<gw, kThreads, 0, s>>>(nd, mr_didx.get(), p.A.ptr.get(), p.A.idx.get(),
                                                        mr_cmap.get(), b_ptr.get());
        if (nf) k_mr_row_counts<<<gw, kThreads, 0, s>>>(nf, mr_fidx.get(), p.AT.ptr.get(), p.AT.idx.get(),
                                                        mr_rmap.get(), bt_ptr.get());
        exclusive_scan(b_ptr.get(), b_ptr.get(), nd + 1, mr_scan.get(), s);
        exclusive_scan(bt_ptr.get(), bt_ptr.get(), nf + 1, mr_scan.get(), s);
        if (nd) k_mr_row_fill<<<gw, kThreads, 0, s>>>(nd, mr_didx.get(), p.A.ptr.get(), p.A.idx.get(),
                                                      p.A.val64.get(), mr_cmap.get(), b_ptr.get(), b_idx.get(),
                                                      b_val.get());
        if (nf) k_mr_row_fill<<<gw, kThreads, 0, s>>>(nf, mr_fidx.get(), p.AT.ptr.get(), p.AT.idx.get(),
                                                      p.AT.val64.get(), mr_rmap.get(), bt_ptr.get(), bt_idx.get(),
                                                      bt_val.get());
        b_ptr_h.resize(nd + 1);
        bt_ptr_h.resize(nf + 1);
        GB_CUDA(cudaMemcpyAsync(b_ptr_h.data(), b_ptr.get(), sizeof(int) * (nd + 1), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaMemcpyAsync(bt_ptr_h.data(), bt_ptr.get(), sizeof(int) * (nf + 1), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        b_s.upload(build_schedule(b_ptr_h.data(), nd, mr_doff_h.data(), K), 1, s);
        bt_s.upload(build_schedule(bt_ptr_h.data(), nf, mr_foff_h.data(), K), 1, s);
        launches += 10;
    }
    CsrView<double> reduced_view(const DevBuf<int>& ptr, const DevBuf<int>& idx, const DevBuf<double>& val,
                                 const DevSchedule& sc, int rows) const {
        CsrView<double> v;
        v.ptr = ptr.get();
        v.idx = idx.get();
        v.val = val.get();
        v.blocks = sc.blocks.get();
        v.slots = sc.slots.get();
        v.counters = sc.counters.get();
        v.bits = sc.bits.get();
        v.rows = rows;
        v.nb = sc.nb;
        v.vec = 1;  // idx / val allocated with padded_nnz
        v.nc = kLoadPlain;
        return v;
    }

    // Per-instance MINRES on K = [[0, B^T], [B, 0]] with B = A'[D, F] read from
    // the codes of step 0 of the resident segment, in the compact index space
    // of (F, D); the solution goes to mr_sol_x / mr_sol_y in the full index
    // space (zero outside F / D); per-instance state left in mst_host.
    // sel (device, may be NULL): only the instances with sel[k] != 0 start a
    // new solve; the others keep their state and full-space solution.
    void minres(const double* rhs_x, const double* rhs_y, const int* sel = nullptr) {
        Problem& p = *P;
        cudaStream_t s = p.stream;
        const size_t smem = spmv_smem_bytes<1, double>();
        build_reduced(sel);
        MrVecs v = mr_vecs();
        k_mr_init<<<p.count, kThreads, 0, s>>>(v, rhs_x, rhs_y, mr_max, mr_tol, sel);
        launches += 1;
        const int nd = mr_doff_h[p.count], nf = mr_foff_h[p.count];
        MrOpArgs oa{reduced_view(b_ptr, b_idx, b_val, b_s, nd), reduced_view(bt_ptr, bt_idx, bt_val, bt_s, nf), v};
        const int nb = oa.A.nb + oa.AT.nb;
        mr_graph.reset();  // it holds the previous system's schedules
        // the whole solve in one launch, one CTA per instance, when every
        // instance's B and B^T are small (GANIT_B200_MR_ONE_LAUNCH=0: never)
        long long widest = 0;
        for (int k = 0; k < p.count; ++k)
            widest = std::max<long long>(widest, (b_ptr_h[mr_doff_h[k + 1]] - b_ptr_h[mr_doff_h[k]]) +
                                                     (bt_ptr_h[mr_foff_h[k + 1]] - bt_ptr_h[mr_foff_h[k]]));
        const bool one_launch = mr_one_launch_enabled() && widest <= kMrOneLaunchNnz;
        if (one_launch) {
            k_mr_solve<<<p.count, kMrSolveThreads, 0, s>>>(oa);
        } else if (host_loop_mode()) {  // the same steps from the host, one state read-back per chunk
            for (;;) {
                for (int c = 0; c < kMrChunk; ++c) {
                    if (nb) k_mr_op<<<nb, kThreads, smem, s>>>(oa);
                    k_mr_update<<<p.count, kThreads, 0, s>>>(v);
                }
                GB_CUDA(cudaMemcpyAsync(mst_host, mst.get(), sizeof(MrState) * p.count, cudaMemcpyDeviceToHost, s));
                GB_CUDA(cudaStreamSynchronize(s));
                bool any = false;
                for (int k = 0; k < p.count; ++k) any |= mst_host[k].done == 0;
                if (!any) break;
            }
        } else {
            // The steps run as one CUDA graph: a conditional while node whose body is
            // kMrChunk steps and a test of the per-instance "done" flags, so the
            // loop needs no host round trip.  Every instance stops at its own step
            // bound (MrState::max_it), so the loop ends.
            if (!mr_graph) {
                auto g = std::make_unique<LevelGraph>();
                GB_CUDA(cudaGraphCreate(&g->graph, 0));
                cudaGraphConditionalHandle h;
                GB_CUDA(cudaGraphConditionalHandleCreate(&h, g->graph, 1, cudaGraphCondAssignDefault));
                cudaGraphNodeParams cp = {};
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = h;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                cudaGraphNode_t node;
                GB_CUDA(cudaGraphAddNode(&node, g->graph, nullptr, 0, &cp));
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                cudaStream_t cs;
                GB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
                GB_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
                for (int c = 0; c < kMrChunk; ++c) {
                    // (plain launches: with programmatic dependent launch the next
                    // step's CTAs wait on SMs the current step needs -- measured
                    // 10-25 % slower)
                    if (nb) k_mr_op<<<nb, kThreads, smem, cs>>>(oa);
                    k_mr_update<<<p.count, kThreads, 0, cs>>>(v);
                }
                k_mr_cond<<<1, kThreads, 0, cs>>>(mst.get(), p.count, static_cast<unsigned long long>(h));
                const cudaError_t e = cudaGetLastError();
                cudaGraph_t done_body = nullptr;
                const cudaError_t e2 = cudaStreamEndCapture(cs, &done_body);
                cudaStreamDestroy(cs);
                if (e != cudaSuccess || e2 != cudaSuccess) {
                    g->graph = nullptr;  // a failed capture: leak the half-built graph rather than destroy it
                    GB_CUDA(e != cudaSuccess ? e : e2);
                }
                GB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
                mr_graph = std::move(g);
            }
            GB_CUDA(cudaGraphLaunch(mr_graph->exec, s));
        }
        k_mr_scatter<<<elem_grid(std::max(p.n, p.m), p.sms), kThreads, 0, s>>>(
            p.n, p.m, p.icol(), p.irow(), sel, mr_cmap.get(), mr_rmap.get(), mr[10].get(), mr[11].get(),
            mr_sol_x.get(), mr_sol_y.get());
        GB_CUDA(cudaMemcpyAsync(mst_host, mst.get(), sizeof(MrState) * p.count, cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        long long steps = 0;
        for (int k = 0; k < p.count; ++k) steps = std::max<long long>(steps, mst_host[k].it);
        launches += 1 + (one_launch ? 1 : ((steps + kMrChunk - 1) / kMrChunk) * (2 * kMrChunk + 1));
    }
};

void diff_alloc(Diff& D) {
    Problem& P = *D.P;
    const size_t n = std::max<size_t>(D.n(), 1), m = std::max<size_t>(D.m(), 1), z = std::max<size_t>(D.nnz(), 1);
    D.tau.reset(P.count);
    D.sig.reset(P.count);
    D.ck_x.reset(n * D.nseg);
    D.ck_y.reset(m * D.nseg);
    D.sx.reset(n * (D.R + 1));
    D.sy.reset(m * (D.R + 1));
    D.sxb.reset(n * D.R);
    D.scx.reset(n * D.R);
    D.scy.reset(m * D.R);
    for (DevBuf<double>* b : {&D.lx, &D.lg, &D.gc, &D.io_n}) b->reset(n);
    for (DevBuf<double>* b : {&D.ly, &D.lq, &D.glo, &D.ghi, &D.io_m, &D.io_m2}) b->reset(m);
    D.ga.reset(z);
    D.io_z.reset(z);
    for (int k = 0; k < 12; ++k) D.mr[k].reset(k % 2 == 0 ? n : m);
    D.mr_sol_x.reset(n);
    D.mr_sol_y.reset(m);
    for (DevBuf<int>* b : {&D.mr_ff, &D.mr_fs}) b->reset(n + 1);
    for (DevBuf<int>* b : {&D.mr_df, &D.mr_ds}) b->reset(m + 1);
    for (DevBuf<int>* b : {&D.mr_cmap, &D.mr_fidx}) b->reset(n);
    for (DevBuf<int>* b : {&D.mr_rmap, &D.mr_didx}) b->reset(m);
    D.mr_foff.reset(P.count + 1);
    D.mr_doff.reset(P.count + 1);
    D.mr_scan.reset(std::max(scan_tiles(n + 1), scan_tiles(m + 1)));
    D.b_ptr.reset(m + 1);
    D.bt_ptr.reset(n + 1);
    D.b_idx.reset(padded_nnz(z));  // B and B^T hold at most A's nonzeros
    D.bt_idx.reset(padded_nnz(z));
    D.b_val.reset(padded_nnz(z));
    D.bt_val.reset(padded_nnz(z));
    D.mst.reset(P.count);
    {  // an instance no solve has selected yet counts as finished
        std::vector<MrState> idle(P.count);
        std::memset(idle.data(), 0, sizeof(MrState) * idle.size());
        for (MrState& st : idle) st.done = 1;
        D.mst.upload(idle.data(), idle.size(), P.stream);
        GB_CUDA(cudaStreamSynchronize(P.stream));
    }
    D.flags.reset(P.count);
    D.mst_host = static_cast<MrState*>(host_alloc(sizeof(MrState) * P.count));
    D.flags_host = static_cast<int*>(host_alloc(sizeof(int) * P.count));
    D.counts.reset(P.count);
    D.counts_host = static_cast<int2*>(host_alloc(sizeof(int2) * P.count));
    D.info.assign(P.count, gb_diff_info{});
}

inline double kkt_err(const Kkt& k) {
    const double e = std::max(k.rel_p, std::max(k.rel_d, k.rel_gap));
    return std::isfinite(e) ? e : INFINITY;
}

// Active-set repair before the polishing solve.  An instance whose active set
// is not square (|D| dual-active rows != |F| free columns; a nondegenerate
// vertex has a square, nonsingular basis B = A'[D, F]) was read off a point
// whose smallest duals or slacks are within the solve tolerance of zero, so
// one PDHG step classified them wrongly, and its reduced system is
// inconsistent (MINRES would run to its step bound).  Its excess rows (|D| > |F|) leave D smallest |y+| first (equality
// rows never leave); its excess columns (|F| > |D|) go to their nearest finite
// bound, nearest first.  The codes are changed in place (they define the
// reduced system and the polished point) and D.flags selects the repaired
// instances.  Returns whether any instance was repaired.
// `cnt` holds (free columns, dual-active rows) per instance (k_code_counts).
bool repair_active_sets(Diff& D, const std::vector<int>& todo, const int2* cnt) {
    Problem& P = *D.P;
    cudaStream_t s = P.stream;
    std::vector<int> fix;
    for (int k = 0; k < P.count; ++k)
        if (todo[k] && cnt[k].x != cnt[k].y) fix.push_back(k);
    if (fix.empty()) return false;
    const size_t n = D.n(), m = D.m();
    std::vector<i8> cx(n), cy(m);
    std::vector<double> x1(n), y1(m), l(n), u(n), lo(m), hi(m);
    GB_CUDA(cudaMemcpyAsync(cx.data(), D.cx_at(0), n, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(cy.data(), D.cy_at(0), m, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(x1.data(), D.x_at(1), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(y1.data(), D.y_at(1), m * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(l.data(), P.l.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(u.data(), P.u.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(lo.data(), P.lo.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaMemcpyAsync(hi.data(), P.hi.get(), m * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < P.count; ++k) D.flags_host[k] = 0;
    bool any = false;
    for (int k : fix) {
        const int c0 = P.col_off[k], c1 = P.col_off[k + 1], r0 = P.row_off[k], r1 = P.row_off[k + 1];
        std::vector<std::pair<double, int>> cand;
        const int excess = cnt[k].y - cnt[k].x;
        if (excess > 0) {
            for (int i = r0; i < r1; ++i)
                if (cy[i] != 0 && lo[i] < hi[i]) cand.push_back({std::fabs(y1[i]), i});
        } else {
            for (int j = c0; j < c1; ++j) {
                if (cx[j] != 1) continue;
                double d = INFINITY;
                if (std::isfinite(l[j])) d = std::min(d, x1[j] - l[j]);
                if (std::isfinite(u[j])) d = std::min(d, u[j] - x1[j]);
                if (std::isfinite(d)) cand.push_back({d, j});
            }
        }
        const int need = std::abs(excess);
        if (static_cast<int>(cand.size()) < need) continue;
        std::partial_sort(cand.begin(), cand.begin() + need, cand.end());
        for (int t = 0; t < need; ++t) {
            const int e = cand[t].second;
            if (excess > 0) cy[e] = 0;
            else cx[e] = (std::isfinite(l[e]) && (!std::isfinite(u[e]) || x1[e] - l[e] <= u[e] - x1[e])) ? 0 : 2;
        }
        D.flags_host[k] = 1;
        D.info[k].active_set_repaired = 1;
        any = true;
    }
    if (!any) return false;
    GB_CUDA(cudaMemcpyAsync(D.cx_at(0), cx.data(), n, cudaMemcpyHostToDevice, s));
    GB_CUDA(cudaMemcpyAsync(D.cy_at(0), cy.data(), m, cudaMemcpyHostToDevice, s));
    D.flags.upload(D.flags_host, P.count, s);
    GB_CUDA(cudaStreamSynchronize(s));  // the host vectors above go out of scope
    return true;
}

// Polishing (the reduced KKT solve of OSQP-style solvers): per instance in
// `todo`, replace the PDHG point by the vertex of the active set one PDHG step
// reads off it -- when that vertex certifies within accept_tol in FP64
// (accept_tol > 0), else when it certifies better than the PDHG point.
// Instances outside `todo` keep their point untouched.
void polish(Diff& D, double accept_tol, const std::vector<int>& todo) {
    Problem& P = *D.P;
    cudaStream_t s = P.stream;
    const int n = P.n, m = P.m;
    const size_t nb = D.n() * sizeof(double), mb = D.m() * sizeof(double);
    const int gv = elem_grid(std::max(n, m), P.sms);
    std::vector<double> err0(P.count);
    for (int k = 0; k < P.count; ++k) err0[k] = kkt_err(P.st_host[k].kcert);
    // PDHG point -> sx[0], sy[0]; one step for the codes
    GB_CUDA(cudaMemcpyAsync(D.x_at(0), P.x64.get(), nb, cudaMemcpyDeviceToDevice, s));
    GB_CUDA(cudaMemcpyAsync(D.y_at(0), P.y64.get(), mb, cudaMemcpyDeviceToDevice, s));
    D.run_segment(1);
    D.seg_valid = -1;
    double* rhs_x = D.lx.get();   // adjoint buffers are free during the forward
    double* rhs_y = D.ly.get();
    double* xn = D.lg.get();
    auto rhs = [&]() {
        k_polish_rhs_cols<<<gv, kThreads, 0, s>>>(n, D.cx_at(0), P.c.get(), P.l.get(), P.u.get(), rhs_x, xn);
        if (P.A.sched.nb) {
            PolishRowEpi e{D.cy_at(0), P.lo.get(), P.hi.get(), rhs_y};
            k_polish_rhs_rows<<<P.A.sched.nb, kThreads, spmv_smem_bytes<1, double>(), s>>>(P.A.view<double>(), xn,
                                                                                           e);
        }
        D.launches += 2;
    };
    StageTrace tr{s, "polish"};
    // A nondegenerate vertex has a square basis (|F| = |D|); a non-square
    // active set makes the reduced system inconsistent, on which MINRES would
    // only stop at its step bound, so it is repaired before the solve.
    k_code_counts<<<P.count, kThreads, 0, s>>>(P.d_col_off.get(), P.d_row_off.get(), D.cx_at(0), D.cy_at(0),
                                               D.counts.get());
    GB_CUDA(cudaMemcpyAsync(D.counts_host, D.counts.get(), sizeof(int2) * P.count, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    repair_active_sets(D, todo, D.counts_host);
    rhs();
    for (int k = 0; k < P.count; ++k) D.flags_host[k] = todo[k];
    D.flags.upload(D.flags_host, P.count, s);
    tr.mark("step + repair + rhs");
    D.minres(rhs_x, rhs_y, D.flags.get());
    tr.mark("minres");
    for (int k = 0; k < P.count; ++k) {
        D.flags_host[k] = todo[k] && D.mst_host[k].converged ? 1 : 0;
        if (todo[k]) D.info[k].polish_iterations = D.mst_host[k].it;
    }
    D.flags.upload(D.flags_host, P.count, s);
    k_polish_point<<<gv, kThreads, 0, s>>>(n, m, P.icol(), P.irow(), D.flags.get(), D.cx_at(0), D.cy_at(0),
                                          D.mr_sol_x.get(), D.mr_sol_y.get(), P.l.get(), P.u.get(), P.x64.get(),
                                          P.y64.get());
    certify(P);
    bool any_restore = false;
    for (int k = 0; k < P.count; ++k) {
        if (!todo[k]) {
            D.flags_host[k] = 0;
            continue;
        }
        const double e = kkt_err(P.st_host[k].kcert);
        const bool keep = D.flags_host[k] && (accept_tol > 0.0 ? e <= accept_tol * 1.0000001 : e < err0[k]);
        D.info[k].polished = keep ? 1 : 0;
        D.flags_host[k] = keep ? 0 : 1;
        any_restore |= !keep;
    }
    if (any_restore) {
        D.flags.upload(D.flags_host, P.count, s);
        k_restore<<<gv, kThreads, 0, s>>>(n, m, P.icol(), P.irow(), D.flags.get(), D.x_at(0), D.y_at(0), P.x64.get(),
                                         P.y64.get());
        D.launches += 1;
    }
    D.launches += 3;
}

// Tolerance at which polishing is first tried when the layer asks for a
// tighter one.  Measured on the 256-LP, 500 x 1000 workload (mixed precision,
// to 1e-6): the vertex read off the 1e-4 point certifies for 251 of 256
// instances, and solving to 1e-4 takes 6,792 iterations at most against 88,200
// to 1e-6.  Forward time by first tolerance (each later round ten times
// tighter): 1e-4 0.238 s, 2e-4 0.176 s, 4e-4 0.170 s (two rounds), 1e-3
// 0.240 s (three rounds); every instance certified and polished each time.
constexpr double kPolishFirstTol = 4e-4;
// Each later round's tolerance over the previous one's.  Measured with the
// first round at 4e-4 (forward, same workload): 0.1 (4e-4, 4e-5) 0.143 s, 0.25
// (4e-4, 1e-4) 0.123 s; from 2e-4 with 0.25 0.126 s, from 1e-3 with 0.25 (four
// rounds) 0.178 s.
constexpr double kPolishRoundFactor = 0.25;

void diff_forward(Diff& D, const gb_options* opt, gb_result* res, double* x_out, double* y_out) {
    Problem& P = *D.P;
    cudaStream_t s = P.stream;
    const int K = P.count;
    const int gv = elem_grid(std::max(P.n, P.m), P.sms);
    std::vector<gb_result> tmp(K);
    gb_result* r = res ? res : tmp.data();
    D.info.assign(K, gb_diff_info{});
    D.tau_h.assign(K, 0.0);
    D.sig_h.assign(K, 0.0);
    // Progressive polishing: solve to a loose tolerance, keep the instances
    // whose polished vertex certifies at the requested one, and go on (warm
    // started from their points, tolerance x kPolishRoundFactor per round) only with the
    // others; the last round solves to the requested tolerance and polishes
    // as a single-round forward does.
    const double target = opt->tol;
    gb_options o = *opt;
    // (only when polishing can succeed: its reduced solve shares the MINRES
    // step bound, and a forward with no polishing keeps one cold solve)
    o.tol = D.polish && D.mr_max > 0 && target < kPolishFirstTol ? kPolishFirstTol : target;
    std::vector<int> todo(K, 1), kept(K, 0);
    // the first round starts cold, whatever an interrupted forward left behind
    P.x_start.release();
    P.y_start.release();
    P.w_start.release();
    std::vector<long long> its(K, 0);
    long long launches = 0;
    bool any_kept = false;
    StageTrace tr{s, "diff forward"};
    char lab[48];
    for (;;) {
        solve_problem(P, &o, r);
        launches += P.launches;
        std::snprintf(lab, sizeof lab, "solve to %.0e", o.tol);
        tr.mark(lab);
        for (int k = 0; k < K; ++k) {
            its[k] += r[k].iterations;
            if (!todo[k]) continue;
            // tail step sizes from the final primal weight (pdhg_impl.hpp:87-91, LP)
            const SolveState& st = P.st_host[k];
            D.tau_h[k] = st.eta / st.w;
            D.sig_h[k] = st.eta * st.w;
        }
        D.tau.upload(D.tau_h.data(), K, s);
        D.sig.upload(D.sig_h.data(), K, s);
        if (!D.polish) break;
        const bool last = o.tol <= target;
        polish(D, last ? -1.0 : target, todo);
        tr.mark("polish");
        if (last) break;
        int left = 0;
        for (int k = 0; k < K; ++k) {
            D.flags_host[k] = todo[k] && D.info[k].polished ? 1 : 0;  // certified at the target: done
            if (D.flags_host[k]) todo[k] = 0, kept[k] = 1, any_kept = true;
            left += todo[k];
        }
        if (!D.kx.get()) {
            D.kx.reset(std::max<size_t>(D.n(), 1));
            D.ky.reset(std::max<size_t>(D.m(), 1));
        }
        D.flags.upload(D.flags_host, K, s);
        k_restore<<<gv, kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), D.flags.get(), P.x64.get(), P.y64.get(),
                                         D.kx.get(), D.ky.get());  // keep the certified vertices
        launches += 1;
        if (left == 0) break;
        // the next round starts every instance from its current point (original units)
        // and primal weight
        k_unscale<<<gv, kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), P.x64.get(), P.y64.get(), P.C.get(),
                                         P.R.get(), P.scal.get(), P.xo.get(), P.yo.get());
        if (!P.x_start.get()) {
            P.x_start.reset(std::max(P.n, 1));
            P.y_start.reset(std::max(P.m, 1));
        }
        {  // and with its final primal weight, not the cold default
            std::vector<double> w(K);
            for (int k = 0; k < K; ++k) w[k] = P.st_host[k].w;
            P.w_start.reset(K);
            P.w_start.upload(w.data(), K, s);
        }
        GB_CUDA(cudaMemcpyAsync(P.x_start.get(), P.xo.get(), D.n() * sizeof(double), cudaMemcpyDeviceToDevice, s));
        GB_CUDA(cudaMemcpyAsync(P.y_start.get(), P.yo.get(), D.m() * sizeof(double), cudaMemcpyDeviceToDevice, s));
        launches += 1;
        o.tol = std::max(target, o.tol * kPolishRoundFactor);
    }
    if (P.x_start.get()) {  // the next forward starts cold again
        P.x_start.release();
        P.y_start.release();
    }
    P.w_start.release();
    if (any_kept) {  // vertices certified in an earlier round replace what later rounds left there
        for (int k = 0; k < K; ++k) D.flags_host[k] = kept[k];
        D.flags.upload(D.flags_host, K, s);
        k_restore<<<gv, kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), D.flags.get(), D.kx.get(), D.ky.get(),
                                         P.x64.get(), P.y64.get());
        launches += 1;
        for (int k = 0; k < K; ++k)
            if (kept[k]) D.info[k].polished = 1;
    }
    for (int k = 0; k < K; ++k) r[k].iterations = its[k];
    D.launches = launches;
    const size_t nb = D.n() * sizeof(double), mb = D.m() * sizeof(double);
    GB_CUDA(cudaMemcpyAsync(D.x_at(0), P.x64.get(), nb, cudaMemcpyDeviceToDevice, s));
    GB_CUDA(cudaMemcpyAsync(D.y_at(0), P.y64.get(), mb, cudaMemcpyDeviceToDevice, s));
    for (int seg = 0; seg < D.nseg; ++seg) {
        if (seg > 0) {
            GB_CUDA(cudaMemcpyAsync(D.x_at(0), D.x_at(D.R), nb, cudaMemcpyDeviceToDevice, s));
            GB_CUDA(cudaMemcpyAsync(D.y_at(0), D.y_at(D.R), mb, cudaMemcpyDeviceToDevice, s));
        }
        GB_CUDA(cudaMemcpyAsync(D.ck_x.get() + seg * D.n(), D.x_at(0), nb, cudaMemcpyDeviceToDevice, s));
        GB_CUDA(cudaMemcpyAsync(D.ck_y.get() + seg * D.m(), D.y_at(0), mb, cudaMemcpyDeviceToDevice, s));
        D.run_segment(D.R);
    }
    D.seg_valid = D.nseg - 1;
    tr.mark("tail");
    // the layer's output z_K, certified in FP64 and unscaled
    GB_CUDA(cudaMemcpyAsync(P.x64.get(), D.x_at(D.R), nb, cudaMemcpyDeviceToDevice, s));
    GB_CUDA(cudaMemcpyAsync(P.y64.get(), D.y_at(D.R), mb, cudaMemcpyDeviceToDevice, s));
    certify(P);
    k_unscale<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), P.x64.get(),
                                                                     P.y64.get(), P.C.get(), P.R.get(), P.scal.get(),
                                                                     P.xo.get(), P.yo.get());
    D.launches += 2;
    if (x_out) GB_CUDA(cudaMemcpyAsync(x_out, P.xo.get(), nb, cudaMemcpyDeviceToHost, s));
    if (y_out) GB_CUDA(cudaMemcpyAsync(y_out, P.yo.get(), mb, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    GB_CUDA(cudaGetLastError());
    for (int k = 0; k < P.count; ++k) {
        const Kkt& f = P.st_host[k].kcert;
        const double sign = P.maximize[k] ? -1.0 : 1.0;
        r[k].pobj = sign * f.pobj;
        r[k].dobj = sign * f.dobj;
        r[k].rel_primal = f.rel_p;
        r[k].rel_dual = f.rel_d;
        r[k].rel_gap = f.rel_gap;
        r[k].iterations += D.K;
        if (r[k].status == GB_OPTIMAL &&
            !(f.rel_p <= opt->tol * 1.0000001 && f.rel_d <= opt->tol * 1.0000001 && f.rel_gap <= opt->tol * 1.0000001))
            r[k].status = GB_NUMERICAL_ERROR;
        gb_diff_info& in = D.info[k];
        in.tau = D.tau_h[k];
        in.sigma = D.sig_h[k];
        in.tail_iterations = D.K;
        in.checkpoint_every = D.R;
        in.free_cols = in.active_rows = -1;
    }
    D.forward_done = true;
    D.backward_done = false;
}

void diff_backward(Diff& D, const double* dl_dx, const double* dl_dy, double* dl_dc, double* dl_dlo, double* dl_dhi,
                   double* dl_dval) {
    GB_REQUIRE(D.forward_done, "gb_diff_backward before gb_diff_forward");
    Problem& P = *D.P;
    cudaStream_t s = P.stream;
    const int n = P.n, m = P.m, nnz = static_cast<int>(P.A.nnz);
    const size_t nb = D.n() * sizeof(double), mb = D.m() * sizeof(double);
    const int gv = elem_grid(std::max(n, m), P.sms), gz = elem_grid(std::max<long long>(nnz, 1), P.sms);
    const int gall = elem_grid(std::max<long long>(std::max(n, m), nnz), P.sms);
    D.launches = 0;
    // upstream adjoint in scaled space
    if (dl_dx) D.io_n.upload(dl_dx, D.n(), s);
    else GB_CUDA(cudaMemsetAsync(D.io_n.get(), 0, nb, s));
    if (dl_dy) D.io_m.upload(dl_dy, D.m(), s);
    else GB_CUDA(cudaMemsetAsync(D.io_m.get(), 0, mb, s));
    k_adjoint_in<<<gv, kThreads, 0, s>>>(n, m, P.icol(), P.irow(), P.scal.get(), P.C.get(), P.R.get(), D.io_n.get(),
                                         D.io_m.get(), D.lx.get(), D.ly.get());
    GB_CUDA(cudaMemsetAsync(D.gc.get(), 0, nb, s));
    GB_CUDA(cudaMemsetAsync(D.glo.get(), 0, mb, s));
    GB_CUDA(cudaMemsetAsync(D.ghi.get(), 0, mb, s));
    GB_CUDA(cudaMemsetAsync(D.ga.get(), 0, D.ga.size() * sizeof(double), s));
    D.launches += 1;

    StageTrace tr{s, "diff backward"};
    // 3. reverse through the tail, last segment first
    const size_t smem = spmv_smem_bytes<1, double>();
    const CsrView<double> A = P.A.view<double>(), AT = P.AT.view<double>();
    for (int seg = D.nseg - 1; seg >= 0; --seg) {
        if (seg != D.seg_valid) D.recompute(seg);
        k_rev_start<<<gv, kThreads, 0, s>>>(m, P.irow(), D.cy_at(D.R - 1), D.sig.get(), D.ly.get(), D.lq.get(),
                                            D.glo.get(), D.ghi.get());
        D.launches += 1;
        for (int k = D.R - 1; k >= 0; --k) {
            if (AT.nb) {
                RevColEpi e{D.cx_at(k), D.tau.get(), D.sig.get(), D.lx.get(), D.lg.get(), D.gc.get(), 0.0, 0.0};
                launch_pdl(k_rev_cols, AT.nb, kThreads, smem, s, AT, static_cast<const double*>(D.lq.get()), e);
            }
            if (nnz)
                launch_pdl(k_rev_da, gz, kThreads, 0, s, nnz, static_cast<const int*>(P.row_of.get()),
                           static_cast<const int*>(P.A.idx.get()), P.irow(), static_cast<const double*>(D.sig.get()),
                           static_cast<const double*>(D.lq.get()), static_cast<const double*>(D.xb_at(k)),
                           static_cast<const double*>(D.y_at(k)), static_cast<const double*>(D.lg.get()), D.ga.get());
            if (A.nb) {
                RevRowEpi e{k > 0 ? D.cy_at(k - 1) : nullptr, D.sig.get(), D.lq.get(), D.ly.get(), D.glo.get(),
                            D.ghi.get(), 0.0};
                launch_pdl(k_rev_rows, A.nb, kThreads, smem, s, A, static_cast<const double*>(D.lg.get()), e);
            }
            D.launches += 3;
        }
    }
    // (lx, ly) now hold mu_0, the adjoint at the tail start; segment 0's step 0 is resident.

    tr.mark("reverse pass");
    // 4. implicit completion
    if (D.mr_max > 0) {
        D.minres(D.lx.get(), D.ly.get());
        tr.mark("completion");
        k_implicit_grads<<<gall, kThreads, 0, s>>>(n, m, nnz, P.row_of.get(), P.A.idx.get(), D.cy_at(0),
                                                   D.mr_sol_x.get(), D.mr_sol_y.get(), D.xb_at(0), D.y_at(0),
                                                   D.gc.get(), D.glo.get(), D.ghi.get(), D.ga.get());
        D.launches += 1;
        for (int k = 0; k < P.count; ++k) {
            const MrState& st = D.mst_host[k];
            gb_diff_info& in = D.info[k];
            in.implicit_iterations = st.it;
            in.implicit_residual = st.beta1 > 0.0 ? st.phibar / st.beta1 : 0.0;
            in.implicit_converged = st.converged;
            in.free_cols = st.free_cols;
            in.active_rows = st.active_rows;
        }
    }

    // 5. back to the original data
    k_grads_out<<<gall, kThreads, 0, s>>>(n, m, nnz, P.icol(), P.irow(), P.row_of.get(), P.A.idx.get(), P.scal.get(),
                                          P.C.get(), P.R.get(), D.gc.get(), D.glo.get(), D.ghi.get(), D.ga.get(),
                                          D.io_n.get(), D.io_m.get(), D.io_m2.get(), D.io_z.get());
    D.launches += 1;
    // an instance whose completion did not converge gets NaN gradients (all bytes 0xff), not unverified values
    if (D.mr_max > 0)
        for (int k = 0; k < P.count; ++k) {
            if (D.mst_host[k].converged) continue;
            const size_t c0 = P.col_off[k], c1 = P.col_off[k + 1], r0 = P.row_off[k], r1 = P.row_off[k + 1];
            const size_t z0 = P.nnz_off[k], z1 = P.nnz_off[k + 1];
            GB_CUDA(cudaMemsetAsync(D.io_n.get() + c0, 0xff, (c1 - c0) * sizeof(double), s));
            GB_CUDA(cudaMemsetAsync(D.io_m.get() + r0, 0xff, (r1 - r0) * sizeof(double), s));
            GB_CUDA(cudaMemsetAsync(D.io_m2.get() + r0, 0xff, (r1 - r0) * sizeof(double), s));
            if (z1 > z0) GB_CUDA(cudaMemsetAsync(D.io_z.get() + z0, 0xff, (z1 - z0) * sizeof(double), s));
        }
    if (dl_dc) GB_CUDA(cudaMemcpyAsync(dl_dc, D.io_n.get(), nb, cudaMemcpyDeviceToHost, s));
    if (dl_dlo) GB_CUDA(cudaMemcpyAsync(dl_dlo, D.io_m.get(), mb, cudaMemcpyDeviceToHost, s));
    if (dl_dhi) GB_CUDA(cudaMemcpyAsync(dl_dhi, D.io_m2.get(), mb, cudaMemcpyDeviceToHost, s));
    if (dl_dval && nnz) GB_CUDA(cudaMemcpyAsync(dl_dval, D.io_z.get(), D.nnz() * sizeof(double), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    GB_CUDA(cudaGetLastError());
    D.backward_done = true;
}

}  // namespace gb

struct gb_diff {
    std::unique_ptr<gb::Diff> d;
};

extern "C" {

void gb_diff_default_options(gb_diff_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->implicit_max_iters = 20000;
    o->implicit_tol = 1e-10;
    o->polish = 1;
}

int gb_diff_create(int count, const gb_lp* lps, const gb_options* opt, int tail_iters, int ckpt_every,
                   gb_diff** out) {
    return gb::guarded([&] {
        GB_REQUIRE(out != nullptr, "out is NULL");
        *out = nullptr;
        GB_REQUIRE(count >= 1 && lps != nullptr, "need at least one problem");
        GB_REQUIRE(tail_iters >= 1 && ckpt_every >= 1 && tail_iters % ckpt_every == 0,
                   "tail_iters must be a positive multiple of ckpt_every");
        for (int k = 0; k < count; ++k)
            GB_REQUIRE(lps[k].q_ptr == nullptr && lps[k].q_rank == 0, "the differentiable layer takes LPs only");
        gb_options o;
        if (opt) o = *opt;
        else gb_default_options(&o);
        auto D = std::make_unique<gb::Diff>();
        D->P.reset(gb::create_problem(count, lps, &o));
        D->K = tail_iters;
        D->R = ckpt_every;
        D->nseg = tail_iters / ckpt_every;
        gb::diff_alloc(*D);
        *out = new gb_diff{std::move(D)};
    });
}

int gb_diff_set_options(gb_diff* d, const gb_diff_options* o) {
    return gb::guarded([&] {
        GB_REQUIRE(d != nullptr && o != nullptr, "null argument");
        GB_REQUIRE(o->implicit_max_iters >= 0 && o->implicit_tol > 0.0,
                   "implicit_max_iters must be >= 0 and implicit_tol > 0");
        d->d->mr_max = o->implicit_max_iters;
        d->d->mr_tol = o->implicit_tol;
        d->d->polish = o->polish != 0;
    });
}

int gb_diff_forward(gb_diff* d, const gb_options* opt, gb_result* results, double* x_out, double* y_out) {
    return gb::guarded([&] {
        GB_REQUIRE(d != nullptr, "null handle");
        gb_options o;
        if (opt) o = *opt;
        else gb_default_options(&o);
        GB_CUDA(cudaSetDevice(d->d->P->device));
        gb::diff_forward(*d->d, &o, results, x_out, y_out);
    });
}

int gb_diff_backward(gb_diff* d, const double* dl_dx, const double* dl_dy, double* dl_dc, double* dl_dlo,
                     double* dl_dhi, double* dl_dval) {
    return gb::guarded([&] {
        GB_REQUIRE(d != nullptr, "null handle");
        GB_CUDA(cudaSetDevice(d->d->P->device));
        gb::diff_backward(*d->d, dl_dx, dl_dy, dl_dc, dl_dlo, dl_dhi, dl_dval);
    });
}

int gb_diff_get_info(gb_diff* d, int i, gb_diff_info* out) {
    return gb::guarded([&] {
        GB_REQUIRE(d != nullptr && out != nullptr, "null argument");
        gb::Diff& D = *d->d;
        GB_REQUIRE(i >= 0 && i < D.P->count, "instance index out of range");
        GB_REQUIRE(D.forward_done, "no forward pass yet");
        *out = D.info[i];
        out->launches = D.launches;
    });
}

int gb_diff_tail_start(gb_diff* d, double* x_scaled, double* y_scaled) {
    return gb::guarded([&] {
        GB_REQUIRE(d != nullptr, "null handle");
        gb::Diff& D = *d->d;
        GB_REQUIRE(D.forward_done, "no forward pass yet");
        cudaStream_t s = D.P->stream;
        if (x_scaled) GB_CUDA(cudaMemcpyAsync(x_scaled, D.ck_x.get(), D.n() * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (y_scaled) GB_CUDA(cudaMemcpyAsync(y_scaled, D.ck_y.get(), D.m() * sizeof(double), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
    });
}

void gb_diff_destroy(gb_diff* d) { delete d; }

}  // extern "C"

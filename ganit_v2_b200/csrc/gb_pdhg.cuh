// Fused restarted-PDHG kernels over a batch of instances (one instance = the
// single-problem case).
//
// A batch is one block-diagonal problem: instance k owns rows
// [row_off[k], row_off[k+1]) of A and columns [col_off[k], col_off[k+1]); every
// row block of the schedules belongs to exactly one instance, so a block reads
// its instance's step sizes and is skipped once that instance has stopped
// iterating.
//
// Per iteration (src/pdhg_impl.hpp:133-139) two launches:
//   k_primal : rows j of the stored transpose: aty_j = (A^T y)_j, then the
//              primal step of src/backend_cpu.cpp:67-80 in the epilogue
//              (x+ = clamp(x - tau (c - aty + qx)), xbar = 2x+ - x, sumx += x+)
//   k_dual   : rows i of A: ax_i = (A xbar)_i, then the dual step of
//              src/backend_cpu.cpp:81-92 (y+ = q + clamp(-q, sigma lo, sigma hi))
// Every check_every iterations (pdhg_impl.hpp:142-190) one k_eval launch
// computes, for the current iterate, the running average and the ray y - y_r,
// all KKT pieces of pdhg_impl.hpp:92-118 in FP64 (one pass over A and one
// over A^T, several right-hand sides per pass) as per-CTA partial sums; then
// the one-CTA k_decide reduces each instance's partials in a fixed order and
// runs, one thread per instance, the whole scalar decision of
// pdhg_impl.hpp:144-189 (convergence, limits, infeasibility certificate,
// stall exit, adaptive restart, primal weight).  The decision is a separate
// kernel because its registers (~100 per thread) would otherwise be
// allocated to every CTA of k_eval's grid.  k_restart applies restarts.  No
// host round trip happens inside a precision phase.
#pragma once
#include "gb_spmv.cuh"

namespace gb {

struct Kkt {
    double pobj, dobj, rel_p, rel_d, rel_gap, err;
};

// Phase exits (pdhg_impl.hpp:65)
enum PhaseExit : int {
    kConverged = 0, kStalled = 1, kIterLimit = 2, kTimeLimit = 3, kInfeasible = 4, kNumerical = 5,
    kUnbounded = 6  // extension: primal ray certificate of dual infeasibility
};
enum EvalMode : int { kEvalInit = 0, kEvalCheck = 1, kEvalCertify = 2 };

// Device-resident solver state of one instance (PdhgShared + PdhgState + loop
// locals of pdhg_impl.hpp:44-63, 120-128).  Scalars are FP64.
struct alignas(16) SolveState {
    // problem constants
    double eta, normA, normQ, obj_scale, obj_const, bnorm, cnorm;
    double phase_tol, infeas_tol, time_limit_s;
    long long max_iter;
    int check_every, stall_checks, stall_exit, has_q;
    unsigned long long t0_ns;
    // carried across phases (PdhgState)
    double w;
    long long it;
    int restarts;
    int checks;
    double carry_restart_err;  // st.restart_err (-1 = none)
    // phase loop locals
    double tau, sigma;
    long long it_since;
    double restart_err, prev_cand, best_err;
    int cwp;                   // checks without progress
    // decision of the last check
    int restart_now, avg_better, done, exit_reason, best_is_avg;
    double inv_avg;
    Kkt best, kcert, kc, ka;
    int active;                // iterating in the current phase
    int in_phase;              // took part in the current phase
    int ran_body;              // iterated during the body that ended at the last check
    int detect_unbounded;      // test the primal ray (extension, LPs)
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// "Active" flag of an instance read before the programmatic-launch wait (a
// prefetching kernel's hint): possibly stale, but inside a phase the flag only
// goes from 1 to 0 (k_decide clears it; it is set only by the phase set-up
// before the phase's graph starts), so a stale value only errs towards true.
__device__ __forceinline__ bool active_hint(const SolveState* st, int inst) {
    return *reinterpret_cast<const volatile int*>(&st[inst].active) != 0;
}

// ---------------------------------------------------------------- iteration kernels
// Minimum resident CTAs per SM requested from the register allocator.
template <class V>
constexpr int kMinCtas = sizeof(V) == 4 ? 8 : 6;

template <class M, class V>
struct PrimalArgs {
    CsrView<M> AT;
    const V* __restrict__ y;     // gathered by column index of A^T (row of A)
    const V* __restrict__ x;
    const V* __restrict__ c;
    const V* __restrict__ l;
    const V* __restrict__ u;
    const V* __restrict__ qx;    // Q x or nullptr
    V* __restrict__ xn;
    V* __restrict__ xbar;
    V* __restrict__ sumx;
    const SolveState* st;       // per instance
};

template <class M, class V>
struct PrimalEpi {
    const PrimalArgs<M, V>* a;  // kernel parameter space (__grid_constant__)
    V tau;
    __device__ __forceinline__ bool begin(int inst) {
        const SolveState& s = a->st[inst];
        tau = static_cast<V>(s.tau);
        return s.active != 0;
    }
    __device__ __forceinline__ bool hint(int inst) const { return active_hint(a->st, inst); }
    __device__ __forceinline__ void l2_prefetch_rows(int r0, int r1) const {
        const size_t k = sizeof(V) * static_cast<size_t>(r1 - r0);
        l2_prefetch(a->x + r0, k);
        l2_prefetch(a->c + r0, k);
        l2_prefetch(a->l + r0, k);
        l2_prefetch(a->u + r0, k);
        l2_prefetch(a->sumx + r0, k);
        if (a->qx) l2_prefetch(a->qx + r0, k);
    }
    struct Pre {
        V x, c, l, u, sumx, qx;
    };
    __device__ __forceinline__ Pre prefetch(int j) const {
        return Pre{a->x[j], a->c[j], a->l[j], a->u[j], a->sumx[j], a->qx ? a->qx[j] : V(0)};
    }
    __device__ __forceinline__ void operator()(int j, const V (&s)[1], const Pre& p) const {
        const V g = p.c - s[0] + p.qx;
        V v = p.x - tau * g;
        v = (v < p.l) ? p.l : v;
        v = (p.u < v) ? p.u : v;
        a->xn[j] = v;
        a->xbar[j] = V(2) * v - p.x;
        a->sumx[j] = p.sumx + v;
    }
};

template <class M, class V, int L = kLoadPlain>
__global__ void __launch_bounds__(kThreads, kMinCtas<V>) k_primal(const __grid_constant__ PrimalArgs<M, V> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    PrimalEpi<M, V> epi{&a, V(0)};
    if constexpr (L == kLoadPrefetch) {
        spmv_run_prefetched<M, V>(a.AT, blockIdx.x, GatherOne<V>{a.y}, epi, smem);
    } else {
        pdl_enter();
        spmv_run_iter<M, V, L == kLoadStream>(a.AT, blockIdx.x, GatherOne<V>{a.y}, epi, smem);
    }
}

template <class M, class V>
struct DualArgs {
    CsrView<M> A;
    const V* __restrict__ xbar;
    const V* __restrict__ y;
    const V* __restrict__ lo;
    const V* __restrict__ hi;
    V* __restrict__ yn;
    V* __restrict__ sumy;
    const SolveState* st;       // per instance
};

template <class M, class V>
struct DualEpi {
    const DualArgs<M, V>* a;  // kernel parameter space (__grid_constant__)
    V sigma;
    __device__ __forceinline__ bool begin(int inst) {
        const SolveState& s = a->st[inst];
        sigma = static_cast<V>(s.sigma);
        return s.active != 0;
    }
    __device__ __forceinline__ bool hint(int inst) const { return active_hint(a->st, inst); }
    __device__ __forceinline__ void l2_prefetch_rows(int r0, int r1) const {
        const size_t k = sizeof(V) * static_cast<size_t>(r1 - r0);
        l2_prefetch(a->y + r0, k);
        l2_prefetch(a->lo + r0, k);
        l2_prefetch(a->hi + r0, k);
        l2_prefetch(a->sumy + r0, k);
    }
    struct Pre {
        V y, lo, hi, sumy;
    };
    __device__ __forceinline__ Pre prefetch(int i) const { return Pre{a->y[i], a->lo[i], a->hi[i], a->sumy[i]}; }
    __device__ __forceinline__ void operator()(int i, const V (&s)[1], const Pre& p) const {
        const V q = p.y - sigma * s[0];
        const V l = sigma * p.lo, h = sigma * p.hi;
        V t = -q;
        t = (t < l) ? l : t;
        t = (h < t) ? h : t;
        const V v = q + t;
        a->yn[i] = v;
        a->sumy[i] = p.sumy + v;
    }
};

template <class M, class V, int L = kLoadPlain>
__global__ void __launch_bounds__(kThreads, kMinCtas<V>) k_dual(const __grid_constant__ DualArgs<M, V> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    DualEpi<M, V> epi{&a, V(0)};
    if constexpr (L == kLoadPrefetch) {
        spmv_run_prefetched<M, V>(a.A, blockIdx.x, GatherOne<V>{a.xbar}, epi, smem);
    } else {
        pdl_enter();
        spmv_run_iter<M, V, L == kLoadStream>(a.A, blockIdx.x, GatherOne<V>{a.xbar}, epi, smem);
    }
}

// ---------------------------------------------------------------- KKT evaluation
// FP64 partial sums written by every CTA of k_eval: the row pass (A) forms
// the first kRowTerms, the column pass (A^T) the rest, so a CTA carries only
// its own pass's accumulators (register pressure sets k_eval's occupancy).
enum Term : int {
    T_RP2_C = 0, T_RP2_A, T_ROBJ_C, T_ROBJ_A, T_ROBJ_R, T_DY2_C, T_DY2_A,
    T_UR2,  // primal ray d = x - x_r: row recession violation^2
    kRowTerms,
    T_RD2_C = kRowTerms, T_VOBJ_C, T_RD2_A, T_VOBJ_A, T_RD2_R, T_VOBJ_R, T_CX_C, T_CX_A, T_XQX_C, T_XQX_A,
    T_DX2_C, T_DX2_A,
    T_UC2, T_CD,  // primal ray: column recession violation^2, c'd
    kTerms
};
constexpr int kColTerms = kTerms - kRowTerms;

template <class M, class V>
struct EvalArgs {
    CsrView<M> A, AT;
    const V* __restrict__ x;
    const V* __restrict__ y;
    const V* __restrict__ sumx;
    const V* __restrict__ sumy;
    const V* __restrict__ xr;
    const V* __restrict__ yr;
    const V* __restrict__ c;
    const V* __restrict__ l;
    const V* __restrict__ u;
    const V* __restrict__ lo;
    const V* __restrict__ hi;
    const V* __restrict__ rres;
    const V* __restrict__ cres;
    const V* __restrict__ qx;    // Q x   (QP) or nullptr
    const V* __restrict__ qxa;   // Q xa  (QP, check mode) or nullptr
    int mode;
    int count;                   // instances
    const int* seg_a;            // instance k owns A blocks [seg_a[k], seg_a[k+1])
    const int* seg_t;            // and A^T blocks [seg_t[k], seg_t[k+1])
    SolveState* st;              // per instance
    double* partials;            // term-major: [kTerms][A.nb + AT.nb]; a pass writes only its own terms
    double* inst_terms;          // [count][kTerms] scratch of k_decide
    unsigned long long cond;     // cudaGraphConditionalHandle of the phase loop
    int use_cond;                // 1 inside the loop body: the decision drives the loop
    unsigned* sync = nullptr;    // k_decide over several CTAs: {arrivals, any instance active}
    int terms_ready = 0;         // single instance: k_terms summed its terms into inst_terms
};

// k_decide's grid: one CTA for a single problem, else one CTA per
// kDecideInst instances (one instance per warp while reducing).
constexpr int kDecideInst = kWarps;
constexpr int kDecideWide = 128;  // blocks above which an instance's terms are summed by a whole CTA
inline int decide_grid(int count) { return count == 1 ? 1 : (count + kDecideInst - 1) / kDecideInst; }

template <class V>
__device__ __forceinline__ V avg_of(const V* s, int k, double inv) {
    return static_cast<V>(inv * static_cast<double>(s[k]));  // scale_into, backend_cpu.cpp:97-100
}

template <class V, int NV>
struct GatherXAvg {  // A side: x, (check) the running average xa, (unbounded test) the ray x - xr
    const V* __restrict__ x;
    const V* __restrict__ sumx;
    const V* __restrict__ xr;
    double inv;
    __device__ __forceinline__ void operator()(int j, V (&o)[NV]) const {
        const V xj = __ldg(x + j);
        o[0] = xj;
        if (NV > 1) o[NV > 1 ? 1 : 0] = avg_of(sumx, j, inv);
        if (NV > 2) o[NV > 2 ? 2 : 0] = xj - __ldg(xr + j);
    }
};

template <class V, int NV>
struct GatherYAvgRay {  // A^T side: y, ya and the ray y - yr
    const V* __restrict__ y;
    const V* __restrict__ sumy;
    const V* __restrict__ yr;
    double inv;
    __device__ __forceinline__ void operator()(int i, V (&o)[NV]) const {
        const V yi = __ldg(y + i);
        o[0] = yi;
        if (NV > 1) {
            o[NV > 1 ? 1 : 0] = avg_of(sumy, i, inv);
            o[NV > 2 ? 2 : 0] = yi - __ldg(yr + i);
        }
    }
};

// 1 / it_since at the coming check of an instance (the average's weight).
__device__ __forceinline__ double avg_weight(const SolveState& s, int mode) {
    return mode == kEvalCheck ? 1.0 / static_cast<double>(s.it_since + s.check_every) : 0.0;
}

// Evaluated instances: every instance when certifying, else the iterating ones.
__device__ __forceinline__ bool eval_includes(const SolveState& s, int mode) {
    return mode == kEvalCertify || s.active != 0;
}

// Per-row terms (backend_cpu.cpp:101-112, 132-142) and restart distances.
template <class M, class V, int NV>
struct EvalRowEpi {
    const EvalArgs<M, V>& a;  // kernel parameter space (__grid_constant__)
    double inv;
    double t[kRowTerms];  // indexed by the row terms
    __device__ __forceinline__ bool begin(int inst) { return eval_includes(a.st[inst], a.mode); }
    __device__ __forceinline__ static double pres2(double ax, double lo, double hi, double r) {
        double p = (ax < lo) ? lo : ax;
        p = (hi < p) ? hi : p;
        const double d = (ax - p) / r;
        return d * d;
    }
    __device__ __forceinline__ static double robj(double yi, double lo, double hi) {
        if (yi > 0 && isfinite(lo)) return yi * lo;
        if (yi < 0 && isfinite(hi)) return yi * hi;
        return 0.0;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int i, const V (&s)[NV], const NoPre&) {
        const double lo = double(a.lo[i]), hi = double(a.hi[i]), r = double(a.rres[i]);
        const V yi = a.y[i];
        t[T_RP2_C] += pres2(double(s[0]), lo, hi, r);
        t[T_ROBJ_C] += robj(double(yi), lo, hi);
        if (NV > 1) {
            const V ya = avg_of(a.sumy, i, inv);
            const V yri = a.yr[i];
            const V ray = yi - yri;
            t[T_RP2_A] += pres2(double(s[NV > 1 ? 1 : 0]), lo, hi, r);
            t[T_ROBJ_A] += robj(double(ya), lo, hi);
            t[T_ROBJ_R] += robj(double(ray), lo, hi);
            const double d0 = double(yi) - double(yri), d1 = double(ya) - double(yri);
            t[T_DY2_C] += d0 * d0;
            t[T_DY2_A] += d1 * d1;
        }
        if (NV > 2) {  // A d must lie in the row's recession cone: >= 0 if lo finite, <= 0 if hi finite
            const double ad = double(s[NV > 2 ? 2 : 0]);
            double v = 0.0;
            if (isfinite(lo) && ad < 0) v -= ad;
            if (isfinite(hi) && ad > 0) v += ad;
            v /= r;
            t[T_UR2] += v * v;
        }
    }
};

// Per-column terms (backend_cpu.cpp:113-131, 143-149).
template <class M, class V, int NV>
struct EvalColEpi {
    const EvalArgs<M, V>& a;  // kernel parameter space (__grid_constant__)
    double inv;
    double t[kColTerms];  // indexed by the column terms - kRowTerms
    __device__ __forceinline__ bool begin(int inst) { return eval_includes(a.st[inst], a.mode); }
    __device__ __forceinline__ static void dres(double z, double lj, double uj, double cres, double& rd2,
                                                double& ob) {
        double r = 0.0;
        if (z > 0) { if (isfinite(lj)) ob += z * lj; else r = z; }
        else if (z < 0) { if (isfinite(uj)) ob += z * uj; else r = z; }
        r /= cres;
        rd2 += r * r;
    }
    __device__ __forceinline__ NoPre prefetch(int) const { return {}; }
    __device__ __forceinline__ void operator()(int j, const V (&s)[NV], const NoPre&) {
        const double cj = double(a.c[j]), lj = double(a.l[j]), uj = double(a.u[j]), cr = double(a.cres[j]);
        const V xj = a.x[j];
        const double qc = a.qx ? double(a.qx[j]) : 0.0;
        dres(1.0 * cj - double(s[0]) + qc, lj, uj, cr, t[T_RD2_C - kRowTerms], t[T_VOBJ_C - kRowTerms]);
        t[T_CX_C - kRowTerms] += cj * double(xj);
        if (a.qx) t[T_XQX_C - kRowTerms] += double(xj) * qc;
        if (NV > 1) {
            const V xa = avg_of(a.sumx, j, inv);
            const V xrj = a.xr[j];
            const double qa = a.qxa ? double(a.qxa[j]) : 0.0;
            dres(1.0 * cj - double(s[NV > 1 ? 1 : 0]) + qa, lj, uj, cr, t[T_RD2_A - kRowTerms],
                 t[T_VOBJ_A - kRowTerms]);
            dres(0.0 * cj - double(s[NV > 2 ? 2 : 0]) + 0.0, lj, uj, cr, t[T_RD2_R - kRowTerms],
                 t[T_VOBJ_R - kRowTerms]);
            t[T_CX_A - kRowTerms] += cj * double(xa);
            if (a.qxa) t[T_XQX_A - kRowTerms] += double(xa) * qa;
            const double d0 = double(xj) - double(xrj), d1 = double(xa) - double(xrj);
            t[T_DX2_C - kRowTerms] += d0 * d0;
            t[T_DX2_A - kRowTerms] += d1 * d1;
            // the ray within the column's recession cone: >= 0 if l finite, <= 0 if u finite
            const double vc = (isfinite(lj) && d0 < 0 ? -d0 : 0.0) + (isfinite(uj) && d0 > 0 ? d0 : 0.0);
            t[T_UC2 - kRowTerms] += vc * vc;
            t[T_CD - kRowTerms] += cj * d0;
        }
    }
};

// KKT from reduced terms (eval lambda, pdhg_impl.hpp:102-107)
__device__ __forceinline__ Kkt make_kkt(const SolveState& s, double cx, double xqx, double robj, double vobj,
                                        double rp2, double rd2) {
    Kkt k;
    k.pobj = (cx + 0.5 * xqx) * s.obj_scale + s.obj_const;
    k.dobj = (robj + vobj - 0.5 * xqx) * s.obj_scale + s.obj_const;
    k.rel_p = sqrt(rp2) / (1.0 + s.bnorm);
    k.rel_d = sqrt(rd2) / (1.0 + s.cnorm);
    k.rel_gap = fabs(k.pobj - k.dobj) / (1.0 + fabs(k.pobj) + fabs(k.dobj));
    k.err = sqrt(k.rel_p * k.rel_p + k.rel_d * k.rel_d + k.rel_gap * k.rel_gap);
    return k;
}
__device__ __forceinline__ bool kkt_finite(const Kkt& k) {
    return isfinite(k.pobj) && isfinite(k.dobj) && isfinite(k.rel_p) && isfinite(k.rel_d);
}
__device__ __forceinline__ bool kkt_conv(const Kkt& k, double tol) {
    return k.rel_p <= tol && k.rel_d <= tol && k.rel_gap <= tol;
}

__device__ __forceinline__ void step_sizes(SolveState& s) {  // pdhg_impl.hpp:87-91
    s.sigma = s.eta * s.w;
    s.tau = s.eta / s.w;
    if (s.has_q) {
        const double tq = 0.998 / (0.5 * s.normQ + s.sigma * s.normA * s.normA);
        s.tau = (tq < s.tau) ? tq : s.tau;
    }
}

// Scalar decision logic of one instance, after its partials are reduced.
static __device__ void decide(SolveState& s, const double (&T)[kTerms], int mode) {
    const Kkt kc = make_kkt(s, T[T_CX_C], T[T_XQX_C], T[T_ROBJ_C], T[T_VOBJ_C], T[T_RP2_C], T[T_RD2_C]);
    if (mode == kEvalCertify) { s.kcert = kc; return; }
    if (mode == kEvalInit) {  // pdhg_impl.hpp:120-128
        double e = kc.err;
        if (s.carry_restart_err > 0) e = (e < s.carry_restart_err) ? s.carry_restart_err : e;
        s.restart_err = e;
        s.prev_cand = INFINITY;
        s.it_since = 0;
        s.best_err = e;
        s.cwp = 0;
        s.done = 0;
        s.exit_reason = kIterLimit;
        s.best_is_avg = 0;
        s.restart_now = 0;
        s.avg_better = 0;
        s.kc = kc;
        step_sizes(s);
        if (s.t0_ns == 0) s.t0_ns = global_ns();
        return;
    }
    // check (pdhg_impl.hpp:144-189)
    const long long it = s.it + s.check_every;
    const long long it_since = s.it_since + s.check_every;
    s.it = it;
    s.checks += 1;
    s.inv_avg = 1.0 / static_cast<double>(it_since);
    const Kkt ka = make_kkt(s, T[T_CX_A], T[T_XQX_A], T[T_ROBJ_A], T[T_VOBJ_A], T[T_RP2_A], T[T_RD2_A]);
    s.kc = kc;
    s.ka = ka;
    s.restart_now = 0;
    const double t = (global_ns() - s.t0_ns) * 1e-9;
    int done = 1;
    const bool avg_better = kkt_finite(ka) && (!kkt_finite(kc) || ka.err < kc.err);
    const Kkt kcand = avg_better ? ka : kc;
    if (!kkt_finite(kc) && !kkt_finite(ka)) { s.exit_reason = kNumerical; s.best = kc; s.best_is_avg = 0; }
    else if (kkt_conv(kc, s.phase_tol)) { s.exit_reason = kConverged; s.best = kc; s.best_is_avg = 0; }
    else if (kkt_conv(ka, s.phase_tol)) { s.exit_reason = kConverged; s.best = ka; s.best_is_avg = 1; }
    else if (it >= s.max_iter) { s.exit_reason = kIterLimit; s.best = kcand; s.best_is_avg = avg_better; }
    else if (t >= s.time_limit_s) { s.exit_reason = kTimeLimit; s.best = kcand; s.best_is_avg = avg_better; }
    else {
        bool infeasible = false;
        if (it_since >= 4LL * s.check_every) {  // primal_infeasible (pdhg_impl.hpp:110-118)
            const double dray = (T[T_ROBJ_R] + T[T_VOBJ_R]) * s.obj_scale;
            infeasible = (dray > 0) && sqrt(T[T_RD2_R]) * (1.0 + s.bnorm) / dray <= s.infeas_tol;
        }
        bool unbounded = false;
        if (!infeasible && s.detect_unbounded && !s.has_q && it_since >= 4LL * s.check_every) {
            // extension: dual infeasibility from the primal ray d = x - x_r
            const double cd = T[T_CD];
            unbounded = cd < 0 && T[T_DX2_C] > 1e-20 && sqrt(T[T_UR2] + T[T_UC2]) / (-cd) <= s.infeas_tol;
        }
        if (infeasible) { s.exit_reason = kInfeasible; s.best = kcand; s.best_is_avg = avg_better; }
        else if (unbounded) { s.exit_reason = kUnbounded; s.best = kcand; s.best_is_avg = avg_better; }
        else {
            done = 0;
            if (kcand.err < 0.8 * s.best_err) { s.best_err = kcand.err; s.cwp = 0; }
            else if (++s.cwp >= s.stall_checks && s.stall_exit) {
                done = 1;
                s.exit_reason = kStalled; s.best = kcand; s.best_is_avg = avg_better;
            }
        }
    }
    s.done = done;
    s.avg_better = avg_better;
    s.it_since = it_since;
    if (!done) {  // adaptive restart (pdhg_impl.hpp:172-189)
        const bool sufficient = kcand.err <= 0.2 * s.restart_err;
        const bool necessary = kcand.err <= 0.8 * s.restart_err && kcand.err > s.prev_cand;
        const bool artificial = static_cast<double>(it_since) >= 0.36 * static_cast<double>(it);
        s.prev_cand = kcand.err;
        if (sufficient || necessary || artificial) {
            const double dx = sqrt(avg_better ? T[T_DX2_A] : T[T_DX2_C]);
            const double dy = sqrt(avg_better ? T[T_DY2_A] : T[T_DY2_C]);
            if (dx > 1e-10 && dy > 1e-10) s.w = exp(0.5 * log(dy / dx) + 0.5 * log(s.w));
            s.restart_now = 1;
            s.it_since = 0;
            s.restart_err = kcand.err;
            s.prev_cand = INFINITY;
            s.restarts += 1;
        }
        step_sizes(s);
    } else {
        s.active = 0;  // this instance leaves the phase
    }
}

template <class M, class V, int NVA, int NVT>
__global__ void __launch_bounds__(kThreads) k_eval(const __grid_constant__ EvalArgs<M, V> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    pdl_enter();
    __shared__ double red[kWarps * kColTerms];
    const int nbA = a.A.nb;
    const size_t nb = static_cast<size_t>(nbA + a.AT.nb);
    double* part = a.partials + blockIdx.x;  // term q of this CTA at part[q * nb]
    if (static_cast<int>(blockIdx.x) < nbA) {
        const double inv = avg_weight(a.st[a.A.blocks[blockIdx.x].inst], a.mode);
        EvalRowEpi<M, V, NVA> epi{a, inv, {}};
#pragma unroll
        for (int k = 0; k < kRowTerms; ++k) epi.t[k] = 0.0;
        spmv_run<NVA, M, V>(a.A, blockIdx.x, GatherXAvg<V, NVA>{a.x, a.sumx, a.xr, inv}, epi, smem);
        block_sum<kRowTerms>(epi.t, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < kRowTerms; ++k) part[k * nb] = epi.t[k];
        }
    } else {
        const int cta = blockIdx.x - nbA;
        const double inv = avg_weight(a.st[a.AT.blocks[cta].inst], a.mode);
        EvalColEpi<M, V, NVT> epi{a, inv, {}};
#pragma unroll
        for (int k = 0; k < kColTerms; ++k) epi.t[k] = 0.0;
        spmv_run<NVT, M, V>(a.AT, cta, GatherYAvgRay<V, NVT>{a.y, a.sumy, a.yr, inv}, epi, smem);
        block_sum<kColTerms>(epi.t, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < kColTerms; ++k) part[(kRowTerms + k) * nb] = epi.t[k];
        }
    }
}

// After k_eval: reduce every instance's partials in a fixed order and run its
// decision.  A single problem is one CTA; a batch gets one CTA per
// kDecideInst instances (decide_grid).  Within a CTA an instance with many
// blocks is reduced by the whole CTA (one at a time); the others by one warp
// each into inst_terms, after which every thread runs the decisions of its own
// instances (the scalar decision code is the long part, so it must not run one
// instance per warp).  With several CTAs the last to arrive sets the phase
// loop's condition from the OR of every CTA's "some instance still active" and
// re-arms the two sync words.
// The term sums of a single instance with more than kDecideWide blocks,
// one CTA per term, before k_decide: CTA q folds term q over the instance's
// blocks exactly as k_decide's whole-CTA path does (thread t takes blocks
// t, t + kThreads, ..., then block_sum), so the sums are the same bits, and
// the 22 folds run side by side instead of in one CTA.
template <class M, class V>
__global__ void __launch_bounds__(kThreads) k_terms(const __grid_constant__ EvalArgs<M, V> a) {
    pdl_enter();
    __shared__ double red[kWarps];
    const int q = blockIdx.x;
    const size_t nb = static_cast<size_t>(a.A.nb + a.AT.nb);
    const int b0 = q < kRowTerms ? a.seg_a[0] : a.A.nb + a.seg_t[0];
    const int b1 = q < kRowTerms ? a.seg_a[1] : a.A.nb + a.seg_t[1];
    double v[1] = {0.0};
    for (int b = b0 + static_cast<int>(threadIdx.x); b < b1; b += kThreads) v[0] += __ldcg(a.partials + q * nb + b);
    block_sum<1>(v, red);
    if (threadIdx.x == 0) a.inst_terms[q] = v[0];
}

template <class M, class V>
__global__ void __launch_bounds__(kThreads) k_decide(const __grid_constant__ EvalArgs<M, V> a) {
    pdl_enter();
    __shared__ double red[kWarps * kTerms];
    const int nbA = a.A.nb;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k0 = gridDim.x == 1 ? 0 : blockIdx.x * kDecideInst;
    const int k1 = gridDim.x == 1 ? a.count : min(a.count, k0 + kDecideInst);
    int any_active = 0;
    auto load_terms = [&](int k, int first, int step, double (&T)[kTerms]) {
#pragma unroll
        for (int q = 0; q < kTerms; ++q) T[q] = 0.0;
        // row terms over the instance's A blocks, column terms over its A^T
        // blocks; consecutive threads read consecutive blocks of one term
        const size_t nb = static_cast<size_t>(nbA + a.AT.nb);
        const int a0 = a.seg_a[k], a1 = a.seg_a[k + 1], t0 = nbA + a.seg_t[k], t1 = nbA + a.seg_t[k + 1];
#pragma unroll
        for (int q = 0; q < kRowTerms; ++q)
            for (int b = a0 + first; b < a1; b += step) T[q] += __ldcg(a.partials + q * nb + b);
#pragma unroll
        for (int q = kRowTerms; q < kTerms; ++q)
            for (int b = t0 + first; b < t1; b += step) T[q] += __ldcg(a.partials + q * nb + b);
    };
    auto finish = [&](SolveState& s, const double (&T)[kTerms]) {
        s.ran_body = (a.mode == kEvalCheck) ? 1 : 0;
        decide(s, T, a.mode);
        any_active |= s.active;
    };
    constexpr int kWide = kDecideWide;
    for (int k = k0; k < k1; ++k) {
        const int nblk = (a.seg_a[k + 1] - a.seg_a[k]) + (a.seg_t[k + 1] - a.seg_t[k]);
        if (nblk <= kWide) continue;
        SolveState& s = a.st[k];
        if (!eval_includes(s, a.mode)) {
            if (threadIdx.x == 0) s.ran_body = 0;
            continue;
        }
        double T[kTerms];
        if (a.terms_ready) {  // k_terms folded them already, in this same order
            if (threadIdx.x == 0) {
#pragma unroll
                for (int q = 0; q < kTerms; ++q) T[q] = __ldcg(a.inst_terms + static_cast<size_t>(k) * kTerms + q);
                finish(s, T);
            }
        } else {
            load_terms(k, threadIdx.x, kThreads, T);
            block_sum<kTerms>(T, red);
            if (threadIdx.x == 0) finish(s, T);
        }
        __syncthreads();
    }
    for (int k = k0 + wid; k < k1; k += kWarps) {
        const int nblk = (a.seg_a[k + 1] - a.seg_a[k]) + (a.seg_t[k + 1] - a.seg_t[k]);
        if (nblk > kWide || !eval_includes(a.st[k], a.mode)) continue;
        double T[kTerms];
        load_terms(k, lane, 32, T);
#pragma unroll
        for (int q = 0; q < kTerms; ++q) T[q] = warp_sum(T[q]);
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < kTerms; ++q) a.inst_terms[static_cast<size_t>(k) * kTerms + q] = T[q];
        }
    }
    __syncthreads();
    for (int k = k0 + threadIdx.x; k < k1; k += kThreads) {
        const int nblk = (a.seg_a[k + 1] - a.seg_a[k]) + (a.seg_t[k + 1] - a.seg_t[k]);
        if (nblk > kWide) continue;
        SolveState& s = a.st[k];
        if (!eval_includes(s, a.mode)) {
            s.ran_body = 0;
            continue;
        }
        double T[kTerms];
#pragma unroll
        for (int q = 0; q < kTerms; ++q) T[q] = a.inst_terms[static_cast<size_t>(k) * kTerms + q];
        finish(s, T);
    }
    any_active = __syncthreads_or(any_active);
    if (threadIdx.x != 0) return;
    if (gridDim.x == 1) {
        if (a.use_cond)
            cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(a.cond), any_active ? 1u : 0u);
        return;
    }
    if (any_active) atomicOr(a.sync + 1, 1u);
    __threadfence();
    if (atomicAdd(a.sync, 1u) == gridDim.x - 1) {  // last CTA: every decision is written
        __threadfence();
        const unsigned any = atomicExch(a.sync + 1, 0u);
        atomicExch(a.sync, 0u);
        if (a.use_cond) cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(a.cond), any ? 1u : 0u);
    }
}

// Restart / buffer bookkeeping after a check (pdhg_impl.hpp:178-185).
// `xc`/`yc` hold the current iterate (buffer 1 when check_every is odd); the
// result always lands in buffer 0 (x0, y0).  Only instances that iterated in
// the body just checked are touched.
template <class V>
struct RestartArgs {
    const V* xc; const V* yc;
    V* x0; V* y0; V* xr; V* yr; V* sumx; V* sumy;
    int n, m;
    const int* inst_col;   // column -> instance (nullptr: one instance)
    const int* inst_row;   // row -> instance
    const SolveState* st;
};

template <class V>
__global__ void k_restart(const RestartArgs<V> a) {
    pdl_enter();
    const bool copy = a.xc != a.x0;
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.n; j += stride) {
        const SolveState& s = a.st[a.inst_col ? a.inst_col[j] : 0];
        if (!s.ran_body) continue;
        const bool restart = s.restart_now != 0;
        if (!restart && !copy) continue;
        V v = a.xc[j];
        if (restart) {
            if (s.avg_better) v = avg_of(a.sumx, j, s.inv_avg);
            a.xr[j] = v;
            a.sumx[j] = V(0);
        }
        a.x0[j] = v;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.m; i += stride) {
        const SolveState& s = a.st[a.inst_row ? a.inst_row[i] : 0];
        if (!s.ran_body) continue;
        const bool restart = s.restart_now != 0;
        if (!restart && !copy) continue;
        V v = a.yc[i];
        if (restart) {
            if (s.avg_better) v = avg_of(a.sumy, i, s.inv_avg);
            a.yr[i] = v;
            a.sumy[i] = V(0);
        }
        a.y0[i] = v;
    }
}

// Phase start: iterate, restart point and zero sums in precision V from the
// FP64 carried state (pdhg_impl.hpp:78-84), for the instances in the phase.
template <class V>
__global__ void k_phase_in(int n, int m, const int* inst_col, const int* inst_row, const SolveState* st,
                           const double* x64, const double* y64, const double* xr64, const double* yr64,
                           int has_r, V* x, V* y, V* xr, V* yr, V* sumx, V* sumy) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        if (!st[inst_col ? inst_col[j] : 0].in_phase) continue;
        x[j] = static_cast<V>(x64[j]);
        xr[j] = static_cast<V>(has_r ? xr64[j] : x64[j]);
        sumx[j] = V(0);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        if (!st[inst_row ? inst_row[i] : 0].in_phase) continue;
        y[i] = static_cast<V>(y64[i]);
        yr[i] = static_cast<V>(has_r ? yr64[i] : y64[i]);
        sumy[i] = V(0);
    }
}

// Phase end: best point (current or average) and restart point to FP64
// (pdhg_impl.hpp:191-194), for the instances in the phase.
template <class V>
__global__ void k_phase_out(int n, int m, const int* inst_col, const int* inst_row, const V* x, const V* y,
                            const V* sumx, const V* sumy, const V* xr, const V* yr, const SolveState* st,
                            double* x64, double* y64, double* xr64, double* yr64) {
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const SolveState& s = st[inst_col ? inst_col[j] : 0];
        if (!s.in_phase) continue;
        x64[j] = static_cast<double>(s.best_is_avg ? avg_of(sumx, j, s.inv_avg) : x[j]);
        xr64[j] = static_cast<double>(xr[j]);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const SolveState& s = st[inst_row ? inst_row[i] : 0];
        if (!s.in_phase) continue;
        y64[i] = static_cast<double>(s.best_is_avg ? avg_of(sumy, i, s.inv_avg) : y[i]);
        yr64[i] = static_cast<double>(yr[i]);
    }
}

}  // namespace gb

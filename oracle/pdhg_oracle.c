/*
 * CPU oracle for GANIT's restarted PDHG -- TEST INFRASTRUCTURE ONLY.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker; the product library never links or calls it.
 *
 * Restates, in plain C:
 *   src/lp.cpp:55-72        transpose
 *   src/scaling.cpp:8-155   norm2, finite_bound_norm, scale_lp, estimate_norm
 *   src/pdhg_impl.hpp       KKT, run_pdhg, status_from (phases in pdhg_phase.inc)
 * Build: see oracle/Makefile (gcc -O2, no -march flags, so no FMA contraction).
 */
#define _POSIX_C_SOURCE 199309L
#include "pdhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    int rows, cols;
    long nnz;
    int* ptr;
    int* idx;
    double* val;
} csr_t;

/* ScaledLP (src/scaling.hpp:8-23) */
typedef struct {
    int m, n;
    csr_t A, AT, Q;
    int has_q;
    double *c, *l, *u, *lo, *hi, *R, *C, *Rres, *Cres;
    double bscale, cscale, normQ, obj_const, bnorm, cnorm;
    int maximize;
} scaled_lp;

/* KKT (pdhg_impl.hpp:36-42) */
typedef struct {
    double pobj, dobj, rel_p, rel_d, rel_gap, err;
} kkt_t;

static int kkt_finite(const kkt_t* k) {
    return isfinite(k->pobj) && isfinite(k->dobj) && isfinite(k->rel_p) && isfinite(k->rel_d);
}
static int kkt_converged(const kkt_t* k, double tol) {
    return k->rel_p <= tol && k->rel_d <= tol && k->rel_gap <= tol;
}

/* PdhgShared (pdhg_impl.hpp:44-53) */
typedef struct {
    const scaled_lp* s;
    const ora_options* opt;
    double eta, normA, obj_scale;
    struct timespec t_solve;
} shared_t;

/* PdhgState (pdhg_impl.hpp:55-63); xr/yr "empty" is has_r == 0 */
typedef struct {
    double *x, *y, *xr, *yr;
    int has_r;
    double restart_err, w;
    long it;
    int restarts;
    kkt_t kkt;
} state_t;

/* PhaseExit (pdhg_impl.hpp:65) */
enum { PX_CONVERGED, PX_STALLED, PX_ITERATION_LIMIT, PX_TIME_LIMIT, PX_INFEASIBLE, PX_NUMERICAL };

static double now_diff(const struct timespec* a) {
    struct timespec b;
    clock_gettime(CLOCK_MONOTONIC, &b);
    return (double)(b.tv_sec - a->tv_sec) + 1e-9 * (double)(b.tv_nsec - a->tv_nsec);
}
static double elapsed_s(const shared_t* sh) { return now_diff(&sh->t_solve); }

/* scaling.cpp:8-12 */
static double norm2(const double* v, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s);
}
/* scaling.cpp:15-24 */
static double finite_bound_norm(const double* lo, const double* hi, int m) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) {
        double a = isfinite(lo[i]) ? fabs(lo[i]) : 0.0;
        double b = isfinite(hi[i]) ? fabs(hi[i]) : 0.0;
        double v = (a < b) ? b : a;
        s += v * v;
    }
    return sqrt(s);
}

static void csr_free(csr_t* a) {
    free(a->ptr); free(a->idx); free(a->val);
    memset(a, 0, sizeof(*a));
}
static int csr_copy(csr_t* d, int rows, int cols, const int* ptr, const int* idx, const double* val) {
    d->rows = rows;
    d->cols = cols;
    d->nnz = ptr[rows];
    d->ptr = (int*)malloc(sizeof(int) * (size_t)(rows + 1));
    d->idx = (int*)malloc(sizeof(int) * (size_t)(d->nnz > 0 ? d->nnz : 1));
    d->val = (double*)malloc(sizeof(double) * (size_t)(d->nnz > 0 ? d->nnz : 1));
    if (!d->ptr || !d->idx || !d->val) return -1;
    memcpy(d->ptr, ptr, sizeof(int) * (size_t)(rows + 1));
    if (d->nnz) {
        memcpy(d->idx, idx, sizeof(int) * (size_t)d->nnz);
        memcpy(d->val, val, sizeof(double) * (size_t)d->nnz);
    }
    return 0;
}

/* lp.cpp:55-72: counting-sort transpose, entries of each output row in
 * increasing source-row order. */
static int csr_transpose(const csr_t* a, csr_t* t) {
    t->rows = a->cols;
    t->cols = a->rows;
    t->nnz = a->nnz;
    t->ptr = (int*)calloc((size_t)a->cols + 1, sizeof(int));
    t->idx = (int*)malloc(sizeof(int) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    t->val = (double*)malloc(sizeof(double) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    int* pos = (int*)malloc(sizeof(int) * (size_t)(a->cols > 0 ? a->cols : 1));
    if (!t->ptr || !t->idx || !t->val || !pos) { free(pos); return -1; }
    for (long p = 0; p < a->nnz; ++p) t->ptr[a->idx[p] + 1]++;
    for (int j = 0; j < a->cols; ++j) t->ptr[j + 1] += t->ptr[j];
    for (int j = 0; j < a->cols; ++j) pos[j] = t->ptr[j];
    for (int i = 0; i < a->rows; ++i)
        for (int p = a->ptr[i]; p < a->ptr[i + 1]; ++p) {
            int q = pos[a->idx[p]]++;
            t->idx[q] = i;
            t->val[q] = a->val[p];
        }
    free(pos);
    return 0;
}

/* scaling.cpp:27-33 */
static void apply_scaling(csr_t* a, const double* rs, const double* cs, double* R, double* C) {
    for (int i = 0; i < a->rows; ++i)
        for (int p = a->ptr[i]; p < a->ptr[i + 1]; ++p) a->val[p] *= rs[i] * cs[a->idx[p]];
    for (int i = 0; i < a->rows; ++i) R[i] *= rs[i];
    for (int j = 0; j < a->cols; ++j) C[j] *= cs[j];
}

static void slp_free(scaled_lp* s) {
    csr_free(&s->A); csr_free(&s->AT); csr_free(&s->Q);
    free(s->c); free(s->l); free(s->u); free(s->lo); free(s->hi);
    free(s->R); free(s->C); free(s->Rres); free(s->Cres);
}

static double* dalloc(int n) { return (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1)); }

/* scale_lp (scaling.cpp:36-129) with bound_obj_rescale = true. */
static int scale_lp(const ora_lp* lp, int ruiz_iters, int pock_chambolle, scaled_lp* s) {
    memset(s, 0, sizeof(*s));
    s->m = lp->m;
    s->n = lp->n;
    if (csr_copy(&s->A, lp->m, lp->n, lp->a_ptr, lp->a_idx, lp->a_val)) return -1;
    s->R = dalloc(lp->m);
    s->C = dalloc(lp->n);
    for (int i = 0; i < lp->m; ++i) s->R[i] = 1.0;
    for (int j = 0; j < lp->n; ++j) s->C[j] = 1.0;
    s->maximize = lp->maximize;
    const double sign = lp->maximize ? -1.0 : 1.0;
    s->bscale = 1.0;
    s->cscale = 1.0;

    double* rs = dalloc(lp->m);
    double* cs = dalloc(lp->n);
    for (int it = 0; it < ruiz_iters; ++it) {
        for (int i = 0; i < lp->m; ++i) rs[i] = 0.0;
        for (int j = 0; j < lp->n; ++j) cs[j] = 0.0;
        for (int i = 0; i < lp->m; ++i)
            for (int p = s->A.ptr[i]; p < s->A.ptr[i + 1]; ++p) {
                double a = fabs(s->A.val[p]);
                rs[i] = (rs[i] < a) ? a : rs[i];
                int j = s->A.idx[p];
                cs[j] = (cs[j] < a) ? a : cs[j];
            }
        for (int i = 0; i < lp->m; ++i) rs[i] = rs[i] > 0 ? 1.0 / sqrt(rs[i]) : 1.0;
        for (int j = 0; j < lp->n; ++j) cs[j] = cs[j] > 0 ? 1.0 / sqrt(cs[j]) : 1.0;
        apply_scaling(&s->A, rs, cs, s->R, s->C);
    }
    if (pock_chambolle) {
        for (int i = 0; i < lp->m; ++i) rs[i] = 0.0;
        for (int j = 0; j < lp->n; ++j) cs[j] = 0.0;
        for (int i = 0; i < lp->m; ++i)
            for (int p = s->A.ptr[i]; p < s->A.ptr[i + 1]; ++p) {
                double a = fabs(s->A.val[p]);
                rs[i] += a;
                cs[s->A.idx[p]] += a;
            }
        for (int i = 0; i < lp->m; ++i) rs[i] = rs[i] > 0 ? 1.0 / sqrt(rs[i]) : 1.0;
        for (int j = 0; j < lp->n; ++j) cs[j] = cs[j] > 0 ? 1.0 / sqrt(cs[j]) : 1.0;
        apply_scaling(&s->A, rs, cs, s->R, s->C);
    }
    free(rs);
    free(cs);
    if (csr_transpose(&s->A, &s->AT)) return -1;

    s->c = dalloc(lp->n); s->l = dalloc(lp->n); s->u = dalloc(lp->n);
    s->lo = dalloc(lp->m); s->hi = dalloc(lp->m);
    for (int j = 0; j < lp->n; ++j) {
        s->c[j] = sign * lp->c[j] * s->C[j];
        s->l[j] = lp->l[j] / s->C[j];
        s->u[j] = lp->u[j] / s->C[j];
    }
    for (int i = 0; i < lp->m; ++i) {
        s->lo[i] = lp->lo[i] * s->R[i];
        s->hi[i] = lp->hi[i] * s->R[i];
    }
    s->bscale = finite_bound_norm(s->lo, s->hi, lp->m) + 1.0;
    s->cscale = norm2(s->c, lp->n) + 1.0;
    for (int j = 0; j < lp->n; ++j) s->c[j] /= s->cscale;
    for (int j = 0; j < lp->n; ++j) s->l[j] /= s->bscale;
    for (int j = 0; j < lp->n; ++j) s->u[j] /= s->bscale;
    for (int i = 0; i < lp->m; ++i) s->lo[i] /= s->bscale;
    for (int i = 0; i < lp->m; ++i) s->hi[i] /= s->bscale;
    s->Rres = dalloc(lp->m);
    s->Cres = dalloc(lp->n);
    for (int i = 0; i < lp->m; ++i) s->Rres[i] = s->R[i] / s->bscale;
    for (int j = 0; j < lp->n; ++j) s->Cres[j] = s->C[j] / s->cscale;
    s->obj_const = sign * lp->obj_const;
    s->has_q = lp->q_ptr != NULL && lp->q_ptr[lp->n] > 0;
    if (s->has_q) {
        if (csr_copy(&s->Q, lp->n, lp->n, lp->q_ptr, lp->q_idx, lp->q_val)) return -1;
        for (int i = 0; i < lp->n; ++i)
            for (int p = s->Q.ptr[i]; p < s->Q.ptr[i + 1]; ++p)
                s->Q.val[p] *= sign * s->C[i] * s->C[s->Q.idx[p]] * s->bscale / s->cscale;
        /* power iteration for ||Q'||_2 (scaling.cpp:108-124) */
        double* v = dalloc(lp->n);
        double* w = dalloc(lp->n);
        for (int j = 0; j < lp->n; ++j) v[j] = 1.0;
        double nv = norm2(v, lp->n);
        for (int j = 0; j < lp->n; ++j) v[j] /= nv;
        double lam = 0.0;
        for (int it = 0; it < 60; ++it) {
            for (int i = 0; i < lp->n; ++i) {
                double t = 0.0;
                for (int p = s->Q.ptr[i]; p < s->Q.ptr[i + 1]; ++p) t += s->Q.val[p] * v[s->Q.idx[p]];
                w[i] = t;
            }
            double nw = norm2(w, lp->n);
            if (nw == 0.0) break;
            lam = nw;
            for (int i = 0; i < lp->n; ++i) v[i] = w[i] / nw;
        }
        s->normQ = lam * 1.01;
        free(v);
        free(w);
    }
    s->bnorm = finite_bound_norm(lp->lo, lp->hi, lp->m);
    s->cnorm = norm2(lp->c, lp->n);
    return 0;
}

/* estimate_norm (scaling.cpp:131-155), iters = 50 */
static double estimate_norm(const scaled_lp* s, int iters) {
    if (s->A.nnz == 0) return 1.0;
    double* v = dalloc(s->n);
    double* w = dalloc(s->m);
    double* z = dalloc(s->n);
    for (int j = 0; j < s->n; ++j) v[j] = 1.0;
    double nv = norm2(v, s->n);
    for (int j = 0; j < s->n; ++j) v[j] /= nv;
    double lambda = 0.0;
    for (int it = 0; it < iters; ++it) {
        for (int i = 0; i < s->m; ++i) {
            double t = 0.0;
            for (int p = s->A.ptr[i]; p < s->A.ptr[i + 1]; ++p) t += s->A.val[p] * v[s->A.idx[p]];
            w[i] = t;
        }
        for (int j = 0; j < s->n; ++j) {
            double t = 0.0;
            for (int p = s->AT.ptr[j]; p < s->AT.ptr[j + 1]; ++p) t += s->AT.val[p] * w[s->AT.idx[p]];
            z[j] = t;
        }
        double nz = norm2(z, s->n);
        if (nz == 0.0) break;
        lambda = nz;
        for (int j = 0; j < s->n; ++j) v[j] = z[j] / nz;
    }
    free(v); free(w); free(z);
    return sqrt(lambda) * 1.01;
}

/* ---- the three precision levels */
#define ORA_M float
#define ORA_V float
#define ORA_SFX l1
#include "pdhg_phase.inc"
#undef ORA_M
#undef ORA_V
#undef ORA_SFX

#define ORA_M float
#define ORA_V double
#define ORA_SFX l2
#include "pdhg_phase.inc"
#undef ORA_M
#undef ORA_V
#undef ORA_SFX

#define ORA_M double
#define ORA_V double
#define ORA_SFX l3
#include "pdhg_phase.inc"
#undef ORA_M
#undef ORA_V
#undef ORA_SFX

/* status_from (pdhg_impl.hpp:232-240) */
static int status_from(int e) {
    switch (e) {
        case PX_CONVERGED: return ORA_OPTIMAL;
        case PX_INFEASIBLE: return ORA_PRIMAL_INFEASIBLE;
        case PX_TIME_LIMIT: return ORA_TIME_LIMIT;
        case PX_NUMERICAL: return ORA_NUMERICAL_ERROR;
        default: return ORA_ITERATION_LIMIT;
    }
}

void ora_default_options(ora_options* o) {
    o->tol = 1e-4;
    o->max_iter = 10000000;
    o->time_limit = 3600.0;
    o->check_every = 64;
    o->ruiz_iters = 10;
    o->pock_chambolle = 1;
    o->infeas_tol = 1e-8;
    o->precision = ORA_DOUBLE;
    o->stall_checks = 12;
    o->stall_checks_l2 = 24;
}

/* finished lambda (pdhg_impl.hpp:278-286) */
static int phase_finished(shared_t* sh, state_t* st, int e) {
    kkt_t k64 = evaluate_l3(sh, st);
    return (e == PX_CONVERGED && kkt_converged(&k64, sh->opt->tol)) || e == PX_TIME_LIMIT ||
           e == PX_ITERATION_LIMIT || e == PX_INFEASIBLE;
}

/* run_pdhg (pdhg_impl.hpp:243-328) */
int ora_solve_pdhg(const ora_lp* lp, const ora_options* opt, ora_result* res, double* x_out, double* y_out) {
    if (!lp || !opt || !res || lp->m < 0 || lp->n < 0 || opt->check_every <= 0) return -1;
    struct timespec t_start;
    clock_gettime(CLOCK_MONOTONIC, &t_start);
    memset(res, 0, sizeof(*res));
    res->status = ORA_NUMERICAL_ERROR;

    scaled_lp s;
    if (scale_lp(lp, opt->ruiz_iters, opt->pock_chambolle, &s)) { slp_free(&s); return -2; }
    const double normA = estimate_norm(&s, 50);
    shared_t sh;
    sh.s = &s;
    sh.opt = opt;
    sh.eta = 0.998 / normA;
    sh.normA = normA;
    sh.obj_scale = s.cscale * s.bscale;

    state_t st;
    memset(&st, 0, sizeof(st));
    st.x = dalloc(s.n); st.y = dalloc(s.m); st.xr = dalloc(s.n); st.yr = dalloc(s.m);
    st.restart_err = -1.0;
    st.w = 1.0;
    for (int j = 0; j < s.n; ++j) {
        double v = (0.0 < s.l[j]) ? s.l[j] : 0.0;  /* std::max(0.0, l) */
        st.x[j] = (s.u[j] < v) ? s.u[j] : v;       /* std::min(., u) */
    }
    for (int i = 0; i < s.m; ++i) st.y[i] = 0.0;
    {
        double cn = norm2(s.c, s.n), bn = finite_bound_norm(s.lo, s.hi, s.m);
        st.w = (cn > 1e-10 && bn > 1e-10) ? cn / bn : 1.0;
    }
    const int mixed = opt->precision != ORA_DOUBLE;
    res->setup_s = now_diff(&t_start);
    clock_gettime(CLOCK_MONOTONIC, &sh.t_solve);

    int ex;
    long fp32_iters = 0;
    if (mixed) {
        ex = phase_l1(&sh, &st, opt->tol, 1, opt->stall_checks);
        fp32_iters = st.it;
        int done = phase_finished(&sh, &st, ex);
        if (!done && opt->precision == ORA_DYNAMIC) {
            ex = phase_l2(&sh, &st, opt->tol, 1, opt->stall_checks_l2);
            res->l2_iterations = st.it - fp32_iters;
            done = phase_finished(&sh, &st, ex);
        }
        if (!done) ex = phase_l3(&sh, &st, opt->tol, 0, 0);
    } else {
        ex = phase_l3(&sh, &st, opt->tol, 0, 0);
    }
    kkt_t fin = evaluate_l3(&sh, &st);
    int status = status_from(ex);
    if (status == ORA_OPTIMAL && !kkt_converged(&fin, opt->tol * 1.0000001)) status = ORA_NUMERICAL_ERROR;

    res->solve_s = elapsed_s(&sh);
    res->status = status;
    res->iterations = st.it;
    res->fp32_iterations = fp32_iters;
    res->restarts = st.restarts;
    res->norm_a = normA;
    res->w_final = st.w;
    const double sign = s.maximize ? -1.0 : 1.0;
    if (x_out)
        for (int j = 0; j < s.n; ++j) x_out[j] = st.x[j] * s.C[j] * s.bscale;
    if (y_out)
        for (int i = 0; i < s.m; ++i) y_out[i] = sign * st.y[i] * s.R[i] * s.cscale;
    res->pobj = sign * fin.pobj;
    res->dobj = sign * fin.dobj;
    res->rel_p = fin.rel_p;
    res->rel_d = fin.rel_d;
    res->rel_gap = fin.rel_gap;

    free(st.x); free(st.y); free(st.xr); free(st.yr);
    slp_free(&s);
    return 0;
}

int ora_scale(const ora_lp* lp, int ruiz_iters, int pock_chambolle, double* a_val_s, double* c_s, double* l_s,
              double* u_s, double* lo_s, double* hi_s, double* R, double* C, double* Rres, double* Cres,
              double* scal) {
    scaled_lp s;
    if (scale_lp(lp, ruiz_iters, pock_chambolle, &s)) { slp_free(&s); return -2; }
    double normA = estimate_norm(&s, 50);
    memcpy(a_val_s, s.A.val, sizeof(double) * (size_t)s.A.nnz);
    memcpy(c_s, s.c, sizeof(double) * (size_t)s.n);
    memcpy(l_s, s.l, sizeof(double) * (size_t)s.n);
    memcpy(u_s, s.u, sizeof(double) * (size_t)s.n);
    memcpy(lo_s, s.lo, sizeof(double) * (size_t)s.m);
    memcpy(hi_s, s.hi, sizeof(double) * (size_t)s.m);
    memcpy(R, s.R, sizeof(double) * (size_t)s.m);
    memcpy(C, s.C, sizeof(double) * (size_t)s.n);
    memcpy(Rres, s.Rres, sizeof(double) * (size_t)s.m);
    memcpy(Cres, s.Cres, sizeof(double) * (size_t)s.n);
    scal[0] = s.bscale;
    scal[1] = s.cscale;
    scal[2] = normA;
    scal[3] = s.normQ;
    scal[4] = s.bnorm;
    scal[5] = s.cnorm;
    scal[6] = s.obj_const;
    slp_free(&s);
    return 0;
}

int ora_plain_iterations(int m, int n, const int* a_ptr, const int* a_idx, const double* a_val,
                         const int* at_ptr, const int* at_idx, const double* at_val, const double* c,
                         const double* l, const double* u, const double* lo, const double* hi, double tau,
                         double sigma, long iters, double* x, double* y) {
    double* aty = dalloc(n);
    double* xn = dalloc(n);
    double* xbar = dalloc(n);
    double* axbar = dalloc(m);
    for (long k = 0; k < iters; ++k) {
        for (int j = 0; j < n; ++j) {
            double t = 0;
            for (int p = at_ptr[j]; p < at_ptr[j + 1]; ++p) t += at_val[p] * y[at_idx[p]];
            aty[j] = t;
        }
        for (int j = 0; j < n; ++j) {
            double g = c[j] - aty[j] + 0.0;
            double v = x[j] - tau * g;
            v = (v < l[j]) ? l[j] : v;
            v = (u[j] < v) ? u[j] : v;
            xn[j] = v;
            xbar[j] = 2.0 * v - x[j];
        }
        for (int i = 0; i < m; ++i) {
            double t = 0;
            for (int p = a_ptr[i]; p < a_ptr[i + 1]; ++p) t += a_val[p] * xbar[a_idx[p]];
            axbar[i] = t;
        }
        for (int i = 0; i < m; ++i) {
            double q = y[i] - sigma * axbar[i];
            double a = -q, lo_s = sigma * lo[i], hi_s = sigma * hi[i];
            double t = (a < lo_s) ? lo_s : a;
            t = (hi_s < t) ? hi_s : t;
            y[i] = q + t;
        }
        memcpy(x, xn, sizeof(double) * (size_t)n);
    }
    free(aty); free(xn); free(xbar); free(axbar);
    return 0;
}

/* FP64 KKT of a point (x, y) of an already-scaled LP: the eval lambda of
 * pdhg_phase (pdhg_impl.hpp:92-109) over the reductions of backend_cpu.cpp:
 * primal_res2 (101-112), dual_res (113-131), row_dual_obj (132-142) and
 * dot_c (143-149), every sum taken in index order.  LPs only.
 * sc[0..3] = obj_scale, obj_const, bnorm, cnorm; out[0..5] = pobj, dobj,
 * rel_p, rel_d, rel_gap, err. */
int ora_eval_kkt(int m, int n, const int* a_ptr, const int* a_idx, const double* a_val, const int* at_ptr,
                 const int* at_idx, const double* at_val, const double* c, const double* l, const double* u,
                 const double* lo, const double* hi, const double* rres, const double* cres, const double* x,
                 const double* y, const double* sc, double* out) {
    double rp2 = 0.0, rd2 = 0.0, vobj = 0.0, robj = 0.0, cx = 0.0;
    for (int i = 0; i < m; ++i) {
        double a = 0.0;
        for (int p = a_ptr[i]; p < a_ptr[i + 1]; ++p) a += a_val[p] * x[a_idx[p]];
        double pr = (a < lo[i]) ? lo[i] : a;
        pr = (hi[i] < pr) ? hi[i] : pr;
        double r = (a - pr) / rres[i];
        rp2 += r * r;
    }
    for (int j = 0; j < n; ++j) {
        double t = 0.0;
        for (int p = at_ptr[j]; p < at_ptr[j + 1]; ++p) t += at_val[p] * y[at_idx[p]];
        double z = c[j] - t + 0.0, r = 0.0;
        if (z > 0) { if (isfinite(l[j])) vobj += z * l[j]; else r = z; }
        else if (z < 0) { if (isfinite(u[j])) vobj += z * u[j]; else r = z; }
        r /= cres[j];
        rd2 += r * r;
    }
    for (int i = 0; i < m; ++i) {
        if (y[i] > 0 && isfinite(lo[i])) robj += y[i] * lo[i];
        else if (y[i] < 0 && isfinite(hi[i])) robj += y[i] * hi[i];
    }
    for (int j = 0; j < n; ++j) cx += c[j] * x[j];
    const double pobj = cx * sc[0] + sc[1];
    const double dobj = (robj + vobj) * sc[0] + sc[1];
    const double rel_p = sqrt(rp2) / (1.0 + sc[2]);
    const double rel_d = sqrt(rd2) / (1.0 + sc[3]);
    const double rel_gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    out[0] = pobj;
    out[1] = dobj;
    out[2] = rel_p;
    out[3] = rel_d;
    out[4] = rel_gap;
    out[5] = sqrt(rel_p * rel_p + rel_d * rel_d + rel_gap * rel_gap);
    return 0;
}

/* lp.cpp:55-72 on caller buffers: t_ptr[cols+1], t_idx / t_val[ptr[rows]]. */
int ora_transpose(int rows, int cols, const int* ptr, const int* idx, const double* val, int* t_ptr, int* t_idx,
                  double* t_val) {
    csr_t a, t;
    if (csr_copy(&a, rows, cols, ptr, idx, val)) { csr_free(&a); return -1; }
    if (csr_transpose(&a, &t)) { csr_free(&a); csr_free(&t); return -1; }
    memcpy(t_ptr, t.ptr, sizeof(int) * (size_t)(cols + 1));
    if (t.nnz) {
        memcpy(t_idx, t.idx, sizeof(int) * (size_t)t.nnz);
        memcpy(t_val, t.val, sizeof(double) * (size_t)t.nnz);
    }
    csr_free(&a);
    csr_free(&t);
    return 0;
}

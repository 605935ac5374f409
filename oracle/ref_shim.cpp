// C-ABI shim around the UNMODIFIED reference CPU implementation -- TEST
// INFRASTRUCTURE ONLY.  oracle/Makefile compiles it together with the
// reference's own sources (src/lp.cpp, src/mps.cpp, src/scaling.cpp,
// src/backend_cpu.cpp, src/simplex.cpp, compiled where they lie) into
// oracle/_ref/libganit_ref.so.  Tests use it to pin the C oracle and to make
// golden fixtures; bench.py's reference arm times ganit::solve_pdhg_cpu
// through it.  Nothing in the product links it.
//
// Wrapped reference entry points:
//   ganit::solve_pdhg_cpu   include/ganit/pdhg.hpp:44, src/backend_cpu.cpp:160
//   ganit::read_mps         include/ganit/lp.hpp:50,  src/mps.cpp:69
//   ganit::DualSimplex      src/simplex.hpp:37-93
//   the strong-branching loop of Mip::select_branch (src/mip.cpp:738-760)
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

#include "ganit/lp.hpp"
#include "ganit/pdhg.hpp"
#include "simplex.hpp"

using namespace ganit;

extern "C" {

struct ref_options {
    double tol;
    long max_iter;
    double time_limit;
    int check_every, ruiz_iters, pock_chambolle;
    double infeas_tol;
    int precision, stall_checks, stall_checks_l2;
};

struct ref_result {
    int status;
    double pobj, dobj, rel_p, rel_d, rel_gap;
    long iterations, fp32_iterations, l2_iterations;
    int restarts;
    double setup_s, solve_s;
};

static LP make_lp(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                  const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                  int maximize, const int* qptr, const int* qidx, const double* qval) {
    LP lp;
    lp.name = "shim";
    lp.m = m;
    lp.n = n;
    lp.A.rows = m;
    lp.A.cols = n;
    lp.A.ptr.assign(ptr, ptr + m + 1);
    lp.A.idx.assign(idx, idx + ptr[m]);
    lp.A.val.assign(val, val + ptr[m]);
    lp.c.assign(c, c + n);
    lp.l.assign(l, l + n);
    lp.u.assign(u, u + n);
    lp.lo.assign(lo, lo + m);
    lp.hi.assign(hi, hi + m);
    lp.obj_const = obj_const;
    lp.maximize = maximize != 0;
    lp.is_int.assign(n, 0);
    if (qptr && qptr[n] > 0) {
        lp.Q.rows = n;
        lp.Q.cols = n;
        lp.Q.ptr.assign(qptr, qptr + n + 1);
        lp.Q.idx.assign(qidx, qidx + qptr[n]);
        lp.Q.val.assign(qval, qval + qptr[n]);
    }
    return lp;
}

int ref_solve_pdhg(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                   const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                   int maximize, const int* qptr, const int* qidx, const double* qval, const ref_options* o,
                   ref_result* r, double* x_out, double* y_out) {
    try {
        LP lp = make_lp(m, n, ptr, idx, val, c, l, u, lo, hi, obj_const, maximize, qptr, qidx, qval);
        Options opt;
        opt.tol = o->tol;
        opt.max_iter = o->max_iter;
        opt.time_limit = o->time_limit;
        opt.check_every = o->check_every;
        opt.ruiz_iters = o->ruiz_iters;
        opt.pock_chambolle = o->pock_chambolle != 0;
        opt.infeas_tol = o->infeas_tol;
        opt.precision = o->precision == 1 ? Precision::Mixed : o->precision == 2 ? Precision::Dynamic
                                                                               : Precision::Double;
        opt.stall_checks = o->stall_checks;
        opt.stall_checks_l2 = o->stall_checks_l2;
        opt.verbose = 0;
        Result res = solve_pdhg_cpu(lp, opt);
        r->status = static_cast<int>(res.status);
        r->pobj = res.pobj;
        r->dobj = res.dobj;
        r->rel_p = res.rel_primal;
        r->rel_d = res.rel_dual;
        r->rel_gap = res.rel_gap;
        r->iterations = res.iterations;
        r->fp32_iterations = res.fp32_iterations;
        r->l2_iterations = res.l2_iterations;
        r->restarts = res.restarts;
        r->setup_s = res.setup_seconds;
        r->solve_s = res.solve_seconds;
        if (x_out) std::memcpy(x_out, res.x.data(), sizeof(double) * n);
        if (y_out) std::memcpy(y_out, res.y.data(), sizeof(double) * m);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ---- MPS reading through the reference reader (src/mps.cpp:69-272)
struct ref_mps {
    LP lp;
};

void* ref_read_mps(const char* path) {
    try {
        auto* h = new ref_mps;
        h->lp = read_mps(path);
        return h;
    } catch (const std::exception&) {
        return nullptr;
    }
}

// dims[0..4] = m, n, nnz(A), nnz(Q), maximize
void ref_mps_dims(void* hp, long* dims) {
    auto* h = static_cast<ref_mps*>(hp);
    dims[0] = h->lp.m;
    dims[1] = h->lp.n;
    dims[2] = h->lp.A.nnz();
    dims[3] = h->lp.Q.nnz();
    dims[4] = h->lp.maximize ? 1 : 0;
}

void ref_mps_copy(void* hp, int* ptr, int* idx, double* val, double* c, double* l, double* u, double* lo,
                  double* hi, double* obj_const, int* qptr, int* qidx, double* qval) {
    auto* h = static_cast<ref_mps*>(hp);
    const LP& lp = h->lp;
    std::memcpy(ptr, lp.A.ptr.data(), sizeof(int) * (lp.m + 1));
    std::memcpy(idx, lp.A.idx.data(), sizeof(int) * lp.A.nnz());
    std::memcpy(val, lp.A.val.data(), sizeof(double) * lp.A.nnz());
    std::memcpy(c, lp.c.data(), sizeof(double) * lp.n);
    std::memcpy(l, lp.l.data(), sizeof(double) * lp.n);
    std::memcpy(u, lp.u.data(), sizeof(double) * lp.n);
    std::memcpy(lo, lp.lo.data(), sizeof(double) * lp.m);
    std::memcpy(hi, lp.hi.data(), sizeof(double) * lp.m);
    *obj_const = lp.obj_const;
    if (lp.Q.nnz() > 0 && qptr) {
        std::memcpy(qptr, lp.Q.ptr.data(), sizeof(int) * (lp.n + 1));
        std::memcpy(qidx, lp.Q.idx.data(), sizeof(int) * lp.Q.nnz());
        std::memcpy(qval, lp.Q.val.data(), sizeof(double) * lp.Q.nnz());
    }
}

// is_int (n bytes) of the reference reader's LP
void ref_mps_is_int(void* hp, unsigned char* out) {
    const LP& lp = static_cast<ref_mps*>(hp)->lp;
    for (int j = 0; j < lp.n; ++j) out[j] = j < (int)lp.is_int.size() && lp.is_int[j] ? 1 : 0;
}

void ref_mps_free(void* hp) { delete static_cast<ref_mps*>(hp); }

// ---- dual simplex (src/simplex.hpp:37-93): exact vertex, basis and duals.
// head_out (m) receives the basic variable of each basis position (j < n:
// structural, n+i: logical of row i); status_out (n+m) the VarStatus codes.
int ref_dual_simplex(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                     const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                     int maximize, double time_limit, double* obj, double* x_out, double* y_out, int* head_out,
                     signed char* status_out, long* iters) {
    try {
        LP lp = make_lp(m, n, ptr, idx, val, c, l, u, lo, hi, obj_const, maximize, nullptr, nullptr, nullptr);
        SimplexOptions so;
        DualSimplex ds(lp, so);
        LpStatus st = ds.solve(-1, kInf, time_limit);
        *obj = ds.objective();
        *iters = ds.iterations();
        std::vector<double> x = ds.primal();
        std::vector<double> y = ds.row_duals_orig();
        if (x_out) std::memcpy(x_out, x.data(), sizeof(double) * n);
        if (y_out) std::memcpy(y_out, y.data(), sizeof(double) * m);
        DualSimplex::Basis b = ds.get_basis();
        if (head_out) for (int r = 0; r < m && r < (int)b.head.size(); ++r) head_out[r] = b.head[r];
        if (status_out)
            for (int j = 0; j < n + m && j < (int)b.status.size(); ++j) status_out[j] = b.status[j];
        return static_cast<int>(st);
    } catch (const std::exception&) {
        return -100;
    }
}

// Strong branching as Mip::select_branch runs it (src/mip.cpp:738-760):
// the node LP solved once (not timed), then per candidate j and side the
// state saved, the child's bounds set ((l_j, floor x_j) / (ceil x_j, u_j)),
// a warm dual-simplex solve with iter_limit (< 0: to optimality), the
// outcome recorded in the reference's mapping (Infeasible / Cutoff -> +inf,
// Optimal -> the objective, else max(z, dual bound) or z), the state
// restored.  Minimisation LPs.  z_out / status_out / iters_out hold 2k
// entries (down, up per candidate); *seconds the loop's wall time.
int ref_strong_branch(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                      const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                      const double* x, const int* cand, int k, long iter_limit, double* z_node, double* z_out,
                      int* status_out, long* iters_out, double* seconds) {
    try {
        LP lp = make_lp(m, n, ptr, idx, val, c, l, u, lo, hi, obj_const, 0, nullptr, nullptr, nullptr);
        DualSimplex S(lp, SimplexOptions{});
        if (S.solve(-1, kInf) != LpStatus::Optimal) return -1;
        const double z = S.objective();
        *z_node = z;
        const auto t0 = std::chrono::steady_clock::now();
        std::unique_ptr<DualSimplex::State> saved = S.save_state();
        for (int t = 0; t < k; ++t) {
            const int j = cand[t];
            const double v = x[j], cl = S.col_lower(j), cu = S.col_upper(j);
            for (int d = 0; d < 2; ++d) {
                const long it0 = S.iterations();
                if (d == 0) S.set_col_bounds(j, cl, std::floor(v));
                else S.set_col_bounds(j, std::ceil(v), cu);
                const LpStatus st = S.solve(iter_limit, kInf);
                double zz;
                if (st == LpStatus::Infeasible || st == LpStatus::Cutoff) zz = kInf;
                else if (st == LpStatus::Optimal) zz = S.objective();
                else {
                    const double db = S.dual_bound_min();
                    zz = std::isfinite(db) ? std::max(z, db) : z;
                }
                z_out[2 * t + d] = zz;
                status_out[2 * t + d] = static_cast<int>(st);
                iters_out[2 * t + d] = S.iterations() - it0;
                S.restore_state(*saved);
            }
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    } catch (const std::exception&) {
        return -100;
    }
}

}  // extern "C"

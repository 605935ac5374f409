// Drop-in demonstration -- TEST INFRASTRUCTURE ONLY.  The reference's own PDHG
// driver (src/pdhg_impl.hpp: run_pdhg, pdhg_phase, pdhg_evaluate), compiled
// UNMODIFIED from the reference sources where they lie, instantiated with the
// B200 Backend adapter (include/ganit_b200_backend.hpp) instead of
// CudaBackend.  oracle/Makefile builds it into oracle/_ref/libganit_dropin.so,
// linked against ganit_v2_b200/libganit_b200.so.
#include <cstring>
#include <exception>

#include "ganit_b200_backend.hpp"
#include "pdhg_impl.hpp"

using namespace ganit;

extern "C" {

struct dropin_options {
    double tol;
    long max_iter;
    double time_limit;
    int check_every, ruiz_iters, pock_chambolle;
    double infeas_tol;
    int precision, stall_checks, stall_checks_l2;
};

struct dropin_result {
    int status;
    double pobj, dobj, rel_p, rel_d, rel_gap;
    long iterations, fp32_iterations, l2_iterations;
    int restarts;
    double setup_s, solve_s;
};

int dropin_solve_b200(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                      const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                      int maximize, const int* qptr, const int* qidx, const double* qval, const dropin_options* o,
                      dropin_result* r, double* x_out, double* y_out) {
    try {
        LP lp;
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
        if (qptr && qptr[n] > 0) {
            lp.Q.rows = n;
            lp.Q.cols = n;
            lp.Q.ptr.assign(qptr, qptr + n + 1);
            lp.Q.idx.assign(qidx, qidx + qptr[n]);
            lp.Q.val.assign(qval, qval + qptr[n]);
        }
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
        Result res = run_pdhg<gb::B200Backend<float, float>, gb::B200Backend<float, double>,
                              gb::B200Backend<double, double>>(lp, opt, "b200");
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

}  // extern "C"

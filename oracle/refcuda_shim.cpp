// C-ABI shim around the UNMODIFIED reference CUDA backend -- BENCHMARK
// INFRASTRUCTURE ONLY.  oracle/Makefile compiles it with nvcc for sm_100a
// together with the reference's own src/backend_cuda.cu, src/lp.cpp and
// src/scaling.cpp (compiled where they lie, with GANIT_HAVE_CUDA as the
// reference's CMakeLists.txt defines it) into oracle/_ref/libganit_refcuda.so.
// bench.py times ganit::solve_pdhg_gpu through it on the same B200 as the
// library, as a comparison leg.  Nothing in the product links it.
//
// Wrapped reference entry point:
//   ganit::solve_pdhg_gpu   include/ganit/pdhg.hpp:45-47, src/backend_cuda.cu:382-393
#include <cstring>
#include <exception>

#include "ganit/lp.hpp"
#include "ganit/pdhg.hpp"

using namespace ganit;

extern "C" {

struct refcuda_options {
    double tol;
    long max_iter;
    double time_limit;
    int check_every, ruiz_iters, pock_chambolle;
    double infeas_tol;
    int precision, stall_checks, stall_checks_l2;
};

struct refcuda_result {
    int status;
    double pobj, dobj, rel_p, rel_d, rel_gap;
    long iterations, fp32_iterations, l2_iterations;
    int restarts;
    double setup_s, solve_s;
};

int refcuda_solve_pdhg_gpu(int m, int n, const int* ptr, const int* idx, const double* val, const double* c,
                           const double* l, const double* u, const double* lo, const double* hi, double obj_const,
                           int maximize, const refcuda_options* o, refcuda_result* r, double* x_out,
                           double* y_out) {
    try {
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
        Result res = solve_pdhg_gpu(lp, opt);
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

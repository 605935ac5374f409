/*
 * CPU oracle for GANIT's restarted PDHG (LP + convex QP) -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithm, used by the test
 * suite and by bench.py's CPU-baseline leg as the checker.  The product path
 * (ganit_v2_b200 / libganit_b200.so) never links, loads or calls it.
 *
 * Followed reference files (paths inside the GANIT_v2 project):
 *   src/scaling.cpp:8-155   norm2, finite_bound_norm, scale_lp, estimate_norm
 *   src/lp.cpp:55-72        transpose
 *   src/backend_cpu.cpp     CPU backend kernels (spmv, primal/dual step, reductions)
 *   src/pdhg_impl.hpp       pdhg_phase, pdhg_evaluate, run_pdhg (restarts, weights,
 *                           infeasibility test, precision phases, certification)
 *   include/ganit/pdhg.hpp  Options / Status / Result
 *
 * Single-threaded and compiled without FMA contraction, so at OMP_NUM_THREADS=1
 * it reproduces the reference CPU build bit for bit (checked by the tests
 * against fixtures produced by the reference itself).
 */
#ifndef GANIT_PDHG_ORACLE_H
#define GANIT_PDHG_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Precision schedule, include/ganit/pdhg.hpp:10 */
enum { ORA_DOUBLE = 0, ORA_MIXED = 1, ORA_DYNAMIC = 2 };
/* Status codes, include/ganit/pdhg.hpp:27 */
enum { ORA_OPTIMAL = 0, ORA_PRIMAL_INFEASIBLE = 1, ORA_ITERATION_LIMIT = 2, ORA_TIME_LIMIT = 3,
       ORA_NUMERICAL_ERROR = 4 };

typedef struct {
    int m, n;
    const int* a_ptr;     /* m+1 */
    const int* a_idx;     /* nnz */
    const double* a_val;  /* nnz */
    const double *c, *l, *u, *lo, *hi;
    double obj_const;
    int maximize;
    const int* q_ptr;     /* n+1, or NULL for an LP (full-storage symmetric Hessian) */
    const int* q_idx;
    const double* q_val;
} ora_lp;

typedef struct {
    double tol;        /* 1e-4 */
    long max_iter;     /* 10000000 */
    double time_limit; /* 3600 */
    int check_every;   /* 64 */
    int ruiz_iters;    /* 10 */
    int pock_chambolle;/* 1 */
    double infeas_tol; /* 1e-8 */
    int precision;     /* ORA_DOUBLE */
    int stall_checks;  /* 12 */
    int stall_checks_l2; /* 24 */
} ora_options;

typedef struct {
    int status;
    double pobj, dobj, rel_p, rel_d, rel_gap;
    long iterations, fp32_iterations, l2_iterations;
    int restarts;
    double setup_s, solve_s;
    double norm_a;     /* ||A'||_2 estimate (scaled matrix) */
    double w_final;    /* primal weight at exit */
} ora_result;

void ora_default_options(ora_options* o);

/* Restarted PDHG, same semantics as ganit::solve_pdhg_cpu.  x_out (n) and
 * y_out (m) receive the unscaled primal solution and row duals.  Returns 0,
 * or a negative value on bad input / allocation failure. */
int ora_solve_pdhg(const ora_lp* lp, const ora_options* opt, ora_result* res, double* x_out, double* y_out);

/* Scaling only (src/scaling.cpp:36-155): writes the scaled data so tests can
 * compare a GPU-side setup with it.  a_val_s (nnz), c_s/l_s/u_s/C/Cres (n),
 * lo_s/hi_s/R/Rres (m); scal[0..6] = bscale, cscale, normA, normQ, bnorm,
 * cnorm, obj_const (scaled sign). */
int ora_scale(const ora_lp* lp, int ruiz_iters, int pock_chambolle, double* a_val_s, double* c_s, double* l_s,
              double* u_s, double* lo_s, double* hi_s, double* R, double* C, double* Rres, double* Cres,
              double* scal);

/* Fixed-length plain PDHG in the scaled space without restarts: from (x0, y0)
 * run `iters` iterations with fixed (tau, sigma) at double precision
 * (pdhg_impl.hpp:133-139 without the check block).  Used to check the
 * GPU iteration kernels and the adjoint tail. */
int ora_plain_iterations(int m, int n, const int* a_ptr, const int* a_idx, const double* a_val,
                         const int* at_ptr, const int* at_idx, const double* at_val, const double* c,
                         const double* l, const double* u, const double* lo, const double* hi, double tau,
                         double sigma, long iters, double* x, double* y);

/* FP64 KKT of a point (x, y) of an already-scaled LP (pdhg_impl.hpp:92-109
 * over backend_cpu.cpp:101-149): sc = {obj_scale, obj_const, bnorm, cnorm};
 * out = {pobj, dobj, rel_p, rel_d, rel_gap, err}.  Checks the device KKT
 * evaluations. */
int ora_eval_kkt(int m, int n, const int* a_ptr, const int* a_idx, const double* a_val, const int* at_ptr,
                 const int* at_idx, const double* at_val, const double* c, const double* l, const double* u,
                 const double* lo, const double* hi, const double* rres, const double* cres, const double* x,
                 const double* y, const double* sc, double* out);

/* Counting-sort transpose (lp.cpp:55-72) into caller buffers: t_ptr[cols+1],
 * t_idx / t_val[ptr[rows]].  Checks the device transpose. */
int ora_transpose(int rows, int cols, const int* ptr, const int* idx, const double* val, int* t_ptr, int* t_idx,
                  double* t_val);

#ifdef __cplusplus
}
#endif
#endif

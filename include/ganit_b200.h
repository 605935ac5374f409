/*
 * ganit_b200.h -- C ABI of the B200-native restarted-PDHG engine (LP + convex QP).
 *
 * Library: ganit_v2_b200/libganit_b200.so (sm_100a).  Every function returns
 * an int status (GB_OK == 0, negative on error) and never throws; the message
 * of the last error on the calling thread is gb_last_error().  Handles are
 * bound to one CUDA device and one stream and are not thread-safe; the caller
 * owns every host buffer, the library owns every device buffer.
 *
 * Three layers, each replacing one reference interface (paths inside the
 * GANIT_v2 project):
 *
 *  1. Fused solver      gb_solve / gb_problem_*        replaces
 *       ganit::solve_pdhg_gpu(const LP&, const Options&)  include/ganit/pdhg.hpp:44-47,
 *       i.e. run_pdhg<CudaBackend...> (src/pdhg_impl.hpp:243-328, src/backend_cuda.cu:382-393).
 *       Scaling, the PDHG iteration, KKT checks, restarts, primal weight,
 *       infeasibility test, precision phases and FP64 certification all run
 *       on the device; one CUDA-graph launch per precision phase.
 *
 *  2. Backend ops       gb_backend_* / gb_vec_* / gb_spmv_* ...  replace the
 *       compile-time Backend concept that pdhg_impl.hpp drives (implemented by
 *       CudaBackend<M,V>, src/backend_cuda.cu:286-378).  A thin C++ adapter
 *       (include/ganit_b200_backend.hpp) satisfies that concept with these
 *       calls, so run_pdhg can drive the B200 kernels unchanged.
 *
 *  3. Batched and differentiable solving  gb_batch_* / gb_diff_*  (no
 *       counterpart in the reference; README.md:196 lists batched GPU solving
 *       as planned).
 */
#ifndef GANIT_B200_H
#define GANIT_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes */
enum {
    GB_OK = 0,
    GB_ERR_INVALID = -1,   /* bad argument or malformed problem */
    GB_ERR_CUDA = -2,      /* CUDA runtime error (message in gb_last_error) */
    GB_ERR_NOMEM = -3,     /* device allocation failed */
    GB_ERR_NODEVICE = -4,  /* no sm_100 device visible */
    GB_ERR_UNSUPPORTED = -5
};

/* ---- solver status, include/ganit/pdhg.hpp:27 (same order) */
enum { GB_OPTIMAL = 0, GB_PRIMAL_INFEASIBLE = 1, GB_ITERATION_LIMIT = 2, GB_TIME_LIMIT = 3, GB_NUMERICAL_ERROR = 4,
       /* extension (gb_options.detect_unbounded): a primal ray certifies that
        * the LP is unbounded (its dual infeasible); the reference has no such
        * test and reports ITERATION_LIMIT or TIME_LIMIT there (README.md:197) */
       GB_DUAL_INFEASIBLE = 5 };

/* ---- precision schedule, include/ganit/pdhg.hpp:10 (same order) */
enum { GB_PREC_DOUBLE = 0, GB_PREC_MIXED = 1, GB_PREC_DYNAMIC = 2,
       /* extension (no reference counterpart): a first phase with BF16 matrix
        * values and FP32 iterates, then FP32, then FP64, each exit certified
        * in FP64; LPs only (a QP starts at the FP32 phase) */
       GB_PREC_MIXED_BF16 = 3 };

/* ---- value types for gb_backend_create */
enum { GB_F32 = 0, GB_F64 = 1 };

/* Problem in GANIT's form (include/ganit/lp.hpp:4-47):
 *   minimise c'x + 0.5 x'Qx + obj_const  s.t.  lo <= A x <= hi,  l <= x <= u.
 * A is host CSR (int32 ptr[m+1], idx[nnz], double val[nnz]); bounds may be
 * +-INFINITY.  Q is either a full-storage symmetric CSR (q_ptr != NULL, as in
 * the reference) or diagonal-plus-low-rank Q = 2 (F F^T + diag(D)) with F an
 * n x q_rank row-major host array (q_rank > 0), or absent. */
typedef struct {
    int32_t m, n;
    const int32_t* a_ptr;
    const int32_t* a_idx;
    const double* a_val;
    const double* c;
    const double* l;
    const double* u;
    const double* lo;
    const double* hi;
    double obj_const;
    int32_t maximize;
    const int32_t* q_ptr;
    const int32_t* q_idx;
    const double* q_val;
    int32_t q_rank;
    const double* q_F;
    const double* q_D;
} gb_lp;

/* ganit::Options (include/ganit/pdhg.hpp:12-25), same meaning and defaults. */
typedef struct {
    double tol;              /* 1e-4 relative KKT tolerance */
    int64_t max_iter;        /* 10000000 */
    double time_limit;       /* 3600 s */
    int32_t check_every;     /* 64 */
    int32_t ruiz_iters;      /* 10 */
    int32_t pock_chambolle;  /* 1 */
    double infeas_tol;       /* 1e-8 */
    int32_t precision;       /* GB_PREC_DOUBLE */
    int32_t stall_checks;    /* 12 */
    int32_t stall_checks_l2; /* 24 */
    int32_t verbose;         /* 0 (the engine prints nothing) */
    /* Extension, off by default (as the reference): test the primal ray
     * d = x - x_r every check once 4 checks have passed since the last
     * restart, and stop with GB_DUAL_INFEASIBLE when c'd < 0 and the
     * violation of d's recession conditions (A d within the rows' recession
     * cones, d within the bounds') divided by -c'd is <= infeas_tol.  LPs. */
    int32_t detect_unbounded;
} gb_options;

/* ganit::Result (include/ganit/pdhg.hpp:30-42) without the vectors, which go
 * to caller buffers; plus engine diagnostics. */
typedef struct {
    int32_t status;
    double pobj, dobj;
    double rel_primal, rel_dual, rel_gap;
    int64_t iterations, fp32_iterations, l2_iterations;
    int32_t restarts;
    double setup_seconds, solve_seconds;
    double norm_a;        /* ||A'||_2 estimate of the scaled matrix */
    double primal_weight; /* final primal weight w */
    int32_t checks;       /* KKT checks performed */
    int32_t phases;       /* precision phases run */
    int64_t bf16_iterations; /* iterations of the BF16-matrix phase (GB_PREC_MIXED_BF16) */
} gb_result;

/* ---------------------------------------------------------------- common */
const char* gb_last_error(void);
/* Device memory: the library keeps the blocks it frees (per device and
 * size, at most GANIT_B200_POOL_BYTES, default 4 GiB) and reuses them for the
 * next problem of the same shape, because cudaMalloc / cudaFree of a
 * problem's buffers can cost more than its solve.  The small pinned host
 * arrays of a problem's state are kept the same way (at most 256 MiB).  A
 * block is cached only after a device synchronisation, as cudaFree would do
 * (one per destroyed problem).  Release returns every cached block, device
 * and pinned host, to the driver; the second call reports the device bytes
 * cached. */
void gb_release_cached_memory(void);
int64_t gb_cached_memory_bytes(void);
int gb_version(void);                       /* 10000*major + 100*minor + patch */
void gb_default_options(gb_options* opt);
/* Selects the CUDA device used by handles created afterwards on this thread. */
int gb_set_device(int device);
/* Transpose of a rows x cols CSR matrix (replaces ganit::transpose,
 * include/ganit/lp.hpp:32, src/lp.cpp:55-72), computed on the device the way
 * the solver builds A^T: every output row lists its entries in increasing
 * source row, so the result equals the reference's counting transpose.
 * ptr: rows + 1 non-decreasing offsets from 0; idx: ptr[rows] column indices
 * in [0, cols) (checked on the host before upload); val / t_val: optional
 * (both or neither).  Outputs: t_ptr (cols + 1), t_idx and t_val (ptr[rows]).
 * Synchronous. */
int gb_csr_transpose(int rows, int cols, const int* ptr, const int* idx, const double* val, int* t_ptr, int* t_idx,
                     double* t_val);

/* ---------------------------------------------------------------- 1. fused solver */
/* One-shot solve of a host problem: upload, scale (on the device), restarted
 * PDHG with the precision schedule of opt, FP64 certification, unscale,
 * download.  x_out[n] / y_out[m] may be NULL.  Same contract as
 * ganit::solve_pdhg_gpu (include/ganit/pdhg.hpp:44-47). */
int gb_solve(const gb_lp* lp, const gb_options* opt, gb_result* res, double* x_out, double* y_out);

typedef struct gb_problem gb_problem;
/* Upload + scale once (scaling options taken from opt: ruiz_iters,
 * pock_chambolle); the scaled problem stays resident in HBM. */
int gb_problem_create(const gb_lp* lp, const gb_options* opt, gb_problem** out);
/* Solve the resident problem from the default start (x0 = proj(0), y0 = 0).
 * Results stay on the device until gb_problem_get_solution. */
int gb_problem_solve(gb_problem* p, const gb_options* opt, gb_result* res);
/* Copy the unscaled solution of the last solve to host buffers (either may be NULL). */
int gb_problem_get_solution(gb_problem* p, double* x_out, double* y_out);
/* Warm start (extension, as gb_batch_set_start): later solves start from
 * (x, y) in original units; both NULL restores the default start. */
int gb_problem_set_start(gb_problem* p, const double* x, const double* y);
void gb_problem_destroy(gb_problem* p);
/* Stream the problem's work is issued on (a cudaStream_t). */
void* gb_problem_stream(gb_problem* p);
/* Kernel-level timing of one precision level (0 = L1, 1 = L2, 2 = L3,
 * 3 = the BF16-matrix level of GB_PREC_MIXED_BF16, LPs only):
 * runs `iters` plain PDHG iterations from the current iterate with CUDA
 * events around every launch and reports the mean duration (ms) of the fused
 * primal kernel (A^T y + primal step) and of the fused dual kernel (A xbar +
 * dual step), and the number of launches issued. */
int gb_problem_time_kernels(gb_problem* p, int level, int iters, double* ms_primal, double* ms_dual,
                            int64_t* launches);
/* Counters of the last gb_problem_solve: kernel launches issued inside the
 * solve, and algorithmic bytes moved by the fused iteration kernels per
 * iteration at each level (index 0..2 = L1..L3). */
int gb_problem_stats(gb_problem* p, int64_t* launches, double* bytes_per_iter_level);
/* Same kernels launched back to back: `iters` launches of the fused primal
 * kernel, then of the fused dual kernel, each captured into a CUDA graph with
 * programmatic dependent launch exactly as the solve loop issues them and
 * timed with two CUDA events; also `iters` full iterations.  Mean ms per
 * launch / per iteration (warm L2). */
int gb_problem_time_kernels_graph(gb_problem* p, int level, int iters, double* ms_primal, double* ms_dual,
                                  double* ms_iteration);
/* Row-split schedule autotuner for one resident problem (see
 * gb_batch_autotune): after a first solve, times candidate (block_nnz,
 * max_rows) cuts of the CSR row blocks -- including cuts into whole waves of
 * resident CTAs -- separately for the FP32/BF16-matrix kernels and the FP64
 * ones, and keeps the fastest of each.  Outputs are pairs [FP32, FP64]
 * (block_nnz[2], max_rows[2], ms_default[2], ms_tuned[2]; any may be NULL).
 * Results stay certified; only the summation grouping inside a row changes. */
int gb_problem_autotune(gb_problem* p, int iters, int* block_nnz, int* max_rows, double* ms_default,
                        double* ms_tuned);

/* ---------------------------------------------------------------- 2. backend ops
 * Mirrors the Backend concept used at src/pdhg_impl.hpp:73-84, 92-118,
 * 133-137, 145-146, 178-194, 207-220.  The problem passed to
 * gb_backend_create is already SCALED (ganit::ScaledLP, src/scaling.hpp:8-23):
 * A and its stored transpose AT, optional CSR Q, and the scaled vectors. */
typedef struct {
    int32_t m, n;
    const int32_t* a_ptr; const int32_t* a_idx; const double* a_val;
    const int32_t* at_ptr; const int32_t* at_idx; const double* at_val;
    const int32_t* q_ptr; const int32_t* q_idx; const double* q_val; /* NULL for LP */
    const double *c, *l, *u, *lo, *hi, *rres, *cres;
} gb_scaled_lp;

typedef struct gb_backend gb_backend;
typedef struct gb_vec gb_vec;

/* CudaBackend<M,V>(const ScaledLP&) (backend_cuda.cu:294-303); mat_type and
 * vec_type are GB_F32 / GB_F64. */
int gb_backend_create(const gb_scaled_lp* s, int mat_type, int vec_type, gb_backend** out);
void gb_backend_destroy(gb_backend* b);
/* zeros(k) (backend_cuda.cu:305) */
int gb_vec_zeros(gb_backend* b, int k, gb_vec** out);
/* from_host(h) (backend_cuda.cu:306) */
int gb_vec_from_host(gb_backend* b, const double* h, int k, gb_vec** out);
/* to_host(v) (backend_cuda.cu:307-315); h must hold gb_vec_size(v) doubles */
int gb_vec_to_host(gb_backend* b, const gb_vec* v, double* h);
int gb_vec_size(const gb_vec* v);
void gb_vec_destroy(gb_vec* v);
/* copy / fill (backend_cuda.cu:316-322) */
int gb_copy(gb_backend* b, const gb_vec* src, gb_vec* dst);
int gb_fill(gb_backend* b, gb_vec* v, double a);
/* spmv_A / spmv_AT / spmv_Q (backend_cuda.cu:324-335) */
int gb_spmv_A(gb_backend* b, const gb_vec* x, gb_vec* ax);
int gb_spmv_AT(gb_backend* b, const gb_vec* y, gb_vec* aty);
int gb_spmv_Q(gb_backend* b, const gb_vec* x, gb_vec* qx);
/* primal_step / dual_step (backend_cuda.cu:337-344); qx may be NULL */
int gb_primal_step(gb_backend* b, const gb_vec* x, const gb_vec* aty, const gb_vec* qx, double tau, gb_vec* xn,
                   gb_vec* xbar, gb_vec* sumx);
int gb_dual_step(gb_backend* b, const gb_vec* y, const gb_vec* axbar, double sigma, gb_vec* yn, gb_vec* sumy);
/* sub / scale_into (backend_cuda.cu:345-350) */
int gb_sub(gb_backend* b, const gb_vec* a, const gb_vec* c, gb_vec* d);
int gb_scale_into(gb_backend* b, const gb_vec* src, double a, gb_vec* dst);
/* FP64-accumulated reductions (backend_cuda.cu:363-377), results to host */
int gb_primal_res2(gb_backend* b, const gb_vec* ax, double* out);
int gb_dual_res(gb_backend* b, const gb_vec* aty, const gb_vec* qx, int with_c, double* rd2, double* vobj);
int gb_row_dual_obj(gb_backend* b, const gb_vec* y, double* out);
int gb_dot(gb_backend* b, const gb_vec* a, const gb_vec* c, double* out);
int gb_dot_c(gb_backend* b, const gb_vec* x, double* out);
int gb_diff2(gb_backend* b, const gb_vec* a, const gb_vec* c, double* out);

/* ---------------------------------------------------------------- KKT check without allocation
 * No counterpart in the reference.  FP64 KKT evaluation of a point (x, y) of
 * an already-scaled LP, for callers that cannot allocate device memory when
 * they need a check: a branch-and-bound worker or solver service working in
 * a fixed device-memory budget, or a latency-critical path where
 * cudaMalloc/cudaFree would synchronise the device and stall other streams.
 *
 * Every pointer member of `dev` (and x[n], y[m]) points to DEVICE memory
 * holding FP64 scaled data as in gb_scaled_lp (q_* must be NULL: LP only);
 * h_a_ptr / h_at_ptr are HOST copies of the two row-pointer arrays.  The
 * scalars are those of the reference's KKT formulas (pdhg_impl.hpp:92-109):
 * obj_scale = cscale*bscale, obj_const (min-sense), and the norms bnorm and
 * cnorm of the original right-hand side and objective.  Work runs on
 * `stream` (a cudaStream_t, NULL = default stream) on the current device and
 * the call returns after the result reached `out`.
 *
 * It calls no cudaMalloc/cudaFree and no allocating library routine: its
 * scratch is a fixed 4 MiB __device__ array inside the library, held on every
 * GPU that loads the library until the process exits.  Limits: at most
 * GB_NOALLOC_MAX_BLOCKS row blocks for A and A^T together (a block is <= 2048
 * nonzeros and <= 256 rows), GB_NOALLOC_MAX_SLOTS chunk slots (a row of
 * A or A^T longer than 4096 nonzeros takes one slot per 2048 nonzeros) and
 * GB_NOALLOC_MAX_LONG_ROWS such rows (each takes one arrival counter);
 * larger problems get GB_ERR_INVALID with a message.  All calls share the
 * array, so calls whose GPU work overlaps (unordered streams or threads)
 * race; the call is synchronous (it waits on `stream` for its result); the
 * first call on a device looks the array up (cudaGetSymbolAddress) and
 * should come before any stream capture. */
#define GB_NOALLOC_MAX_BLOCKS 16384
#define GB_NOALLOC_MAX_SLOTS 8192
#define GB_NOALLOC_MAX_LONG_ROWS 4096
typedef struct {
    double obj_scale, obj_const, bnorm, cnorm;
} gb_kkt_scalars;
typedef struct {  /* KKT of src/pdhg_impl.hpp:36-42 */
    double pobj, dobj, rel_p, rel_d, rel_gap, err;
} gb_kkt;
int gb_eval_kkt_noalloc(const gb_scaled_lp* dev, const int32_t* h_a_ptr, const int32_t* h_at_ptr, const double* x,
                        const double* y, const gb_kkt_scalars* sc, void* stream, gb_kkt* out);

/* ---------------------------------------------------------------- 3a. batched solving
 * Many independent LPs (no Q) resident as ONE block-diagonal problem: every
 * kernel launch covers all instances (a row block never straddles two), and
 * each instance keeps its own scaling, step sizes, KKT checks, restarts,
 * primal weight, infeasibility test, precision phases and FP64
 * certification -- per-instance state lives on the device and a finished
 * instance's row blocks return at once.  Each precision phase is one CUDA
 * graph whose body repeats in a device-side loop.  opt->precision as for
 * gb_solve; every result is certified in FP64. */
typedef struct gb_batch gb_batch;
int gb_batch_create(int count, const gb_lp* lps, const gb_options* opt, gb_batch** out);
/* Solve every instance; results[count] receives per-instance results. */
int gb_batch_solve(gb_batch* b, const gb_options* opt, gb_result* results);
/* Unscaled solution of instance i (either buffer may be NULL). */
int gb_batch_get_solution(gb_batch* b, int i, double* x_out, double* y_out);
/* Schedule chosen by the autotuner: threads per block, blocks per SM, and
 * the row-split group sizes picked per instance (written to groups[count*2]
 * when groups != NULL: group size for A rows, for A^T rows). */
int gb_batch_schedule(gb_batch* b, int* threads, int* blocks_per_sm, int* groups);
/* Row-split schedule autotuner: per class of instance sizes (four classes of
 * equal total nonzeros), picks (block_nnz, max_rows) of the CSR row blocks by
 * timing `iters` fused iterations per candidate with CUDA events -- once for
 * the schedule of the FP32/BF16-matrix kernels (timed at FP32), once for that
 * of the FP64 kernels (timed at FP64).  Writes the chosen values per instance
 * (arrays of 2 * count: FP32 schedule then FP64; may be NULL) and the
 * per-iteration kernel time of the default and tuned schedules (ms, [2]). */
int gb_batch_autotune(gb_batch* b, int iters, int* block_nnz, int* max_rows, double* ms_default, double* ms_tuned);
/* Load variant of the fused iteration kernels, per matrix and precision
 * class: modes[0..3] = A (FP32/BF16 kernels), A^T (FP32/BF16), A (FP64),
 * A^T (FP64); GB_LOAD_PLAIN: 16-byte idx / value loads through L1;
 * GB_LOAD_STREAM: the same loads without L1 allocation; GB_LOAD_PREFETCH:
 * the streaming loads after a bulk L2 prefetch of each row block's window,
 * issued before the kernel waits for its predecessor.  Untuned, a matrix
 * streams when an iteration's data exceeds the L2 (126 MB) and loads plainly
 * otherwise (GANIT_B200_LOADS=plain|stream|prefetch forces one); the
 * autotuners time all three per matrix and keep the fastest. */
enum { GB_LOAD_PLAIN = 0, GB_LOAD_STREAM = 1, GB_LOAD_PREFETCH = 2 };
int gb_batch_load_modes(gb_batch* b, int* modes);
int gb_problem_load_modes(gb_problem* p, int* modes);
/* Average device time of the two fused iteration kernels over `iters`
 * iterations at a precision level (0 = FP32, 1 = FP32 matrix / FP64 vectors,
 * 3 = BF16 matrix / FP32 vectors,
 * 2 = FP64), all instances active, and the algorithmic bytes of one iteration. */
int gb_batch_time_kernels(gb_batch* b, int level, int iters, double* ms_primal, double* ms_dual, int64_t* launches,
                          double* bytes_per_iter);
int gb_batch_time_kernels_graph(gb_batch* b, int level, int iters, double* ms_primal, double* ms_dual,
                                double* ms_iteration);
void gb_batch_destroy(gb_batch* b);
/* Warm start (extension; the reference always starts from the projection of
 * 0 and y = 0): instance i starts every later solve from x (n_i) / y (m_i)
 * in original units, x projected onto its bounds; a NULL side or a NaN entry
 * keeps the default.  gb_batch_clear_start drops every start. */
int gb_batch_set_start(gb_batch* b, int i, const double* x, const double* y);
int gb_batch_clear_start(gb_batch* b);

/* ---------------------------------------------------------------- 3c. problem files
 * Replaces ganit::read_mps (src/mps.cpp:69-272) for callers that feed the
 * engine directly from an MPS / QPS file, with the same format rules
 * (sections, N rows, RHS / RANGES / BOUNDS semantics, QUADOBJ mirrored).
 * gb_model_lp returns a view of the model, valid until gb_model_free, that
 * gb_solve / gb_problem_create accept; gb_model_is_int its integrality (n
 * bytes, 1 = integer: columns between 'MARKER' INTORG / INTEND lines and
 * columns with a UI, LI or BV bound, as src/mps.cpp:149-229), which the LP
 * solvers ignore (they solve the relaxation). */
typedef struct gb_model gb_model;
int gb_read_mps(const char* path, gb_model** out);
const gb_lp* gb_model_lp(const gb_model* model);
const char* gb_model_name(const gb_model* model);
const unsigned char* gb_model_is_int(const gb_model* model);
void gb_model_free(gb_model* model);

/* Factor-model rewrite (no reference counterpart).  A QP with a diagonal CSR
 * Hessian in the lifted form of a factor risk model -- free columns f_k with
 * curvature q_k > 0, each in exactly one equality row a_k f_k + g'x = b_k
 * that holds no other such column (the form bench/gen_portfolio.py of the
 * reference writes) -- is rewritten over x alone with Q = 2 (F F^T + diag(D)),
 * F[:, k] = sqrt(q_k / 2) (-row_k / a_k), D = diag(Q_xx) / 2, for the engine's
 * diagonal-plus-low-rank kernel.  GB_ERR_UNSUPPORTED when no such structure
 * (or more than 128 factors, or a non-diagonal / indefinite Hessian, or a
 * maximisation).  gb_factor_expand maps a solution (x, y) of the rewritten
 * problem back: x_full (n of the input), y_full (m of the input), with
 * f_k = (b_k - g'x) / a_k and y_k = (c_k + q_k f_k) / a_k. */
typedef struct gb_factor gb_factor;
int gb_factor_detect(const gb_lp* qp, gb_factor** out);
const gb_lp* gb_factor_lp(const gb_factor* f);
int gb_factor_expand(const gb_factor* f, const double* x, const double* y, double* x_full, double* y_full);
void gb_factor_free(gb_factor* f);

/* ---------------------------------------------------------------- 3d. strong branching
 * Replaces the per-candidate strong-branching loop of Mip::select_branch
 * (src/mip.cpp:727-783), where each child LP is a warm dual-simplex re-solve
 * followed by Mip::safe_bound (src/mip.cpp:356-410).  Here the 2 * count
 * children of the candidate columns cand[] of the node LP `lp` (its column
 * bounds are the node's) -- down: u_j = floor(x_j), up: l_j = ceil(x_j) --
 * are solved together as one gb_batch with `opt`, and each child's rigorous
 * Lagrangian lower bound is formed on the device from its duals with
 * directed rounding.  1 <= count <= 32767; every x[cand[k]] must be finite
 * and not integral (GB_ERR_INVALID otherwise); a Hessian gives
 * GB_ERR_UNSUPPORTED (LPs only).
 * y (may be NULL): the node's row duals (minimisation form, as x and y of a
 * gb_solve of the node LP after negating a maximisation); given, every
 * entry of x and y must be finite and every child starts from (x, y), x
 * projected onto its bounds (the default start otherwise; an extension --
 * the reference's dual simplex starts warm).
 * Objectives are in minimisation form (a maximisation LP's are negated), and
 * node_obj / cutoff are too (cutoff = INFINITY: no incumbent).
 * Per child (index 0 = down, 1 = up), as src/mip.cpp:750-763: z = +INF when
 * the child is primal infeasible (also when its bounds cross), when its
 * certified bound is >= cutoff, or when it is GB_OPTIMAL with an objective
 * >= cutoff (the reference's dual simplex stops with Cutoff there); else its
 * objective when GB_OPTIMAL; else max(node_obj, cert), or node_obj when
 * cert = -INF (not certifiable).
 * The certified bound uses the child's own column bounds: unlike
 * Mip::safe_bound (src/mip.cpp:361-364), no implied bounds replace infinite
 * ones, so a child with an unbounded column whose reduced-cost interval has
 * the wrong sign gets cert = -INF where the reference may certify a finite
 * bound. */
typedef struct {
    double z[2];          /* child objective estimate */
    double cert[2];       /* certified lower bound (+INF: infeasible; -INF: none) */
    int32_t status[2];    /* GB_OPTIMAL ... of the child solve */
    int64_t iterations[2];
    double score;         /* max(z0 - node_obj, 1e-6) * max(z1 - node_obj, 1e-6); 0 if a z is +INF */
} gb_branch_cand;
/* The decision select_branch takes, scanning cand[] in order: the first
 * candidate with both children +INF makes the node infeasible, the first
 * with one makes the column tightened to the other side; else the largest
 * score wins (first on ties). */
enum { GB_BRANCH_VAR = 0, GB_BRANCH_TIGHTEN = -1, GB_BRANCH_NODE_INFEASIBLE = -2 };
typedef struct {
    int32_t action;       /* GB_BRANCH_* (the return value of select_branch) */
    int32_t var;          /* column branched on / tightened / found infeasible */
    double lo, hi;        /* GB_BRANCH_TIGHTEN: the column's new bounds */
    double est[2];        /* GB_BRANCH_VAR: est_down / est_up of the chosen column */
    double cert[2];       /* GB_BRANCH_VAR: cert_down / cert_up of the chosen column */
    int32_t children_solved; /* children in the batch (bounds that cross need no solve) */
    double seconds;       /* wall time of the call */
} gb_branch_decision;
int gb_strong_branch(const gb_lp* lp, const double* x, const double* y, int32_t count, const int32_t* cand,
                     double node_obj, double cutoff, const gb_options* opt, gb_branch_cand* out,
                     gb_branch_decision* decision);

/* ---------------------------------------------------------------- 3b. differentiable solving
 * No counterpart in the reference (it differentiates run_pdhg,
 * src/pdhg_impl.hpp:243-328).  LPs only.
 * Forward: the batch engine solves every instance to opt->tol, then
 * `tail_iters` (K) plain PDHG iterations run in FP64 with the final step
 * sizes and no restart, keeping a checkpoint of (x, y) every `ckpt_every` (R)
 * iterations; the outputs are the last tail iterate (x*, y*) in original
 * units, certified again in FP64 (results[] report that point's KKT).
 * Unless switched off, the tail starts from a POLISHED point: the active set
 * one PDHG step reads off the solver's point defines a reduced KKT system
 * (B^T y_D = c_F, B x_F = b_D - A[D,N] x_N, B = A[D,F]), solved per instance by
 * MINRES; the vertex it gives replaces the PDHG point when it certifies
 * better in FP64 (OSQP-style polishing).  A polished start is a fixed point of
 * the PDHG map, so the tail then reproduces it.  When the active set is not
 * square (|D| != |F|, impossible at a nondegenerate vertex: a dual or a slack
 * within the tolerance of zero was misread, and the reduced system is
 * inconsistent), the excess rows leave D smallest |y| first (equality rows
 * stay) or the excess free columns go to their nearest finite bound before
 * the solve (info.active_set_repaired).  With polishing on
 * (and implicit_max_iters > 0) and opt->tol below 4e-4, the solve goes in
 * rounds: first to 4e-4; every instance whose polished vertex certifies at
 * opt->tol keeps it; the rest continue, warm-started from their points, at a
 * tolerance four times tighter per round, down to opt->tol, where the last
 * round polishes as above (results[].iterations counts every round).
 * Backward: given dL/dx* and dL/dy*, exact reverse mode through the K tail
 * iterations (each R-segment recomputed from its checkpoint; projections,
 * extrapolation and the scaling are differentiated), then -- unless switched
 * off -- an implicit completion that accounts for the tail start being a
 * fixed point of the PDHG map: a per-instance MINRES solve on the projection
 * masks of that point (for a nondegenerate vertex this is the basis
 * sensitivity).  Returns dL/dc, dL/dlo, dL/dhi and dL/d(A values) (CSR order
 * of the input A) in original units; scaling factors are held constant.
 * An instance whose completion did not converge (info.implicit_converged = 0)
 * gets NaN in all of its gradient entries rather than an unverified value. */
typedef struct gb_diff gb_diff;
typedef struct {
    int64_t implicit_max_iters;     /* MINRES steps per instance at most (0: truncated gradient,
                                       the exact gradient of the K-step map with its start held fixed);
                                       also bounds the polishing solve */
    double implicit_tol;            /* relative residual at which MINRES stops */
    int32_t polish;                 /* polish the solver's point before the tail */
    int32_t pad;
} gb_diff_options;
void gb_diff_default_options(gb_diff_options* o); /* 20000, 1e-10, polish on */
typedef struct {
    double tau, sigma;              /* tail step sizes (scaled problem) */
    int64_t tail_iterations;        /* K */
    int64_t checkpoint_every;       /* R */
    int64_t implicit_iterations;    /* MINRES steps of the last backward */
    double implicit_residual;       /* its final relative residual */
    int32_t implicit_converged;     /* residual <= implicit_tol reached */
    int32_t free_cols;              /* columns strictly inside their box at the tail start (-1: unknown) */
    int32_t active_rows;            /* rows whose dual is not projected to 0 there (-1: unknown) */
    int32_t polished;               /* the tail started from the polished vertex */
    int32_t active_set_repaired;    /* polishing repaired a non-square active set (see gb_diff_forward) */
    int32_t pad;
    int64_t polish_iterations;      /* MINRES steps of the polishing solve */
    int64_t launches;               /* kernel launches of the last forward / backward call */
} gb_diff_info;
int gb_diff_create(int count, const gb_lp* lps, const gb_options* opt, int tail_iters, int ckpt_every,
                   gb_diff** out);
int gb_diff_set_options(gb_diff* d, const gb_diff_options* o);
/* x_out: concatenation of the instances' x (sum n), y_out: of y (sum m). */
int gb_diff_forward(gb_diff* d, const gb_options* opt, gb_result* results, double* x_out, double* y_out);
/* dl_dx (sum n), dl_dy (sum m) in (NULL = zero); dl_dc (sum n), dl_dlo /
 * dl_dhi (sum m), dl_dval (sum nnz) out.  Any output may be NULL. */
int gb_diff_backward(gb_diff* d, const double* dl_dx, const double* dl_dy, double* dl_dc, double* dl_dlo,
                     double* dl_dhi, double* dl_dval);
int gb_diff_get_info(gb_diff* d, int i, gb_diff_info* out);
/* Scaled tail start point z_0 (sum n, sum m), for checking the K-step map. */
int gb_diff_tail_start(gb_diff* d, double* x_scaled, double* y_scaled);
void gb_diff_destroy(gb_diff* d);

#ifdef __cplusplus
}
#endif
#endif /* GANIT_B200_H */

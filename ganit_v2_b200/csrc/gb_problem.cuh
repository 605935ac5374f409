// Host-side engine state for a resident batch of problems (one problem is a
// batch of one): upload, device setup, precision phases driven by per-level
// CUDA graphs whose body (check_every iterations + KKT check + restart)
// repeats inside a device-side while loop.
#pragma once
#include <chrono>
#include <memory>
#include <type_traits>

#include "../../include/ganit_b200.h"
#include "gb_pdhg.cuh"
#include "gb_setup.cuh"

namespace gb {

struct DevMat {
    int rows = 0, cols = 0;
    long long nnz = 0;
    DevBuf<int> ptr, idx;
    DevBuf<double> val64;
    DevBuf<float> val32;
    DevBuf<__nv_bfloat16> valbf;  // made on the first solve that asks for the BF16 phase
    DevSchedule sched;    // row blocks of the FP64-matrix kernels (and of all kernels until tuned)
    DevSchedule sched32;  // row blocks tuned for the FP32 / BF16-matrix kernels (empty: use sched)
    int stream_nc[2] = {0, 0};  // CsrView::nc (LoadMode) for the FP32 / BF16 views and for the FP64 view
    int default_nc[2] = {0, 0}; // the untuned choice (from the iteration's bytes against the L2)
    std::vector<int> host_ptr;
    // The schedule the kernels of matrix type M run on: FP32 and BF16 kernels
    // keep more CTAs resident per SM than FP64 ones, so the best cut differs.
    template <class M>
    const DevSchedule& sched_for() const {
        return (!std::is_same<M, double>::value && sched32.nb) ? sched32 : sched;
    }
    template <class M>
    CsrView<M> view() const {
        const DevSchedule& sc = sched_for<M>();
        CsrView<M> v;
        v.ptr = ptr.get();
        v.idx = idx.get();
        v.val = val<M>();
        v.blocks = sc.blocks.get();
        v.slots = sc.slots.get();
        v.counters = sc.counters.get();
        v.bits = sc.bits.get();
        v.rows = rows;
        v.nb = sc.nb;
        v.vec = 1;  // upload_mat / device_transpose / cvt32 allocate padded_nnz, cudaMalloc aligns
        v.nc = stream_nc[sizeof(M) == 8 ? 1 : 0];
        return v;
    }
    template <class M>
    const M* val() const;
};
template <>
inline const double* DevMat::val<double>() const { return val64.get(); }
template <>
inline const float* DevMat::val<float>() const { return val32.get(); }
template <>
inline const __nv_bfloat16* DevMat::val<__nv_bfloat16>() const { return valbf.get(); }

// Problem data and iterate buffers in vector precision V.
template <class V>
struct VecSet {
    DevBuf<V> c, l, u, lo, hi, rres, cres;
    DevBuf<V> x0, x1, xbar, y0, y1, sumx, sumy, xr, yr, qx, qxa;
    DevBuf<V> F, D;  // DPLR factor (n x k) and diagonal in precision V
    void alloc(int n, int m, int qk, bool has_q) {
        for (DevBuf<V>* b : {&c, &l, &u, &cres, &x0, &x1, &xbar, &sumx, &xr}) b->reset(n ? n : 1);
        for (DevBuf<V>* b : {&lo, &hi, &rres, &y0, &y1, &sumy, &yr}) b->reset(m ? m : 1);
        if (has_q) {
            qx.reset(n ? n : 1);
            qxa.reset(n ? n : 1);
        }
        if (qk > 0) {
            F.reset(static_cast<size_t>(n) * qk);
            D.reset(n);
        }
    }
};

struct LevelGraph {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int check_every = 0;
    int ray = 0;  // the check also forms A (x - x_r) (unbounded test)
    // block lists the iteration kernels were captured with (Problem::list_*;
    // their contents may change between phases, their buffers and lengths not)
    const RowBlock* list_a = nullptr;
    const RowBlock* list_t = nullptr;
    int list_na = 0, list_nt = 0;
    long long launches_per_body = 0;
    ~LevelGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// Per-instance outcome of a solve.
struct InstanceResult {
    int status = GB_NUMERICAL_ERROR;
    long long bf16_iters = 0, fp32_iters = 0, l2_iters = 0;
    int phases = 0;
};

struct Problem {
    FreeBatchEnd free_batch;              // first member, destroyed last: closes the teardown's free batch
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    int count = 1;                        // instances
    int m = 0, n = 0;                     // totals
    std::vector<int> row_off, col_off, nnz_off;  // instance boundaries (count + 1)
    DevBuf<int> d_row_off, d_col_off, d_nnz_off;
    DevBuf<int> inst_row, inst_col;       // row / column -> instance (empty for one instance)
    std::vector<char> maximize;
    std::vector<double> obj_const;
    DevMat A, AT, Q;
    bool has_q = false, dplr = false;
    int qk = 0;
    DevBuf<int> perm, row_of, q_row_of;
    DevBuf<double> c, l, u, lo, hi, R, C, Rres, Cres;  // scaled FP64 data
    DevBuf<double> F64, D64;                            // scaled DPLR factor
    DevBuf<double> scal;                                // count x kScal per-instance scalars
    std::vector<double> scal_host;
    DevBuf<double> red_partials;
    DevBuf<unsigned> red_arrivals;        // k_red's arrival counter (re-armed by its last CTA)
    DevBuf<double> x64, y64, xr64, yr64, xo, yo;
    DevBuf<double> x_start, y_start;      // warm start in original units (NaN: default start); empty: none
    DevBuf<double> work1, work2;          // n / m FP64 scratch
    DevBuf<double> ftx;                   // F^T x of the DPLR Hessian (2 x qk, FP64)
    DevBuf<unsigned> decide_sync;         // k_decide's {arrivals, any active} (re-armed by its last CTA)
    VecSet<float> v32;
    VecSet<double> v64;
    DevBuf<SolveState> st;                // per instance
    SolveState* st_host = nullptr;        // pinned mirror (count entries)
    DevBuf<int> phase_flags;              // per-instance flags uploaded for a phase
    int* phase_flags_host = nullptr;      // pinned
    DevBuf<double> partials;
    // Phase graphs: levels <f32,f32>, <f32,f64>, <f64,f64>, <bf16,f32>, then the
    // same four for phases that run on block lists.
    std::unique_ptr<LevelGraph> graphs[8];
    DevBuf<double> w_start;               // per-instance primal weight of a warm start (<= 0: the default)
    // Row blocks of the current phase when only some instances of a batch take
    // part and their blocks are at most half of all: copies of those
    // instances' RowBlocks, which the iteration kernels of level list_level
    // run alone (list_level -1: none).
    DevBuf<RowBlock> list_a, list_t;
    int list_na = 0, list_nt = 0, list_level = -1;
    double setup_seconds = 0.0;
    long long launches = 0;               // kernel launches of the last solve
    std::vector<InstanceResult> results;
    bool solved = false;
    bool detect_unbounded = false;        // option of the current solve (LPs)
    // row-split schedule tunables per instance and schedule (index 0: FP32 /
    // BF16 kernels, 1: FP64 kernels); set by the autotuner
    std::vector<int> tune_block_nnz[2], tune_max_rows[2];

    const int* icol() const { return count > 1 ? inst_col.get() : nullptr; }
    const int* irow() const { return count > 1 ? inst_row.get() : nullptr; }

    ~Problem() {
        cudaSetDevice(device);
        begin_free_batch();  // one device synchronisation for all the buffers freed below
        free_batch.open = true;
        for (auto& g : graphs) g.reset();
        host_free(st_host);
        host_free(phase_flags_host);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Engine entry points (gb_engine.cu) shared with the differentiable layer.
extern thread_local std::string g_last_error;
Problem* create_problem(int count, const gb_lp* lps, const gb_options* opt);
void solve_problem(Problem& P, const gb_options* opt, gb_result* res);
void set_start(Problem& P, int inst, const double* x, const double* y);
void clear_start(Problem& P);
// GANIT_B200_LAUNCH=stream: loops that otherwise run as conditional CUDA
// graphs are driven from the host (kernel profilers see their kernels).
bool host_loop_mode();
void certify(Problem& P);  // FP64 KKT of (x64, y64) of every instance into st_host[k].kcert

// Runs f, turning exceptions into the ABI's status codes (message in g_last_error).
template <class F>
int guarded(F&& f) {
    try {
        f();
        return GB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return GB_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GB_ERR_INVALID;
    }
}

}  // namespace gb

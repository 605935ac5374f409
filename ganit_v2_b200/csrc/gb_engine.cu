// Engine for a resident batch of problems and the C ABI of the fused solver
// (include/ganit_b200.h).  One problem is a batch of one.
//
// gb_solve / gb_problem_*  : restarted PDHG with every step on the device
//                            (replaces ganit::solve_pdhg_gpu, backend_cuda.cu:382-393)
// gb_batch_*               : many independent LPs as one block-diagonal problem,
//                            each instance with its own scaling, step sizes,
//                            restarts, primal weight, phases and certification
#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>

#include "gb_problem.cuh"
#include "gb_qp.cuh"

namespace gb {

thread_local std::string g_last_error;
thread_local int g_device = 0;

// Compute capability and SM count of a device, looked up once per device
// (cudaDeviceGetAttribute; a full cudaGetDeviceProperties costs milliseconds).
inline void check_device(int dev, int* sms) {
    static std::mutex mu;
    static std::vector<std::array<int, 3>> seen;  // device, major*10+minor, SMs
    {
        std::lock_guard<std::mutex> g(mu);
        for (const auto& d : seen)
            if (d[0] == dev) {
                *sms = d[2];
                return;
            }
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw Error(GB_ERR_NODEVICE, "no CUDA device");
    GB_REQUIRE(dev >= 0 && dev < count, "device index out of range");
    int major = 0, minor = 0, nsm = 0;
    GB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    GB_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
    GB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (major < 10) throw Error(GB_ERR_NODEVICE, "libganit_b200 is built for sm_100a (B200); found sm_" +
                                                     std::to_string(major) + std::to_string(minor));
    std::lock_guard<std::mutex> g(mu);
    seen.push_back({dev, major * 10 + minor, nsm});
    *sms = nsm;
}

// Opt a kernel into the dynamic shared memory it needs.
template <class K>
void set_smem(K kernel, size_t bytes) {
    GB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
}

void validate_lp(const gb_lp* lp) {
    GB_REQUIRE(lp != nullptr, "lp is NULL");
    GB_REQUIRE(lp->m > 0 && lp->n > 0, "need m > 0 and n > 0");
    GB_REQUIRE(lp->a_ptr && lp->c && lp->l && lp->u, "missing A/c/l/u");
    GB_REQUIRE(lp->lo && lp->hi, "missing lo/hi");
    GB_REQUIRE(lp->a_ptr[0] == 0, "A.ptr[0] must be 0");
    for (int i = 0; i < lp->m; ++i) GB_REQUIRE(lp->a_ptr[i + 1] >= lp->a_ptr[i], "A.ptr must be nondecreasing");
    const long long nnz = lp->a_ptr[lp->m];
    GB_REQUIRE(nnz == 0 || (lp->a_idx && lp->a_val), "missing A.idx/val");
    if (lp->q_rank > 0) {
        GB_REQUIRE(lp->q_F && lp->q_D, "DPLR Hessian needs q_F and q_D");
        GB_REQUIRE(lp->q_rank <= kMaxRank, "DPLR rank above 128");
        GB_REQUIRE(!lp->maximize, "DPLR Hessian supports minimisation only");
    }
    if (lp->q_ptr) {
        GB_REQUIRE(lp->q_ptr[0] == 0, "Q.ptr[0] must be 0");
        for (int i = 0; i < lp->n; ++i) GB_REQUIRE(lp->q_ptr[i + 1] >= lp->q_ptr[i], "Q.ptr must be nondecreasing");
        const long long qn = lp->q_ptr[lp->n];
        for (long long p = 0; p < qn; ++p) GB_REQUIRE(lp->q_idx[p] >= 0 && lp->q_idx[p] < lp->n, "Q.idx out of range");
    }
}

// The entry checks of validate_lp's problem (column indices in range, l <= u):
// the long passes, run while the upload of the same arrays is in flight and
// before any kernel indexes with A.idx.
void validate_entries(const gb_lp* lp) {
    const long long nnz = lp->a_ptr[lp->m];
    int lo_idx = 0, hi_idx = 0;  // one vectorisable min / max pass instead of a branch per entry
    for (long long p = 0; p < nnz; ++p) {
        lo_idx = std::min(lo_idx, lp->a_idx[p]);
        hi_idx = std::max(hi_idx, lp->a_idx[p]);
    }
    GB_REQUIRE(lo_idx >= 0 && (nnz == 0 || hi_idx < lp->n), "A.idx out of range");
    for (int j = 0; j < lp->n; ++j) GB_REQUIRE(!(lp->l[j] > lp->u[j]), "column bound l > u");
}

void upload_mat(DevMat& M, int rows, int cols, const int* ptr, const int* idx, const double* val, cudaStream_t s) {
    M.rows = rows;
    M.cols = cols;
    M.nnz = ptr[rows];
    M.host_ptr.assign(ptr, ptr + rows + 1);
    M.ptr.reset(rows + 1);
    M.ptr.upload(ptr, rows + 1, s);
    M.idx.reset(padded_nnz(M.nnz));
    M.val64.reset(padded_nnz(M.nnz));
    if (M.nnz) {
        M.idx.upload(idx, M.nnz, s);
        M.val64.upload(val, M.nnz, s);
    }
}

// Transpose of a rows x cols CSR matrix on the device (lp.cpp:55-72): row_of
// = source row of each nonzero; perm = the stable order of the column keys,
// so every output row lists its entries in increasing source row; t_ptr =
// the exclusive scan of the column counts; t_idx (and t_val when val and
// t_val are given) gathered through perm.  Column indices must lie in
// [0, cols).  The scratch buffers stay with the caller until it synchronises.
struct TransposeScratch {
    DevBuf<int> cnt, tile_sum;
    SortScratch sort;
};
// With host_ptr, t_ptr is also copied to that pageable host array as soon as
// it is formed: the copy returns then, and the sort and gather are enqueued
// after it, so the caller works on t_ptr while they run.
void transpose_csr(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val, int* row_of,
                   int* perm, int* t_ptr, int* t_idx, double* t_val, int sms, TransposeScratch& w, cudaStream_t s,
                   int* host_ptr = nullptr) {
    const int g = elem_grid(std::max<long long>(nnz, static_cast<long long>(rows) * 32), sms);
    if (rows) k_row_of<<<g, kThreads, 0, s>>>(rows, ptr, row_of);
    w.cnt.reset(cols + 1);
    w.tile_sum.reset(scan_tiles(cols + 1));
    GB_CUDA(cudaMemsetAsync(w.cnt.get(), 0, sizeof(int) * (cols + 1), s));
    if (nnz) k_count_cols<<<elem_grid(nnz, sms), kThreads, 0, s>>>(nnz, idx, w.cnt.get());
    exclusive_scan(w.cnt.get(), t_ptr, cols + 1, w.tile_sum.get(), s);
    if (host_ptr)
        GB_CUDA(cudaMemcpyAsync(host_ptr, t_ptr, sizeof(int) * (cols + 1), cudaMemcpyDeviceToHost, s));
    if (nnz) {
        int bits = 0;  // column keys lie in [0, 2^bits)
        while ((1LL << bits) < cols) ++bits;
        stable_sort_index(idx, nnz, bits, perm, sms, w.sort, s);
        k_gather_transpose<<<elem_grid(nnz, sms), kThreads, 0, s>>>(nnz, perm, row_of, val, t_idx, t_val);
    }
}

// A^T of a problem: its structure now, its values after the scaling
// (k_gather_transpose through perm again).  Returns with A^T's row pointers
// on the host while the sort may still run; `w` must outlive it.
void device_transpose(Problem& P, TransposeScratch& w, cudaStream_t s) {
    const int nnz = static_cast<int>(P.A.nnz), n = P.n, m = P.m;
    P.AT.rows = n;
    P.AT.cols = m;
    P.AT.nnz = nnz;
    P.row_of.reset(nnz ? nnz : 1);
    P.perm.reset(nnz ? nnz : 1);
    P.AT.ptr.reset(n + 1);
    P.AT.idx.reset(padded_nnz(nnz));
    P.AT.val64.reset(padded_nnz(nnz));
    P.AT.host_ptr.resize(n + 1);
    // (a pageable destination: the copy returns once done, before the sort)
    transpose_csr(m, n, nnz, P.A.ptr.get(), P.A.idx.get(), nullptr, P.row_of.get(), P.perm.get(), P.AT.ptr.get(),
                  P.AT.idx.get(), nullptr, P.sms, w, s, P.AT.host_ptr.data());
}

// Per-instance fixed-order reduction into scal[k][slot]: rows (m) or columns (n).
template <class F, class Post>
void inst_reduce(Problem& P, bool rows, F f, int slot, Post post, cudaStream_t s) {
    if (P.count == 1) {
        reduce_to(s, rows ? P.m : P.n, f, P.red_partials.get(), P.red_arrivals.get(), P.scal.get() + slot, post);
    } else {
        launch_pdl(k_seg_red<F, Post>, P.count, kThreads, 0, s,
                   static_cast<const int*>(rows ? P.d_row_off.get() : P.d_col_off.get()), f, P.scal.get() + slot, post);
    }
}

// Power iteration on the scaled data, per instance (scaling.cpp:131-155 for
// A'^T A', scaling.cpp:108-124 for Q').
void qx_dplr_f64(Problem& P, const double* x, double* out, cudaStream_t s);

void power_iteration(Problem& P, bool q, cudaStream_t s) {
    const int n = P.n;
    double* v = P.x64.get();  // FP64 vectors double as scratch before the solve
    double* w = P.work2.get();
    double* z = P.work1.get();
    double* sc = P.scal.get();
    const int gi = div_up(P.count, kThreads);
    k_fill<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, 1.0, v);
    inst_reduce(P, false, Sq{v}, S_PW_NORM, PostSqrt{}, s);
    k_power_reset<<<gi, kThreads, 0, s>>>(P.count, sc);
    k_power_vec<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, P.icol(), sc, v, v, 0);  // v /= ||v||
    const size_t sm1 = spmv_smem_bytes<1, double>();
    const int iters = q ? 60 : 50;
    for (int it = 0; it < iters; ++it) {
        if (q) {
            if (P.dplr) qx_dplr_f64(P, v, z, s);
            else k_spmv<double, double><<<P.Q.sched.nb, kThreads, sm1, s>>>(P.Q.view<double>(), v, z);
        } else {
            launch_pdl(k_spmv<double, double>, P.A.sched.nb, kThreads, sm1, s, P.A.view<double>(),
                       static_cast<const double*>(v), w);
            launch_pdl(k_spmv<double, double>, P.AT.sched.nb, kThreads, sm1, s, P.AT.view<double>(),
                       static_cast<const double*>(w), z);
        }
        inst_reduce(P, false, Sq{z}, S_PW_NORM, PostSqrt{}, s);
        launch_pdl(k_power_vec, elem_grid(n, P.sms), kThreads, 0, s, n, P.icol(), sc, static_cast<const double*>(z), v,
                   static_cast<int>(P.count));
    }
    k_finish_norms<<<gi, kThreads, 0, s>>>(P.count, P.d_nnz_off.get(), sc, q ? 1 : 0);
}

// DPLR product in FP64 used by the setup power iteration.
void qx_dplr_f64(Problem& P, const double* x, double* out, cudaStream_t s) {
    double* part = P.partials.get();
    double* t = P.ftx.get();
    k_ftx_partial<double, 1><<<kFtxGrid, kThreads, 0, s>>>(P.n, P.qk, P.F64.get(), x, nullptr, nullptr, part);
    k_ftx_final<<<P.qk, 32, 0, s>>>(kFtxGrid, part, t);
    k_dplr_expand<double, 1><<<expand_grid(P.n), kExpandWarps * 32, expand_smem_bytes<double, 1>(P.qk), s>>>(
        P.n, P.qk, P.F64.get(), P.D64.get(), t, x, nullptr, nullptr, out, nullptr);
}

template <class V>
void convert_data(Problem& P, VecSet<V>& vs, cudaStream_t s) {
    const int n = P.n, m = P.m;
    auto cv = [&](const double* src, V* dst, long long k) {
        if (k) k_convert<V><<<elem_grid(k, P.sms), kThreads, 0, s>>>(k, src, dst);
    };
    cv(P.c.get(), vs.c.get(), n);
    cv(P.l.get(), vs.l.get(), n);
    cv(P.u.get(), vs.u.get(), n);
    cv(P.Cres.get(), vs.cres.get(), n);
    cv(P.lo.get(), vs.lo.get(), m);
    cv(P.hi.get(), vs.hi.get(), m);
    cv(P.Rres.get(), vs.rres.get(), m);
    if (P.dplr) {
        cv(P.F64.get(), vs.F.get(), static_cast<long long>(n) * P.qk);
        cv(P.D64.get(), vs.D.get(), n);
    }
}

// Kernels whose dynamic shared memory exceeds the 48 KB default opt in.
void init_kernel_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        set_smem(k_eval<float, float, 2, 3>, spmv_smem_bytes<3, float>());
        set_smem(k_eval<float, double, 2, 3>, spmv_smem_bytes<3, double>());
        set_smem(k_eval<double, double, 2, 3>, spmv_smem_bytes<3, double>());
        // checks that also form A (x - x_r) for the unbounded test
        set_smem(k_eval<float, float, 3, 3>, spmv_smem_bytes<3, float>());
        set_smem(k_eval<float, double, 3, 3>, spmv_smem_bytes<3, double>());
        set_smem(k_eval<double, double, 3, 3>, spmv_smem_bytes<3, double>());
        set_smem(k_spmv_q2<float, double>, spmv_smem_bytes<2, double>());
        // DPLR expansion: rows of F staged per warp, up to the largest rank
        set_smem(k_dplr_expand<float, 1>, expand_smem_bytes<float, 1>(kMaxRank));
        set_smem(k_dplr_expand<float, 2>, expand_smem_bytes<float, 2>(kMaxRank));
        set_smem(k_dplr_expand<double, 1>, expand_smem_bytes<double, 1>(kMaxRank));
        set_smem(k_dplr_expand<double, 2>, expand_smem_bytes<double, 2>(kMaxRank));
        set_smem(k_spmv_q2<double, double>, spmv_smem_bytes<2, double>());
    });
}

// Instance index of every element of [0, off[count]).
__global__ void k_fill_segments(const int* off, int* out) {
    const int k = blockIdx.x;
    for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) out[i] = k;
}

constexpr double kL2StreamBytes = 126.0e6;  // the B200's L2

// Load mode of the iteration kernels forced by GANIT_B200_LOADS (plain,
// stream or prefetch); -1 (unset or "auto"): chosen per matrix and precision
// from the iteration's bytes against the L2.
int load_mode_override() {
    static const int mode = [] {
        const char* v = std::getenv("GANIT_B200_LOADS");
        if (v == nullptr) return -1;
        const std::string s(v);
        if (s == "plain") return static_cast<int>(kLoadPlain);
        if (s == "stream") return static_cast<int>(kLoadStream);
        if (s == "prefetch") return static_cast<int>(kLoadPrefetch);
        return -1;
    }();
    return mode;
}

void prebuild_graphs(Problem& P, const gb_options* opt);

// Upload + device setup (scale_lp + estimate_norm + run_pdhg's start point)
// of `count` instances.
Problem* create_problem(int count, const gb_lp* lps, const gb_options* opt) {
    GB_REQUIRE(count >= 1 && lps != nullptr, "need at least one problem");
    const auto t0 = std::chrono::steady_clock::now();  // setup_seconds covers validation too
    for (int k = 0; k < count; ++k) validate_lp(&lps[k]);
    if (count > 1)
        for (int k = 0; k < count; ++k)
            GB_REQUIRE(lps[k].q_ptr == nullptr && lps[k].q_rank == 0, "batched solving takes LPs only (no Hessian)");
    auto P = std::make_unique<Problem>();
    P->device = g_device;
    GB_CUDA(cudaSetDevice(P->device));
    check_device(P->device, &P->sms);
    init_kernel_attrs();
    GB_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
    cudaStream_t s = P->stream;
    StageTrace tr{s, "setup"};
    tr.mark("stream");
    P->count = count;
    P->row_off.assign(count + 1, 0);
    P->col_off.assign(count + 1, 0);
    P->nnz_off.assign(count + 1, 0);
    P->maximize.resize(count);
    P->obj_const.resize(count);
    for (int k = 0; k < count; ++k) {
        P->row_off[k + 1] = P->row_off[k] + lps[k].m;
        P->col_off[k + 1] = P->col_off[k] + lps[k].n;
        const long long z = static_cast<long long>(P->nnz_off[k]) + lps[k].a_ptr[lps[k].m];
        GB_REQUIRE(z < (1LL << 31) - 16, "more than 2^31 nonzeros in one problem");
        P->nnz_off[k + 1] = static_cast<int>(z);
        P->maximize[k] = lps[k].maximize != 0;
        P->obj_const[k] = lps[k].obj_const;
    }
    const int m = P->row_off[count], n = P->col_off[count];
    P->m = m;
    P->n = n;

    // Host layout of the block-diagonal problem (a single problem is used in place).
    std::vector<int> hptr, hidx;
    std::vector<double> hval, hc, hl, hu, hlo, hhi;
    const int *ap = lps[0].a_ptr, *ai = lps[0].a_idx;
    const double *av = lps[0].a_val, *vc = lps[0].c, *vl = lps[0].l, *vu = lps[0].u, *vlo = lps[0].lo,
                 *vhi = lps[0].hi;
    if (count > 1) {
        hptr.resize(m + 1);
        hidx.resize(P->nnz_off[count]);
        hval.resize(P->nnz_off[count]);
        for (auto* v : {&hc, &hl, &hu}) v->resize(n);
        for (auto* v : {&hlo, &hhi}) v->resize(m);
        for (int k = 0; k < count; ++k) {
            const gb_lp& L = lps[k];
            const int r0 = P->row_off[k], c0 = P->col_off[k], z0 = P->nnz_off[k];
            for (int i = 0; i <= L.m; ++i) hptr[r0 + i] = z0 + L.a_ptr[i];
            const int nz = L.a_ptr[L.m];
            for (int p = 0; p < nz; ++p) {
                hidx[z0 + p] = c0 + L.a_idx[p];
                hval[z0 + p] = L.a_val[p];
            }
            std::copy(L.c, L.c + L.n, hc.begin() + c0);
            std::copy(L.l, L.l + L.n, hl.begin() + c0);
            std::copy(L.u, L.u + L.n, hu.begin() + c0);
            std::copy(L.lo, L.lo + L.m, hlo.begin() + r0);
            std::copy(L.hi, L.hi + L.m, hhi.begin() + r0);
        }
        ap = hptr.data(); ai = hidx.data(); av = hval.data();
        vc = hc.data(); vl = hl.data(); vu = hu.data(); vlo = hlo.data(); vhi = hhi.data();
    }
    auto upi = [&](DevBuf<int>& d, const std::vector<int>& h) {
        d.reset(h.size());
        d.upload(h.data(), h.size(), s);
    };
    upi(P->d_row_off, P->row_off);
    upi(P->d_col_off, P->col_off);
    upi(P->d_nnz_off, P->nnz_off);
    if (count > 1) {
        P->inst_row.reset(m);
        P->inst_col.reset(n);
        k_fill_segments<<<count, kThreads, 0, s>>>(P->d_row_off.get(), P->inst_row.get());
        k_fill_segments<<<count, kThreads, 0, s>>>(P->d_col_off.get(), P->inst_col.get());
    }

    upload_mat(P->A, m, n, ap, ai, av, s);
    auto up = [&](DevBuf<double>& d, const double* h, int k) {
        d.reset(k ? k : 1);
        d.upload(h, k, s);
    };
    DevBuf<double> c0, l0, u0, lo0, hi0;
    up(c0, vc, n);
    up(l0, vl, n);
    up(u0, vu, n);
    up(lo0, vlo, m);
    up(hi0, vhi, m);
    for (int k = 0; k < count; ++k) validate_entries(&lps[k]);  // overlaps the uploads from pinned memory
    tr.mark("upload+entries");
    for (DevBuf<double>* b : {&P->c, &P->l, &P->u, &P->C, &P->Cres, &P->x64, &P->xr64, &P->xo, &P->work1})
        b->reset(n);
    for (DevBuf<double>* b : {&P->lo, &P->hi, &P->R, &P->Rres, &P->y64, &P->yr64, &P->yo, &P->work2}) b->reset(m);
    P->scal.reset(static_cast<size_t>(count) * kScal);
    P->scal_host.assign(static_cast<size_t>(count) * kScal, 0.0);
    for (int k = 0; k < count; ++k) {
        P->scal_host[static_cast<size_t>(k) * kScal + S_SIGN] = P->maximize[k] ? -1.0 : 1.0;
        P->scal_host[static_cast<size_t>(k) * kScal + S_OBJC] = (P->maximize[k] ? -1.0 : 1.0) * P->obj_const[k];
    }
    P->scal.upload(P->scal_host.data(), P->scal_host.size(), s);
    P->red_partials.reset(kRedGrid);
    P->red_arrivals.reset(1);
    GB_CUDA(cudaMemsetAsync(P->red_arrivals.get(), 0, sizeof(unsigned), s));
    P->st.reset(count);
    GB_CUDA(cudaMemsetAsync(P->st.get(), 0, sizeof(SolveState) * count, s));

    // schedules (host, from the row-length histogram, per instance) and transpose
    for (int w = 0; w < 2; ++w) {
        P->tune_block_nnz[w].assign(count, kBlockNnz);
        P->tune_max_rows[w].assign(count, kThreads);
    }
    P->A.sched.upload(build_schedule(P->A.host_ptr.data(), m, P->row_off.data(), count), 3, s);
    tr.mark("allocs+A schedule");
    TransposeScratch tw;  // lives until the set-up's final synchronisation
    device_transpose(*P, tw, s);
    tr.mark("transpose");

    // Ruiz equilibration + Pock-Chambolle (scaling.cpp:47-72); row and column
    // factors are per row / column, so the block-diagonal matrix scales every
    // instance exactly as it would alone.
    const int gw = elem_grid(static_cast<long long>(std::max(m, n)) * 32, P->sms);
    const int ge = elem_grid(std::max<long long>(P->A.nnz, 1), P->sms);
    DevBuf<double> rs(m), cs(n);
    k_fill<<<elem_grid(m, P->sms), kThreads, 0, s>>>(m, 1.0, P->R.get());
    k_fill<<<elem_grid(n, P->sms), kThreads, 0, s>>>(n, 1.0, P->C.get());
    const int passes = opt->ruiz_iters + (opt->pock_chambolle ? 1 : 0);
    // lanes per row for the maxima: the average row length, rounded up to a power of two
    auto lanes_lg = [](long long nnz, int rows) {
        int lg = 0;
        while (lg < 5 && (1LL << lg) * rows < nnz) ++lg;
        return lg;
    };
    const int lg_a = lanes_lg(P->A.nnz, m), lg_at = lanes_lg(P->A.nnz, n);
    for (int it = 0; it < passes; ++it) {
        const int mode = it < opt->ruiz_iters ? 0 : 1;
        launch_pdl(k_row_norm_factor, gw, kThreads, 0, s, m, static_cast<const int*>(P->A.ptr.get()),
                   static_cast<const int*>(nullptr), static_cast<const double*>(P->A.val64.get()), mode, rs.get(),
                   mode == 0 ? lg_a : 5);
        launch_pdl(k_row_norm_factor, gw, kThreads, 0, s, n, static_cast<const int*>(P->AT.ptr.get()),
                   static_cast<const int*>(P->perm.get()), static_cast<const double*>(P->A.val64.get()), mode, cs.get(),
                   mode == 0 ? lg_at : 5);
        launch_pdl(k_apply_scaling, std::max(ge, elem_grid(std::max(m, n), P->sms)), kThreads, 0, s,
                   static_cast<int>(P->A.nnz), static_cast<const int*>(P->row_of.get()),
                   static_cast<const int*>(P->A.idx.get()), static_cast<const double*>(rs.get()),
                   static_cast<const double*>(cs.get()), P->A.val64.get(), m, P->R.get(), n, P->C.get());
    }
    if (P->A.nnz)
        k_gather_transpose<<<ge, kThreads, 0, s>>>(static_cast<int>(P->A.nnz), P->perm.get(), P->row_of.get(),
                                                  P->A.val64.get(), P->AT.idx.get(), P->AT.val64.get());
    // vectors (scaling.cpp:75-101)
    const int gv = elem_grid(std::max(m, n), P->sms);
    double* sc = P->scal.get();
    k_scale_vectors<<<gv, kThreads, 0, s>>>(n, m, P->icol(), sc, c0.get(), l0.get(), u0.get(), lo0.get(), hi0.get(),
                                            P->R.get(), P->C.get(), P->c.get(), P->l.get(), P->u.get(), P->lo.get(),
                                            P->hi.get());
    inst_reduce(*P, true, FiniteBoundSq{P->lo.get(), P->hi.get()}, S_BSCALE, PostSqrtPlus1{}, s);
    inst_reduce(*P, false, Sq{P->c.get()}, S_CSCALE, PostSqrtPlus1{}, s);
    k_rescale<<<gv, kThreads, 0, s>>>(n, m, P->icol(), P->irow(), sc, P->R.get(), P->C.get(), P->c.get(), P->l.get(),
                                      P->u.get(), P->lo.get(), P->hi.get(), P->Rres.get(), P->Cres.get());
    // norms of the ORIGINAL data (scaling.cpp:126-127)
    inst_reduce(*P, true, FiniteBoundSq{lo0.get(), hi0.get()}, S_BNORM, PostSqrt{}, s);
    inst_reduce(*P, false, Sq{c0.get()}, S_CNORM, PostSqrt{}, s);

    tr.mark("scaling");
    // A^T's schedule, built on the host while the scaling kernels run (the
    // power iteration is its first user)
    P->AT.sched.upload(build_schedule(P->AT.host_ptr.data(), n, P->col_off.data(), count), 3, s);
    tr.mark("A^T schedule");

    // Hessian (single problem only)
    const gb_lp& L0 = lps[0];
    P->has_q = count == 1 && ((L0.q_ptr && L0.q_ptr[n] > 0) || L0.q_rank > 0);
    P->dplr = P->has_q && L0.q_rank > 0;
    P->qk = P->dplr ? L0.q_rank : 0;
    P->partials.reset(std::max<size_t>(static_cast<size_t>(kFtxGrid) * 2 * kMaxRank,
                                       static_cast<size_t>(P->A.sched.nb + P->AT.sched.nb + count) * kTerms));
    P->ftx.reset(2 * kMaxRank);
    P->decide_sync.reset(2);
    GB_CUDA(cudaMemsetAsync(P->decide_sync.get(), 0, 2 * sizeof(unsigned), s));
    P->v32.alloc(n, m, P->qk, P->has_q);
    P->v64.alloc(n, m, P->qk, P->has_q);
    if (P->has_q && !P->dplr) {
        upload_mat(P->Q, n, n, L0.q_ptr, L0.q_idx, L0.q_val, s);
        P->Q.sched.upload(build_schedule(P->Q.host_ptr.data(), n), 3, s);
        P->q_row_of.reset(P->Q.nnz ? P->Q.nnz : 1);
        k_row_of<<<elem_grid((long long)n * 32, P->sms), kThreads, 0, s>>>(n, P->Q.ptr.get(), P->q_row_of.get());
        k_scale_q<<<elem_grid(P->Q.nnz, P->sms), kThreads, 0, s>>>(static_cast<int>(P->Q.nnz), P->q_row_of.get(),
                                                                 P->Q.idx.get(), P->C.get(), sc, P->Q.val64.get());
    } else if (P->dplr) {
        P->F64.reset(static_cast<size_t>(n) * P->qk);
        P->F64.upload(L0.q_F, static_cast<size_t>(n) * P->qk, s);
        up(P->D64, L0.q_D, n);
        k_scale_dplr<<<elem_grid((long long)n * P->qk, P->sms), kThreads, 0, s>>>(n, P->qk, P->C.get(), sc,
                                                                                  P->F64.get(), P->D64.get());
    }
    if (P->has_q) power_iteration(*P, true, s);
    power_iteration(*P, false, s);  // ||A'|| (scaling.cpp:131-155)
    tr.mark("power iteration");
    // w0 from the scaled data (pdhg_impl.hpp:258-261)
    inst_reduce(*P, false, Sq{P->c.get()}, S_CN, PostSqrt{}, s);
    inst_reduce(*P, true, FiniteBoundSq{P->lo.get(), P->hi.get()}, S_BN, PostSqrt{}, s);
    k_w0<<<div_up(count, kThreads), kThreads, 0, s>>>(count, sc);
    // FP32 copies of the matrix values and data
    auto cvt32 = [&](DevMat& M) {
        M.val32.reset(padded_nnz(M.nnz));
        if (M.nnz) k_convert<float><<<elem_grid(M.nnz, P->sms), kThreads, 0, s>>>(M.nnz, M.val64.get(), M.val32.get());
    };
    cvt32(P->A);
    cvt32(P->AT);
    // Matrix streams that cannot stay in L2 across iterations skip L1
    // allocation (CsrView::nc): per-iteration bytes of the LP iteration at
    // FP32 and at FP64 against the 126 MB L2.
    for (int w = 0; w < 2; ++w) {
        const double sm = w ? 8.0 : 4.0, sv = w ? 8.0 : 4.0;
        const double iter = 2.0 * static_cast<double>(P->A.nnz) * (sm + 4.0) + 4.0 * (m + n + 2) + sv * (9.0 * n + 7.0 * m);
        const int forced = load_mode_override();
        const int nc = forced >= 0 ? forced : (iter > kL2StreamBytes ? kLoadStream : kLoadPlain);
        P->A.stream_nc[w] = P->AT.stream_nc[w] = nc;
        P->A.default_nc[w] = P->AT.default_nc[w] = nc;
    }
    if (P->has_q && !P->dplr) cvt32(P->Q);
    convert_data(*P, P->v32, s);
    convert_data(*P, P->v64, s);
    // The phase graphs these options run, captured and instantiated on the
    // host while the set-up kernels above execute.
    prebuild_graphs(*P, opt);
    tr.mark("fp32 copies+graphs");
    P->st_host = static_cast<SolveState*>(host_alloc(sizeof(SolveState) * count));
    P->phase_flags_host = static_cast<int*>(host_alloc(sizeof(int) * count));
    tr.mark("pinned state");
    P->phase_flags.reset(count);
    GB_CUDA(cudaMemcpyAsync(P->scal_host.data(), sc, sizeof(double) * P->scal_host.size(), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    GB_CUDA(cudaGetLastError());
    P->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return P.release();
}

// ---------------------------------------------------------------- phase runner
template <class M, class V>
struct Level {
    static VecSet<V>& vs(Problem& P);
};
template <>
VecSet<float>& Level<float, float>::vs(Problem& P) { return P.v32; }
template <>
VecSet<double>& Level<float, double>::vs(Problem& P) { return P.v64; }
template <>
VecSet<double>& Level<double, double>::vs(Problem& P) { return P.v64; }
template <>
VecSet<float>& Level<__nv_bfloat16, float>::vs(Problem& P) { return P.v32; }
template <class M, class V>
constexpr int level_index() {
    return std::is_same<M, __nv_bfloat16>::value
               ? 3
               : (std::is_same<M, double>::value ? 2 : (std::is_same<V, double>::value ? 1 : 0));
}

// BF16 copies of the scaled matrix values (A and A^T), made once.  After
// Ruiz / Pock-Chambolle scaling every value is O(1), far inside BF16's
// (FP32's) exponent range; what BF16 gives up is precision (8-bit
// significand), so its phase ends by the same stall rule as the FP32 one.
void ensure_bf16(Problem& P) {
    auto cvt = [&](DevMat& M) {
        if (M.valbf.get()) return;
        M.valbf.reset(padded_nnz(M.nnz));
        if (M.nnz)
            k_convert<__nv_bfloat16><<<elem_grid(M.nnz, P.sms), kThreads, 0, P.stream>>>(M.nnz, M.val64.get(),
                                                                                        M.valbf.get());
    };
    cvt(P.A);
    cvt(P.AT);
    GB_CUDA(cudaGetLastError());
}

template <class M, class V>
void launch_qx(Problem& P, VecSet<V>& vs, const V* x, V* qx, cudaStream_t s, long long& nl) {
    if (P.dplr) {
        double* part = P.partials.get();
        double* t = P.ftx.get();  // FP64 F^T x at every level
        const V* none = nullptr;
        V* none_out = nullptr;
        const SolveState* no_st = nullptr;
        launch_pdl(k_ftx_partial<V, 1>, kFtxGrid, kThreads, 0, s, P.n, P.qk, vs.F.get(), x, none, no_st, part);
        launch_pdl(k_ftx_final, P.qk, 32, 0, s, kFtxGrid, part, t);
        launch_pdl(k_dplr_expand<V, 1>, expand_grid(P.n), kExpandWarps * 32, expand_smem_bytes<V, 1>(P.qk), s, P.n,
                   P.qk, vs.F.get(), vs.D.get(), t, x, none, no_st, qx, none_out);
        nl += 3;
    } else {
        k_spmv<M, V><<<P.Q.sched.nb, kThreads, spmv_smem_bytes<1, V>(), s>>>(P.Q.view<M>(), x, qx);
        nl += 1;
    }
}

template <class M, class V>
void launch_qx2(Problem& P, VecSet<V>& vs, const V* x, cudaStream_t s, long long& nl) {
    if (P.dplr) {
        double* part = P.partials.get();
        double* t = P.ftx.get();
        launch_pdl(k_ftx_partial<V, 2>, kFtxGrid, kThreads, 0, s, P.n, P.qk, vs.F.get(), x, vs.sumx.get(), P.st.get(),
                   part);
        launch_pdl(k_ftx_final, 2 * P.qk, 32, 0, s, kFtxGrid, part, t);
        launch_pdl(k_dplr_expand<V, 2>, expand_grid(P.n), kExpandWarps * 32, expand_smem_bytes<V, 2>(P.qk), s, P.n,
                   P.qk, vs.F.get(), vs.D.get(), t, x, vs.sumx.get(), P.st.get(), vs.qx.get(), vs.qxa.get());
        nl += 3;
    } else {
        k_spmv_q2<M, V><<<P.Q.sched.nb, kThreads, spmv_smem_bytes<2, V>(), s>>>(P.Q.view<M>(), x, vs.sumx.get(),
                                                                            P.st.get(), vs.qx.get(), vs.qxa.get());
        nl += 1;
    }
}

template <class M, class V>
EvalArgs<M, V> eval_args(Problem& P, VecSet<V>& vs, const V* x, const V* y, int mode, bool with_q) {
    EvalArgs<M, V> a;
    a.A = P.A.view<M>();
    a.AT = P.AT.view<M>();
    a.x = x;
    a.y = y;
    a.sumx = vs.sumx.get();
    a.sumy = vs.sumy.get();
    a.xr = vs.xr.get();
    a.yr = vs.yr.get();
    a.c = vs.c.get();
    a.l = vs.l.get();
    a.u = vs.u.get();
    a.lo = vs.lo.get();
    a.hi = vs.hi.get();
    a.rres = vs.rres.get();
    a.cres = vs.cres.get();
    a.qx = with_q ? vs.qx.get() : nullptr;
    a.qxa = (with_q && mode == kEvalCheck) ? vs.qxa.get() : nullptr;
    a.mode = mode;
    a.count = P.count;
    a.seg_a = P.A.sched_for<M>().seg_block.get();
    a.seg_t = P.AT.sched_for<M>().seg_block.get();
    a.st = P.st.get();
    a.partials = P.partials.get();
    a.inst_terms = P.partials.get() + static_cast<size_t>(a.A.nb + a.AT.nb) * kTerms;
    a.sync = P.decide_sync.get();
    a.cond = 0;
    a.use_cond = 0;
    return a;
}

// Arguments of the two kernels of the k-th iteration inside a body (buffers by parity).
template <class M, class V>
void iteration_args(Problem& P, VecSet<V>& vs, int k, PrimalArgs<M, V>& pa, DualArgs<M, V>& da) {
    const V* xin = (k & 1) ? vs.x1.get() : vs.x0.get();
    V* xout = (k & 1) ? vs.x0.get() : vs.x1.get();
    const V* yin = (k & 1) ? vs.y1.get() : vs.y0.get();
    V* yout = (k & 1) ? vs.y0.get() : vs.y1.get();
    pa = PrimalArgs<M, V>{P.AT.view<M>(), yin, xin, vs.c.get(), vs.l.get(), vs.u.get(),
                          P.has_q ? vs.qx.get() : nullptr, xout, vs.xbar.get(), vs.sumx.get(), P.st.get()};
    da = DualArgs<M, V>{P.A.view<M>(), vs.xbar.get(), yin, vs.lo.get(), vs.hi.get(), yout, vs.sumy.get(),
                        P.st.get()};
    if (P.list_level == level_index<M, V>()) {  // a phase of some instances only
        pa.AT.blocks = P.list_t.get();
        pa.AT.nb = P.list_nt;
        da.A.blocks = P.list_a.get();
        da.A.nb = P.list_na;
    }
}

// The fused iteration kernels at their matrix view's load mode (CsrView::nc).
template <class M, class V>
void launch_primal(const PrimalArgs<M, V>& pa, cudaStream_t s) {
    if (pa.AT.nc == kLoadPrefetch)
        launch_pdl(k_primal<M, V, kLoadPrefetch>, pa.AT.nb, kThreads, spmv_seg_smem_bytes<V>(), s, pa);
    else if (pa.AT.nc == kLoadStream)
        launch_pdl(k_primal<M, V, kLoadStream>, pa.AT.nb, kThreads, spmv_seg_smem_bytes<V>(), s, pa);
    else
        launch_pdl(k_primal<M, V>, pa.AT.nb, kThreads, spmv_seg_smem_bytes<V>(), s, pa);
}
template <class M, class V>
void launch_dual(const DualArgs<M, V>& da, cudaStream_t s) {
    if (da.A.nc == kLoadPrefetch)
        launch_pdl(k_dual<M, V, kLoadPrefetch>, da.A.nb, kThreads, spmv_seg_smem_bytes<V>(), s, da);
    else if (da.A.nc == kLoadStream)
        launch_pdl(k_dual<M, V, kLoadStream>, da.A.nb, kThreads, spmv_seg_smem_bytes<V>(), s, da);
    else
        launch_pdl(k_dual<M, V>, da.A.nb, kThreads, spmv_seg_smem_bytes<V>(), s, da);
}

// One PDHG iteration (k-th inside the body) on buffers selected by parity.
template <class M, class V>
void launch_iteration(Problem& P, VecSet<V>& vs, int k, cudaStream_t s, long long& nl, cudaEvent_t mid = nullptr) {
    PrimalArgs<M, V> pa;
    DualArgs<M, V> da;
    iteration_args<M, V>(P, vs, k, pa, da);
    if (P.has_q) launch_qx<M, V>(P, vs, pa.x, vs.qx.get(), s, nl);
    launch_primal<M, V>(pa, s);
    if (mid) GB_CUDA(cudaEventRecord(mid, s));
    launch_dual<M, V>(da, s);
    nl += 2;
}

// k_decide, preceded for a single problem with more than kDecideWide row
// blocks by k_terms (its term sums, one CTA per term; same bits).  Returns
// the launches.
template <class M, class V>
int launch_decide(Problem& P, EvalArgs<M, V>& ea, cudaStream_t s, bool pdl) {
    int nl = 1;
    ea.terms_ready = 0;
    if (P.count == 1 && ea.A.nb + ea.AT.nb > kDecideWide) {
        ea.terms_ready = 1;
        if (pdl) launch_pdl(k_terms<M, V>, kTerms, kThreads, 0, s, ea);
        else k_terms<M, V><<<kTerms, kThreads, 0, s>>>(ea);
        nl += 1;
    }
    if (pdl) launch_pdl(k_decide<M, V>, decide_grid(P.count), kThreads, 0, s, ea);
    else k_decide<M, V><<<decide_grid(P.count), kThreads, 0, s>>>(ea);
    return nl;
}

// Body of the phase loop: check_every iterations, KKT check, restart.
// use_cond = 0 when the body is launched from the host loop instead of the graph.
template <class M, class V>
long long capture_body(Problem& P, int ce, cudaGraphConditionalHandle cond, cudaStream_t s, int use_cond = 1) {
    VecSet<V>& vs = Level<M, V>::vs(P);
    long long nl = 0;
    for (int k = 0; k < ce; ++k) launch_iteration<M, V>(P, vs, k, s, nl);
    const bool odd = (ce & 1) != 0;
    const V* xc = odd ? vs.x1.get() : vs.x0.get();
    const V* yc = odd ? vs.y1.get() : vs.y0.get();
    if (P.has_q) launch_qx2<M, V>(P, vs, xc, s, nl);
    EvalArgs<M, V> ea = eval_args<M, V>(P, vs, xc, yc, kEvalCheck, P.has_q);
    ea.cond = cond;
    ea.use_cond = use_cond;
    const int grid = ea.A.nb + ea.AT.nb;
    if (P.detect_unbounded && !P.has_q)  // third right-hand side of the A pass: the primal ray
        launch_pdl(k_eval<M, V, 3, 3>, grid, kThreads, spmv_smem_bytes<3, V>(), s, ea);
    else
        launch_pdl(k_eval<M, V, 2, 3>, grid, kThreads, spmv_smem_bytes<3, V>(), s, ea);
    nl += launch_decide<M, V>(P, ea, s, true);
    RestartArgs<V> ra{xc, yc, vs.x0.get(), vs.y0.get(), vs.xr.get(), vs.yr.get(), vs.sumx.get(), vs.sumy.get(),
                      P.n, P.m, P.icol(), P.irow(), P.st.get()};
    launch_pdl(k_restart<V>, elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s, ra);
    nl += 2;
    return nl;
}

template <class M, class V>
LevelGraph* level_graph(Problem& P, int ce) {
    constexpr int li = level_index<M, V>();
    const bool lists = P.list_level == li;
    auto& slot = P.graphs[li + (lists ? 4 : 0)];
    const int ray = P.detect_unbounded && !P.has_q ? 1 : 0;
    const RowBlock* la = lists ? P.list_a.get() : nullptr;
    const RowBlock* lt = lists ? P.list_t.get() : nullptr;
    const int na = lists ? P.list_na : 0, nt = lists ? P.list_nt : 0;
    if (slot && slot->check_every == ce && slot->ray == ray && slot->list_a == la && slot->list_t == lt &&
        slot->list_na == na && slot->list_nt == nt)
        return slot.get();
    slot.reset(new LevelGraph);
    LevelGraph* g = slot.get();
    g->check_every = ce;
    g->ray = ray;
    g->list_a = la;
    g->list_t = lt;
    g->list_na = na;
    g->list_nt = nt;
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
    long long nl = 0;
    try {
        nl = capture_body<M, V>(P, ce, h, cs);
    } catch (...) {
        // A failed launch invalidated the capture: end it, and drop this
        // LevelGraph without tearing down its half-built graph (a handle is
        // leaked on this error path rather than destroyed in an unknown state).
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(cs, &dummy);
        cudaGetLastError();
        cudaStreamDestroy(cs);
        g->graph = nullptr;
        g->exec = nullptr;
        slot.reset();
        throw;
    }
    GB_CUDA(cudaStreamEndCapture(cs, &body));
    GB_CUDA(cudaStreamDestroy(cs));
    GB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
    GB_CUDA(cudaGraphUpload(g->exec, P.stream));
    g->launches_per_body = nl;
    return g;
}

// GANIT_B200_LAUNCH=stream runs each phase loop from the host (same kernels,
// one state read-back per check) instead of the device-side while loop of a
// conditional CUDA graph; kernel profilers need it to see the loop's kernels.
bool host_loop_mode() {
    static const bool host = [] {
        const char* v = std::getenv("GANIT_B200_LAUNCH");
        return v != nullptr && std::string(v) == "stream";
    }();
    return host;
}

// Graphs of the precision levels a solve with `opt` runs (the BF16 trial
// level is built on its first use, with its matrix copy).
void prebuild_graphs(Problem& P, const gb_options* opt) {
    if (host_loop_mode() || opt->check_every <= 0) return;
    P.detect_unbounded = opt->detect_unbounded != 0;
    if (opt->precision != GB_PREC_DOUBLE) {
        level_graph<float, float>(P, opt->check_every);
        if (opt->precision == GB_PREC_DYNAMIC) level_graph<float, double>(P, opt->check_every);
    }
    level_graph<double, double>(P, opt->check_every);
}

// Phase set-up of every instance: in_phase / active from flags.
__global__ void k_set_phase(int count, SolveState* st, const int* flags, double tol, int stall_checks,
                            int stall_exit, int first_phase) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    SolveState& s = st[k];
    s.in_phase = flags[k];
    s.active = flags[k];
    s.ran_body = 0;
    if (!flags[k]) return;
    s.phase_tol = tol;
    s.stall_checks = stall_checks;
    s.stall_exit = stall_exit;
    s.carry_restart_err = first_phase ? -1.0 : s.restart_err;
}

__global__ void k_init_state(int count, SolveState* st, const double* sc, int has_q, int check_every,
                             long long max_iter, double time_limit, double infeas_tol, int detect_unbounded) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double* s0 = sc + static_cast<size_t>(k) * kScal;
    SolveState s;
    memset(&s, 0, sizeof(s));
    s.normA = s0[S_NORMA];
    s.eta = 0.998 / s.normA;
    s.normQ = s0[S_NORMQ];
    s.obj_scale = s0[S_CSCALE] * s0[S_BSCALE];
    s.obj_const = s0[S_OBJC];
    s.bnorm = s0[S_BNORM];
    s.cnorm = s0[S_CNORM];
    s.w = s0[S_W0];
    s.infeas_tol = infeas_tol;
    s.time_limit_s = time_limit;
    s.max_iter = max_iter;
    s.check_every = check_every;
    s.has_q = has_q;
    s.detect_unbounded = detect_unbounded;
    s.carry_restart_err = -1.0;
    s.restart_err = -1.0;
    s.t0_ns = global_ns();
    st[k] = s;
}

// Primal weight of a warm start (Problem::w_start, entries > 0), over k_init_state's w0.
__global__ void k_set_w(int count, SolveState* st, const double* w) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count && w[k] > 0.0) st[k].w = w[k];
}

__global__ void k_activate_all(int count, SolveState* st) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) st[k].active = st[k].in_phase = 1;
}

void sync_state(Problem& P) {
    GB_CUDA(cudaMemcpyAsync(P.st_host, P.st.get(), sizeof(SolveState) * P.count, cudaMemcpyDeviceToHost, P.stream));
    GB_CUDA(cudaStreamSynchronize(P.stream));
}

// Block lists of a batch phase that only some instances take part in
// (phase_flags_host): the iteration kernels of level <M,V> then launch the
// row blocks of those instances alone (copies of their RowBlocks, which carry
// their own slot and counter indices), instead of every block with the
// others' CTAs returning at once -- same blocks, same arithmetic, fewer CTAs.
// Used when the phase's blocks are at most half of all.
// GANIT_B200_PHASE_LISTS=0 turns it off.
bool phase_lists_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("GANIT_B200_PHASE_LISTS");
        return v == nullptr || std::string(v) != "0";
    }();
    return on;
}
template <class M, class V>
void set_phase_lists(Problem& P) {
    P.list_level = -1;
    if (P.count <= 1 || !phase_lists_enabled()) return;
    const DevSchedule& sa = P.A.template sched_for<M>();
    const DevSchedule& st = P.AT.template sched_for<M>();
    std::vector<RowBlock> la, lt;
    for (int k = 0; k < P.count; ++k) {
        if (!P.phase_flags_host[k]) continue;
        for (int b = sa.host_seg_block[k]; b < sa.host_seg_block[k + 1]; ++b) la.push_back(sa.host_blocks[b]);
        for (int b = st.host_seg_block[k]; b < st.host_seg_block[k + 1]; ++b) lt.push_back(st.host_blocks[b]);
    }
    if (la.empty() || lt.empty() || 2 * (la.size() + lt.size()) > static_cast<size_t>(sa.nb + st.nb)) return;
    auto put = [&](DevBuf<RowBlock>& d, const std::vector<RowBlock>& h) {
        if (d.size() < h.size()) d.reset(h.size());  // a buffer only grows: graphs keep their pointer
        d.upload(h.data(), h.size(), P.stream);
    };
    put(P.list_a, la);
    put(P.list_t, lt);
    P.list_na = static_cast<int>(la.size());
    P.list_nt = static_cast<int>(lt.size());
    P.list_level = level_index<M, V>();
    if (trace_enabled())
        std::fprintf(stderr, "[gb trace] phase lists: %d + %d of %d row blocks\n", P.list_na, P.list_nt,
                     sa.nb + st.nb);
}
struct PhaseListsOff {  // the lists end with the phase, also on an error
    Problem& P;
    ~PhaseListsOff() { P.list_level = -1; }
};

template <class M, class V>
void run_phase(Problem& P, const gb_options* opt, double tol, int stall_exit, int stall_checks, bool first,
               bool has_r) {
    cudaStream_t s = P.stream;
    VecSet<V>& vs = Level<M, V>::vs(P);
    const int gv = elem_grid(std::max(P.n, P.m), P.sms);
    long long checks_before = 0;
    if (!first)
        for (int k = 0; k < P.count; ++k) checks_before = std::max<long long>(checks_before, P.st_host[k].checks);
    GB_CUDA(cudaMemcpyAsync(P.phase_flags.get(), P.phase_flags_host, sizeof(int) * P.count, cudaMemcpyHostToDevice,
                            s));
    k_set_phase<<<div_up(P.count, kThreads), kThreads, 0, s>>>(P.count, P.st.get(), P.phase_flags.get(), tol,
                                                               stall_checks, stall_exit, first ? 1 : 0);
    set_phase_lists<M, V>(P);
    PhaseListsOff lists_off{P};
    k_phase_in<V><<<gv, kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), P.st.get(), P.x64.get(), P.y64.get(),
                                         P.xr64.get(), P.yr64.get(), has_r ? 1 : 0, vs.x0.get(), vs.y0.get(),
                                         vs.xr.get(), vs.yr.get(), vs.sumx.get(), vs.sumy.get());
    P.launches += 2;
    if (P.has_q) launch_qx<M, V>(P, vs, vs.x0.get(), vs.qx.get(), s, P.launches);
    EvalArgs<M, V> ea = eval_args<M, V>(P, vs, vs.x0.get(), vs.y0.get(), kEvalInit, P.has_q);
    k_eval<M, V, 1, 1><<<ea.A.nb + ea.AT.nb, kThreads, spmv_smem_bytes<1, V>(), s>>>(ea);
    P.launches += 1 + launch_decide<M, V>(P, ea, s, false);
    long long per_body = 0;
    long long bodies = 0;
    if (host_loop_mode()) {
        // Same kernels, launched from a host loop with one state read-back per
        // check (profilers cannot see kernels inside conditional graphs).
        for (;;) {
            per_body = capture_body<M, V>(P, opt->check_every, 0, s, 0);
            ++bodies;
            sync_state(P);
            bool any = false;
            for (int k = 0; k < P.count; ++k) any |= P.st_host[k].active != 0;
            if (!any) break;
        }
    } else {
        StageTrace tr{s, level_index<M, V>() == 2 ? "phase f64" : "phase"};
        tr.mark("phase entry");
        LevelGraph* g = level_graph<M, V>(P, opt->check_every);
        tr.mark("graph build");
        GB_CUDA(cudaGraphLaunch(g->exec, s));
        per_body = g->launches_per_body;
        tr.mark("graph run");
    }
    k_phase_out<V><<<gv, kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), vs.x0.get(), vs.y0.get(), vs.sumx.get(),
                                          vs.sumy.get(), vs.xr.get(), vs.yr.get(), P.st.get(), P.x64.get(),
                                          P.y64.get(), P.xr64.get(), P.yr64.get());
    sync_state(P);
    if (!host_loop_mode()) {
        long long checks_after = 0;
        for (int k = 0; k < P.count; ++k) checks_after = std::max<long long>(checks_after, P.st_host[k].checks);
        bodies = checks_after - checks_before;
    }
    P.launches += 1 + bodies * per_body;
    GB_CUDA(cudaGetLastError());
}

// pdhg_evaluate<Bd> (pdhg_impl.hpp:202-230) of the carried FP64 state of every instance.
void certify(Problem& P) {
    cudaStream_t s = P.stream;
    VecSet<double>& vs = P.v64;
    if (P.has_q) launch_qx<double, double>(P, vs, P.x64.get(), vs.qx.get(), s, P.launches);
    EvalArgs<double, double> ea = eval_args<double, double>(P, vs, P.x64.get(), P.y64.get(), kEvalCertify, P.has_q);
    k_eval<double, double, 1, 1><<<ea.A.nb + ea.AT.nb, kThreads, spmv_smem_bytes<1, double>(), s>>>(ea);
    P.launches += 1 + launch_decide<double, double>(P, ea, s, false);
    sync_state(P);
}

inline bool kkt_conv_h(const Kkt& k, double tol) { return k.rel_p <= tol && k.rel_d <= tol && k.rel_gap <= tol; }

int status_from(int e) {  // pdhg_impl.hpp:232-240
    switch (e) {
        case kConverged: return GB_OPTIMAL;
        case kInfeasible: return GB_PRIMAL_INFEASIBLE;
        case kUnbounded: return GB_DUAL_INFEASIBLE;
        case kTimeLimit: return GB_TIME_LIMIT;
        case kNumerical: return GB_NUMERICAL_ERROR;
        default: return GB_ITERATION_LIMIT;
    }
}

// run_pdhg (pdhg_impl.hpp:243-328) of every instance with device-resident state.
void solve_problem(Problem& P, const gb_options* opt, gb_result* res) {
    GB_REQUIRE(opt->check_every > 0, "check_every must be positive");
    GB_REQUIRE(opt->precision >= 0 && opt->precision <= 3, "unknown precision");
    GB_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = P.stream;
    const auto t0 = std::chrono::steady_clock::now();
    const int K = P.count;
    P.launches = 0;
    P.detect_unbounded = opt->detect_unbounded != 0;
    k_init_state<<<div_up(K, kThreads), kThreads, 0, s>>>(K, P.st.get(), P.scal.get(), P.has_q ? 1 : 0,
                                                          opt->check_every, opt->max_iter, opt->time_limit,
                                                          opt->infeas_tol, P.detect_unbounded ? 1 : 0);
    k_start_point<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(P.n, P.m, P.l.get(), P.u.get(),
                                                                         P.x64.get(), P.y64.get());
    P.launches += 2;
    if (P.x_start.get()) {
        k_warm_point<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(
            P.n, P.m, P.icol(), P.irow(), P.l.get(), P.u.get(), P.C.get(), P.R.get(), P.scal.get(),
            P.x_start.get(), P.y_start.get(), P.x64.get(), P.y64.get());
        P.launches += 1;
        if (P.w_start.get()) {
            k_set_w<<<div_up(K, kThreads), kThreads, 0, s>>>(K, P.st.get(), P.w_start.get());
            P.launches += 1;
        }
    }
    P.results.assign(K, InstanceResult{});
    std::vector<int> ex(K, kIterLimit), done(K, 0);
    auto set_flags = [&](auto pred) {
        int any = 0;
        for (int k = 0; k < K; ++k) any |= (P.phase_flags_host[k] = pred(k) ? 1 : 0);
        return any != 0;
    };
    auto collect = [&]() {
        for (int k = 0; k < K; ++k)
            if (P.phase_flags_host[k]) {
                ex[k] = P.st_host[k].exit_reason;
                P.results[k].phases += 1;
            }
    };
    // finished lambda (pdhg_impl.hpp:278-286) after the FP64 certification
    auto finished = [&]() {
        certify(P);
        for (int k = 0; k < K; ++k) {
            if (!P.phase_flags_host[k] || done[k]) continue;
            const int e = ex[k];
            done[k] = (e == kConverged && kkt_conv_h(P.st_host[k].kcert, opt->tol)) || e == kTimeLimit ||
                      e == kIterLimit || e == kInfeasible || e == kUnbounded;
        }
    };
    if (opt->precision != GB_PREC_DOUBLE) {
        set_flags([](int) { return true; });
        bool first = true;
        if (opt->precision == GB_PREC_MIXED_BF16 && !P.has_q) {
            ensure_bf16(P);
            run_phase<__nv_bfloat16, float>(P, opt, opt->tol, 1, opt->stall_checks, true, false);
            collect();
            for (int k = 0; k < K; ++k) P.results[k].bf16_iters = P.st_host[k].it;
            finished();
            first = false;
        }
        if (set_flags([&](int k) { return !done[k]; })) {
            run_phase<float, float>(P, opt, opt->tol, 1, opt->stall_checks, first, !first);
            collect();
        }
        for (int k = 0; k < K; ++k) P.results[k].fp32_iters = P.st_host[k].it - P.results[k].bf16_iters;
        finished();
        if (opt->precision == GB_PREC_DYNAMIC && set_flags([&](int k) { return !done[k]; })) {
            run_phase<float, double>(P, opt, opt->tol, 1, opt->stall_checks_l2, false, true);
            collect();
            for (int k = 0; k < K; ++k)
                if (P.phase_flags_host[k]) P.results[k].l2_iters = P.st_host[k].it - P.results[k].fp32_iters;
            finished();
        }
        if (set_flags([&](int k) { return !done[k]; })) {
            run_phase<double, double>(P, opt, opt->tol, 0, 0, false, true);
            collect();
        }
    } else {
        set_flags([](int) { return true; });
        run_phase<double, double>(P, opt, opt->tol, 0, 0, true, false);
        collect();
    }
    // Final FP64 certification of the returned points.
    StageTrace tr{s, "solve"};
    tr.mark("phases");
    certify(P);
    k_unscale<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(P.n, P.m, P.icol(), P.irow(), P.x64.get(),
                                                                     P.y64.get(), P.C.get(), P.R.get(),
                                                                     P.scal.get(), P.xo.get(), P.yo.get());
    P.launches += 1;
    GB_CUDA(cudaStreamSynchronize(s));
    GB_CUDA(cudaGetLastError());
    tr.mark("certify+unscale");
    const double solve_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int k = 0; k < K; ++k) {
        const SolveState& st = P.st_host[k];
        const Kkt& fin = st.kcert;
        int status = status_from(ex[k]);
        if (status == GB_OPTIMAL && !kkt_conv_h(fin, opt->tol * 1.0000001)) status = GB_NUMERICAL_ERROR;
        P.results[k].status = status;
        if (!res) continue;
        gb_result& r = res[k];
        const double sign = P.maximize[k] ? -1.0 : 1.0;
        std::memset(&r, 0, sizeof(r));
        r.status = status;
        r.pobj = sign * fin.pobj;
        r.dobj = sign * fin.dobj;
        r.rel_primal = fin.rel_p;
        r.rel_dual = fin.rel_d;
        r.rel_gap = fin.rel_gap;
        r.iterations = st.it;
        r.fp32_iterations = P.results[k].fp32_iters;
        r.l2_iterations = P.results[k].l2_iters;
        r.bf16_iterations = P.results[k].bf16_iters;
        r.restarts = st.restarts;
        r.setup_seconds = P.setup_seconds;
        r.solve_seconds = solve_s;
        r.norm_a = P.scal_host[static_cast<size_t>(k) * kScal + S_NORMA];
        r.primal_weight = st.w;
        r.checks = st.checks;
        r.phases = P.results[k].phases;
    }
    P.solved = true;
}

// ---------------------------------------------------------------- kernel timing
template <class M_, class V_>
struct Tag {
    using M = M_;
    using V = V_;
};

template <class M, class V>
void time_level(Problem& P, int iters, double* msp, double* msd, int64_t* launches) {
    cudaStream_t s = P.stream;
    VecSet<V>& vs = Level<M, V>::vs(P);
    k_activate_all<<<div_up(P.count, kThreads), kThreads, 0, s>>>(P.count, P.st.get());
    k_phase_in<V><<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(
        P.n, P.m, P.icol(), P.irow(), P.st.get(), P.x64.get(), P.y64.get(), P.x64.get(), P.y64.get(), 0,
        vs.x0.get(), vs.y0.get(), vs.xr.get(), vs.yr.get(), vs.sumx.get(), vs.sumy.get());
    std::vector<cudaEvent_t> ev(2 * iters + 1);
    for (auto& e : ev) GB_CUDA(cudaEventCreate(&e));
    long long nl = 0;
    for (int k = 0; k < 4; ++k) launch_iteration<M, V>(P, vs, k, s, nl);  // warm-up
    GB_CUDA(cudaEventRecord(ev[0], s));
    for (int k = 0; k < iters; ++k) {
        launch_iteration<M, V>(P, vs, k, s, nl, ev[2 * k + 1]);
        GB_CUDA(cudaEventRecord(ev[2 * k + 2], s));
    }
    GB_CUDA(cudaStreamSynchronize(s));
    double tp = 0, td = 0;
    for (int k = 0; k < iters; ++k) {
        float a = 0, b = 0;
        GB_CUDA(cudaEventElapsedTime(&a, ev[2 * k], ev[2 * k + 1]));
        GB_CUDA(cudaEventElapsedTime(&b, ev[2 * k + 1], ev[2 * k + 2]));
        tp += a;
        td += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    *msp = tp / iters;
    *msd = td / iters;
    *launches = nl;
}

// Average device time of k_primal and of k_dual when launched back to back
// (each captured `iters` times into a CUDA graph with programmatic dependent
// launch, as the solve loop issues them, and the graph timed with two CUDA
// events), and of one full iteration (the pair, alternating buffers).  Every
// instance is active.  Warm L2: the same matrix and vectors every launch.
// msp / msd may be NULL (only the iteration is timed then).
template <class M, class V>
void time_level_graph(Problem& P, int iters, double* msp, double* msd, double* msi) {
    cudaStream_t s = P.stream;
    VecSet<V>& vs = Level<M, V>::vs(P);
    k_activate_all<<<div_up(P.count, kThreads), kThreads, 0, s>>>(P.count, P.st.get());
    k_phase_in<V><<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(
        P.n, P.m, P.icol(), P.irow(), P.st.get(), P.x64.get(), P.y64.get(), P.x64.get(), P.y64.get(), 0,
        vs.x0.get(), vs.y0.get(), vs.xr.get(), vs.yr.get(), vs.sumx.get(), vs.sumy.get());
    PrimalArgs<M, V> pa;
    DualArgs<M, V> da;
    iteration_args<M, V>(P, vs, 0, pa, da);
    auto timed_graph = [&](auto&& body) {
        cudaStream_t cs;
        GB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        GB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        try {
            body(cs);
        } catch (...) {
            cudaStreamEndCapture(cs, &g);
            cudaGetLastError();
            cudaStreamDestroy(cs);
            throw;
        }
        GB_CUDA(cudaStreamEndCapture(cs, &g));
        GB_CUDA(cudaStreamDestroy(cs));
        GB_CUDA(cudaGraphInstantiate(&ge, g, 0));
        cudaEvent_t e0, e1;
        GB_CUDA(cudaEventCreate(&e0));
        GB_CUDA(cudaEventCreate(&e1));
        GB_CUDA(cudaGraphLaunch(ge, s));  // warm-up
        GB_CUDA(cudaEventRecord(e0, s));
        GB_CUDA(cudaGraphLaunch(ge, s));
        GB_CUDA(cudaEventRecord(e1, s));
        GB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        GB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaGraphExecDestroy(ge);
        cudaGraphDestroy(g);
        return static_cast<double>(ms) / iters;
    };
    if (msp)
        *msp = timed_graph([&](cudaStream_t cs) {
            for (int k = 0; k < iters; ++k) launch_primal<M, V>(pa, cs);
        });
    if (msd)
        *msd = timed_graph([&](cudaStream_t cs) {
            for (int k = 0; k < iters; ++k) launch_dual<M, V>(da, cs);
        });
    *msi = timed_graph([&](cudaStream_t cs) {
        long long nl = 0;
        for (int k = 0; k < iters; ++k) launch_iteration<M, V>(P, vs, k, cs, nl);
    });
    GB_CUDA(cudaGetLastError());
}

template <class F>
void by_level(int level, Problem& P, F&& f) {
    if (level == 0) f(Tag<float, float>{});
    else if (level == 1) f(Tag<float, double>{});
    else if (level == 2) f(Tag<double, double>{});
    else {
        GB_REQUIRE(!P.has_q, "the BF16 level takes LPs only");
        ensure_bf16(P);
        f(Tag<__nv_bfloat16, float>{});
    }
}

// Rebuild the row-block schedules of A and A^T for kernel class w (0: FP32 /
// BF16 matrix, 1: FP64 matrix) from the per-instance tunables; captured
// graphs hold the old schedules and are dropped.
void rebuild_schedules(Problem& P, int w) {
    cudaStream_t s = P.stream;
    GB_CUDA(cudaStreamSynchronize(s));
    for (auto& g : P.graphs) g.reset();
    DevSchedule& sa = w == 0 ? P.A.sched32 : P.A.sched;
    DevSchedule& st = w == 0 ? P.AT.sched32 : P.AT.sched;
    sa.upload(build_schedule(P.A.host_ptr.data(), P.row_off.data(), P.count, P.tune_block_nnz[w].data(),
                             P.tune_max_rows[w].data()),
              3, s);
    st.upload(build_schedule(P.AT.host_ptr.data(), P.col_off.data(), P.count, P.tune_block_nnz[w].data(),
                             P.tune_max_rows[w].data()),
              3, s);
    const int nb = std::max(P.A.sched.nb + P.AT.sched.nb, P.A.sched32.nb + P.AT.sched32.nb);
    const size_t need = static_cast<size_t>(nb + P.count) * kTerms;
    if (P.partials.size() < need) P.partials.reset(need);
    GB_CUDA(cudaStreamSynchronize(s));
}

// Row-split schedule autotuner, run once per kernel class (w = 0: the FP32
// schedule, timed with the FP32 iteration kernels; w = 1: the FP64 one,
// timed with the FP64 kernels).  Instances are binned into (at most) four
// classes of equal total nonzeros by instance size; for each class in turn
// every candidate (block_nnz, max_rows) -- block_nnz bounds the nonzeros a
// STREAM block stages (<= kBlockNnz, the shared-memory product buffer),
// max_rows the rows it reduces and hence the lanes per row -- is tried with
// the other classes at their incumbents, by timing `iters` fused iterations
// (CUDA events around k_primal + k_dual), and kept when it is more than 1%
// faster.  The per-row group size inside a block still follows the block's
// row count (the row-length histogram).  Besides a fixed grid of candidates,
// block sizes that cut the nonzeros into whole waves of resident CTAs are
// tried: a launch of 1.2 waves leaves most SMs idle during its second wave.
void autotune_class(Problem& P, int w, int iters, double* ms_default, double* ms_tuned) {
    std::vector<std::array<int, 2>> cand = {{2048, 256}, {2048, 128}, {2048, 64}, {1024, 256}, {1024, 128},
                                            {1024, 64},  {1024, 32},  {512, 64},  {512, 32}};
    int per_sm = 0;
    if (w == 0)
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dual<float, float>, kThreads,
                                                              spmv_smem_bytes<1, float>()));
    else
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dual<double, double>, kThreads,
                                                              spmv_smem_bytes<1, double>()));
    const long long wave = static_cast<long long>(std::max(per_sm, 1)) * P.sms;
    for (int k = 1; k <= 4; ++k) {
        long long b = (P.A.nnz + k * wave - 1) / (k * wave);
        b = (b + 31) / 32 * 32;
        if (b >= 256 && b <= kBlockNnz) cand.push_back({static_cast<int>(b), kThreads});
    }
    auto measure = [&]() {  // ms per iteration, back to back in a CUDA graph as the solve loop issues them
        double best = INFINITY;
        for (int rep = 0; rep < 2; ++rep) {
            double mi = 0;
            if (w == 0) time_level_graph<float, float>(P, iters, nullptr, nullptr, &mi);
            else time_level_graph<double, double>(P, iters, nullptr, nullptr, &mi);
            best = std::min(best, mi);
        }
        return best;
    };
    auto& tb = P.tune_block_nnz[w];
    auto& tr = P.tune_max_rows[w];
    tb.assign(P.count, kBlockNnz);
    tr.assign(P.count, kThreads);
    P.A.stream_nc[w] = P.A.default_nc[w];
    P.AT.stream_nc[w] = P.AT.default_nc[w];
    rebuild_schedules(P, w);
    double best = measure();
    if (ms_default) *ms_default = best;
    // load mode of each matrix's kernel (k_dual reads A, k_primal A^T), the
    // other at its incumbent
    for (DevMat* mat : {&P.A, &P.AT}) {
        const int inc = mat->stream_nc[w];
        int win = inc;
        for (int mode : {kLoadPlain, kLoadStream, kLoadPrefetch}) {
            if (mode == inc) continue;
            mat->stream_nc[w] = mode;
            for (auto& g : P.graphs) g.reset();
            const double t = measure();
            if (t < 0.97 * best) {  // 3%: run-to-run noise of one measurement is ~1%
                best = t;
                win = mode;
            }
        }
        mat->stream_nc[w] = win;
        for (auto& g : P.graphs) g.reset();
    }
    std::vector<int> order(P.count);
    std::iota(order.begin(), order.end(), 0);
    auto nnz_of = [&](int k) { return static_cast<long long>(P.nnz_off[k + 1]) - P.nnz_off[k]; };
    std::sort(order.begin(), order.end(), [&](int a, int b) { return nnz_of(a) < nnz_of(b); });
    const long long total = P.nnz_off[P.count];
    const int nclass = std::min(4, P.count);
    std::vector<std::vector<int>> cls(nclass);
    long long acc = 0;
    for (int k : order) {
        const int c = std::min(nclass - 1, static_cast<int>(total ? (acc * nclass) / total : 0));
        cls[c].push_back(k);
        acc += nnz_of(k);
    }
    for (const auto& members : cls) {
        if (members.empty()) continue;
        const int inc_b = tb[members[0]], inc_r = tr[members[0]];
        int win_b = inc_b, win_r = inc_r;
        for (const auto& c : cand) {
            if (c[0] == inc_b && c[1] == inc_r) continue;
            for (int k : members) {
                tb[k] = c[0];
                tr[k] = c[1];
            }
            rebuild_schedules(P, w);
            const double t = measure();
            if (t < 0.99 * best) {
                best = t;
                win_b = c[0];
                win_r = c[1];
            }
        }
        for (int k : members) {
            tb[k] = win_b;
            tr[k] = win_r;
        }
    }
    rebuild_schedules(P, w);
    if (ms_tuned) *ms_tuned = measure();
}

// Both classes; outputs [FP32, FP64].
void autotune(Problem& P, int iters, double* ms_default, double* ms_tuned) {
    for (int w = 0; w < 2; ++w)
        autotune_class(P, w, iters, ms_default ? ms_default + w : nullptr, ms_tuned ? ms_tuned + w : nullptr);
}

void problem_stats(const Problem& P, int64_t* launches, double* bpi) {
    if (launches) *launches = P.launches;
    if (bpi) {
        // fused iteration: 2 nnz (s_M + 4) + 4 (m + n + 2) + s_V (9 n + 7 m)  (+ Q for QP)
        const double nnz = static_cast<double>(P.A.nnz), n = P.n, m = P.m;
        const double sm[3] = {4, 4, 8}, sv[3] = {4, 8, 8};
        for (int l = 0; l < 3; ++l) {
            double b = 2 * nnz * (sm[l] + 4) + 4 * (m + n + 2) + sv[l] * (9 * n + 7 * m);
            if (P.has_q) {
                if (P.dplr) b += 2.0 * n * P.qk * sv[l] + 2 * n * sv[l];
                else b += static_cast<double>(P.Q.nnz) * (sm[l] + 4) + 4 * (n + 1) + sv[l] * 2 * n;
            }
            bpi[l] = b;
        }
    }
}

}  // namespace gb

// ==================================================================== C ABI
using namespace gb;

namespace gb {
// Warm start of instance `inst` (original units; NULL keeps that side's
// default start, NaN entries too).  Applies to every later solve.
void set_start(Problem& P, int inst, const double* x, const double* y) {
    GB_REQUIRE(inst >= 0 && inst < P.count, "instance index out of range");
    GB_CUDA(cudaSetDevice(P.device));
    const int c0 = P.col_off[inst], c1 = P.col_off[inst + 1], r0 = P.row_off[inst], r1 = P.row_off[inst + 1];
    if (x)
        for (int j = 0; j < c1 - c0; ++j) GB_REQUIRE(!std::isinf(x[j]), "start point has an infinite entry");
    if (y)
        for (int i = 0; i < r1 - r0; ++i) GB_REQUIRE(!std::isinf(y[i]), "start point has an infinite entry");
    if (!P.x_start.get()) {
        P.x_start.reset(std::max(P.n, 1));
        P.y_start.reset(std::max(P.m, 1));
        // all-ones bytes are a NaN: every entry starts as "default"
        GB_CUDA(cudaMemsetAsync(P.x_start.get(), 0xff, sizeof(double) * P.x_start.size(), P.stream));
        GB_CUDA(cudaMemsetAsync(P.y_start.get(), 0xff, sizeof(double) * P.y_start.size(), P.stream));
    }
    if (x && c1 > c0)
        GB_CUDA(cudaMemcpyAsync(P.x_start.get() + c0, x, sizeof(double) * (c1 - c0), cudaMemcpyHostToDevice, P.stream));
    if (y && r1 > r0)
        GB_CUDA(cudaMemcpyAsync(P.y_start.get() + r0, y, sizeof(double) * (r1 - r0), cudaMemcpyHostToDevice, P.stream));
    GB_CUDA(cudaStreamSynchronize(P.stream));
}

void clear_start(Problem& P) {
    P.x_start.release();
    P.y_start.release();
}
}  // namespace gb

struct gb_problem {
    Problem* p;
};
struct gb_batch {
    Problem* p;
};

extern "C" {

const char* gb_last_error(void) { return g_last_error.c_str(); }
int gb_version(void) { return 10000; }

void gb_default_options(gb_options* o) {
    o->tol = 1e-4;
    o->max_iter = 10000000;
    o->time_limit = 3600.0;
    o->check_every = 64;
    o->ruiz_iters = 10;
    o->pock_chambolle = 1;
    o->infeas_tol = 1e-8;
    o->precision = GB_PREC_DOUBLE;
    o->stall_checks = 12;
    o->stall_checks_l2 = 24;
    o->verbose = 0;
    o->detect_unbounded = 0;
}

int gb_set_device(int device) {
    return guarded([&] {
        int sms;
        check_device(device, &sms);
        g_device = device;
        GB_CUDA(cudaSetDevice(device));
    });
}

int gb_csr_transpose(int rows, int cols, const int* ptr, const int* idx, const double* val, int* t_ptr, int* t_idx,
                     double* t_val) {
    return guarded([&] {
        GB_REQUIRE(rows >= 0 && cols >= 0 && ptr != nullptr && t_ptr != nullptr, "bad arguments");
        GB_REQUIRE(ptr[0] == 0, "ptr[0] must be 0");
        for (int i = 0; i < rows; ++i) GB_REQUIRE(ptr[i + 1] >= ptr[i], "ptr must be non-decreasing");
        const int nnz = ptr[rows];
        GB_REQUIRE(nnz < (1 << 30), "more than 2^30 nonzeros");
        GB_REQUIRE(nnz == 0 || (idx != nullptr && t_idx != nullptr), "idx / t_idx missing");
        GB_REQUIRE((val == nullptr) == (t_val == nullptr), "val and t_val go together");
        for (int p = 0; p < nnz; ++p) GB_REQUIRE(idx[p] >= 0 && idx[p] < cols, "column index out of range");
        int sms;
        check_device(g_device, &sms);
        GB_CUDA(cudaSetDevice(g_device));
        cudaStream_t s;
        GB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
        } sg{s};
        const size_t z = nnz ? nnz : 1;
        DevBuf<int> d_ptr(rows + 1), d_idx(z), row_of(z), perm(z), d_tptr(cols + 1), d_tidx(z);
        DevBuf<double> d_val, d_tval;
        d_ptr.upload(ptr, rows + 1, s);
        d_idx.upload(idx, nnz, s);
        if (val) {
            d_val.reset(z);
            d_tval.reset(z);
            d_val.upload(val, nnz, s);
        }
        TransposeScratch w;
        transpose_csr(rows, cols, nnz, d_ptr.get(), d_idx.get(), d_val.get(), row_of.get(), perm.get(),
                      d_tptr.get(), d_tidx.get(), d_tval.get(), sms, w, s);
        d_tptr.download(t_ptr, cols + 1, s);
        d_tidx.download(t_idx, nnz, s);
        if (val) d_tval.download(t_val, nnz, s);
        GB_CUDA(cudaStreamSynchronize(s));
        GB_CUDA(cudaGetLastError());
    });
}

int gb_problem_create(const gb_lp* lp, const gb_options* opt, gb_problem** out) {
    return guarded([&] {
        GB_REQUIRE(out != nullptr, "out is NULL");
        gb_options def;
        gb_default_options(&def);
        Problem* p = create_problem(1, lp, opt ? opt : &def);
        *out = new gb_problem{p};
    });
}

int gb_problem_solve(gb_problem* p, const gb_options* opt, gb_result* res) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr, "problem is NULL");
        gb_options def;
        gb_default_options(&def);
        solve_problem(*p->p, opt ? opt : &def, res);
    });
}

int gb_problem_get_solution(gb_problem* p, double* x_out, double* y_out) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr && p->p->solved, "no solution available");
        Problem& P = *p->p;
        if (x_out) P.xo.download(x_out, P.n, P.stream);
        if (y_out) P.yo.download(y_out, P.m, P.stream);
        GB_CUDA(cudaStreamSynchronize(P.stream));
    });
}

void gb_problem_destroy(gb_problem* p) {
    if (!p) return;
    delete p->p;
    delete p;
}

void* gb_problem_stream(gb_problem* p) { return p ? static_cast<void*>(p->p->stream) : nullptr; }

int gb_problem_time_kernels(gb_problem* p, int level, int iters, double* ms_primal, double* ms_dual,
                            int64_t* launches) {
    return guarded([&] {
        GB_REQUIRE(p && iters > 0 && level >= 0 && level <= 3, "bad arguments");
        Problem& P = *p->p;
        GB_REQUIRE(P.solved, "solve once before timing (step sizes come from the solve)");
        GB_REQUIRE(level != 3 || !P.has_q, "the BF16 level takes LPs only");
        if (level == 0) time_level<float, float>(P, iters, ms_primal, ms_dual, launches);
        else if (level == 1) time_level<float, double>(P, iters, ms_primal, ms_dual, launches);
        else if (level == 2) time_level<double, double>(P, iters, ms_primal, ms_dual, launches);
        else {
            ensure_bf16(P);
            time_level<__nv_bfloat16, float>(P, iters, ms_primal, ms_dual, launches);
        }
    });
}

int gb_problem_stats(gb_problem* p, int64_t* launches, double* bpi) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr, "problem is NULL");
        problem_stats(*p->p, launches, bpi);
    });
}

int gb_solve(const gb_lp* lp, const gb_options* opt, gb_result* res, double* x_out, double* y_out) {
    return guarded([&] {
        gb_options def;
        gb_default_options(&def);
        const gb_options* o = opt ? opt : &def;
        std::unique_ptr<Problem> P(create_problem(1, lp, o));
        solve_problem(*P, o, res);
        StageTrace tr{P->stream, "gb_solve"};
        if (x_out) P->xo.download(x_out, P->n, P->stream);
        if (y_out) P->yo.download(y_out, P->m, P->stream);
        GB_CUDA(cudaStreamSynchronize(P->stream));
        tr.mark("download");
        tr.s = nullptr;  // the stream goes with the problem
        P.reset();
        tr.mark("teardown");
    });
}

// ---- batched solving (one block-diagonal resident problem)
int gb_batch_create(int count, const gb_lp* lps, const gb_options* opt, gb_batch** out) {
    return guarded([&] {
        GB_REQUIRE(out != nullptr && count >= 1, "bad arguments");
        gb_options def;
        gb_default_options(&def);
        Problem* p = create_problem(count, lps, opt ? opt : &def);
        *out = new gb_batch{p};
    });
}

int gb_batch_solve(gb_batch* b, const gb_options* opt, gb_result* results) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr, "batch is NULL");
        gb_options def;
        gb_default_options(&def);
        solve_problem(*b->p, opt ? opt : &def, results);
    });
}

int gb_problem_set_start(gb_problem* p, const double* x, const double* y) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr, "problem is NULL");
        if (!x && !y) clear_start(*p->p);
        else set_start(*p->p, 0, x, y);
    });
}

int gb_batch_set_start(gb_batch* b, int i, const double* x, const double* y) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr, "batch is NULL");
        set_start(*b->p, i, x, y);
    });
}

int gb_batch_clear_start(gb_batch* b) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr, "batch is NULL");
        clear_start(*b->p);
    });
}

int gb_batch_get_solution(gb_batch* b, int i, double* x_out, double* y_out) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr && b->p->solved, "no solution available");
        Problem& P = *b->p;
        GB_REQUIRE(i >= 0 && i < P.count, "instance index out of range");
        const int c0 = P.col_off[i], c1 = P.col_off[i + 1], r0 = P.row_off[i], r1 = P.row_off[i + 1];
        if (x_out && c1 > c0)
            GB_CUDA(cudaMemcpyAsync(x_out, P.xo.get() + c0, sizeof(double) * (c1 - c0), cudaMemcpyDeviceToHost,
                                    P.stream));
        if (y_out && r1 > r0)
            GB_CUDA(cudaMemcpyAsync(y_out, P.yo.get() + r0, sizeof(double) * (r1 - r0), cudaMemcpyDeviceToHost,
                                    P.stream));
        GB_CUDA(cudaStreamSynchronize(P.stream));
    });
}

int gb_batch_schedule(gb_batch* b, int* threads, int* blocks_per_sm, int* groups) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr, "batch is NULL");
        Problem& P = *b->p;
        if (threads) *threads = kThreads;
        if (blocks_per_sm) {
            int o = 0;
            GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_dual<float, float>, kThreads,
                                                                  spmv_smem_bytes<1, float>()));
            *blocks_per_sm = o;
        }
        if (groups) {
            // group size (lanes per row) used by most of an instance's STREAM-block nonzeros
            const DevSchedule& sa = P.A.sched_for<float>();
            const DevSchedule& sb = P.AT.sched_for<float>();
            std::vector<RowBlock> ba(sa.nb), bt(sb.nb);
            sa.blocks.download(ba.data(), ba.size(), P.stream);
            sb.blocks.download(bt.data(), bt.size(), P.stream);
            GB_CUDA(cudaStreamSynchronize(P.stream));
            auto mode_g = [](const std::vector<RowBlock>& bl, int b0, int b1) {
                int cnt[6] = {0};
                for (int i = b0; i < b1; ++i)
                    if (bl[i].kind == kStream) cnt[std::min(bl[i].lg, 5)] += bl[i].p1 - bl[i].p0;
                return 1 << static_cast<int>(std::max_element(cnt, cnt + 6) - cnt);
            };
            for (int k = 0; k < P.count; ++k) {
                groups[2 * k] = mode_g(ba, sa.host_seg_block[k], sa.host_seg_block[k + 1]);
                groups[2 * k + 1] = mode_g(bt, sb.host_seg_block[k], sb.host_seg_block[k + 1]);
            }
        }
    });
}

static void load_modes_of(const Problem& P, int* modes) {
    modes[0] = P.A.stream_nc[0];
    modes[1] = P.AT.stream_nc[0];
    modes[2] = P.A.stream_nc[1];
    modes[3] = P.AT.stream_nc[1];
}

int gb_batch_load_modes(gb_batch* b, int* modes) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr && modes != nullptr, "null argument");
        load_modes_of(*b->p, modes);
    });
}

int gb_problem_load_modes(gb_problem* p, int* modes) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr && modes != nullptr, "null argument");
        load_modes_of(*p->p, modes);
    });
}

int gb_batch_autotune(gb_batch* b, int iters, int* block_nnz, int* max_rows, double* ms_default, double* ms_tuned) {
    return guarded([&] {
        GB_REQUIRE(b != nullptr && iters > 0, "bad arguments");
        Problem& P = *b->p;
        autotune(P, iters, ms_default, ms_tuned);
        for (int w = 0; w < 2; ++w)
            for (int k = 0; k < P.count; ++k) {
                if (block_nnz) block_nnz[w * P.count + k] = P.tune_block_nnz[w][k];
                if (max_rows) max_rows[w * P.count + k] = P.tune_max_rows[w][k];
            }
    });
}

int gb_problem_autotune(gb_problem* p, int iters, int* block_nnz, int* max_rows, double* ms_default,
                        double* ms_tuned) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr && iters > 0, "bad arguments");
        Problem& P = *p->p;
        GB_REQUIRE(P.solved, "solve once before tuning (the iterate and step sizes come from the solve)");
        autotune(P, iters, ms_default, ms_tuned);
        for (int w = 0; w < 2; ++w) {
            if (block_nnz) block_nnz[w] = P.tune_block_nnz[w][0];
            if (max_rows) max_rows[w] = P.tune_max_rows[w][0];
        }
    });
}

int gb_problem_time_kernels_graph(gb_problem* p, int level, int iters, double* ms_primal, double* ms_dual,
                                  double* ms_iteration) {
    return guarded([&] {
        GB_REQUIRE(p && iters > 0 && level >= 0 && level <= 3, "bad arguments");
        Problem& P = *p->p;
        GB_REQUIRE(P.solved, "solve once before timing (step sizes come from the solve)");
        by_level(level, P, [&](auto t) {
            using T = decltype(t);
            time_level_graph<typename T::M, typename T::V>(P, iters, ms_primal, ms_dual, ms_iteration);
        });
    });
}

int gb_batch_time_kernels_graph(gb_batch* b, int level, int iters, double* ms_primal, double* ms_dual,
                                double* ms_iteration) {
    return guarded([&] {
        GB_REQUIRE(b && iters > 0 && level >= 0 && level <= 3, "bad arguments");
        Problem& P = *b->p;
        by_level(level, P, [&](auto t) {
            using T = decltype(t);
            time_level_graph<typename T::M, typename T::V>(P, iters, ms_primal, ms_dual, ms_iteration);
        });
    });
}

int gb_batch_time_kernels(gb_batch* b, int level, int iters, double* ms_primal, double* ms_dual, int64_t* launches,
                          double* bytes_per_iter) {
    return guarded([&] {
        GB_REQUIRE(b && iters > 0 && level >= 0 && level <= 3, "bad arguments");
        Problem& P = *b->p;
        if (level == 0) time_level<float, float>(P, iters, ms_primal, ms_dual, launches);
        else if (level == 1) time_level<float, double>(P, iters, ms_primal, ms_dual, launches);
        else if (level == 2) time_level<double, double>(P, iters, ms_primal, ms_dual, launches);
        else {
            ensure_bf16(P);
            time_level<__nv_bfloat16, float>(P, iters, ms_primal, ms_dual, launches);
        }
        if (bytes_per_iter) {
            double bpi[3];
            problem_stats(P, nullptr, bpi);
            // BF16 level: 2 bytes per matrix value instead of FP32's 4
            *bytes_per_iter = level < 3 ? bpi[level] : bpi[0] - 2.0 * 2.0 * static_cast<double>(P.A.nnz);
        }
    });
}

void gb_batch_destroy(gb_batch* b) {
    if (!b) return;
    delete b->p;
    delete b;
}

}  // extern "C"

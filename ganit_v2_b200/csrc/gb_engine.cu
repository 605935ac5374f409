// Single-problem engine and the C ABI (include/ganit_b200.h).
//
// gb_solve / gb_problem_*  : restarted PDHG with every step on the device
//                            (replaces ganit::solve_pdhg_gpu, backend_cuda.cu:382-393)
// gb_backend_* / gb_vec_*  : the Backend concept ops that src/pdhg_impl.hpp
//                            drives (replaces CudaBackend, backend_cuda.cu:286-378)
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "gb_problem.cuh"
#include "gb_qp.cuh"

namespace gb {

thread_local std::string g_last_error;
thread_local int g_device = 0;

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

inline void check_device(int dev, int* sms) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw Error(GB_ERR_NODEVICE, "no CUDA device");
    GB_REQUIRE(dev >= 0 && dev < count, "device index out of range");
    cudaDeviceProp prop;
    GB_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) throw Error(GB_ERR_NODEVICE, "libganit_b200 is built for sm_100a (B200); found sm_" +
                                                          std::to_string(prop.major) + std::to_string(prop.minor));
    *sms = prop.multiProcessorCount;
}

// Opt every SpMV-based kernel into the dynamic shared memory it needs.
template <class K>
void set_smem(K kernel, size_t bytes) {
    GB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
}

void validate_lp(const gb_lp* lp) {
    GB_REQUIRE(lp != nullptr, "lp is NULL");
    GB_REQUIRE(lp->m > 0 && lp->n > 0, "need m > 0 and n > 0");
    GB_REQUIRE(lp->a_ptr && lp->c && lp->l && lp->u, "missing A/c/l/u");
    GB_REQUIRE(lp->m == 0 || (lp->lo && lp->hi), "missing lo/hi");
    GB_REQUIRE(lp->a_ptr[0] == 0, "A.ptr[0] must be 0");
    for (int i = 0; i < lp->m; ++i) GB_REQUIRE(lp->a_ptr[i + 1] >= lp->a_ptr[i], "A.ptr must be nondecreasing");
    const long long nnz = lp->a_ptr[lp->m];
    GB_REQUIRE(nnz == 0 || (lp->a_idx && lp->a_val), "missing A.idx/val");
    for (long long p = 0; p < nnz; ++p) GB_REQUIRE(lp->a_idx[p] >= 0 && lp->a_idx[p] < lp->n, "A.idx out of range");
    for (int j = 0; j < lp->n; ++j) GB_REQUIRE(!(lp->l[j] > lp->u[j]), "column bound l > u");
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

void upload_mat(DevMat& M, int rows, int cols, const int* ptr, const int* idx, const double* val, cudaStream_t s) {
    M.rows = rows;
    M.cols = cols;
    M.nnz = ptr[rows];
    M.host_ptr.assign(ptr, ptr + rows + 1);
    M.ptr.reset(rows + 1);
    M.ptr.upload(ptr, rows + 1, s);
    M.idx.reset(padded_nnz(M.nnz));
    M.val64.reset(padded_nnz(M.nnz));
    GB_CUDA(cudaMemsetAsync(M.idx.get(), 0, M.idx.size() * sizeof(int), s));
    GB_CUDA(cudaMemsetAsync(M.val64.get(), 0, M.val64.size() * sizeof(double), s));
    if (M.nnz) {
        M.idx.upload(idx, M.nnz, s);
        M.val64.upload(val, M.nnz, s);
    }
}

// Device transpose (lp.cpp:55-72): stable radix sort of column keys keeps the
// entries of every output row in increasing source-row order.
void device_transpose(Problem& P, cudaStream_t s) {
    const int nnz = static_cast<int>(P.A.nnz), n = P.n, m = P.m;
    P.AT.rows = n;
    P.AT.cols = m;
    P.AT.nnz = nnz;
    P.row_of.reset(nnz ? nnz : 1);
    P.perm.reset(nnz ? nnz : 1);
    P.AT.ptr.reset(n + 1);
    P.AT.idx.reset(padded_nnz(nnz));
    P.AT.val64.reset(padded_nnz(nnz));
    GB_CUDA(cudaMemsetAsync(P.AT.idx.get(), 0, P.AT.idx.size() * sizeof(int), s));
    GB_CUDA(cudaMemsetAsync(P.AT.val64.get(), 0, P.AT.val64.size() * sizeof(double), s));
    const int g = elem_grid(std::max(nnz, m * 32), P.sms);
    if (m) k_row_of<<<g, kThreads, 0, s>>>(m, P.A.ptr.get(), P.row_of.get());
    DevBuf<int> cnt(n + 1), keys_out, iota;
    DevBuf<unsigned char> tmp;
    GB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * (n + 1), s));
    if (nnz) {
        k_count_cols<<<elem_grid(nnz, P.sms), kThreads, 0, s>>>(nnz, P.A.idx.get(), cnt.get());
        keys_out.reset(nnz);
        iota.reset(nnz);
        k_iota<<<elem_grid(nnz, P.sms), kThreads, 0, s>>>(nnz, iota.get());
        size_t tmp_bytes = 0;
        int bits = 1;
        while ((1LL << bits) < n) ++bits;
        GB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, P.A.idx.get(), keys_out.get(), iota.get(),
                                                P.perm.get(), nnz, 0, bits, s));
        tmp.reset(tmp_bytes ? tmp_bytes : 1);
        GB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, P.A.idx.get(), keys_out.get(), iota.get(),
                                                P.perm.get(), nnz, 0, bits, s));
        k_gather_transpose<<<elem_grid(nnz, P.sms), kThreads, 0, s>>>(nnz, P.perm.get(), P.row_of.get(), nullptr,
                                                                     P.AT.idx.get(), nullptr);
    }
    size_t scan_bytes = 0;
    GB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.get(), P.AT.ptr.get(), n + 1, s));
    DevBuf<unsigned char> stmp(scan_bytes ? scan_bytes : 1);
    GB_CUDA(cub::DeviceScan::ExclusiveSum(stmp.get(), scan_bytes, cnt.get(), P.AT.ptr.get(), n + 1, s));
    P.AT.host_ptr.resize(n + 1);
    GB_CUDA(cudaMemcpyAsync(P.AT.host_ptr.data(), P.AT.ptr.get(), sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
}

__global__ void k_finish_norms(double* sc, int empty) {
    // sc[2] = sqrt(lambda) * 1.01, or 1 for an empty matrix (scaling.cpp:132, 153-154)
    sc[2] = empty ? 1.0 : sqrt(sc[8]) * 1.01;
}
__global__ void k_finish_normq(double* sc) { sc[3] = sc[8] * 1.01; }  // scaling.cpp:124
__global__ void k_w0(double* sc, const double* cn, const double* bn) {
    // w0 = ||c'|| / ||b'||_finite (pdhg_impl.hpp:258-261)
    const double c = *cn, b = *bn;
    sc[6] = (c > 1e-10 && b > 1e-10) ? c / b : 1.0;
}

// Power iteration on the scaled data (scaling.cpp:131-155 for A'^T A',
// scaling.cpp:108-124 for Q').  ||A'|| lands in P.scal[2].
void power_norm_A(Problem& P, cudaStream_t s) {
    const int n = P.n;
    double* pw = P.scal.get() + 7;  // [0] norm, [1] lambda, [2] stopped
    GB_CUDA(cudaMemsetAsync(pw, 0, 3 * sizeof(double), s));
    if (P.A.nnz == 0) {
        k_finish_norms<<<1, 1, 0, s>>>(P.scal.get(), 1);
        return;
    }
    double* v = P.x64.get();  // reuse FP64 vectors as scratch before the solve
    double* w = P.work2.get();
    double* z = P.work1.get();
    k_fill<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, 1.0, v);
    reduce_to(s, n, Sq{v}, P.red_partials.get(), pw, PostSqrt{});
    k_power_step<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, v, v, pw);  // v /= ||v|| (lambda overwritten below)
    GB_CUDA(cudaMemsetAsync(pw + 1, 0, 2 * sizeof(double), s));
    const size_t sm1 = spmv_smem_bytes<1, double>();
    for (int it = 0; it < 50; ++it) {
        k_spmv<double, double><<<P.A.sched.nb, kThreads, sm1, s>>>(P.A.view<double>(), v, w);
        k_spmv<double, double><<<P.AT.sched.nb, kThreads, sm1, s>>>(P.AT.view<double>(), w, z);
        reduce_to(s, n, Sq{z}, P.red_partials.get(), pw, PostSqrt{});
        k_power_step<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, z, v, pw);
    }
    k_finish_norms<<<1, 1, 0, s>>>(P.scal.get(), 0);
}

void qx_dplr_f64(Problem& P, const double* x, double* out, cudaStream_t s);

void power_norm_Q(Problem& P, cudaStream_t s) {
    const int n = P.n;
    double* pw = P.scal.get() + 7;
    double* v = P.x64.get();
    double* w = P.work1.get();
    GB_CUDA(cudaMemsetAsync(pw, 0, 3 * sizeof(double), s));
    k_fill<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, 1.0, v);
    reduce_to(s, n, Sq{v}, P.red_partials.get(), pw, PostSqrt{});
    k_power_step<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, v, v, pw);
    GB_CUDA(cudaMemsetAsync(pw + 1, 0, 2 * sizeof(double), s));
    const size_t sm1 = spmv_smem_bytes<1, double>();
    for (int it = 0; it < 60; ++it) {
        if (P.dplr)
            qx_dplr_f64(P, v, w, s);
        else
            k_spmv<double, double><<<P.Q.sched.nb, kThreads, sm1, s>>>(P.Q.view<double>(), v, w);
        reduce_to(s, n, Sq{w}, P.red_partials.get(), pw, PostSqrt{});
        k_power_step<<<elem_grid(n, P.sms), kThreads, 0, s>>>(n, w, v, pw);
    }
    k_finish_normq<<<1, 1, 0, s>>>(P.scal.get());
}

// DPLR product in FP64 used by the setup power iteration (st == nullptr: one vector).
void qx_dplr_f64(Problem& P, const double* x, double* out, cudaStream_t s) {
    double* part = P.partials.get();
    double* t = P.v64.ftx.get();
    k_ftx_partial<double, 1><<<kFtxGrid, kThreads, 0, s>>>(P.n, P.qk, P.F64.get(), x, nullptr, nullptr, part);
    k_ftx_final<<<1, kThreads, 0, s>>>(kFtxGrid, P.qk, part, t);
    k_dplr_expand<double, 1><<<elem_grid((long long)P.n * 32, P.sms), kThreads, 0, s>>>(
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
        set_smem(k_spmv_q2<float, double>, spmv_smem_bytes<2, double>());
        set_smem(k_spmv_q2<double, double>, spmv_smem_bytes<2, double>());
    });
}

// Upload + device setup (scale_lp + estimate_norm + run_pdhg's start point).
Problem* create_problem(const gb_lp* lp, const gb_options* opt) {
    validate_lp(lp);
    auto P = std::make_unique<Problem>();
    P->device = g_device;
    GB_CUDA(cudaSetDevice(P->device));
    check_device(P->device, &P->sms);
    init_kernel_attrs();
    GB_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
    cudaStream_t s = P->stream;
    const auto t0 = std::chrono::steady_clock::now();
    const int m = lp->m, n = lp->n;
    P->m = m;
    P->n = n;
    P->maximize = lp->maximize != 0;
    P->obj_const = lp->obj_const;
    const double sign = P->maximize ? -1.0 : 1.0;

    upload_mat(P->A, m, n, lp->a_ptr, lp->a_idx, lp->a_val, s);
    auto up = [&](DevBuf<double>& d, const double* h, int k) {
        d.reset(k ? k : 1);
        d.upload(h, k, s);
    };
    DevBuf<double> c0, l0, u0, lo0, hi0;
    up(c0, lp->c, n);
    up(l0, lp->l, n);
    up(u0, lp->u, n);
    up(lo0, lp->lo, m);
    up(hi0, lp->hi, m);
    for (DevBuf<double>* b : {&P->c, &P->l, &P->u, &P->C, &P->Cres, &P->x64, &P->xr64, &P->xo, &P->work1})
        b->reset(n ? n : 1);
    for (DevBuf<double>* b : {&P->lo, &P->hi, &P->R, &P->Rres, &P->y64, &P->yr64, &P->yo, &P->work2})
        b->reset(m ? m : 1);
    P->scal.reset(16);
    GB_CUDA(cudaMemsetAsync(P->scal.get(), 0, 16 * sizeof(double), s));
    P->red_partials.reset(kRedGrid);

    // schedules (host, from the row-length histogram) and transpose
        P->st.reset(1);
    GB_CUDA(cudaMemsetAsync(P->st.get(), 0, sizeof(SolveState), s));
    P->A.sched.upload(build_schedule(P->A.host_ptr.data(), m), 3, s);
    device_transpose(*P, s);
    P->AT.sched.upload(build_schedule(P->AT.host_ptr.data(), n), 3, s);

    // Ruiz equilibration + Pock-Chambolle (scaling.cpp:47-72)
    const int gw = elem_grid(static_cast<long long>(std::max(m, n)) * 32, P->sms);
    const int ge = elem_grid(std::max<long long>(P->A.nnz, 1), P->sms);
    DevBuf<double> rs(m ? m : 1), cs(n);
    k_fill<<<elem_grid(m, P->sms), kThreads, 0, s>>>(m, 1.0, P->R.get());
    k_fill<<<elem_grid(n, P->sms), kThreads, 0, s>>>(n, 1.0, P->C.get());
    const int passes = opt->ruiz_iters + (opt->pock_chambolle ? 1 : 0);
    for (int it = 0; it < passes; ++it) {
        const int mode = it < opt->ruiz_iters ? 0 : 1;
        if (m) k_row_norm_factor<<<gw, kThreads, 0, s>>>(m, P->A.ptr.get(), nullptr, P->A.val64.get(), mode, rs.get());
        k_row_norm_factor<<<gw, kThreads, 0, s>>>(n, P->AT.ptr.get(), P->perm.get(), P->A.val64.get(), mode, cs.get());
        if (P->A.nnz)
            k_apply_scaling<<<ge, kThreads, 0, s>>>(static_cast<int>(P->A.nnz), P->row_of.get(), P->A.idx.get(),
                                                    rs.get(), cs.get(), P->A.val64.get());
        if (m) k_mul_into<<<elem_grid(m, P->sms), kThreads, 0, s>>>(m, rs.get(), P->R.get());
        k_mul_into<<<elem_grid(n, P->sms), kThreads, 0, s>>>(n, cs.get(), P->C.get());
    }
    if (P->A.nnz)
        k_gather_transpose<<<ge, kThreads, 0, s>>>(static_cast<int>(P->A.nnz), P->perm.get(), P->row_of.get(),
                                                  P->A.val64.get(), P->AT.idx.get(), P->AT.val64.get());
    // vectors (scaling.cpp:75-101)
    const int gv = elem_grid(std::max(m, n), P->sms);
    k_scale_vectors<<<gv, kThreads, 0, s>>>(n, m, sign, c0.get(), l0.get(), u0.get(), lo0.get(), hi0.get(),
                                            P->R.get(), P->C.get(), P->c.get(), P->l.get(), P->u.get(), P->lo.get(),
                                            P->hi.get());
    double* sc = P->scal.get();
    reduce_to(s, m, FiniteBoundSq{P->lo.get(), P->hi.get()}, P->red_partials.get(), sc + 0, PostSqrtPlus1{});
    reduce_to(s, n, Sq{P->c.get()}, P->red_partials.get(), sc + 1, PostSqrtPlus1{});
    k_rescale<<<gv, kThreads, 0, s>>>(n, m, sc, P->R.get(), P->C.get(), P->c.get(), P->l.get(), P->u.get(),
                                      P->lo.get(), P->hi.get(), P->Rres.get(), P->Cres.get());
    // norms of the ORIGINAL data (scaling.cpp:126-127)
    reduce_to(s, m, FiniteBoundSq{lo0.get(), hi0.get()}, P->red_partials.get(), sc + 4, PostSqrt{});
    reduce_to(s, n, Sq{c0.get()}, P->red_partials.get(), sc + 5, PostSqrt{});

    // Hessian
    P->has_q = (lp->q_ptr && lp->q_ptr[n] > 0) || lp->q_rank > 0;
    P->dplr = lp->q_rank > 0;
    P->qk = P->dplr ? lp->q_rank : 0;
    P->partials.reset(std::max<size_t>(static_cast<size_t>(kFtxGrid) * 2 * kMaxRank,
                                       static_cast<size_t>(P->A.sched.nb + P->AT.sched.nb) * kTerms));
    P->v32.alloc(n, m, P->qk, P->has_q);
    P->v64.alloc(n, m, P->qk, P->has_q);
    if (P->has_q && !P->dplr) {
        upload_mat(P->Q, n, n, lp->q_ptr, lp->q_idx, lp->q_val, s);
        P->Q.sched.upload(build_schedule(P->Q.host_ptr.data(), n), 3, s);
        P->q_row_of.reset(P->Q.nnz ? P->Q.nnz : 1);
        k_row_of<<<elem_grid((long long)n * 32, P->sms), kThreads, 0, s>>>(n, P->Q.ptr.get(), P->q_row_of.get());
        k_scale_q<<<elem_grid(P->Q.nnz, P->sms), kThreads, 0, s>>>(static_cast<int>(P->Q.nnz), P->q_row_of.get(),
                                                                 P->Q.idx.get(), sign, P->C.get(), sc,
                                                                 P->Q.val64.get());
    } else if (P->dplr) {
        P->F64.reset(static_cast<size_t>(n) * P->qk);
        P->F64.upload(lp->q_F, static_cast<size_t>(n) * P->qk, s);
        up(P->D64, lp->q_D, n);
        k_scale_dplr<<<elem_grid((long long)n * P->qk, P->sms), kThreads, 0, s>>>(n, P->qk, P->C.get(), sc,
                                                                                  P->F64.get(), P->D64.get());
    }
    if (P->has_q) power_norm_Q(*P, s);
    // ||A'|| (scaling.cpp:131-155)
    power_norm_A(*P, s);
    // w0 from the scaled data (pdhg_impl.hpp:258-261)
    reduce_to(s, n, Sq{P->c.get()}, P->red_partials.get(), sc + 10, PostSqrt{});
    reduce_to(s, m, FiniteBoundSq{P->lo.get(), P->hi.get()}, P->red_partials.get(), sc + 11, PostSqrt{});
    k_w0<<<1, 1, 0, s>>>(sc, sc + 10, sc + 11);
    // FP32 copies of the matrix values and data
    auto cvt32 = [&](DevMat& M) {
        M.val32.reset(padded_nnz(M.nnz));
        GB_CUDA(cudaMemsetAsync(M.val32.get(), 0, M.val32.size() * sizeof(float), s));
        if (M.nnz) k_convert<float><<<elem_grid(M.nnz, P->sms), kThreads, 0, s>>>(M.nnz, M.val64.get(), M.val32.get());
    };
    cvt32(P->A);
    cvt32(P->AT);
    if (P->has_q && !P->dplr) cvt32(P->Q);
    convert_data(*P, P->v32, s);
    convert_data(*P, P->v64, s);
    GB_CUDA(cudaMallocHost(&P->st_host, sizeof(SolveState)));
    GB_CUDA(cudaMemcpyAsync(P->scal_host, sc, 10 * sizeof(double), cudaMemcpyDeviceToHost, s));
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
template <class M, class V>
constexpr int level_index() {
    return std::is_same<M, double>::value ? 2 : (std::is_same<V, double>::value ? 1 : 0);
}

template <class M, class V>
void launch_qx(Problem& P, VecSet<V>& vs, const V* x, V* qx, cudaStream_t s, long long& nl) {
    if (P.dplr) {
        double* part = P.partials.get();
        double* t = P.v64.ftx.get();  // FP64 F^T x of any level
        k_ftx_partial<V, 1><<<kFtxGrid, kThreads, 0, s>>>(P.n, P.qk, vs.F.get(), x, nullptr, nullptr, part);
        k_ftx_final<<<1, kThreads, 0, s>>>(kFtxGrid, P.qk, part, t);
        k_dplr_expand<V, 1><<<elem_grid((long long)P.n * 32, P.sms), kThreads, 0, s>>>(
            P.n, P.qk, vs.F.get(), vs.D.get(), t, x, nullptr, nullptr, qx, nullptr);
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
        double* t = P.v64.ftx.get();
        k_ftx_partial<V, 2><<<kFtxGrid, kThreads, 0, s>>>(P.n, P.qk, vs.F.get(), x, vs.sumx.get(), P.st.get(), part);
        k_ftx_final<<<1, kThreads, 0, s>>>(kFtxGrid, 2 * P.qk, part, t);
        k_dplr_expand<V, 2><<<elem_grid((long long)P.n * 32, P.sms), kThreads, 0, s>>>(
            P.n, P.qk, vs.F.get(), vs.D.get(), t, x, vs.sumx.get(), P.st.get(), vs.qx.get(), vs.qxa.get());
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
    a.st = P.st.get();
    a.partials = P.partials.get();
    a.cond = 0;
    a.use_cond = 0;
    return a;
}

// One PDHG iteration (k-th inside the body) on buffers selected by parity.
template <class M, class V>
void launch_iteration(Problem& P, VecSet<V>& vs, int k, cudaStream_t s, long long& nl) {
    const V* xin = (k & 1) ? vs.x1.get() : vs.x0.get();
    V* xout = (k & 1) ? vs.x0.get() : vs.x1.get();
    const V* yin = (k & 1) ? vs.y1.get() : vs.y0.get();
    V* yout = (k & 1) ? vs.y0.get() : vs.y1.get();
    if (P.has_q) launch_qx<M, V>(P, vs, xin, vs.qx.get(), s, nl);
    constexpr size_t sm = spmv_smem_bytes<1, V>();
    PrimalArgs<M, V> pa{P.AT.view<M>(), yin, xin, vs.c.get(), vs.l.get(), vs.u.get(),
                        P.has_q ? vs.qx.get() : nullptr, xout, vs.xbar.get(), vs.sumx.get(), P.st.get()};
    k_primal<M, V><<<P.AT.sched.nb, kThreads, sm, s>>>(pa);
    DualArgs<M, V> da{P.A.view<M>(), vs.xbar.get(), yin, vs.lo.get(), vs.hi.get(), yout, vs.sumy.get(),
                      P.st.get()};
    k_dual<M, V><<<P.A.sched.nb, kThreads, sm, s>>>(da);
    nl += 2;
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
    const int grid = P.A.sched.nb + P.AT.sched.nb;
    k_eval<M, V, 2, 3><<<grid, kThreads, spmv_smem_bytes<3, V>(), s>>>(ea);
    RestartArgs<V> ra{xc, yc, vs.x0.get(), vs.y0.get(), vs.xr.get(), vs.yr.get(), vs.sumx.get(), vs.sumy.get(),
                      P.n, P.m, P.st.get()};
    k_restart<V><<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(ra);
    nl += 2;
    return nl;
}

template <class M, class V>
LevelGraph* level_graph(Problem& P, int ce) {
    constexpr int li = level_index<M, V>();
    auto& slot = P.graphs[li];
    if (slot && slot->check_every == ce) return slot.get();
    slot.reset(new LevelGraph);
    LevelGraph* g = slot.get();
    g->check_every = ce;
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
        cudaGraph_t dummy;
        cudaStreamEndCapture(cs, &dummy);
        cudaStreamDestroy(cs);
        throw;
    }
    GB_CUDA(cudaStreamEndCapture(cs, &body));
    GB_CUDA(cudaStreamDestroy(cs));
    GB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
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

__global__ void k_set_phase(SolveState* st, double tol, int stall_checks, int stall_exit, int first_phase) {
    st->phase_tol = tol;
    st->stall_checks = stall_checks;
    st->stall_exit = stall_exit;
    st->carry_restart_err = first_phase ? -1.0 : st->restart_err;
}

__global__ void k_init_state(SolveState* st, const double* sc, double obj_const, int has_q, int check_every,
                             long long max_iter, double time_limit, double infeas_tol) {
    SolveState s;
    memset(&s, 0, sizeof(s));
    s.normA = sc[2];
    s.eta = 0.998 / s.normA;
    s.normQ = sc[3];
    s.obj_scale = sc[1] * sc[0];
    s.obj_const = obj_const;
    s.bnorm = sc[4];
    s.cnorm = sc[5];
    s.w = sc[6];
    s.infeas_tol = infeas_tol;
    s.time_limit_s = time_limit;
    s.max_iter = max_iter;
    s.check_every = check_every;
    s.has_q = has_q;
    s.carry_restart_err = -1.0;
    s.restart_err = -1.0;
    *st = s;
}

void sync_state(Problem& P) {
    GB_CUDA(cudaMemcpyAsync(P.st_host, P.st.get(), sizeof(SolveState), cudaMemcpyDeviceToHost, P.stream));
    GB_CUDA(cudaStreamSynchronize(P.stream));
}

template <class M, class V>
int run_phase(Problem& P, const gb_options* opt, double tol, int stall_exit, int stall_checks, bool first,
              bool has_r) {
    cudaStream_t s = P.stream;
    VecSet<V>& vs = Level<M, V>::vs(P);
    const int gv = elem_grid(std::max(P.n, P.m), P.sms);
    k_phase_in<V><<<gv, kThreads, 0, s>>>(P.n, P.m, P.x64.get(), P.y64.get(), has_r ? P.xr64.get() : P.x64.get(),
                                         has_r ? P.yr64.get() : P.y64.get(), vs.x0.get(), vs.y0.get(), vs.xr.get(),
                                         vs.yr.get(), vs.sumx.get(), vs.sumy.get());
    k_set_phase<<<1, 1, 0, s>>>(P.st.get(), tol, stall_checks, stall_exit, first ? 1 : 0);
    P.launches += 2;
    if (P.has_q) launch_qx<M, V>(P, vs, vs.x0.get(), vs.qx.get(), s, P.launches);
    EvalArgs<M, V> ea = eval_args<M, V>(P, vs, vs.x0.get(), vs.y0.get(), kEvalInit, P.has_q);
    k_eval<M, V, 1, 1><<<P.A.sched.nb + P.AT.sched.nb, kThreads, spmv_smem_bytes<1, V>(), s>>>(ea);
    P.launches += 1;
    const int checks_before = first ? 0 : P.st_host->checks;
    long long per_body = 0;
    if (host_loop_mode()) {
        // Same kernels, launched from a host loop with one state read-back per
        // check (profilers cannot see kernels inside conditional graphs).
        for (;;) {
            per_body = capture_body<M, V>(P, opt->check_every, 0, s, 0);
            sync_state(P);
            if (P.st_host->done) break;
        }
    } else {
        LevelGraph* g = level_graph<M, V>(P, opt->check_every);
        GB_CUDA(cudaGraphLaunch(g->exec, s));
        per_body = g->launches_per_body;
    }
    k_phase_out<V><<<gv, kThreads, 0, s>>>(P.n, P.m, vs.x0.get(), vs.y0.get(), vs.sumx.get(), vs.sumy.get(),
                                          vs.xr.get(), vs.yr.get(), P.st.get(), P.x64.get(), P.y64.get(),
                                          P.xr64.get(), P.yr64.get());
    sync_state(P);
    P.launches += 1 + static_cast<long long>(P.st_host->checks - checks_before) * per_body;
    GB_CUDA(cudaGetLastError());
    return P.st_host->exit_reason;
}

// pdhg_evaluate<Bd> (pdhg_impl.hpp:202-230) of the carried FP64 state.
Kkt certify(Problem& P) {
    cudaStream_t s = P.stream;
    VecSet<double>& vs = P.v64;
    if (P.has_q) launch_qx<double, double>(P, vs, P.x64.get(), vs.qx.get(), s, P.launches);
    EvalArgs<double, double> ea = eval_args<double, double>(P, vs, P.x64.get(), P.y64.get(), kEvalCertify, P.has_q);
    k_eval<double, double, 1, 1><<<P.A.sched.nb + P.AT.sched.nb, kThreads,
                                   spmv_smem_bytes<1, double>(), s>>>(ea);
    P.launches += 1;
    sync_state(P);
    return P.st_host->kcert;
}

inline bool kkt_conv_h(const Kkt& k, double tol) { return k.rel_p <= tol && k.rel_d <= tol && k.rel_gap <= tol; }

int status_from(int e) {  // pdhg_impl.hpp:232-240
    switch (e) {
        case kConverged: return GB_OPTIMAL;
        case kInfeasible: return GB_PRIMAL_INFEASIBLE;
        case kTimeLimit: return GB_TIME_LIMIT;
        case kNumerical: return GB_NUMERICAL_ERROR;
        default: return GB_ITERATION_LIMIT;
    }
}

// run_pdhg (pdhg_impl.hpp:243-328) with device-resident state.
void solve_problem(Problem& P, const gb_options* opt, gb_result* res) {
    GB_REQUIRE(opt->check_every > 0, "check_every must be positive");
    GB_REQUIRE(opt->precision >= 0 && opt->precision <= 2, "unknown precision");
    GB_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = P.stream;
    const auto t0 = std::chrono::steady_clock::now();
    P.launches = 0;
    k_init_state<<<1, 1, 0, s>>>(P.st.get(), P.scal.get(), P.maximize ? -P.obj_const : P.obj_const,
                                 P.has_q ? 1 : 0, opt->check_every, opt->max_iter, opt->time_limit, opt->infeas_tol);
    k_start_point<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(P.n, P.m, P.l.get(), P.u.get(),
                                                                         P.x64.get(), P.y64.get());
    k_mark_start<<<1, 1, 0, s>>>(P.st.get());
    P.launches += 3;
    int ex;
    long long fp32_iters = 0, l2_iters = 0;
    int phases = 0;
    auto finished = [&](int e) {
        const Kkt k64 = certify(P);
        return (e == kConverged && kkt_conv_h(k64, opt->tol)) || e == kTimeLimit || e == kIterLimit ||
               e == kInfeasible;
    };
    if (opt->precision != GB_PREC_DOUBLE) {
        ex = run_phase<float, float>(P, opt, opt->tol, 1, opt->stall_checks, true, false);
        ++phases;
        fp32_iters = P.st_host->it;
        bool done = finished(ex);
        if (!done && opt->precision == GB_PREC_DYNAMIC) {
            ex = run_phase<float, double>(P, opt, opt->tol, 1, opt->stall_checks_l2, false, true);
            ++phases;
            l2_iters = P.st_host->it - fp32_iters;
            done = finished(ex);
        }
        if (!done) {
            ex = run_phase<double, double>(P, opt, opt->tol, 0, 0, false, true);
            ++phases;
        }
    } else {
        ex = run_phase<double, double>(P, opt, opt->tol, 0, 0, true, false);
        ++phases;
    }
    const Kkt fin = certify(P);
    int status = status_from(ex);
    if (status == GB_OPTIMAL && !kkt_conv_h(fin, opt->tol * 1.0000001)) status = GB_NUMERICAL_ERROR;
    const double sign = P.maximize ? -1.0 : 1.0;
    k_unscale<<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(P.n, P.m, sign, P.x64.get(), P.y64.get(),
                                                                     P.C.get(), P.R.get(), P.scal.get(),
                                                                     P.xo.get(), P.yo.get());
    P.launches += 1;
    GB_CUDA(cudaStreamSynchronize(s));
    GB_CUDA(cudaGetLastError());
    const SolveState& st = *P.st_host;
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->status = status;
        res->pobj = sign * fin.pobj;
        res->dobj = sign * fin.dobj;
        res->rel_primal = fin.rel_p;
        res->rel_dual = fin.rel_d;
        res->rel_gap = fin.rel_gap;
        res->iterations = st.it;
        res->fp32_iterations = fp32_iters;
        res->l2_iterations = l2_iters;
        res->restarts = st.restarts;
        res->setup_seconds = P.setup_seconds;
        res->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        res->norm_a = P.scal_host[2];
        res->primal_weight = st.w;
        res->checks = st.checks;
        res->phases = phases;
    }
    P.solved = true;
}

// ---------------------------------------------------------------- kernel timing
template <class M, class V>
void time_level(Problem& P, int iters, double* msp, double* msd, int64_t* launches) {
    cudaStream_t s = P.stream;
    VecSet<V>& vs = Level<M, V>::vs(P);
    // a valid iterate: the start point with current step sizes
    k_phase_in<V><<<elem_grid(std::max(P.n, P.m), P.sms), kThreads, 0, s>>>(
        P.n, P.m, P.x64.get(), P.y64.get(), P.x64.get(), P.y64.get(), vs.x0.get(), vs.y0.get(), vs.xr.get(),
        vs.yr.get(), vs.sumx.get(), vs.sumy.get());
    std::vector<cudaEvent_t> ev(2 * iters + 1);
    for (auto& e : ev) GB_CUDA(cudaEventCreate(&e));
    long long nl = 0;
    // warm-up
    for (int k = 0; k < 4; ++k) launch_iteration<M, V>(P, vs, k, s, nl);
    GB_CUDA(cudaEventRecord(ev[0], s));
    for (int k = 0; k < iters; ++k) {
        const V* xin = (k & 1) ? vs.x1.get() : vs.x0.get();
        V* xout = (k & 1) ? vs.x0.get() : vs.x1.get();
        const V* yin = (k & 1) ? vs.y1.get() : vs.y0.get();
        V* yout = (k & 1) ? vs.y0.get() : vs.y1.get();
        if (P.has_q) launch_qx<M, V>(P, vs, xin, vs.qx.get(), s, nl);
        constexpr size_t sm = spmv_smem_bytes<1, V>();
        PrimalArgs<M, V> pa{P.AT.view<M>(), yin, xin, vs.c.get(), vs.l.get(), vs.u.get(),
                            P.has_q ? vs.qx.get() : nullptr, xout, vs.xbar.get(), vs.sumx.get(), P.st.get()};
        k_primal<M, V><<<P.AT.sched.nb, kThreads, sm, s>>>(pa);
        GB_CUDA(cudaEventRecord(ev[2 * k + 1], s));
        DualArgs<M, V> da{P.A.view<M>(), vs.xbar.get(), yin, vs.lo.get(), vs.hi.get(), yout, vs.sumy.get(),
                          P.st.get()};
        k_dual<M, V><<<P.A.sched.nb, kThreads, sm, s>>>(da);
        GB_CUDA(cudaEventRecord(ev[2 * k + 2], s));
        nl += 2;
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

}  // namespace gb

// ==================================================================== C ABI
using namespace gb;

struct gb_problem {
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
}

int gb_set_device(int device) {
    return guarded([&] {
        int sms;
        check_device(device, &sms);
        g_device = device;
        GB_CUDA(cudaSetDevice(device));
    });
}

int gb_problem_create(const gb_lp* lp, const gb_options* opt, gb_problem** out) {
    return guarded([&] {
        GB_REQUIRE(out != nullptr, "out is NULL");
        gb_options def;
        gb_default_options(&def);
        Problem* p = create_problem(lp, opt ? opt : &def);
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
        GB_REQUIRE(p && iters > 0 && level >= 0 && level <= 2, "bad arguments");
        Problem& P = *p->p;
        GB_REQUIRE(P.solved, "solve once before timing (step sizes come from the solve)");
        if (level == 0) time_level<float, float>(P, iters, ms_primal, ms_dual, launches);
        else if (level == 1) time_level<float, double>(P, iters, ms_primal, ms_dual, launches);
        else time_level<double, double>(P, iters, ms_primal, ms_dual, launches);
    });
}

int gb_problem_stats(gb_problem* p, int64_t* launches, double* bpi) {
    return guarded([&] {
        GB_REQUIRE(p != nullptr, "problem is NULL");
        Problem& P = *p->p;
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
    });
}

int gb_solve(const gb_lp* lp, const gb_options* opt, gb_result* res, double* x_out, double* y_out) {
    return guarded([&] {
        gb_options def;
        gb_default_options(&def);
        const gb_options* o = opt ? opt : &def;
        std::unique_ptr<Problem> P(create_problem(lp, o));
        solve_problem(*P, o, res);
        if (x_out) P->xo.download(x_out, P->n, P->stream);
        if (y_out) P->yo.download(y_out, P->m, P->stream);
        GB_CUDA(cudaStreamSynchronize(P->stream));
    });
}

}  // extern "C"

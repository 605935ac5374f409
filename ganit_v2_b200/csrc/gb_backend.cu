// Backend-concept operations behind the C ABI (gb_backend_* / gb_vec_*).
//
// One entry point per member of the Backend concept that src/pdhg_impl.hpp
// drives (implemented in the reference by CudaBackend<M,V>,
// src/backend_cuda.cu:286-378, and CpuBackendT<M,R>, src/backend_cpu.cpp:38-156).
// Matrix products use the row-block SpMV of gb_spmv.cuh; reductions are
// fixed-order two-pass FP64 sums (the reference uses atomicAdd, so its
// results vary run to run; these do not).
#include <cstring>
#include <memory>

#include "../../include/ganit_b200.h"
#include "gb_setup.cuh"

namespace gb {
extern thread_local std::string g_last_error;
extern thread_local int g_device;

template <class F>
int guarded_b(F&& f) {
    try {
        f();
        return GB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GB_ERR_INVALID;
    }
}

// ---- elementwise kernels (backend_cpu.cpp:67-100)
template <class V>
__global__ void kb_primal_step(int n, const V* x, const V* aty, const V* qx, const V* c, const V* l, const V* u,
                               V tau, V* xn, V* xbar, V* sumx) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const V xj = x[j];
        const V g = c[j] - aty[j] + (qx ? qx[j] : V(0));
        V v = xj - tau * g;
        v = (v < l[j]) ? l[j] : v;
        v = (u[j] < v) ? u[j] : v;
        xn[j] = v;
        xbar[j] = V(2) * v - xj;
        sumx[j] += v;
    }
}
template <class V>
__global__ void kb_dual_step(int m, const V* y, const V* axbar, const V* lo, const V* hi, V sigma, V* yn,
                             V* sumy) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const V q = y[i] - sigma * axbar[i];
        const V a = sigma * lo[i], b = sigma * hi[i];
        V t = -q;
        t = (t < a) ? a : t;
        t = (b < t) ? b : t;
        const V v = q + t;
        yn[i] = v;
        sumy[i] += v;
    }
}
template <class V>
__global__ void kb_sub(int n, const V* a, const V* b, V* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = a[i] - b[i];
}
template <class V>
__global__ void kb_scale(int n, double a, const V* s, V* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        d[i] = static_cast<V>(a * static_cast<double>(s[i]));
}
template <class V>
__global__ void kb_fill(int n, double a, V* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = static_cast<V>(a);
}
template <class V>
__global__ void kb_to_double(int n, const V* s, double* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = double(s[i]);
}

// ---- two-channel fixed-order reductions (backend_cpu.cpp:101-155)
template <class F>
__global__ void __launch_bounds__(kThreads) kb_red1(int n, F f, double* part) {
    __shared__ double sh[kWarps * 2];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        double a = 0.0, b = 0.0;
        f(i, a, b);
        v[0] += a;
        v[1] += b;
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = v[0];
        part[2 * blockIdx.x + 1] = v[1];
    }
}
__global__ void __launch_bounds__(kThreads) kb_red2(int np, const double* part, double* out) {
    __shared__ double sh[kWarps * 2];
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < np; i += kThreads) {
        v[0] += part[2 * i];
        v[1] += part[2 * i + 1];
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        out[0] = v[0];
        out[1] = v[1];
    }
}

template <class V>
struct FPrimalRes {
    const V *ax, *lo, *hi, *r;
    __device__ void operator()(int i, double& a, double& b) const {
        const double x = double(ax[i]), l = double(lo[i]), h = double(hi[i]);
        double p = (x < l) ? l : x;
        p = (h < p) ? h : p;
        const double d = (x - p) / double(r[i]);
        a = d * d;
        b = 0.0;
    }
};
template <class V>
struct FDualRes {
    const V *aty, *qx, *c, *l, *u, *cres;
    double cw;
    __device__ void operator()(int j, double& a, double& b) const {
        const double z = cw * double(c[j]) - double(aty[j]) + (qx ? double(qx[j]) : 0.0);
        const double lj = double(l[j]), uj = double(u[j]);
        double r = 0.0, ob = 0.0;
        if (z > 0) { if (isfinite(lj)) ob = z * lj; else r = z; }
        else if (z < 0) { if (isfinite(uj)) ob = z * uj; else r = z; }
        r /= double(cres[j]);
        a = r * r;
        b = ob;
    }
};
template <class V>
struct FRowDualObj {
    const V *y, *lo, *hi;
    __device__ void operator()(int i, double& a, double& b) const {
        const double yi = double(y[i]), l = double(lo[i]), h = double(hi[i]);
        a = 0.0;
        if (yi > 0 && isfinite(l)) a = yi * l;
        else if (yi < 0 && isfinite(h)) a = yi * h;
        b = 0.0;
    }
};
template <class V>
struct FDot {
    const V *x, *y;
    __device__ void operator()(int i, double& a, double& b) const {
        a = double(x[i]) * double(y[i]);
        b = 0.0;
    }
};
template <class V>
struct FDiff2 {
    const V *x, *y;
    __device__ void operator()(int i, double& a, double& b) const {
        const double d = double(x[i]) - double(y[i]);
        a = d * d;
        b = 0.0;
    }
};

struct Vec {
    int k = 0;
    int esize = 8;
    DevBuf<unsigned char> buf;
    template <class V>
    V* p() const { return reinterpret_cast<V*>(buf.get()); }
};

struct Backend {
    FreeBatchEnd free_batch;  // first member, destroyed last: closes the teardown's free batch
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    int mat_type = GB_F64, vec_type = GB_F64;
    int m = 0, n = 0;
    bool has_q = false;
    // matrices: structure + values in the matrix type
    DevBuf<int> a_ptr, a_idx, at_ptr, at_idx, q_ptr, q_idx;
    DevBuf<unsigned char> a_val, at_val, q_val;
    DevSchedule a_s, at_s, q_s;
    // data in the vector type
    Vec c, l, u, lo, hi, rres, cres;
    DevBuf<double> part, out;
    double* out_host = nullptr;
    ~Backend() {
        cudaSetDevice(device);
        begin_free_batch();
        free_batch.open = true;
        host_free(out_host);
        if (stream) cudaStreamDestroy(stream);
    }
};

template <class M>
CsrView<M> bview(const DevBuf<int>& ptr, const DevBuf<int>& idx, const DevBuf<unsigned char>& val,
                 const DevSchedule& s, int rows) {
    CsrView<M> v;
    v.ptr = ptr.get();
    v.idx = idx.get();
    v.val = reinterpret_cast<const M*>(val.get());
    v.blocks = s.blocks.get();
    v.slots = s.slots.get();
    v.counters = s.counters.get();
    v.bits = s.bits.get();
    v.rows = rows;
    v.nb = s.nb;
    return v;
}

void upload_values(Backend& B, DevBuf<unsigned char>& dst, const double* h, long long k) {
    const int es = B.mat_type == GB_F32 ? 4 : 8;
    dst.reset(static_cast<size_t>(k ? k : 1) * es);
    if (!k) return;
    DevBuf<double> tmp(k);
    tmp.upload(h, k, B.stream);
    if (es == 4) k_convert<float><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, tmp.get(), reinterpret_cast<float*>(dst.get()));
    else k_convert<double><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, tmp.get(), reinterpret_cast<double*>(dst.get()));
    GB_CUDA(cudaStreamSynchronize(B.stream));
}

void vec_from_host(Backend& B, Vec& v, const double* h, int k) {
    v.k = k;
    v.esize = B.vec_type == GB_F32 ? 4 : 8;
    v.buf.reset(static_cast<size_t>(k ? k : 1) * v.esize);
    if (!k) return;
    if (!h) {
        GB_CUDA(cudaMemsetAsync(v.buf.get(), 0, static_cast<size_t>(k) * v.esize, B.stream));
        return;
    }
    DevBuf<double> tmp(k);
    tmp.upload(h, k, B.stream);
    if (v.esize == 4) k_convert<float><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, tmp.get(), v.p<float>());
    else GB_CUDA(cudaMemcpyAsync(v.buf.get(), tmp.get(), sizeof(double) * k, cudaMemcpyDeviceToDevice, B.stream));
    GB_CUDA(cudaStreamSynchronize(B.stream));
}

template <class F>
std::pair<double, double> reduce2(Backend& B, int k, F f) {
    if (k > 0) {
        kb_red1<F><<<kRedGrid, kThreads, 0, B.stream>>>(k, f, B.part.get());
        kb_red2<<<1, kThreads, 0, B.stream>>>(kRedGrid, B.part.get(), B.out.get());
    } else {
        GB_CUDA(cudaMemsetAsync(B.out.get(), 0, 2 * sizeof(double), B.stream));
    }
    GB_CUDA(cudaMemcpyAsync(B.out_host, B.out.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, B.stream));
    GB_CUDA(cudaStreamSynchronize(B.stream));
    GB_CUDA(cudaGetLastError());
    return {B.out_host[0], B.out_host[1]};
}

template <class M, class V>
void spmv_t(Backend& B, int which, const Vec& x, Vec& y) {
    const DevBuf<int>& ptr = which == 0 ? B.a_ptr : which == 1 ? B.at_ptr : B.q_ptr;
    const DevBuf<int>& idx = which == 0 ? B.a_idx : which == 1 ? B.at_idx : B.q_idx;
    const DevBuf<unsigned char>& val = which == 0 ? B.a_val : which == 1 ? B.at_val : B.q_val;
    const DevSchedule& s = which == 0 ? B.a_s : which == 1 ? B.at_s : B.q_s;
    const int rows = which == 0 ? B.m : B.n;
    if (rows == 0 || s.nb == 0) return;
    static_assert(spmv_smem_bytes<1, double>() <= 48 * 1024, "single-vector SpMV fits the default smem limit");
    k_spmv<M, V><<<s.nb, kThreads, spmv_smem_bytes<1, V>(), B.stream>>>(bview<M>(ptr, idx, val, s, rows), x.p<V>(),
                                                                     y.p<V>());
    GB_CUDA(cudaGetLastError());
}

}  // namespace gb

using namespace gb;

struct gb_backend {
    Backend b;
};
struct gb_vec {
    gb_backend* owner;
    Vec v;
};

#define GB_DISPATCH_V(B, ...)                                 \
    do {                                                      \
        if ((B).vec_type == GB_F32) {                         \
            using V = float;                                  \
            __VA_ARGS__;                                      \
        } else {                                              \
            using V = double;                                 \
            __VA_ARGS__;                                      \
        }                                                     \
    } while (0)

extern "C" {

int gb_backend_create(const gb_scaled_lp* s, int mat_type, int vec_type, gb_backend** out) {
    return guarded_b([&] {
        GB_REQUIRE(s && out, "NULL argument");
        GB_REQUIRE(s->m > 0 && s->n > 0, "need m > 0 and n > 0");
        GB_REQUIRE((mat_type == GB_F32 || mat_type == GB_F64) && (vec_type == GB_F32 || vec_type == GB_F64),
                   "types must be GB_F32 or GB_F64");
        GB_REQUIRE(!(mat_type == GB_F64 && vec_type == GB_F32), "matrix FP64 with vectors FP32 is not a level");
        auto h = std::make_unique<gb_backend>();
        Backend& B = h->b;
        B.device = g_device;
        GB_CUDA(cudaSetDevice(B.device));
        cudaDeviceProp prop;
        GB_CUDA(cudaGetDeviceProperties(&prop, B.device));
        GB_REQUIRE(prop.major >= 10, "libganit_b200 is built for sm_100a");
        B.sms = prop.multiProcessorCount;
        GB_CUDA(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
        B.mat_type = mat_type;
        B.vec_type = vec_type;
        B.m = s->m;
        B.n = s->n;
        const int nnz = s->a_ptr[s->m];
        GB_REQUIRE(s->at_ptr[s->n] == nnz, "A and AT differ in nnz");
        auto upi = [&](DevBuf<int>& d, const int* h, long long k) {
            d.reset(k ? k : 1);
            d.upload(h, k, B.stream);
        };
        upi(B.a_ptr, s->a_ptr, s->m + 1);
        upi(B.a_idx, s->a_idx, nnz);
        upi(B.at_ptr, s->at_ptr, s->n + 1);
        upi(B.at_idx, s->at_idx, nnz);
        upload_values(B, B.a_val, s->a_val, nnz);
        upload_values(B, B.at_val, s->at_val, nnz);
        B.a_s.upload(build_schedule(s->a_ptr, s->m), 1, B.stream);
        B.at_s.upload(build_schedule(s->at_ptr, s->n), 1, B.stream);
        B.has_q = s->q_ptr != nullptr && s->q_ptr[s->n] > 0;
        if (B.has_q) {
            const int qn = s->q_ptr[s->n];
            upi(B.q_ptr, s->q_ptr, s->n + 1);
            upi(B.q_idx, s->q_idx, qn);
            upload_values(B, B.q_val, s->q_val, qn);
            B.q_s.upload(build_schedule(s->q_ptr, s->n), 1, B.stream);
        }
        vec_from_host(B, B.c, s->c, s->n);
        vec_from_host(B, B.l, s->l, s->n);
        vec_from_host(B, B.u, s->u, s->n);
        vec_from_host(B, B.cres, s->cres, s->n);
        vec_from_host(B, B.lo, s->lo, s->m);
        vec_from_host(B, B.hi, s->hi, s->m);
        vec_from_host(B, B.rres, s->rres, s->m);
        B.part.reset(2 * kRedGrid);
        B.out.reset(2);
        B.out_host = static_cast<double*>(host_alloc(2 * sizeof(double)));
        GB_CUDA(cudaStreamSynchronize(B.stream));
        *out = h.release();
    });
}

void gb_backend_destroy(gb_backend* b) { delete b; }

int gb_vec_zeros(gb_backend* b, int k, gb_vec** out) {
    return guarded_b([&] {
        GB_REQUIRE(b && out && k >= 0, "bad arguments");
        auto v = std::make_unique<gb_vec>();
        v->owner = b;
        vec_from_host(b->b, v->v, nullptr, k);
        GB_CUDA(cudaStreamSynchronize(b->b.stream));
        *out = v.release();
    });
}

int gb_vec_from_host(gb_backend* b, const double* h, int k, gb_vec** out) {
    return guarded_b([&] {
        GB_REQUIRE(b && out && k >= 0 && (h || k == 0), "bad arguments");
        auto v = std::make_unique<gb_vec>();
        v->owner = b;
        vec_from_host(b->b, v->v, h, k);
        *out = v.release();
    });
}

int gb_vec_to_host(gb_backend* b, const gb_vec* v, double* h) {
    return guarded_b([&] {
        GB_REQUIRE(b && v && (h || v->v.k == 0), "bad arguments");
        Backend& B = b->b;
        const int k = v->v.k;
        if (!k) return;
        DevBuf<double> tmp(k);
        GB_DISPATCH_V(B, kb_to_double<V><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, v->v.p<V>(), tmp.get()));
        tmp.download(h, k, B.stream);
        GB_CUDA(cudaStreamSynchronize(B.stream));
    });
}

int gb_vec_size(const gb_vec* v) { return v ? v->v.k : 0; }
void gb_vec_destroy(gb_vec* v) { delete v; }

int gb_copy(gb_backend* b, const gb_vec* src, gb_vec* dst) {
    return guarded_b([&] {
        GB_REQUIRE(b && src && dst && dst->v.k >= src->v.k, "bad arguments");
        if (src->v.k)
            GB_CUDA(cudaMemcpyAsync(dst->v.buf.get(), src->v.buf.get(), static_cast<size_t>(src->v.k) * src->v.esize,
                                    cudaMemcpyDeviceToDevice, b->b.stream));
    });
}

int gb_fill(gb_backend* b, gb_vec* v, double a) {
    return guarded_b([&] {
        GB_REQUIRE(b && v, "bad arguments");
        Backend& B = b->b;
        if (v->v.k) GB_DISPATCH_V(B, kb_fill<V><<<elem_grid(v->v.k, B.sms), kThreads, 0, B.stream>>>(v->v.k, a, v->v.p<V>()));
    });
}

static int spmv_entry(gb_backend* b, int which, const gb_vec* x, gb_vec* y) {
    return guarded_b([&] {
        GB_REQUIRE(b && x && y, "bad arguments");
        Backend& B = b->b;
        GB_REQUIRE(which != 2 || B.has_q, "no Hessian uploaded");
        const int rows = which == 0 ? B.m : B.n, cols = which == 1 ? B.m : B.n;
        GB_REQUIRE(x->v.k >= cols && y->v.k >= rows, "vector sizes do not match the matrix");
        if (B.mat_type == GB_F32 && B.vec_type == GB_F32) spmv_t<float, float>(B, which, x->v, y->v);
        else if (B.mat_type == GB_F32) spmv_t<float, double>(B, which, x->v, y->v);
        else spmv_t<double, double>(B, which, x->v, y->v);
    });
}
int gb_spmv_A(gb_backend* b, const gb_vec* x, gb_vec* ax) { return spmv_entry(b, 0, x, ax); }
int gb_spmv_AT(gb_backend* b, const gb_vec* y, gb_vec* aty) { return spmv_entry(b, 1, y, aty); }
int gb_spmv_Q(gb_backend* b, const gb_vec* x, gb_vec* qx) { return spmv_entry(b, 2, x, qx); }

int gb_primal_step(gb_backend* b, const gb_vec* x, const gb_vec* aty, const gb_vec* qx, double tau, gb_vec* xn,
                   gb_vec* xbar, gb_vec* sumx) {
    return guarded_b([&] {
        GB_REQUIRE(b && x && aty && xn && xbar && sumx, "bad arguments");
        Backend& B = b->b;
        const int n = B.n;
        GB_DISPATCH_V(B, kb_primal_step<V><<<elem_grid(n, B.sms), kThreads, 0, B.stream>>>(
                             n, x->v.p<V>(), aty->v.p<V>(), qx ? qx->v.p<V>() : nullptr, B.c.p<V>(), B.l.p<V>(),
                             B.u.p<V>(), static_cast<V>(tau), xn->v.p<V>(), xbar->v.p<V>(), sumx->v.p<V>()));
    });
}

int gb_dual_step(gb_backend* b, const gb_vec* y, const gb_vec* axbar, double sigma, gb_vec* yn, gb_vec* sumy) {
    return guarded_b([&] {
        GB_REQUIRE(b && y && axbar && yn && sumy, "bad arguments");
        Backend& B = b->b;
        const int m = B.m;
        GB_DISPATCH_V(B, kb_dual_step<V><<<elem_grid(m, B.sms), kThreads, 0, B.stream>>>(
                             m, y->v.p<V>(), axbar->v.p<V>(), B.lo.p<V>(), B.hi.p<V>(), static_cast<V>(sigma),
                             yn->v.p<V>(), sumy->v.p<V>()));
    });
}

int gb_sub(gb_backend* b, const gb_vec* a, const gb_vec* c, gb_vec* d) {
    return guarded_b([&] {
        GB_REQUIRE(b && a && c && d, "bad arguments");
        Backend& B = b->b;
        const int k = a->v.k;
        if (k) GB_DISPATCH_V(B, kb_sub<V><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, a->v.p<V>(), c->v.p<V>(), d->v.p<V>()));
    });
}

int gb_scale_into(gb_backend* b, const gb_vec* src, double a, gb_vec* dst) {
    return guarded_b([&] {
        GB_REQUIRE(b && src && dst, "bad arguments");
        Backend& B = b->b;
        const int k = src->v.k;
        if (k) GB_DISPATCH_V(B, kb_scale<V><<<elem_grid(k, B.sms), kThreads, 0, B.stream>>>(k, a, src->v.p<V>(), dst->v.p<V>()));
    });
}

int gb_primal_res2(gb_backend* b, const gb_vec* ax, double* out) {
    return guarded_b([&] {
        GB_REQUIRE(b && ax && out, "bad arguments");
        Backend& B = b->b;
        GB_DISPATCH_V(B, *out = reduce2(B, B.m, FPrimalRes<V>{ax->v.p<V>(), B.lo.p<V>(), B.hi.p<V>(), B.rres.p<V>()}).first);
    });
}

int gb_dual_res(gb_backend* b, const gb_vec* aty, const gb_vec* qx, int with_c, double* rd2, double* vobj) {
    return guarded_b([&] {
        GB_REQUIRE(b && aty && rd2 && vobj, "bad arguments");
        Backend& B = b->b;
        std::pair<double, double> r;
        GB_DISPATCH_V(B, r = reduce2(B, B.n, FDualRes<V>{aty->v.p<V>(), qx ? qx->v.p<V>() : nullptr, B.c.p<V>(),
                                                         B.l.p<V>(), B.u.p<V>(), B.cres.p<V>(), with_c ? 1.0 : 0.0}));
        *rd2 = r.first;
        *vobj = r.second;
    });
}

int gb_row_dual_obj(gb_backend* b, const gb_vec* y, double* out) {
    return guarded_b([&] {
        GB_REQUIRE(b && y && out, "bad arguments");
        Backend& B = b->b;
        GB_DISPATCH_V(B, *out = reduce2(B, B.m, FRowDualObj<V>{y->v.p<V>(), B.lo.p<V>(), B.hi.p<V>()}).first);
    });
}

int gb_dot(gb_backend* b, const gb_vec* a, const gb_vec* c, double* out) {
    return guarded_b([&] {
        GB_REQUIRE(b && a && c && out, "bad arguments");
        Backend& B = b->b;
        GB_DISPATCH_V(B, *out = reduce2(B, a->v.k, FDot<V>{a->v.p<V>(), c->v.p<V>()}).first);
    });
}

int gb_dot_c(gb_backend* b, const gb_vec* x, double* out) {
    return guarded_b([&] {
        GB_REQUIRE(b && x && out, "bad arguments");
        Backend& B = b->b;
        GB_DISPATCH_V(B, *out = reduce2(B, B.n, FDot<V>{B.c.p<V>(), x->v.p<V>()}).first);
    });
}

int gb_diff2(gb_backend* b, const gb_vec* a, const gb_vec* c, double* out) {
    return guarded_b([&] {
        GB_REQUIRE(b && a && c && out, "bad arguments");
        Backend& B = b->b;
        GB_DISPATCH_V(B, *out = reduce2(B, a->v.k, FDiff2<V>{a->v.p<V>(), c->v.p<V>()}).first);
    });
}

}  // extern "C"

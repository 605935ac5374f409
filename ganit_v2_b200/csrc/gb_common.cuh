// Common pieces of the B200 PDHG engine: error plumbing, device buffers,
// deterministic block reductions.  Built with -fmad=false so that every
// vector update rounds exactly like the reference's scalar C++ code
// (src/backend_cpu.cpp), i.e. no silent FMA contraction.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace gb {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define GB_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e__ = (call);                                                                       \
        if (e__ != cudaSuccess)                                                                         \
            throw ::gb::Error(e__ == cudaErrorMemoryAllocation ? -3 : -2,                               \
                              std::string("CUDA error ") + cudaGetErrorString(e__) + " at " __FILE__ ":" + \
                                  std::to_string(__LINE__));                                            \
    } while (0)

#define GB_REQUIRE(cond, msg)                                        \
    do {                                                             \
        if (!(cond)) throw ::gb::Error(-1, std::string(msg));        \
    } while (0)

// Stage timer of the set-up and solve paths, on when GANIT_B200_TRACE=1:
// mark() waits for the stream and prints the host time since the previous
// mark to stderr (so a stage's time includes its device work).  Off, it does
// nothing, and no synchronisation is added.
bool trace_enabled();
struct StageTrace {
    cudaStream_t s;
    const char* what;
    bool on = trace_enabled();
    double t = now_ms();
    static double now_ms();
    void mark(const char* stage) {
        if (!on) return;
        if (s) cudaStreamSynchronize(s);
        const double u = now_ms();
        std::fprintf(stderr, "[gb trace] %s %-22s %8.3f ms\n", what, stage, u - t);
        t = u;
    }
};

// Device memory of the library (gb_pool.cu): cudaMalloc / cudaFree behind a
// per-process cache of freed blocks (same device, same rounded size), so
// that creating and destroying problems of the same shape -- the one-shot
// gb_solve path -- does not pay the driver's allocation cost each time.
void* dev_alloc(size_t bytes);
void dev_free(void* p);
// Pinned host memory behind the same kind of cache (a cudaMallocHost /
// cudaFreeHost pair of a problem's small state arrays measured 1.5-4 ms on
// the B200 host, as long as the set-up kernels).
void* host_alloc(size_t bytes);
void host_free(void* p);
// A freed block is cached only once no kernel or copy can still use it:
// dev_free / host_free synchronise the device first, unless a free batch is
// open on this thread -- a teardown that synchronised once and then frees
// many buffers (FreeBatch, destroyed last).
void begin_free_batch();
void end_free_batch();
struct FreeBatchEnd {
    bool open = false;
    ~FreeBatchEnd() {
        if (open) end_free_batch();
    }
};

// Owning device buffer (move-only).
template <class T>
class DevBuf {
   public:
    DevBuf() = default;
    explicit DevBuf(size_t n) { reset(n); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    void reset(size_t n) {
        release();
        n_ = n;
        if (n_) p_ = static_cast<T*>(dev_alloc(n_ * sizeof(T)));
    }
    void release() {
        if (p_) dev_free(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    void upload(const T* h, size_t n, cudaStream_t s) {
        if (n) GB_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T* h, size_t n, cudaStream_t s) const {
        if (n) GB_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    }

   private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// Programmatic dependent launch (sm_90+).  A kernel of the iteration loop
// first lets its successor launch (launch_dependents: the successor's CTAs may
// be scheduled once every CTA of this grid has started, filling SMs this
// grid's last wave leaves idle), then waits (wait: blocks until the
// predecessor grid has completed and its memory is visible) before touching
// any memory.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch with the programmatic-stream-serialization attribute (the kernel
// calls pdl_enter()).
template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GB_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

constexpr int kThreads = 256;  // CTA size of every streaming kernel
constexpr int kWarps = kThreads / 32;

inline int div_up(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }
__host__ __device__ __forceinline__ int div_up_dev(int a, int b) { return (a + b - 1) / b; }

// grid for an elementwise kernel: at most 8 CTAs per SM worth of work per
// launch, grid-stride beyond that (148 SMs on B200).
inline int elem_grid(long long n, int sms) {
    long long g = (n + kThreads - 1) / kThreads;
    long long cap = static_cast<long long>(sms) * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of K doubles held by every thread.  Result valid in
// thread 0.  `sh` must hold kWarps*K doubles.  Order: shuffle tree inside each
// warp, then warps 0..7 sequentially.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double t = warp_sum(v[k]);
        if (lane == 0) sh[wid * K + k] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = 0.0;
            for (int w = 0; w < kWarps; ++w) t += sh[w * K + k];
            v[k] = t;
        }
    }
    __syncthreads();
}

}  // namespace gb

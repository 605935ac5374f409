// gb_eval_kkt_noalloc: FP64 KKT evaluation that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree at the point
// where they want a solution checked -- e.g. a branch-and-bound worker or a
// solver service that hands the library a fixed device-memory budget up
// front, or code on a latency-critical path where cudaMalloc/cudaFree would
// synchronise the whole device and stall other streams.  They keep their
// scaled problem and candidate point in their own device buffers; this entry
// point evaluates the point with the same kernel (k_eval, certify mode) that
// the solver uses for its FP64 certification, and its scratch memory lives
// in a file-scope __device__ array instead of being allocated.
//
// The array (kNoAllocScratchBytes = 4 MiB) exists on every GPU that loads the
// library until the process exits.  All calls share it: two calls whose work
// overlaps on the GPU (different streams, different threads without ordering)
// race on it, and each call keeps the previous call's contents, so whatever
// must start at zero (chunk counters, the arrival counter) is cleared here.
#include <cstring>
#include <mutex>

#include "../../include/ganit_b200.h"
#include "gb_pdhg.cuh"

namespace gb {
extern thread_local std::string g_last_error;

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;
constexpr int kNoAllocMaxDevices = 64;

// Scratch layout (byte offsets, 256-aligned)
constexpr size_t kOffState = 0;
constexpr size_t kOffBlocks = 512;
constexpr size_t kOffPartials = kOffBlocks + sizeof(RowBlock) * GB_NOALLOC_MAX_BLOCKS;
constexpr size_t kOffSlots = kOffPartials + sizeof(double) * kTerms * GB_NOALLOC_MAX_BLOCKS;
constexpr size_t kOffCounters = kOffSlots + sizeof(double) * GB_NOALLOC_MAX_SLOTS;
constexpr size_t kOffSeg = kOffCounters + sizeof(unsigned) * GB_NOALLOC_MAX_LONG_ROWS;  // 2 x int[2]
constexpr size_t kOffTerms = kOffSeg + 64;  // k_decide's per-instance sums (one instance)
constexpr size_t kOffEnd = kOffTerms + sizeof(double) * kTerms;
static_assert(kOffTerms % alignof(double) == 0, "term slot misaligned");
static_assert(sizeof(SolveState) <= kOffBlocks, "state slot too small");
static_assert(kOffEnd <= kNoAllocScratchBytes, "scratch layout exceeds the array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host-side address of g_noalloc_scratch per device, looked up once per device
// (the array's host-side name is not a device address).
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kNoAllocMaxDevices] = {};
// Host staging of the schedule: fixed static storage, no allocation.
static RowBlock g_noalloc_blocks[GB_NOALLOC_MAX_BLOCKS];

static unsigned char* scratch_for_current_device() {
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    GB_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, "device index beyond the no-alloc table");
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw Error(GB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                                         cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_addr[dev]);
}

}  // namespace gb

using namespace gb;

extern "C" int gb_eval_kkt_noalloc(const gb_scaled_lp* dev, const int32_t* h_a_ptr, const int32_t* h_at_ptr,
                                   const double* x, const double* y, const gb_kkt_scalars* sc, void* stream,
                                   gb_kkt* out) {
    try {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        GB_REQUIRE(dev && h_a_ptr && h_at_ptr && x && y && sc && out, "NULL argument");
        GB_REQUIRE(dev->m > 0 && dev->n > 0, "need m > 0 and n > 0");
        GB_REQUIRE(dev->q_ptr == nullptr, "gb_eval_kkt_noalloc evaluates LPs only (q_ptr must be NULL)");
        GB_REQUIRE(h_a_ptr[0] == 0 && h_at_ptr[0] == 0 && h_a_ptr[dev->m] == h_at_ptr[dev->n],
                   "row pointers of A and AT disagree");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // schedules of A and AT into the fixed host staging array
        int nb = 0, nslots = 0, ncounters = 0;
        bool overflow = false;
        auto emit = [&](const RowBlock& b) {
            if (nb >= GB_NOALLOC_MAX_BLOCKS) { overflow = true; return; }
            g_noalloc_blocks[nb++] = b;
        };
        schedule_rows(h_a_ptr, 0, dev->m, kBlockNnz, kThreads, &nslots, &ncounters, 0, emit);
        const int nbA = nb;
        const int slotsA = nslots, countersA = ncounters;
        int nslotsT = 0, ncountersT = 0;
        schedule_rows(h_at_ptr, 0, dev->n, kBlockNnz, kThreads, &nslotsT, &ncountersT, 0, emit);
        if (overflow || nslots + nslotsT > GB_NOALLOC_MAX_SLOTS || ncounters + ncountersT > GB_NOALLOC_MAX_LONG_ROWS)
            throw Error(GB_ERR_INVALID,
                        "problem too large for gb_eval_kkt_noalloc: needs " + std::to_string(nb) + "+ row blocks, " +
                            std::to_string(nslots + nslotsT) + " chunk slots and " +
                            std::to_string(ncounters + ncountersT) + " long rows (limits " +
                            std::to_string(GB_NOALLOC_MAX_BLOCKS) + ", " + std::to_string(GB_NOALLOC_MAX_SLOTS) +
                            ", " + std::to_string(GB_NOALLOC_MAX_LONG_ROWS) + ")");
        unsigned char* base = scratch_for_current_device();
        SolveState* st = reinterpret_cast<SolveState*>(base + kOffState);
        RowBlock* blocks = reinterpret_cast<RowBlock*>(base + kOffBlocks);
        double* partials = reinterpret_cast<double*>(base + kOffPartials);
        double* slots = reinterpret_cast<double*>(base + kOffSlots);
        unsigned* counters = reinterpret_cast<unsigned*>(base + kOffCounters);
        int* seg = reinterpret_cast<int*>(base + kOffSeg);  // A blocks [0, nbA), A^T blocks [0, nb - nbA)
        const int hseg[4] = {0, nbA, 0, nb - nbA};
        static_assert(sizeof(hseg) <= 32, "segment slot");
        GB_CUDA(cudaMemcpyAsync(blocks, g_noalloc_blocks, sizeof(RowBlock) * nb, cudaMemcpyHostToDevice, s));
        GB_CUDA(cudaMemsetAsync(counters, 0, sizeof(unsigned) * GB_NOALLOC_MAX_LONG_ROWS, s));
        GB_CUDA(cudaMemcpyAsync(seg, hseg, sizeof(hseg), cudaMemcpyHostToDevice, s));
        SolveState h;
        std::memset(&h, 0, sizeof(h));
        h.obj_scale = sc->obj_scale;
        h.obj_const = sc->obj_const;
        h.bnorm = sc->bnorm;
        h.cnorm = sc->cnorm;
        GB_CUDA(cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, s));

        EvalArgs<double, double> a;
        std::memset(&a, 0, sizeof(a));
        a.A.ptr = dev->a_ptr; a.A.idx = dev->a_idx; a.A.val = dev->a_val;
        a.A.blocks = blocks; a.A.slots = slots; a.A.counters = counters; a.A.rows = dev->m; a.A.nb = nbA;
        a.AT.ptr = dev->at_ptr; a.AT.idx = dev->at_idx; a.AT.val = dev->at_val;
        a.AT.blocks = blocks + nbA; a.AT.slots = slots + slotsA; a.AT.counters = counters + countersA;
        a.AT.rows = dev->n; a.AT.nb = nb - nbA;
        a.x = x; a.y = y;
        a.c = dev->c; a.l = dev->l; a.u = dev->u; a.lo = dev->lo; a.hi = dev->hi; a.rres = dev->rres; a.cres = dev->cres;
        a.mode = kEvalCertify;
        a.count = 1;
        a.seg_a = seg;
        a.seg_t = seg + 2;
        a.st = st;
        a.partials = partials;
        a.inst_terms = reinterpret_cast<double*>(base + kOffTerms);
        a.use_cond = 0;
        k_eval<double, double, 1, 1><<<nb, kThreads, spmv_smem_bytes<1, double>(), s>>>(a);
        k_decide<double, double><<<1, kThreads, 0, s>>>(a);
        GB_CUDA(cudaGetLastError());
        Kkt k;
        GB_CUDA(cudaMemcpyAsync(&k, &st->kcert, sizeof(Kkt), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        out->pobj = k.pobj;
        out->dobj = k.dobj;
        out->rel_p = k.rel_p;
        out->rel_d = k.rel_d;
        out->rel_gap = k.rel_gap;
        out->err = k.err;
        return GB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GB_ERR_INVALID;
    }
}

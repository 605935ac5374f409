// CSR SpMV with a fused per-row epilogue, scheduled by row blocks.
//
// Method: CSR-Adaptive (Greathouse & Daga, SC'14).  At upload time the rows
// of a matrix are cut, from its row-length histogram, into blocks:
//   * STREAM  consecutive rows whose nonzeros total <= kBlockNnz and whose
//             count <= kThreads.  The CTA streams the block's contiguous
//             idx/val range with coalesced loads, stages the products
//             val*x[idx] in shared memory, then reduces each row with a group
//             of G lanes (G = power of two chosen from the rows per block).
//             A block closes before the G it would get leaves a lane of its
//             longest row more than kMaxLaneSum products to add: one long
//             row among many short ones (the capacity rows of a blending LP)
//             otherwise keeps its warp -- and the CTA -- adding hundreds of
//             products in sequence after every other row is done.
//   * LONG    one row with more than min(kBlockNnz, 32 kMaxLaneSum)
//             nonzeros, reduced by the whole CTA (<= kLongSingle nonzeros) or
//   * CHUNK   a slice of a very long row: each CTA writes its partial sum to a
//             fixed slot and the last CTA to arrive adds the slots in chunk
//             order and runs the epilogue (no spin-waits, deterministic).
// Every row is reduced in a fixed order, so results are bit-reproducible run
// to run.  The epilogue functor receives (row, sums) once per row, which is
// what lets the PDHG steps fuse into the product kernels.
//
// Launch: one CTA per block, 256 threads, kept lean (<= 32-40 registers) so
// that 6-8 CTAs are resident per SM: the kernels are latency-bound (dependent
// idx -> x[idx] loads, a barrier between the product and reduction phases),
// and measured on B200 this beats a persistent one-wave grid with TMA bulk
// double-buffering, whose larger shared-memory and register footprint halves
// the resident warps.  Each row's epilogue operands are loaded before the
// block's products are formed, so their latency overlaps the stream.
#pragma once
#include <algorithm>

#include "gb_common.cuh"

namespace gb {

constexpr int kBlockNnz = 2048;     // nonzeros per STREAM block
constexpr int kLongSingle = 4096;   // longest row one CTA reduces alone
constexpr int kChunkNnz = 2048;     // slice of a longer row per CTA
constexpr int kMaxLaneSum = 32;     // STREAM: most products one lane of a row's group adds (16..64 measured)

enum BlockKind : int { kStream = 0, kLong = 1, kChunk = 2 };

struct alignas(16) RowBlock {
    int r0, r1;         // rows [r0, r1)
    int p0, p1;         // nonzeros [p0, p1)
    int kind, lg;       // BlockKind, log2 of the group size (STREAM)
    int chunk, nchunks; // CHUNK: index and count
    int slot_base;      // CHUNK: first slot of the row
    int counter;        // CHUNK: arrival counter of the row
    int inst;           // instance (batch member) the rows belong to
    int pad1;
};

// Host: row-length-driven schedule.  `block_nnz` / `max_rows` are the
// tunables (the batch autotuner varies them).  Blocks never straddle two
// instances of a batch; seg_block[k] .. seg_block[k+1] are instance k's blocks.
struct Schedule {
    std::vector<RowBlock> blocks;
    std::vector<int> seg_block;
    int nslots = 0, ncounters = 0;
    int max_lg = 0;
    // Row-start bitmaps of the STREAM blocks (the iteration kernels' segmented
    // reduction, spmv_run_seg): block b's words start at b.slot_base; bit t of
    // its window (t = element - 4 floor(p0 / 4)) is set where a non-empty row
    // begins.
    std::vector<unsigned> bits;
};

// Appends the row-start bitmap of a STREAM block to s.bits and records its
// offset in b.slot_base (a field CHUNK blocks use for their slots).
// Row starts increase along the block, so each word is gathered in a
// register and stored once.
inline void add_stream_bits(Schedule& s, const int* ptr, RowBlock& b) {
    const int a = b.p0 & 3, nq = ((b.p1 + 3) >> 2) - (b.p0 >> 2);
    const size_t off = s.bits.size();
    s.bits.resize(off + (4 * static_cast<size_t>(nq) + 31) / 32, 0u);
    unsigned* w = s.bits.data() + off;
    const int base = a - b.p0;
    int cur = -1;
    unsigned acc = 0u;
    for (int i = b.r0; i < b.r1; ++i) {
        const int p = ptr[i];
        if (ptr[i + 1] > p) {
            const int t = p + base, k = t >> 5;
            if (k != cur) {
                if (cur >= 0) w[cur] |= acc;
                cur = k;
                acc = 0u;
            }
            acc |= 1u << (t & 31);
        }
    }
    if (cur >= 0) w[cur] |= acc;
    b.slot_base = static_cast<int>(off);
}

inline int floor_log2(int v) {
    int l = 0;
    while ((2 << l) <= v) ++l;
    return l;
}

// Lanes per row of a STREAM block of `nr` rows: the largest power of two
// <= min(32, kThreads / nr) (a table: the packing loop asks once per row).
struct LaneGroups {
    int g[kThreads + 1];
    constexpr LaneGroups() : g{} {
        for (int nr = 1; nr <= kThreads; ++nr) {
            int v = kThreads / nr < 32 ? kThreads / nr : 32, p = 1;
            while (p * 2 <= v) p *= 2;
            g[nr] = p;
        }
    }
};
constexpr LaneGroups kLaneGroups{};

// Walks rows [r_begin, r_end) once and hands every block to `emit`; slot and
// counter ids are numbered from *nslots / *ncounters on; blocks get `inst`.
template <class Emit>
inline void schedule_rows(const int* ptr, int r_begin, int r_end, int block_nnz, int max_rows, int* nslots,
                          int* ncounters, int inst, Emit&& emit) {
    int i = r_begin;
    while (i < r_end) {
        const int len = ptr[i + 1] - ptr[i];
        if (len > block_nnz || len > 32 * kMaxLaneSum) {
            if (len <= kLongSingle) {
                RowBlock b{};
                b.r0 = i; b.r1 = i + 1; b.p0 = ptr[i]; b.p1 = ptr[i + 1]; b.kind = kLong; b.inst = inst;
                emit(b);
            } else {
                const int nch = div_up(len, kChunkNnz);
                for (int c = 0; c < nch; ++c) {
                    RowBlock b{};
                    b.r0 = i; b.r1 = i + 1;
                    b.p0 = ptr[i] + c * kChunkNnz;
                    b.p1 = std::min(ptr[i + 1], b.p0 + kChunkNnz);
                    b.kind = kChunk; b.chunk = c; b.nchunks = nch;
                    b.slot_base = *nslots; b.counter = *ncounters; b.inst = inst;
                    emit(b);
                }
                *nslots += nch;
                *ncounters += 1;
            }
            ++i;
            continue;
        }
        const int r0 = i, start = ptr[i];
        int maxlen = 0;
        while (i < r_end && (i - r0) < max_rows && ptr[i + 1] - start <= block_nnz) {
            const int l = ptr[i + 1] - ptr[i];
            // ceil(maxlen / g) > kMaxLaneSum  <=>  maxlen > kMaxLaneSum * g
            if (i > r0 && std::max(maxlen, l) > kMaxLaneSum * kLaneGroups.g[i - r0 + 1]) break;
            maxlen = std::max(maxlen, l);
            ++i;
        }
        RowBlock b{};
        b.r0 = r0; b.r1 = i; b.p0 = start; b.p1 = ptr[i]; b.kind = kStream; b.inst = inst;
        const int nrows = i - r0;
        int g = kThreads / nrows;  // lanes available per row
        if (g > 32) g = 32;
        b.lg = floor_log2(g < 1 ? 1 : g);
        emit(b);
    }
}

// Schedule of a matrix whose rows are cut into `nseg` instances at
// seg_off[0..nseg] (nseg = 1: one instance, rows [0, rows)).
inline Schedule build_schedule(const int* ptr, int rows, const int* seg_off = nullptr, int nseg = 1,
                               int block_nnz = kBlockNnz, int max_rows = kThreads) {
    Schedule s;
    s.seg_block.assign(nseg + 1, 0);
    s.bits.reserve(static_cast<size_t>(ptr[seg_off ? seg_off[nseg] : rows]) / 8 + 64);  // ~4 words per 128 nonzeros
    for (int k = 0; k < nseg; ++k) {
        s.seg_block[k] = static_cast<int>(s.blocks.size());
        const int r0 = seg_off ? seg_off[k] : 0, r1 = seg_off ? seg_off[k + 1] : rows;
        schedule_rows(ptr, r0, r1, block_nnz, max_rows, &s.nslots, &s.ncounters, k, [&](const RowBlock& b) {
            s.blocks.push_back(b);
            if (b.kind == kStream) add_stream_bits(s, ptr, s.blocks.back());
            s.max_lg = std::max(s.max_lg, b.lg);
        });
    }
    s.seg_block[nseg] = static_cast<int>(s.blocks.size());
    return s;
}

// Same with per-instance tunables (block_nnz <= kBlockNnz, max_rows <= kThreads).
inline Schedule build_schedule(const int* ptr, const int* seg_off, int nseg, const int* block_nnz,
                               const int* max_rows) {
    Schedule s;
    s.seg_block.assign(nseg + 1, 0);
    s.bits.reserve(static_cast<size_t>(ptr[seg_off[nseg]]) / 8 + 64);
    for (int k = 0; k < nseg; ++k) {
        s.seg_block[k] = static_cast<int>(s.blocks.size());
        schedule_rows(ptr, seg_off[k], seg_off[k + 1], block_nnz[k], max_rows[k], &s.nslots, &s.ncounters, k,
                      [&](const RowBlock& b) {
                          s.blocks.push_back(b);
                          if (b.kind == kStream) add_stream_bits(s, ptr, s.blocks.back());
                          s.max_lg = std::max(s.max_lg, b.lg);
                      });
    }
    s.seg_block[nseg] = static_cast<int>(s.blocks.size());
    return s;
}

// Device-resident schedule of one matrix.
struct DevSchedule {
    DevBuf<RowBlock> blocks;
    DevBuf<int> seg_block;  // per-instance block ranges
    DevBuf<double> slots;
    DevBuf<unsigned> counters;
    DevBuf<unsigned> bits;  // Schedule::bits
    int nb = 0;
    int nslots = 0;
    std::vector<int> host_seg_block;
    std::vector<RowBlock> host_blocks;  // for the block lists of partial phases
    void upload(const Schedule& s, int nv_max, cudaStream_t st) {
        nb = static_cast<int>(s.blocks.size());
        host_blocks = s.blocks;
        blocks.reset(nb ? nb : 1);
        blocks.upload(s.blocks.data(), nb, st);
        host_seg_block = s.seg_block;
        seg_block.reset(host_seg_block.size());
        seg_block.upload(host_seg_block.data(), host_seg_block.size(), st);
        nslots = s.nslots;
        slots.reset(static_cast<size_t>(s.nslots ? s.nslots : 1) * nv_max);
        counters.reset(s.ncounters ? s.ncounters : 1);
        GB_CUDA(cudaMemsetAsync(counters.get(), 0, counters.size() * sizeof(unsigned), st));
        bits.reset(s.bits.empty() ? 1 : s.bits.size());
        bits.upload(s.bits.data(), s.bits.size(), st);
    }
};

// Raw view of a CSR matrix on the device.
template <class M>
struct CsrView {
    const int* __restrict__ ptr;
    const int* __restrict__ idx;
    const M* __restrict__ val;
    const RowBlock* __restrict__ blocks;
    double* slots;
    unsigned* counters;
    const unsigned* __restrict__ bits;  // row-start bitmaps of the STREAM blocks (Schedule::bits), or nullptr
    int rows;
    int nb;
    // 1: idx / val are 16-byte aligned and readable 3 elements past the last
    // nonzero (allocated with padded_nnz), so STREAM blocks use 16-byte loads.
    // Views of caller-owned arrays leave it 0 (scalar loads).
    int vec = 0;
    // Load mode of the iteration kernels (LoadMode; a template choice, not a
    // branch: a branch in the loop costs the 32-register kernels spills).
    // kLoadStream: the 16-byte idx / val loads skip L1 allocation
    // (ld.global.nc with L1::no_allocate), for iterations whose data at this
    // precision does not fit in L2 and so streams from HBM.  Measured on
    // B200: -15% per iteration on the 512-LP batch (207 MB per FP32
    // iteration), neutral to +8% per kernel on the blending LP at FP64
    // (104 MB), +20% on it at FP32 (64 MB, L2-resident).  kLoadPrefetch: the
    // same loads after bulk L2 prefetches (spmv_run_prefetched).
    int nc = 0;
};

enum LoadMode : int { kLoadPlain = 0, kLoadStream = 1, kLoadPrefetch = 2 };

// Element count of idx / val arrays allocated for 16-byte loads (CsrView::vec).
inline long long padded_nnz(long long nnz) { return ((nnz + 3) & ~3LL) + 4; }

// Four consecutive matrix values from a 16-byte-aligned address.
__device__ __forceinline__ void load4(const float* p, float (&o)[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void load4(const __nv_bfloat16* p, __nv_bfloat16 (&o)[4]) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));  // 8 bytes; 4q elements are 8-byte aligned
    const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&v.x);
    const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&v.y);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void load4(const double* p, double (&o)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// The same 16-byte loads without L1 allocation (CsrView::nc).
__device__ __forceinline__ int4 ld_stream(const int4* p) {
    int4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}
__device__ __forceinline__ void load4_stream(const float* p, float (&o)[4]) {
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3])
                 : "l"(p));
}
__device__ __forceinline__ void load4_stream(const double* p, double (&o)[4]) {
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(o[0]), "=d"(o[1]) : "l"(p));
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(o[2]), "=d"(o[3]) : "l"(p + 2));
}
__device__ __forceinline__ void load4_stream(const __nv_bfloat16* p, __nv_bfloat16 (&o)[4]) { load4(p, o); }

// Bulk prefetch of [p, p + bytes) into L2 (cp.async.bulk.prefetch.L2,
// sm_90+): one instruction, no shared memory, no registers held and nothing
// to wait for -- a hint that starts the DRAM reads early.  The range is cut
// to the whole 16-byte units inside it (the instruction wants a 16-byte
// aligned start and a size in 16-byte units), so no byte outside
// [p, p + bytes) is touched.
__device__ __forceinline__ void l2_prefetch(const void* p, size_t bytes) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    const unsigned long long s = (a + 15ull) & ~15ull, e = (a + bytes) & ~15ull;
    if (e > s)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(s), "r"(static_cast<unsigned>(e - s))
                     : "memory");
}

// Gather of a single right-hand side.
template <class V>
struct GatherOne {
    const V* __restrict__ v;
    __device__ __forceinline__ void operator()(int j, V (&o)[1]) const { o[0] = __ldg(v + j); }
};

// Epilogue prefetch payload for epilogues that need nothing early.
struct NoPre {};

// Products are staged with one padding word per 32 entries so that rows of
// a constant even length (8, 16, ...) reduced by one lane each do not all hit
// the same shared-memory banks.
__host__ __device__ constexpr int padded(int k) { return k + (k >> 5); }
constexpr int kProdStride = padded(kBlockNnz);

// Dynamic shared memory of spmv_run for NV vectors of type V.
template <int NV, class V>
constexpr size_t spmv_smem_bytes() {
    return sizeof(V) * NV * kProdStride + sizeof(double) * kWarps * NV + 64;
}


// LONG / CHUNK block: whole CTA strides over the slice, block reduction,
// epilogue by thread 0 (CHUNK: the last CTA to arrive).  `red` holds
// kWarps * NV values of V.
template <int NV, class M, class V, class Gather, class Epi>
__device__ __forceinline__ void long_block(const CsrView<M>& A, const RowBlock& b, const Gather& g, Epi& epi,
                                           V* red) {
    const int tid = threadIdx.x;
    V acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = V(0);
    for (int p = b.p0 + tid; p < b.p1; p += kThreads) {
        const int j = __ldg(A.idx + p);
        const V a = static_cast<V>(__ldg(A.val + p));
        V xv[NV];
        g(j, xv);
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] += a * xv[v];
    }
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        V t = warp_sum(acc[v]);
        if (lane == 0) red[wid * NV + v] = t;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            V t = V(0);
            for (int w = 0; w < kWarps; ++w) t += red[w * NV + v];
            acc[v] = t;
        }
        if (b.kind == kLong) {
            const auto pre = epi.prefetch(b.r0);
            epi(b.r0, acc, pre);
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) A.slots[static_cast<size_t>(b.slot_base + b.chunk) * NV + v] = double(acc[v]);
            __threadfence();
            const unsigned prev = atomicAdd(A.counters + b.counter, 1u);
            if (prev == static_cast<unsigned>(b.nchunks - 1)) {
                __threadfence();
                V tot[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) tot[v] = V(0);
                for (int c = 0; c < b.nchunks; ++c) {
#pragma unroll
                    for (int v = 0; v < NV; ++v)
                        tot[v] += static_cast<V>(__ldcg(A.slots + static_cast<size_t>(b.slot_base + c) * NV + v));
                }
                A.counters[b.counter] = 0u;  // re-armed for the next launch (stream order)
                const auto pre = epi.prefetch(b.r0);
                epi(b.r0, tot, pre);
            }
        }
    }
    __syncthreads();
}

// Reduce the staged products of a STREAM block row by row and run the
// epilogue (rows are handled in one pass: nrows <= kThreads >> lg).
template <int NV, class V, class Epi, class Pre>
__device__ __forceinline__ void reduce_rows(const RowBlock& b, const V* prod, int s, int e, bool act, const Pre& pre,
                                            Epi& epi) {
    const int lg = b.lg, G = 1 << lg;
    const int lane_g = threadIdx.x & (G - 1);
    V acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = V(0);
    for (int k = s + lane_g; k < e; k += G) {
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] += prod[v * kProdStride + padded(k)];
    }
    for (int o = G >> 1; o > 0; o >>= 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o, G);
    }
    if (act && lane_g == 0) epi(b.r0 + (threadIdx.x >> lg), acc, pre);
}

// CTA `cta` runs block `cta`.  Gather g(col, V(&)[NV]) supplies the NV vector
// values of a column; epi.begin(inst) returns false to skip a block of an
// instance that is not iterating (and loads per-instance scalars);
// epi.prefetch(row) loads a row's epilogue operands (issued before the
// block's products) and epi(row, const V(&)[NV], pre) consumes a finished row.
template <int NV, class M, class V, bool NC = false, class Gather, class Epi>
__device__ __forceinline__ void spmv_run(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                         unsigned char* smem) {
    V* prod = reinterpret_cast<V*>(smem);
    V* red = reinterpret_cast<V*>(smem + sizeof(V) * NV * kProdStride);
    const RowBlock b = A.blocks[cta];
    if (!epi.begin(b.inst)) return;  // instance not iterating (uniform over the CTA)
    if (b.kind != kStream) {
        long_block<NV, M, V>(A, b, g, epi, red);
        return;
    }
    const int tid = threadIdx.x, grp = tid >> b.lg;
    const bool act = grp < b.r1 - b.r0;
    int s = 0, e = 0;
    decltype(epi.prefetch(0)) pre{};
    if (act) {
        const int r = b.r0 + grp;
        s = __ldg(A.ptr + r) - b.p0;
        e = __ldg(A.ptr + r + 1) - b.p0;
        if ((tid & ((1 << b.lg) - 1)) == 0) pre = epi.prefetch(r);
    }
    const int cnt = b.p1 - b.p0;
    if (A.vec) {
        // 16-byte loads over the 4-aligned window around [p0, p1); lanes of a
        // group outside the block neither gather nor store.  (Loading two
        // groups ahead of their gathers needs more registers than the 6-8
        // resident CTAs per SM leave once the epilogue operands are in flight.)
        const int q0 = b.p0 >> 2, q1 = (b.p1 + 3) >> 2;
#pragma unroll 1
        for (int q = q0 + tid; q < q1; q += kThreads) {
            int4 j4;
            M a4[4];
            if constexpr (NC) {
                j4 = ld_stream(reinterpret_cast<const int4*>(A.idx) + q);
                load4_stream(A.val + 4 * q, a4);
            } else {
                j4 = __ldg(reinterpret_cast<const int4*>(A.idx) + q);
                load4(A.val + 4 * q, a4);
            }
            const int js[4] = {j4.x, j4.y, j4.z, j4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = 4 * q + e - b.p0;
                if (k >= 0 && k < cnt) {
                    V xv[NV];
                    g(js[e], xv);
#pragma unroll
                    for (int v = 0; v < NV; ++v) prod[v * kProdStride + padded(k)] = static_cast<V>(a4[e]) * xv[v];
                }
            }
        }
    } else {
#pragma unroll 4
        for (int k = tid; k < cnt; k += kThreads) {
            const int p = b.p0 + k;
            const V a = static_cast<V>(__ldg(A.val + p));
            V xv[NV];
            g(__ldg(A.idx + p), xv);
#pragma unroll
            for (int v = 0; v < NV; ++v) prod[v * kProdStride + padded(k)] = a * xv[v];
        }
    }
    __syncthreads();
    reduce_rows<NV, V>(b, prod, s, e, act, pre, epi);
}

// ---------------------------------------------------------------- warp-segmented STREAM blocks
// The FP64 iteration kernels' STREAM blocks (one right-hand side) reduce their
// rows in registers instead of staging every product in shared memory (see
// spmv_run_iter for the measured choice).  Measured on B200 (ncu, 512-LP
// batch), the staged form spends ~1/3 of the L1TEX data-pipe wavefronts -- the
// unit that bounds these kernels -- on the product stores and on row
// reductions whose rows start at random banks.  Here:
//   * a bitmap over the block's 4-aligned window (positions 0 .. 4 nq - 1),
//     built with the schedule (Schedule::bits), marks each non-empty row's
//     first element;
//   * warp w takes chunks c = w, w + 8, ... of 32 quads (128 positions); each
//     lane forms its quad's products and a segmented prefix within the quad,
//     and the warp a segmented inclusive scan of the lanes' open parts (the
//     head of a lane is its last row start, found with a ballot), so every
//     element knows the sum of its row from the row's start, or from the
//     chunk's start if the row began earlier, up to itself;
//   * an element that ends its row's part of the chunk (the next element
//     starts a row, the row ends, or the chunk ends) stores that sum at its
//     own position;
//   * thread i then adds, for row i, the parts stored at the ends of its
//     pieces in each chunk it reaches, in chunk order, and runs the epilogue.
// Every sum is taken in a fixed order (within a quad, the scan's fixed tree,
// then chunk order), so results are reproducible run to run; the order
// differs from spmv_run's, so the bits do too.
constexpr int kWinQuads = kBlockNnz / 4 + 1;          // quads of a STREAM block's 4-aligned window
constexpr int kSegPos = 4 * kWinQuads;                // window positions
// Dynamic shared memory of the iteration kernels with segmented STREAM blocks
// (the row parts at their window positions; LONG / CHUNK blocks keep
// spmv_run's layout, which is larger).
template <class V>
constexpr size_t spmv_seg_smem_bytes() {
    return sizeof(V) * kSegPos > spmv_smem_bytes<1, V>() ? sizeof(V) * kSegPos : spmv_smem_bytes<1, V>();
}

template <class M, class V, bool NC, class Gather, class Epi>
__device__ __forceinline__ void spmv_run_seg(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                             unsigned char* smem) {
    const RowBlock b = A.blocks[cta];
    if (!epi.begin(b.inst)) return;  // instance not iterating (uniform over the CTA)
    if (b.kind != kStream) {
        long_block<1, M, V>(A, b, g, epi, reinterpret_cast<V*>(smem + sizeof(V) * kProdStride));
        return;
    }
    const unsigned* __restrict__ bits = A.bits + b.slot_base;  // this block's row-start bitmap
    V* part = reinterpret_cast<V*>(smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nrows = b.r1 - b.r0;                                   // <= kThreads
    const int a = b.p0 & 3, q0 = b.p0 >> 2, nq = ((b.p1 + 3) >> 2) - q0, cnt = b.p1 - b.p0;  // nq <= kWinQuads
    const bool act = tid < nrows;
    const int nchunks = (nq + 31) >> 5;
#pragma unroll 1
    for (int c = warp; c < nchunks; c += kWarps) {  // warp-uniform
        const int q = 32 * c + lane;                 // this lane's window quad
        V p[4] = {V(0), V(0), V(0), V(0)};
        unsigned f = 0u;                             // row starts among the quad's 4 positions
        if (q < nq) {
            f = (__ldg(bits + (q >> 3)) >> ((4 * q) & 31)) & 0xFu;
            int js[4];
            M a4[4];
            if (A.vec) {
                int4 j4;
                if constexpr (NC) {
                    j4 = ld_stream(reinterpret_cast<const int4*>(A.idx) + q0 + q);
                    load4_stream(A.val + 4 * (q0 + q), a4);
                } else {
                    j4 = __ldg(reinterpret_cast<const int4*>(A.idx) + q0 + q);
                    load4(A.val + 4 * (q0 + q), a4);
                }
                js[0] = j4.x; js[1] = j4.y; js[2] = j4.z; js[3] = j4.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = 4 * q + u - a;
                    js[u] = (k >= 0 && k < cnt) ? __ldg(A.idx + b.p0 + k) : 0;
                    a4[u] = (k >= 0 && k < cnt) ? __ldg(A.val + b.p0 + k) : M(0);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = 4 * q + u - a;
                if (k >= 0 && k < cnt) {
                    V xv[1];
                    g(js[u], xv);
                    p[u] = static_cast<V>(a4[u]) * xv[0];
                }
            }
        }
        // segmented prefix inside the quad; `v` = the lane's open part at its end
        V v = V(0);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if ((f >> u) & 1u) v = V(0);
            v += p[u];
            p[u] = v;
        }
        // segmented inclusive scan over the lanes: a lane adds its left
        // neighbour's partial only while no row starts in between
        const unsigned heads = __ballot_sync(0xffffffffu, f != 0u);
        const unsigned upto_lane = heads & ((2u << lane) - 1u);   // heads in lanes 0..lane
        const int hl = upto_lane ? 31 - __clz(upto_lane) : -1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const V pv = __shfl_up_sync(0xffffffffu, v, d);
            if (lane - d >= hl && lane >= d) v = pv + v;
        }
        V cin = __shfl_up_sync(0xffffffffu, v, 1);
        if (lane == 0) cin = V(0);
        const unsigned first = __ballot_sync(0xffffffffu, (f & 1u) != 0u);  // lanes whose quad opens with a start
        const bool next_starts = lane < 31 && ((first >> (lane + 1)) & 1u) != 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (!(f & ((2u << u) - 1u))) p[u] = cin + p[u];  // no start up to u in this quad
            const int k = 4 * q + u - a;
            const bool end = (u < 3 ? ((f >> (u + 1)) & 1u) != 0u : (lane == 31 || next_starts)) || k == cnt - 1;
            if (end && k >= 0 && k < cnt) part[4 * q + u] = p[u];
        }
    }
    // the rows' bounds and epilogue operands are loaded only now (holding them
    // through the chunk loop costs the 32-register kernels spills); their
    // latency overlaps the barrier
    int s = 0, e = 0;
    decltype(epi.prefetch(0)) pre{};
    if (act) {
        s = __ldg(A.ptr + b.r0 + tid) - b.p0;
        e = __ldg(A.ptr + b.r0 + tid + 1) - b.p0;
        pre = epi.prefetch(b.r0 + tid);
    }
    __syncthreads();
    if (act) {
        V tot[1] = {V(0)};
        if (e > s) {
            const int pe = e - 1 + a, cs = (s + a) >> 7, ce = pe >> 7;
            tot[0] = part[min(pe, 128 * cs + 127)];
            for (int cc = cs + 1; cc <= ce; ++cc) tot[0] += part[min(pe, 128 * cc + 127)];
        }
        epi(b.r0 + tid, tot, pre);
    }
}

// STREAM-block reduction of the iteration kernels, by vector type.  Measured
// on B200 (CUDA graphs of back-to-back launches, 512-LP batch / blending LP):
// the segmented form is 11% / 3% faster per FP64 iteration (87.0 vs 98.2 µs,
// 28.2 vs 29.1 µs) and the same / 9% slower per FP32 iteration (53.2 vs
// 53.6 µs, 17.1 vs 15.7 µs) as staging the products in shared memory.
template <class M, class V, bool NC, class Gather, class Epi>
__device__ __forceinline__ void spmv_run_iter(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                              unsigned char* smem) {
    if constexpr (sizeof(V) == 8) spmv_run_seg<M, V, NC>(A, cta, g, epi, smem);
    else spmv_run<1, M, V, NC>(A, cta, g, epi, smem);
}

// Load mode kLoadPrefetch of the iteration kernels (which must NOT call
// pdl_enter themselves): the schedule and the matrix are written once at
// set-up, so before the programmatic-launch wait one thread reads the CTA's
// block and asks L2 for its whole idx / val window and for the rows'
// epilogue operands (epi.l2_prefetch_rows) with bulk prefetches.  The DRAM
// reads then overlap the previous kernel's last wave and this CTA's own
// dependent start-up loads, and the loop's 16-byte loads find the data in
// L2 -- without the shared memory a staging copy would take from the L1
// carve-out the gathers hit.  L2 is the coherence point of device memory, so
// prefetching vectors that the previous kernel may still be writing is only
// a hint, never a stale read.  epi.hint(inst) may read stale per-instance
// state (it runs before the wait) and must only err towards true.  Results
// are bit-identical to spmv_run_seg's.
template <class M, class V, class Gather, class Epi>
__device__ __forceinline__ void spmv_run_prefetched(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                                    unsigned char* smem) {
    if (threadIdx.x == 0) {
        const RowBlock b = A.blocks[cta];
        if (epi.hint(b.inst)) {
            const size_t cnt = static_cast<size_t>(b.p1 - b.p0);
            l2_prefetch(A.idx + b.p0, sizeof(int) * cnt);
            l2_prefetch(A.val + b.p0, sizeof(M) * cnt);
            epi.l2_prefetch_rows(b.r0, b.r1);
        }
    }
    pdl_enter();
    spmv_run_iter<M, V, true>(A, cta, g, epi, smem);
}

}  // namespace gb

// CSR SpMV with a fused per-row epilogue, scheduled by row blocks.
//
// Method: CSR-Adaptive (Greathouse & Daga, SC'14).  At upload time the rows
// of a matrix are cut, from its row-length histogram, into blocks:
//   * STREAM  consecutive rows whose nonzeros total <= kBlockNnz and whose
//             count <= kThreads.  The CTA streams the block's contiguous
//             idx/val range with coalesced loads, stages the products
//             val*x[idx] in shared memory, then reduces each row with a group
//             of G lanes (G = power of two chosen from the rows per block).
//   * LONG    one row with more than kBlockNnz nonzeros, reduced by the whole
//             CTA (<= kLongSingle nonzeros) or
//   * CHUNK   a slice of a very long row: each CTA writes its partial sum to a
//             fixed slot and the last CTA to arrive adds the slots in chunk
//             order and runs the epilogue (no spin-waits, deterministic).
// Every row is reduced in a fixed order, so results are bit-reproducible run
// to run.  The epilogue functor receives (row, sums) once per row, which is
// what lets the PDHG steps fuse into the product kernels.
//
// Launch: persistent.  The grid is one full wave (SMs x resident CTAs) and
// every CTA owns a contiguous, work-balanced range of blocks (no partial
// wave).  Inside a CTA the STREAM blocks' idx/val ranges are double-buffered
// in shared memory by TMA bulk copies (cp.async.bulk, completion on an
// mbarrier) that one thread issues a block ahead, so the nonzero stream costs
// no registers and overlaps the reduction; each row's epilogue operands are
// prefetched before its products are formed.  A plain mode (one CTA per
// block, direct loads) serves caller-owned arrays that are not padded.
#pragma once
#include "gb_common.cuh"

namespace gb {

constexpr int kBlockNnz = 2048;     // nonzeros per STREAM block
constexpr int kLongSingle = 16384;  // longest row one CTA reduces alone
constexpr int kChunkNnz = 8192;     // slice of a longer row per CTA

enum BlockKind : int { kStream = 0, kLong = 1, kChunk = 2 };

struct alignas(16) RowBlock {
    int r0, r1;         // rows [r0, r1)
    int p0, p1;         // nonzeros [p0, p1)
    int kind, lg;       // BlockKind, log2 of the group size (STREAM)
    int chunk, nchunks; // CHUNK: index and count
    int slot_base;      // CHUNK: first slot of the row
    int counter;        // CHUNK: arrival counter of the row
    int pad0, pad1;
};

// Host: row-length-driven schedule.  `block_nnz` / `max_rows` are the
// tunables (the batch autotuner varies them).
struct Schedule {
    std::vector<RowBlock> blocks;
    int nslots = 0, ncounters = 0;
    int max_lg = 0;
};

inline int floor_log2(int v) {
    int l = 0;
    while ((2 << l) <= v) ++l;
    return l;
}

// Walks the rows once and hands every block to `emit`; slot and counter ids
// are numbered from *nslots / *ncounters on.
template <class Emit>
inline void schedule_rows(const int* ptr, int rows, int block_nnz, int max_rows, int* nslots, int* ncounters,
                          Emit&& emit) {
    int i = 0;
    while (i < rows) {
        const int len = ptr[i + 1] - ptr[i];
        if (len > block_nnz) {
            if (len <= kLongSingle) {
                RowBlock b{};
                b.r0 = i; b.r1 = i + 1; b.p0 = ptr[i]; b.p1 = ptr[i + 1]; b.kind = kLong;
                emit(b);
            } else {
                const int nch = div_up(len, kChunkNnz);
                for (int c = 0; c < nch; ++c) {
                    RowBlock b{};
                    b.r0 = i; b.r1 = i + 1;
                    b.p0 = ptr[i] + c * kChunkNnz;
                    b.p1 = std::min(ptr[i + 1], b.p0 + kChunkNnz);
                    b.kind = kChunk; b.chunk = c; b.nchunks = nch;
                    b.slot_base = *nslots; b.counter = *ncounters;
                    emit(b);
                }
                *nslots += nch;
                *ncounters += 1;
            }
            ++i;
            continue;
        }
        const int r0 = i, start = ptr[i];
        while (i < rows && (i - r0) < max_rows && ptr[i + 1] - start <= block_nnz) ++i;
        RowBlock b{};
        b.r0 = r0; b.r1 = i; b.p0 = start; b.p1 = ptr[i]; b.kind = kStream;
        const int nrows = i - r0;
        int g = kThreads / nrows;  // lanes available per row
        if (g > 32) g = 32;
        b.lg = floor_log2(g < 1 ? 1 : g);
        emit(b);
    }
}

inline Schedule build_schedule(const int* ptr, int rows, int block_nnz = kBlockNnz, int max_rows = kThreads) {
    Schedule s;
    schedule_rows(ptr, rows, block_nnz, max_rows, &s.nslots, &s.ncounters, [&](const RowBlock& b) {
        s.blocks.push_back(b);
        s.max_lg = std::max(s.max_lg, b.lg);
    });
    return s;
}

// Contiguous, work-balanced assignment of blocks to `grid` persistent CTAs:
// cta_start[c] .. cta_start[c+1] are the blocks of CTA c.  Work of a block =
// its nonzeros + 4 per row (epilogue) + a fixed 64 (block set-up).
inline std::vector<int> assign_ctas(const std::vector<RowBlock>& blocks, int grid) {
    std::vector<int> start(grid + 1, static_cast<int>(blocks.size()));
    double total = 0;
    for (const RowBlock& b : blocks) total += (b.p1 - b.p0) + 4.0 * (b.r1 - b.r0) + 64.0;
    double acc = 0;
    int c = 0;
    start[0] = 0;
    for (int i = 0; i < static_cast<int>(blocks.size()); ++i) {
        const RowBlock& b = blocks[i];
        // block i goes to the CTA whose share contains the block's midpoint
        const double w = (b.p1 - b.p0) + 4.0 * (b.r1 - b.r0) + 64.0;
        const double mid = acc + 0.5 * w;
        const int owner = std::min(grid - 1, static_cast<int>(mid * grid / total));
        while (c < owner) start[++c] = i;
        acc += w;
    }
    while (c < grid) start[++c] = static_cast<int>(blocks.size());
    return start;
}

// Number of persistent partitions a schedule keeps (one per precision level,
// since the resident CTAs per SM differ with the value types).
constexpr int kPartitions = 3;

// Device-resident schedule of one matrix.
struct DevSchedule {
    DevBuf<RowBlock> blocks;
    DevBuf<int> cta_start[kPartitions];
    DevBuf<double> slots;
    DevBuf<unsigned> counters;
    int nb = 0;
    int grid[kPartitions] = {0, 0, 0};  // persistent CTAs per partition (0: one CTA per block)
    int nslots = 0;
    // grids[k] > 0 builds persistent partition k with that many CTAs
    void upload(const Schedule& s, int nv_max, cudaStream_t st, const int* grids = nullptr) {
        nb = static_cast<int>(s.blocks.size());
        blocks.reset(nb ? nb : 1);
        blocks.upload(s.blocks.data(), nb, st);
        for (int k = 0; k < kPartitions; ++k) {
            grid[k] = 0;
            if (grids && grids[k] > 0 && nb > 0) {
                grid[k] = std::min(grids[k], nb);
                std::vector<int> cs = assign_ctas(s.blocks, grid[k]);
                cta_start[k].reset(grid[k] + 1);
                cta_start[k].upload(cs.data(), grid[k] + 1, st);
                GB_CUDA(cudaStreamSynchronize(st));  // cs is a host temporary
            }
        }
        nslots = s.nslots;
        slots.reset(static_cast<size_t>(s.nslots ? s.nslots : 1) * nv_max);
        counters.reset(s.ncounters ? s.ncounters : 1);
        GB_CUDA(cudaMemsetAsync(counters.get(), 0, counters.size() * sizeof(unsigned), st));
    }
    int ctas(int part) const { return grid[part] > 0 ? grid[part] : nb; }
};

// Raw view of a CSR matrix on the device.  With cta_start set (persistent
// mode) idx and val must be readable up to nnz rounded up to 4 elements + 4,
// because blocks are fetched as 16-byte-aligned bulk copies.
template <class M>
struct CsrView {
    const int* __restrict__ ptr;
    const int* __restrict__ idx;
    const M* __restrict__ val;
    const RowBlock* __restrict__ blocks;
    const int* __restrict__ cta_start;  // nullptr: CTA c runs block c with plain loads
    double* slots;
    unsigned* counters;
    unsigned* err;                      // set to 1 if a bounded wait gave up (persistent mode)
    int rows;
    int nb;
    int ncta;                           // CTAs this matrix is launched with
};

// Padded element count of idx / val arrays used in persistent mode.
inline long long padded_nnz(long long nnz) { return ((nnz + 3) & ~3LL) + 4; }

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

// One pipeline stage: a STREAM block's idx and val, fetched with 16-byte
// alignment (up to 3 leading and 3 trailing extra entries).
constexpr int kStageElems = kBlockNnz + 8;
template <class M>
struct Stage {
    static constexpr size_t idx_bytes = sizeof(int) * kStageElems;
    static constexpr size_t bytes = idx_bytes + sizeof(M) * kStageElems;
};
constexpr size_t kMbarBytes = 64;

// Dynamic shared memory: plain mode / persistent (two TMA stages) mode.
template <int NV, class V>
constexpr size_t spmv_smem_bytes() {
    return sizeof(V) * NV * kProdStride + sizeof(double) * kWarps * NV + 64;
}
template <int NV, class M, class V>
constexpr size_t spmv_smem_bytes_tma() {
    return kMbarBytes + 2 * Stage<M>::bytes + spmv_smem_bytes<NV, V>();
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

// Plain mode: CTA `cta` runs block `cta` with direct global loads.
template <int NV, class M, class V, class Gather, class Epi>
__device__ __forceinline__ void spmv_plain(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                           unsigned char* smem) {
    V* prod = reinterpret_cast<V*>(smem);
    V* red = reinterpret_cast<V*>(smem + sizeof(V) * NV * kProdStride);
    const RowBlock b = A.blocks[cta];
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
#pragma unroll 4
    for (int k = tid; k < cnt; k += kThreads) {
        const int p = b.p0 + k;
        const V a = static_cast<V>(__ldg(A.val + p));
        V xv[NV];
        g(__ldg(A.idx + p), xv);
#pragma unroll
        for (int v = 0; v < NV; ++v) prod[v * kProdStride + padded(k)] = a * xv[v];
    }
    __syncthreads();
    reduce_rows<NV, V>(b, prod, s, e, act, pre, epi);
}

// Thread 0: fetch STREAM block b into a stage (idx then val) on `bar`.
template <class M>
__device__ __forceinline__ void issue_stage(const CsrView<M>& A, const RowBlock& b, unsigned char* stage,
                                            unsigned long long* bar) {
    const int p0a = b.p0 & ~3, p1a = (b.p1 + 3) & ~3;
    const unsigned cnt = static_cast<unsigned>(p1a - p0a);
    const unsigned bi = cnt * sizeof(int), bv = cnt * sizeof(M);
    mbar_arrive_expect_tx(bar, bi + bv);
    if (cnt) {
        bulk_g2s(stage, A.idx + p0a, bi, bar);
        bulk_g2s(stage + Stage<M>::idx_bytes, A.val + p0a, bv, bar);
    }
}

// Run every block of CTA `cta` of matrix A.  Gather g(col, V(&)[NV]) supplies
// the NV vector values of a column; epi.prefetch(row) loads a row's epilogue
// operands early and epi(row, const V(&)[NV], pre) consumes a finished row.
// Persistent mode double-buffers the STREAM blocks' nonzeros in shared memory
// with TMA bulk copies issued one block ahead by thread 0.
template <int NV, class M, class V, class Gather, class Epi>
__device__ __forceinline__ void spmv_run(const CsrView<M>& A, int cta, const Gather& g, Epi& epi,
                                         unsigned char* smem) {
    if (A.cta_start == nullptr) {
        spmv_plain<NV, M, V>(A, cta, g, epi, smem);
        return;
    }
    const int b0 = A.cta_start[cta], b1 = A.cta_start[cta + 1];
    if (b0 >= b1) return;
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
    unsigned char* stages = smem + kMbarBytes;
    V* prod = reinterpret_cast<V*>(stages + 2 * Stage<M>::bytes);
    V* red = prod + NV * kProdStride;
    const int tid = threadIdx.x;
    int next_issue = b0;  // thread 0: next block index to consider for a copy
    int nissued = 0;      // thread 0: STREAM copies issued
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        for (int k = 0; k < 2; ++k) {
            while (next_issue < b1 && A.blocks[next_issue].kind != kStream) ++next_issue;
            if (next_issue >= b1) break;
            issue_stage(A, A.blocks[next_issue], stages + (nissued & 1) * Stage<M>::bytes, &bars[nissued & 1]);
            ++nissued;
            ++next_issue;
        }
    }
    __syncthreads();
    int nconsumed = 0;
    for (int bi = b0; bi < b1; ++bi) {
        const RowBlock b = A.blocks[bi];
        if (b.kind != kStream) {
            long_block<NV, M, V>(A, b, g, epi, red);
            continue;
        }
        const int sidx = nconsumed & 1;
        const unsigned parity = static_cast<unsigned>(nconsumed >> 1) & 1u;
        const int grp = tid >> b.lg;
        const bool act = grp < b.r1 - b.r0;
        int s = 0, e = 0;
        decltype(epi.prefetch(0)) pre{};
        if (act) {
            const int r = b.r0 + grp;
            s = __ldg(A.ptr + r) - b.p0;
            e = __ldg(A.ptr + r + 1) - b.p0;
            if ((tid & ((1 << b.lg) - 1)) == 0) pre = epi.prefetch(r);
        }
        if (!mbar_wait_bounded(&bars[sidx], parity)) {
            atomicOr(A.err, 1u);                  // report, then give the copy one more bounded wait
            mbar_wait_bounded(&bars[sidx], parity);
        }
        const unsigned char* st = stages + sidx * Stage<M>::bytes;
        const int* sI = reinterpret_cast<const int*>(st) + (b.p0 & 3);
        const M* sV = reinterpret_cast<const M*>(st + Stage<M>::idx_bytes) + (b.p0 & 3);
        const int cnt = b.p1 - b.p0;
#pragma unroll 4
        for (int k = tid; k < cnt; k += kThreads) {
            V xv[NV];
            g(sI[k], xv);
            const V a = static_cast<V>(sV[k]);
#pragma unroll
            for (int v = 0; v < NV; ++v) prod[v * kProdStride + padded(k)] = a * xv[v];
        }
        __syncthreads();
        if (tid == 0) {  // stage sidx is free again: fetch the next STREAM block into it
            while (next_issue < b1 && A.blocks[next_issue].kind != kStream) ++next_issue;
            if (next_issue < b1) {
                fence_proxy_async_smem();
                issue_stage(A, A.blocks[next_issue], stages + (nissued & 1) * Stage<M>::bytes, &bars[nissued & 1]);
                ++nissued;
                ++next_issue;
            }
        }
        reduce_rows<NV, V>(b, prod, s, e, act, pre, epi);
        __syncthreads();
        ++nconsumed;
    }
}

}  // namespace gb

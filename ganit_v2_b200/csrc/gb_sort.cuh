// Device exclusive scan and stable LSD radix sort of int keys: the two
// pieces of the stored transpose (src/lp.cpp:55-72) -- the scan turns column
// counts into A^T's row pointers, the sort gives every nonzero its slot in
// A^T with the source order kept inside each column.  Integer work, so the
// result is the same on every run whatever the scheduling.
//
// Scan: tiles of kScanTile ints -- per-tile sums, one CTA scans the sums,
// then each tile scans itself from its offset (in == out allowed).
//
// Sort: 8-bit digits, least significant first, each pass over tiles of
// kRadixTile keys:
//   k_radix_hist     digit histogram of each tile, digit-major (hist[d][tile]),
//                    so the exclusive scan of the whole array is, for every
//                    (digit, tile), the first output slot of that tile's keys
//                    of that digit;
//   k_radix_scatter  each tile walks its keys in index order, kThreads at a
//                    time: a key's slot is its (digit, tile) offset, plus the
//                    keys of its digit in the tile's earlier rounds, in lower
//                    warps of this round, and in lower lanes of its warp
//                    (__match_any_sync peers).  Ties keep index order, which
//                    is what makes the passes compose into a stable sort.
#pragma once
#include <algorithm>

#include "gb_common.cuh"

namespace gb {

constexpr int kScanItems = 4;
constexpr int kScanTile = kThreads * kScanItems;
constexpr int kRadixBins = 256;
constexpr int kRadixItems = 8;
constexpr int kRadixTile = kThreads * kRadixItems;
static_assert(kThreads == kRadixBins, "one thread per digit in the scatter's prefix step");

// Exclusive prefix of one int per thread over the CTA; *total gets the sum.
__device__ __forceinline__ int cta_exclusive_scan(int v, int* sh, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kWarps; ++w) {
            const int t = sh[w];
            sh[w] = run;
            run += t;
        }
        sh[kWarps] = run;
    }
    __syncthreads();
    const int r = sh[wid] + x - v;
    *total = sh[kWarps];
    __syncthreads();  // sh is reused by the caller's next scan
    return r;
}

static __global__ void __launch_bounds__(kThreads) k_scan_tiles(const int* __restrict__ in, long long n,
                                                                int* __restrict__ tile_sum) {
    __shared__ int sh[kWarps + 1];
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
    int acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + static_cast<long long>(k) * kThreads + threadIdx.x;
        if (i < n) acc += in[i];
    }
    int total;
    cta_exclusive_scan(acc, sh, &total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// One CTA: tile_sum <- its exclusive prefix, kThreads entries per round.
static __global__ void __launch_bounds__(kThreads) k_scan_top(int ntiles, int* tile_sum) {
    __shared__ int sh[kWarps + 1];
    int carry = 0;
    for (int b = 0; b < ntiles; b += kThreads) {
        const int i = b + static_cast<int>(threadIdx.x);
        const int v = i < ntiles ? tile_sum[i] : 0;
        int total;
        const int e = cta_exclusive_scan(v, sh, &total);
        if (i < ntiles) tile_sum[i] = carry + e;
        carry += total;
    }
}

// Each thread owns kScanItems consecutive entries of its tile.
static __global__ void __launch_bounds__(kThreads) k_scan_apply(const int* in, int* out, long long n,
                                                                const int* __restrict__ tile_off) {
    __shared__ int sh[kWarps + 1];
    const long long first = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = first + k < n ? in[first + k] : 0;
        acc += v[k];
    }
    int total;
    int run = cta_exclusive_scan(acc, sh, &total) + tile_off[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (first + k < n) {
            out[first + k] = run;
            run += v[k];
        }
}

inline int scan_tiles(long long n) { return static_cast<int>((n + kScanTile - 1) / kScanTile); }

// out[i] = in[0] + ... + in[i-1]; `tile_sum` holds scan_tiles(n) ints.
inline void exclusive_scan(const int* in, int* out, long long n, int* tile_sum, cudaStream_t s) {
    if (n <= 0) return;
    const int nt = scan_tiles(n);
    k_scan_tiles<<<nt, kThreads, 0, s>>>(in, n, tile_sum);
    k_scan_top<<<1, kThreads, 0, s>>>(nt, tile_sum);
    k_scan_apply<<<nt, kThreads, 0, s>>>(in, out, n, tile_sum);
}

static __global__ void __launch_bounds__(kThreads) k_radix_hist(const int* __restrict__ keys, int n, int shift,
                                                                int ntiles, int* __restrict__ hist) {
    __shared__ int cnt[kRadixBins];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long base = static_cast<long long>(blockIdx.x) * kRadixTile;
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
        const long long i = base + r * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & (kRadixBins - 1)], 1);
    }
    __syncthreads();
    hist[static_cast<long long>(threadIdx.x) * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// vals == nullptr: the value of key i is i.  keys_out == nullptr: keys are
// not written (the last pass needs only the permutation).
static __global__ void __launch_bounds__(kThreads) k_radix_scatter(const int* __restrict__ keys,
                                                                   const int* __restrict__ vals, int n, int shift,
                                                                   int ntiles, const int* __restrict__ offs,
                                                                   int* __restrict__ keys_out,
                                                                   int* __restrict__ vals_out) {
    __shared__ int next[kRadixBins];             // next free slot of each digit for this tile
    __shared__ int wcnt[kWarps][kRadixBins];     // this round: keys per (warp, digit), then their first slot
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    next[tid] = offs[static_cast<long long>(tid) * ntiles + blockIdx.x];
    const long long base = static_cast<long long>(blockIdx.x) * kRadixTile;
    for (int r = 0; r < kRadixItems; ++r) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wcnt[w][tid] = 0;
        __syncthreads();
        const long long i = base + r * kThreads + tid;
        const bool valid = i < n;
        const int key = valid ? keys[i] : 0;
        const int val = valid ? (vals ? vals[i] : static_cast<int>(i)) : 0;
        const int d = valid ? (key >> shift) & (kRadixBins - 1) : kRadixBins;  // out-of-range lanes group apart
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[wid][d] = __popc(peers);
        __syncthreads();
        int run = next[tid];  // thread tid owns digit tid
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const int c = wcnt[w][tid];
            wcnt[w][tid] = run;
            run += c;
        }
        next[tid] = run;
        __syncthreads();
        if (valid) {
            const int pos = wcnt[wid][d] + rank;
            if (keys_out) keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();  // this round's slots are read before the next round clears them
    }
}

static __global__ void k_iota_index(int n, int* v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Temporary buffers of a sort, owned by the caller so that they are
// released (a device synchronisation each, in the device cache) only after
// the caller's own synchronisation.
struct SortScratch {
    DevBuf<int> hist, tile_sum, ka, kb, va, vb;
};

// perm[q] = index of the q-th key in ascending order, ties in index order,
// for keys in [0, 2^bits).
inline void stable_sort_index(const int* keys, int n, int bits, int* perm, int sms, SortScratch& w, cudaStream_t s) {
    if (n <= 0) return;
    const int passes = (bits + 7) / 8;
    if (passes == 0) {  // every key is 0
        k_iota_index<<<std::min(div_up(n, kThreads), 8 * sms), kThreads, 0, s>>>(n, perm);
        return;
    }
    const int ntiles = div_up(n, kRadixTile);
    const long long hn = static_cast<long long>(kRadixBins) * ntiles;
    DevBuf<int>&hist = w.hist, &ka = w.ka, &kb = w.kb, &va = w.va, &vb = w.vb;
    hist.reset(hn);
    w.tile_sum.reset(scan_tiles(hn));
    DevBuf<int>& tile_sum = w.tile_sum;
    if (passes > 1) {
        ka.reset(n);
        va.reset(n);
    }
    if (passes > 2) {
        kb.reset(n);
        vb.reset(n);
    }
    const int* kin = keys;
    const int* vin = nullptr;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1;
        int* kout = last ? nullptr : (p % 2 ? kb.get() : ka.get());
        int* vout = last ? perm : (p % 2 ? vb.get() : va.get());
        k_radix_hist<<<ntiles, kThreads, 0, s>>>(kin, n, 8 * p, ntiles, hist.get());
        exclusive_scan(hist.get(), hist.get(), hn, tile_sum.get(), s);
        k_radix_scatter<<<ntiles, kThreads, 0, s>>>(kin, vin, n, 8 * p, ntiles, hist.get(), kout, vout);
        kin = kout;
        vin = vout;
    }
}

}  // namespace gb

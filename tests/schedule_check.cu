// Host-only checker of the row-block scheduler (ganit_v2_b200/csrc/gb_spmv.cuh),
// compiled and run by tests/test_schedule.py; no GPU involved.  For a set of
// row-length patterns it builds schedules and checks the invariants the SpMV
// kernels rely on; it prints one line per pattern and exits non-zero on the
// first violation.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "../ganit_v2_b200/csrc/gb_spmv.cuh"

using gb::RowBlock;

static int fail(const std::string& what, const std::string& pattern) {
    std::printf("FAIL %s: %s\n", pattern.c_str(), what.c_str());
    return 1;
}

static int check(const std::string& name, const std::vector<int>& len, int block_nnz, int max_rows) {
    std::vector<int> ptr(len.size() + 1, 0);
    for (size_t i = 0; i < len.size(); ++i) ptr[i + 1] = ptr[i] + len[i];
    const int rows = static_cast<int>(len.size());
    const gb::Schedule s = gb::build_schedule(ptr.data(), rows, nullptr, 1, block_nnz, max_rows);
    // every nonzero exactly once, in order; every row in exactly one STREAM/LONG
    // block or in consecutive CHUNK slices
    int next_row = 0, next_nz = 0, slots = 0, counters = 0;
    for (size_t k = 0; k < s.blocks.size(); ++k) {
        const RowBlock& b = s.blocks[k];
        if (b.p0 != next_nz) return fail("nonzeros not contiguous at block " + std::to_string(k), name);
        if (b.r0 != next_row) return fail("rows not contiguous at block " + std::to_string(k), name);
        next_nz = b.p1;
        if (b.kind == gb::kStream) {
            const int nr = b.r1 - b.r0;
            if (nr < 1 || nr > max_rows) return fail("STREAM row count", name);
            if (b.p1 - b.p0 > block_nnz) return fail("STREAM nonzeros above block_nnz", name);
            if (b.p0 != ptr[b.r0] || b.p1 != ptr[b.r1]) return fail("STREAM bounds", name);
            int maxlen = 0;
            for (int r = b.r0; r < b.r1; ++r) maxlen = std::max(maxlen, len[r]);
            const int g = gb::kLaneGroups.g[nr];
            if ((1 << b.lg) != g) return fail("lane group of a STREAM block", name);
            if ((maxlen + g - 1) / g > gb::kMaxLaneSum)
                return fail("a lane sums more than kMaxLaneSum products", name);
            next_row = b.r1;
        } else if (b.kind == gb::kLong) {
            if (b.r1 != b.r0 + 1) return fail("LONG covers one row", name);
            if (len[b.r0] <= std::min(block_nnz, 32 * gb::kMaxLaneSum)) return fail("short row made LONG", name);
            if (len[b.r0] > gb::kLongSingle) return fail("LONG row above kLongSingle", name);
            next_row = b.r1;
        } else if (b.kind == gb::kChunk) {
            if (b.r1 != b.r0 + 1 || len[b.r0] <= gb::kLongSingle) return fail("CHUNK of a short row", name);
            if (b.p1 - b.p0 > gb::kChunkNnz) return fail("CHUNK above kChunkNnz", name);
            if (b.chunk == 0) {
                if (b.slot_base != slots || b.counter != counters) return fail("CHUNK slot / counter ids", name);
                slots += b.nchunks;
                counters += 1;
            }
            if (b.chunk == b.nchunks - 1) {
                if (b.p1 != ptr[b.r0 + 1]) return fail("CHUNK slices do not end at the row's end", name);
                next_row = b.r1;
            }
        } else {
            return fail("unknown block kind", name);
        }
    }
    if (next_row != rows || next_nz != ptr[rows]) return fail("schedule does not cover the matrix", name);
    if (s.nslots != slots || s.ncounters != counters) return fail("slot / counter totals", name);
    std::printf("ok %s rows=%d nnz=%d blocks=%zu\n", name.c_str(), rows, ptr[rows], s.blocks.size());
    return 0;
}

int main() {
    // the lane-group table is the largest power of two <= min(32, kThreads / nr)
    for (int nr = 1; nr <= gb::kThreads; ++nr) {
        const int want = 1 << gb::floor_log2(std::min(32, gb::kThreads / nr));
        if (gb::kLaneGroups.g[nr] != want) return fail("kLaneGroups at " + std::to_string(nr), "table");
    }
    std::mt19937 rng(7);
    std::vector<std::pair<std::string, std::vector<int>>> cases;
    {  // uniform short rows
        std::vector<int> l(20000);
        for (int& v : l) v = 1 + static_cast<int>(rng() % 12);
        cases.push_back({"short", l});
    }
    {  // one 960-nonzero row among ~60 short rows, repeated (a blending LP period)
        std::vector<int> l;
        for (int t = 0; t < 200; ++t) {
            l.push_back(960);
            for (int k = 0; k < 60; ++k) l.push_back(18);
            for (int k = 0; k < 80; ++k) l.push_back(60);
        }
        cases.push_back({"blending_like", l});
    }
    {  // heavy tail: a few rows past every threshold, empty rows included
        std::vector<int> l;
        for (int k = 0; k < 5000; ++k) {
            const int r = static_cast<int>(rng() % 1000);
            l.push_back(r < 5 ? 0 : r < 990 ? 1 + static_cast<int>(rng() % 40)
                                            : 500 + static_cast<int>(rng() % 30000));
        }
        l.push_back(100000);  // one row in many CHUNK slices
        l.push_back(4096);    // the longest single-CTA row
        l.push_back(4097);    // the shortest chunked row
        l.push_back(1024);
        l.push_back(1025);
        cases.push_back({"heavy_tail", l});
    }
    int bad = 0;
    for (const auto& c : cases) {
        bad |= check(c.first, c.second, gb::kBlockNnz, gb::kThreads);
        bad |= check(c.first + "_tuned", c.second, 1248, 64);
    }
    return bad;
}

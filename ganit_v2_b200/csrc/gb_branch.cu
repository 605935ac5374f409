// Batched strong branching for a MILP node (gb_strong_branch).
//
// The reference's Mip::select_branch (src/mip.cpp:668-783) strong-branches
// its candidates one at a time: for each fractional column j it sets the
// down child's bounds (l_j, floor x_j), re-solves with a warm dual simplex,
// restores, sets the up child's (ceil x_j, u_j), re-solves, restores, and
// certifies each child's bound from its duals (Mip::safe_bound,
// src/mip.cpp:356-410).  Here all 2k children of the k candidates are ONE
// resident batch of the block-diagonal engine (per-child scaling, restarts,
// precision phases and FP64 certification), and the rigorous Lagrangian
// bound of every child is formed on the device from the batch's unscaled
// duals with directed rounding (__dmul_rd / __dadd_rd and the _ru forms):
//   c'x >= sum_i min(y_i lo_i, y_i hi_i) + sum_j min_{x_j in [l_j, u_j]} d_j x_j,
//   d = c - A'y carried as an interval [d_lo, d_hi],
// with y_i clamped to the sign a one-sided row allows.  Each partial sum is
// rounded toward -inf (toward +inf for the upper end of d), so the result is
// a lower bound of the exact value in any summation order.  One deliberate
// difference from the reference: a column term that overflows to -inf makes
// the child uncertifiable (the reference resets a non-finite column minimum
// to 0, which is right only for d = [0, 0] on a free column).
//
// Child outcome (the reference's mapping, src/mip.cpp:750-763, with the
// PDHG statuses): primal infeasible -> +inf; certified bound >= cutoff
// (the analogue of the dual simplex's cutoff stop) -> +inf; optimal -> the
// child's objective; otherwise max(node objective, certified bound), or the
// node objective when no bound could be certified.  The decision then scans
// the candidates in the caller's order as select_branch does: both children
// +inf -> node infeasible; one -> tighten the column to the other side;
// else the largest score max(z_down - z, 1e-6) * max(z_up - z, 1e-6), the
// first candidate winning ties.
//
// Given the node's duals y as well, every child starts from the node's point
// (x, y) -- x projected onto the child's bounds -- instead of the default
// start (an extension: the reference's PDHG always starts from the
// projection of 0, and the dual simplex it replaces here starts warm).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <vector>

#include "gb_problem.cuh"

namespace gb {
namespace {

constexpr int kBoundThreads = 256;
constexpr double kScoreEps = 1e-6;  // src/mip.cpp:673

struct BoundArgs {
    int m, n, children;
    const int* at_ptr;      // A^T in CSR (one row per column of A)
    const int* at_idx;
    const double* at_val;
    const double* c;        // minimisation-form costs
    const double* l;
    const double* u;
    const double* lo;
    const double* hi;
    const int* col;         // per child: the branched column
    const double* col_lo;   // per child: its bounds in the child
    const double* col_hi;
    const int* inst;        // per child: instance index in the batch (its duals at inst * m)
    const double* y;        // batch duals, unscaled
    double* yadj;           // children x m: duals clamped to the rows' allowed signs
    double* part_rows;      // children x row_blocks
    double* part_cols;      // children x col_blocks
    int* bad;               // children: 1 when the bound cannot be certified
    double* cert;           // children: the certified bound
    double obj_const;
    int row_blocks, col_blocks;
};

// Block sum rounded toward -inf at every addition (result in thread 0).
__device__ double block_sum_rd(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rd(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < static_cast<int>(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = __dadd_rd(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    return v;
}

// Row part: clamp y, sum min(y_i lo_i, y_i hi_i) rounded down.
__global__ void __launch_bounds__(kBoundThreads) k_bound_rows(const __grid_constant__ BoundArgs a) {
    __shared__ double sh[kBoundThreads / 32];
    const int s = blockIdx.y;
    const double* y = a.y + static_cast<size_t>(a.inst[s]) * a.m;
    double* ya = a.yadj + static_cast<size_t>(s) * a.m;
    double acc = 0.0;
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.m; i += gridDim.x * blockDim.x) {
        double yi = y[i];
        const double lo = a.lo[i], hi = a.hi[i];
        if (!isfinite(lo)) yi = fmin(yi, 0.0);
        if (!isfinite(hi)) yi = fmax(yi, 0.0);
        ya[i] = yi;
        if (yi == 0.0) continue;
        const double t = yi > 0.0 ? __dmul_rd(yi, lo) : __dmul_rd(yi, hi);
        if (!isfinite(t)) bad = true;
        else acc = __dadd_rd(acc, t);
    }
    if (bad) a.bad[s] = 1;
    acc = block_sum_rd(acc, sh);
    if (threadIdx.x == 0) a.part_rows[static_cast<size_t>(s) * a.row_blocks + blockIdx.x] = acc;
}

// Column part: d_j = c_j - (A'y)_j as an interval, then min over the
// column's box of d_j x_j, rounded down.
__global__ void __launch_bounds__(kBoundThreads) k_bound_cols(const __grid_constant__ BoundArgs a) {
    __shared__ double sh[kBoundThreads / 32];
    const int s = blockIdx.y;
    const double* ya = a.yadj + static_cast<size_t>(s) * a.m;
    const int jc = a.col[s];
    double acc = 0.0;
    bool bad = false;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.n; j += gridDim.x * blockDim.x) {
        double s_up = 0.0, s_dn = 0.0;
        for (int t = a.at_ptr[j]; t < a.at_ptr[j + 1]; ++t) {
            const double yi = ya[a.at_idx[t]];
            if (yi == 0.0) continue;
            const double v = a.at_val[t];
            s_up = __dadd_ru(s_up, __dmul_ru(yi, v));
            s_dn = __dadd_rd(s_dn, __dmul_rd(yi, v));
        }
        const double dlo = __dsub_rd(a.c[j], s_up), dhi = __dsub_ru(a.c[j], s_dn);
        const double l = j == jc ? a.col_lo[s] : a.l[j], u = j == jc ? a.col_hi[s] : a.u[j];
        if ((!isfinite(l) && dhi > 0.0) || (!isfinite(u) && dlo < 0.0) || isnan(dlo) || isnan(dhi)) {
            bad = true;
            continue;
        }
        double best = INFINITY;
        if (isfinite(l)) best = fmin(__dmul_rd(dlo, l), __dmul_rd(dhi, l));
        if (isfinite(u)) best = fmin(best, fmin(__dmul_rd(dlo, u), __dmul_rd(dhi, u)));
        if (best == INFINITY) best = 0.0;  // free column with d = [0, 0]
        if (!isfinite(best)) bad = true;
        else acc = __dadd_rd(acc, best);
    }
    if (bad) a.bad[s] = 1;
    acc = block_sum_rd(acc, sh);
    if (threadIdx.x == 0) a.part_cols[static_cast<size_t>(s) * a.col_blocks + blockIdx.x] = acc;
}

// One thread per child: add the partial sums (rounded down) and the
// objective constant.
__global__ void k_bound_final(const __grid_constant__ BoundArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.children) return;
    double r = 0.0, c = 0.0;
    for (int b = 0; b < a.row_blocks; ++b) r = __dadd_rd(r, a.part_rows[static_cast<size_t>(s) * a.row_blocks + b]);
    for (int b = 0; b < a.col_blocks; ++b) c = __dadd_rd(c, a.part_cols[static_cast<size_t>(s) * a.col_blocks + b]);
    a.cert[s] = a.bad[s] ? -INFINITY : __dadd_rd(__dadd_rd(r, c), a.obj_const);
}

// Column-major copy of a host CSR matrix (stable: rows increase within a column).
void host_transpose(const gb_lp& lp, std::vector<int>& ptr, std::vector<int>& idx, std::vector<double>& val) {
    const int m = lp.m, n = lp.n;
    const long long nnz = m ? lp.a_ptr[m] : 0;
    ptr.assign(n + 1, 0);
    for (long long t = 0; t < nnz; ++t) ++ptr[lp.a_idx[t] + 1];
    for (int j = 0; j < n; ++j) ptr[j + 1] += ptr[j];
    idx.resize(nnz);
    val.resize(nnz);
    std::vector<int> pos(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < m; ++i)
        for (int t = lp.a_ptr[i]; t < lp.a_ptr[i + 1]; ++t) {
            const int p = pos[lp.a_idx[t]]++;
            idx[p] = i;
            val[p] = lp.a_val[t];
        }
}

struct Child {
    int cand, dir, col;
    double lo, hi;     // the branched column's bounds in this child
    int inst = -1;     // index in the batch (-1: bounds cross, not solved)
};

void strong_branch(const gb_lp& lp, const double* x, const double* y, int count, const int32_t* cand, double node_obj,
                   double cutoff, const gb_options* opt, gb_branch_cand* out, gb_branch_decision* dec) {
    const auto t0 = std::chrono::steady_clock::now();
    GB_REQUIRE(count >= 1 && count <= 32767, "need 1 to 32767 candidates");  // children index the grid's y dimension
    GB_REQUIRE(lp.m >= 0 && lp.n >= 1 && lp.c && lp.l && lp.u && (lp.m == 0 || (lp.a_ptr && lp.lo && lp.hi)),
               "incomplete LP");
    if (lp.q_ptr || lp.q_rank > 0) throw Error(GB_ERR_UNSUPPORTED, "strong branching takes LPs only (no Hessian)");
    GB_REQUIRE(!std::isnan(node_obj) && !std::isnan(cutoff), "node objective and cutoff must not be NaN");
    const int n = lp.n;
    for (int k = 0; k < count; ++k) {
        const int j = cand[k];
        GB_REQUIRE(j >= 0 && j < n, "candidate column out of range");
        GB_REQUIRE(std::isfinite(x[j]), "candidate value is not finite");
        GB_REQUIRE(std::floor(x[j]) != x[j], "candidate value is integral");
    }
    if (y) {
        for (int j = 0; j < n; ++j) GB_REQUIRE(std::isfinite(x[j]), "node point has a non-finite entry");
        for (int i = 0; i < lp.m; ++i) GB_REQUIRE(std::isfinite(y[i]), "node point has a non-finite entry");
    }
    // minimisation form: the reference branches on zmin() = sign * objective
    const double sign = lp.maximize ? -1.0 : 1.0;
    std::vector<double> cmin(lp.c, lp.c + n);
    if (lp.maximize)
        for (double& v : cmin) v = -v;
    gb_lp base = lp;
    base.c = cmin.data();
    base.maximize = 0;
    base.obj_const = sign * lp.obj_const;

    std::vector<Child> ch;
    ch.reserve(2 * static_cast<size_t>(count));
    for (int k = 0; k < count; ++k) {
        const int j = cand[k];
        const double v = x[j];
        ch.push_back({k, 0, j, lp.l[j], std::floor(v)});
        ch.push_back({k, 1, j, std::ceil(v), lp.u[j]});
    }
    // one modified bound array per solved child; the other side is shared
    std::vector<std::vector<double>> bnd;
    std::vector<gb_lp> views;
    std::vector<int> solved;
    for (size_t s = 0; s < ch.size(); ++s) {
        Child& c = ch[s];
        if (!(c.lo <= c.hi)) continue;  // bounds cross: infeasible without a solve
        c.inst = static_cast<int>(views.size());
        gb_lp v = base;
        bnd.emplace_back(c.dir == 0 ? lp.u : lp.l, (c.dir == 0 ? lp.u : lp.l) + n);
        bnd.back()[c.col] = c.dir == 0 ? c.hi : c.lo;
        views.push_back(v);
        solved.push_back(static_cast<int>(s));
    }
    for (size_t b = 0; b < views.size(); ++b) {
        const Child& c = ch[solved[b]];
        (c.dir == 0 ? views[b].u : views[b].l) = bnd[b].data();
    }

    const int S = static_cast<int>(views.size());
    std::vector<gb_result> res(S);
    std::vector<double> cert(S, -INFINITY);
    if (S > 0) {
        std::unique_ptr<Problem> P(create_problem(S, views.data(), opt));
        if (y) {
            // every child starts from the node's point (x projected onto the
            // child's bounds on the device); the duals in minimisation form
            std::vector<double> xs(static_cast<size_t>(S) * n), ys(static_cast<size_t>(S) * std::max(lp.m, 1));
            for (int b = 0; b < S; ++b) {
                std::copy(x, x + n, xs.begin() + static_cast<size_t>(b) * n);
                for (int i = 0; i < lp.m; ++i) ys[static_cast<size_t>(b) * lp.m + i] = sign * y[i];
            }
            P->x_start.reset(xs.size());
            P->y_start.reset(ys.size());
            P->x_start.upload(xs.data(), xs.size(), P->stream);
            P->y_start.upload(ys.data(), ys.size(), P->stream);
        }
        solve_problem(*P, opt, res.data());
        bnd.clear();
        bnd.shrink_to_fit();
        for (int b = 0; b < S; ++b)
            GB_REQUIRE(P->row_off[b] == b * lp.m, "unexpected instance layout of the batch");
        // certified bounds of every solved child, on the device
        cudaStream_t s = P->stream;
        std::vector<int> tp, ti;
        std::vector<double> tv;
        host_transpose(lp, tp, ti, tv);
        DevBuf<int> at_ptr(tp.size()), at_idx(std::max<size_t>(ti.size(), 1));
        DevBuf<double> at_val(std::max<size_t>(tv.size(), 1));
        at_ptr.upload(tp.data(), tp.size(), s);
        at_idx.upload(ti.data(), ti.size(), s);
        at_val.upload(tv.data(), tv.size(), s);
        const size_t mm = std::max(lp.m, 1);
        DevBuf<double> c(n), l(n), u(n), lo(mm), hi(mm);
        c.upload(cmin.data(), n, s);
        l.upload(lp.l, n, s);
        u.upload(lp.u, n, s);
        lo.upload(lp.lo, lp.m, s);
        hi.upload(lp.hi, lp.m, s);
        std::vector<int> hcol(S), hinst(S);
        std::vector<double> hlo(S), hhi(S);
        for (int b = 0; b < S; ++b) {
            const Child& cb = ch[solved[b]];
            hcol[b] = cb.col;
            hinst[b] = b;
            hlo[b] = cb.lo;
            hhi[b] = cb.hi;
        }
        DevBuf<int> dcol(S), dinst(S), dbad(S);
        DevBuf<double> dlo(S), dhi(S), dcert(S);
        dcol.upload(hcol.data(), S, s);
        dinst.upload(hinst.data(), S, s);
        dlo.upload(hlo.data(), S, s);
        dhi.upload(hhi.data(), S, s);
        GB_CUDA(cudaMemsetAsync(dbad.get(), 0, sizeof(int) * S, s));
        const int row_blocks = std::max(1, std::min(div_up(lp.m, kBoundThreads), 64));
        const int col_blocks = std::max(1, std::min(div_up(n, kBoundThreads), 64));
        DevBuf<double> yadj(static_cast<size_t>(S) * mm), prow(static_cast<size_t>(S) * row_blocks),
            pcol(static_cast<size_t>(S) * col_blocks);
        BoundArgs a{};
        a.m = lp.m;
        a.n = n;
        a.children = S;
        a.at_ptr = at_ptr.get();
        a.at_idx = at_idx.get();
        a.at_val = at_val.get();
        a.c = c.get();
        a.l = l.get();
        a.u = u.get();
        a.lo = lo.get();
        a.hi = hi.get();
        a.col = dcol.get();
        a.col_lo = dlo.get();
        a.col_hi = dhi.get();
        a.inst = dinst.get();
        a.y = P->yo.get();
        a.yadj = yadj.get();
        a.part_rows = prow.get();
        a.part_cols = pcol.get();
        a.bad = dbad.get();
        a.cert = dcert.get();
        a.obj_const = base.obj_const;
        a.row_blocks = row_blocks;
        a.col_blocks = col_blocks;
        k_bound_rows<<<dim3(row_blocks, S), kBoundThreads, 0, s>>>(a);
        GB_CUDA(cudaGetLastError());
        k_bound_cols<<<dim3(col_blocks, S), kBoundThreads, 0, s>>>(a);
        GB_CUDA(cudaGetLastError());
        k_bound_final<<<div_up(S, 128), 128, 0, s>>>(a);
        GB_CUDA(cudaGetLastError());
        dcert.download(cert.data(), S, s);
        GB_CUDA(cudaStreamSynchronize(s));
    }

    // per-child outcome (src/mip.cpp:750-763)
    for (int k = 0; k < count; ++k) out[k] = gb_branch_cand{};
    for (size_t s = 0; s < ch.size(); ++s) {
        const Child& c = ch[s];
        gb_branch_cand& o = out[c.cand];
        const int d = c.dir;
        if (c.inst < 0) {
            o.status[d] = GB_PRIMAL_INFEASIBLE;
            o.z[d] = INFINITY;
            o.cert[d] = INFINITY;
            continue;
        }
        const gb_result& r = res[c.inst];
        o.status[d] = r.status;
        o.iterations[d] = r.iterations;
        if (r.status == GB_PRIMAL_INFEASIBLE) {
            o.z[d] = INFINITY;
            o.cert[d] = INFINITY;
            continue;
        }
        const double cb = cert[c.inst];
        o.cert[d] = cb;
        // pruned when the certified bound reaches the cutoff, and -- as the
        // reference's dual simplex returns Cutoff once its objective reaches
        // it (src/mip.cpp:755) -- when a solved child's objective does
        if (cb >= cutoff || (r.status == GB_OPTIMAL && r.pobj >= cutoff)) o.z[d] = INFINITY;
        else if (r.status == GB_OPTIMAL) o.z[d] = r.pobj;  // minimisation form (children are)
        else o.z[d] = std::isfinite(cb) ? std::max(node_obj, cb) : node_obj;
    }
    for (int k = 0; k < count; ++k) {
        gb_branch_cand& o = out[k];
        o.score = std::isfinite(o.z[0]) && std::isfinite(o.z[1])
                      ? std::max(o.z[0] - node_obj, kScoreEps) * std::max(o.z[1] - node_obj, kScoreEps)
                      : 0.0;
    }

    // decision (src/mip.cpp:764-783): the first candidate with an infinite
    // side ends the scan
    gb_branch_decision D{};
    D.action = GB_BRANCH_VAR;
    D.var = cand[0];
    D.est[0] = D.est[1] = node_obj;
    D.cert[0] = D.cert[1] = -INFINITY;
    double best = -1.0;
    for (int k = 0; k < count; ++k) {
        const gb_branch_cand& o = out[k];
        const int j = cand[k];
        const bool inf0 = !std::isfinite(o.z[0]), inf1 = !std::isfinite(o.z[1]);
        if (inf0 && inf1) {
            D.action = GB_BRANCH_NODE_INFEASIBLE;
            D.var = j;
            break;
        }
        if (inf0 || inf1) {
            D.action = GB_BRANCH_TIGHTEN;
            D.var = j;
            D.lo = inf0 ? std::ceil(x[j]) : lp.l[j];
            D.hi = inf0 ? lp.u[j] : std::floor(x[j]);
            break;
        }
        if (o.score > best) {
            best = o.score;
            D.var = j;
            D.est[0] = o.z[0];
            D.est[1] = o.z[1];
            D.cert[0] = o.cert[0];
            D.cert[1] = o.cert[1];
        }
    }
    D.children_solved = S;
    D.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (dec) *dec = D;
}

}  // namespace
}  // namespace gb

extern "C" int gb_strong_branch(const gb_lp* lp, const double* x, const double* y, int32_t count, const int32_t* cand,
                                double node_obj, double cutoff, const gb_options* opt, gb_branch_cand* out,
                                gb_branch_decision* decision) {
    return gb::guarded([&] {
        GB_REQUIRE(lp && x && cand && out, "null argument");
        gb_options def;
        gb_default_options(&def);
        gb::strong_branch(*lp, x, y, count, cand, node_obj, cutoff, opt ? opt : &def, out, decision);
    });
}

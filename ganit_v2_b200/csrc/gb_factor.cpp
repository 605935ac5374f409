// Factor-model detection (gb_factor_*): a convex QP written in the lifted form
// of a factor risk model -- free variables f_k with their own curvature,
// each defined by one equality row  a_k f_k + sum_i a_ki x_i = b_k  -- is
// rewritten over x alone with the diagonal-plus-low-rank Hessian the engine's
// Q x kernel takes (Q = 2 (F F^T + diag(D))), and its solution mapped back.
// The reference reads such files (its bench/gen_portfolio.py writes them)
// and solves the lifted form with a CSR Hessian; it has no such rewrite.
//
// With f_k = h_k + g_k' x  (g_ki = -a_ki / a_k, h_k = b_k / a_k):
//   1/2 q_k f_k^2 + c_k f_k = 1/2 q_k (g_k' x)^2 + (q_k h_k + c_k) g_k' x
//                             + 1/2 q_k h_k^2 + c_k h_k,
// so  F[:, k] = sqrt(q_k / 2) g_k,  D = diag(Q_xx) / 2,  c_x += (q_k h_k + c_k) g_k.
// Back: f_k = h_k + g_k' x, and the eliminated row's dual from f_k's
// stationarity (reduced cost c + Q x - A' y = 0): y_k = (c_k + q_k f_k) / a_k.
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ganit_b200.h"

namespace gb {
extern thread_local std::string g_last_error;
namespace {

constexpr int kMaxFactors = 128;  // rank limit of the engine's DPLR kernels

struct Factor {
    int col, row;        // eliminated column f_k and its defining row
    double a, h, q, c;   // a_k, h_k = b_k / a_k, curvature q_k, linear cost c_k
};

}  // namespace

struct FactorModel {
    int n_full = 0, m_full = 0;
    std::vector<int> xcol;          // reduced column -> original column
    std::vector<int> keep_row;      // reduced row -> original row
    std::vector<Factor> fac;
    std::vector<std::vector<std::pair<int, double>>> g;  // per factor: (reduced column, g_ki)
    // reduced problem
    std::vector<int32_t> ptr, idx;
    std::vector<double> val, c, l, u, lo, hi, F, D;
    gb_lp view{};
};

namespace {

std::unique_ptr<FactorModel> detect(const gb_lp& p) {
    if (!p.q_ptr || p.q_rank > 0) throw std::invalid_argument("no CSR Hessian to rewrite");
    if (p.maximize) throw std::invalid_argument("maximisation problems are not rewritten");
    const int m = p.m, n = p.n;
    // diagonal Hessian only
    std::vector<double> qd(n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int t = p.q_ptr[j]; t < p.q_ptr[j + 1]; ++t) {
            if (p.q_idx[t] != j) throw std::invalid_argument("Hessian is not diagonal");
            qd[j] += p.q_val[t];
        }
    for (int j = 0; j < n; ++j)
        if (qd[j] < 0.0) throw std::invalid_argument("Hessian diagonal has a negative entry");
    // column occurrences
    std::vector<int> cnt(n, 0), only_row(n, -1);
    std::vector<double> only_val(n, 0.0);
    for (int i = 0; i < m; ++i)
        for (int t = p.a_ptr[i]; t < p.a_ptr[i + 1]; ++t) {
            const int j = p.a_idx[t];
            if (cnt[j]++ == 0) {
                only_row[j] = i;
                only_val[j] = p.a_val[t];
            }
        }
    std::vector<int> factor_of_row(m, -1);
    std::vector<char> is_factor(n, 0);
    auto model = std::make_unique<FactorModel>();
    for (int j = 0; j < n; ++j) {
        const int r = only_row[j];
        if (!(cnt[j] == 1 && qd[j] > 0.0 && std::isinf(p.l[j]) && p.l[j] < 0 && std::isinf(p.u[j]) && p.u[j] > 0))
            continue;
        if (!(p.lo[r] == p.hi[r] && std::isfinite(p.lo[r]) && only_val[j] != 0.0)) continue;
        if (factor_of_row[r] >= 0) {  // a second candidate in the row: neither is a clean factor
            is_factor[model->fac[factor_of_row[r]].col] = 0;
            factor_of_row[r] = -2;
            continue;
        }
        if (factor_of_row[r] == -2) continue;
        factor_of_row[r] = static_cast<int>(model->fac.size());
        is_factor[j] = 1;
        model->fac.push_back({j, r, only_val[j], p.lo[r] / only_val[j], qd[j], p.c[j]});
    }
    // drop candidates invalidated by a second candidate in their row
    std::vector<Factor> kept;
    for (const Factor& f : model->fac)
        if (is_factor[f.col]) kept.push_back(f);
    model->fac.swap(kept);
    const int K = static_cast<int>(model->fac.size());
    if (K == 0) throw std::invalid_argument("no factor structure found");
    if (K > kMaxFactors) throw std::invalid_argument("more than 128 factors");
    std::vector<int> red_col(n, -1), red_row(m, -1);
    std::vector<char> drop_row(m, 0);
    for (const Factor& f : model->fac) drop_row[f.row] = 1;
    for (int j = 0; j < n; ++j)
        if (!is_factor[j]) {
            red_col[j] = static_cast<int>(model->xcol.size());
            model->xcol.push_back(j);
        }
    for (int i = 0; i < m; ++i)
        if (!drop_row[i]) {
            red_row[i] = static_cast<int>(model->keep_row.size());
            model->keep_row.push_back(i);
        }
    const int nx = static_cast<int>(model->xcol.size()), mr = static_cast<int>(model->keep_row.size());
    model->n_full = n;
    model->m_full = m;
    // g_k from the defining rows
    model->g.resize(K);
    for (int k = 0; k < K; ++k) {
        const Factor& f = model->fac[k];
        for (int t = p.a_ptr[f.row]; t < p.a_ptr[f.row + 1]; ++t) {
            const int j = p.a_idx[t];
            if (j == f.col) continue;
            model->g[k].emplace_back(red_col[j], -p.a_val[t] / f.a);
        }
    }
    // reduced problem
    FactorModel& R = *model;
    R.ptr.assign(mr + 1, 0);
    for (int r = 0; r < mr; ++r) {
        const int i = R.keep_row[r];
        for (int t = p.a_ptr[i]; t < p.a_ptr[i + 1]; ++t) {
            const int j = p.a_idx[t];
            if (is_factor[j]) throw std::invalid_argument("a factor column appears in a kept row");
            R.idx.push_back(red_col[j]);
            R.val.push_back(p.a_val[t]);
        }
        R.ptr[r + 1] = static_cast<int32_t>(R.idx.size());
        R.lo.push_back(p.lo[i]);
        R.hi.push_back(p.hi[i]);
    }
    R.c.resize(nx);
    R.l.resize(nx);
    R.u.resize(nx);
    R.D.resize(nx);
    for (int t = 0; t < nx; ++t) {
        const int j = R.xcol[t];
        R.c[t] = p.c[j];
        R.l[t] = p.l[j];
        R.u[t] = p.u[j];
        R.D[t] = 0.5 * qd[j];
    }
    R.F.assign(static_cast<size_t>(nx) * K, 0.0);
    double obj_const = p.obj_const;
    for (int k = 0; k < K; ++k) {
        const Factor& f = R.fac[k];
        const double s = std::sqrt(0.5 * f.q), lin = f.q * f.h + f.c;
        for (const auto& [t, gv] : R.g[k]) {
            R.F[static_cast<size_t>(t) * K + k] += s * gv;
            R.c[t] += lin * gv;
        }
        obj_const += 0.5 * f.q * f.h * f.h + f.c * f.h;
    }
    gb_lp& v = R.view;
    std::memset(&v, 0, sizeof(v));
    v.m = mr;
    v.n = nx;
    v.a_ptr = R.ptr.data();
    v.a_idx = R.idx.data();
    v.a_val = R.val.data();
    v.c = R.c.data();
    v.l = R.l.data();
    v.u = R.u.data();
    v.lo = R.lo.data();
    v.hi = R.hi.data();
    v.obj_const = obj_const;
    v.q_rank = K;
    v.q_F = R.F.data();
    v.q_D = R.D.data();
    return model;
}

}  // namespace
}  // namespace gb

struct gb_factor {
    std::unique_ptr<gb::FactorModel> m;
};

extern "C" {

int gb_factor_detect(const gb_lp* qp, gb_factor** out) {
    try {
        if (!qp || !out) throw std::runtime_error("null argument");
        *out = nullptr;
        auto m = gb::detect(*qp);
        *out = new gb_factor{std::move(m)};
        return GB_OK;
    } catch (const std::invalid_argument& e) {
        gb::g_last_error = e.what();
        return GB_ERR_UNSUPPORTED;
    } catch (const std::bad_alloc&) {
        gb::g_last_error = "host allocation failed";
        return GB_ERR_NOMEM;
    } catch (const std::exception& e) {
        gb::g_last_error = e.what();
        return GB_ERR_INVALID;
    }
}

const gb_lp* gb_factor_lp(const gb_factor* f) { return f ? &f->m->view : nullptr; }

int gb_factor_expand(const gb_factor* f, const double* x, const double* y, double* x_full, double* y_full) {
    if (!f || !x || !y || !x_full || !y_full) {
        gb::g_last_error = "null argument";
        return GB_ERR_INVALID;
    }
    const gb::FactorModel& R = *f->m;
    for (size_t t = 0; t < R.xcol.size(); ++t) x_full[R.xcol[t]] = x[t];
    for (size_t r = 0; r < R.keep_row.size(); ++r) y_full[R.keep_row[r]] = y[r];
    for (size_t k = 0; k < R.fac.size(); ++k) {
        const auto& fk = R.fac[k];
        double v = fk.h;
        for (const auto& [t, gv] : R.g[k]) v += gv * x[t];
        x_full[fk.col] = v;
        y_full[fk.row] = (fk.c + fk.q * v) / fk.a;
    }
    return GB_OK;
}

void gb_factor_free(gb_factor* f) { delete f; }

}  // extern "C"

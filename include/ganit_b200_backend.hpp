// ganit_b200_backend.hpp -- the Backend concept of GANIT's PDHG driver on B200 kernels.
//
// src/pdhg_impl.hpp (run_pdhg / pdhg_phase / pdhg_evaluate) is written against a
// duck-typed backend B (used at pdhg_impl.hpp:73-84, 92-118, 133-137, 145-146,
// 178-194, 207-220; implemented in the reference by CudaBackend<M,V>,
// src/backend_cuda.cu:286-378, and CpuBackendT<M,R>, src/backend_cpu.cpp:38-156).
// B200Backend<M,V> implements that concept with the gb_backend_* entry points of
// ganit_b200.h, so the reference's own driver runs unchanged on B200:
//
//     #include "pdhg_impl.hpp"
//     #include "ganit_b200_backend.hpp"
//     ganit::Result r = ganit::run_pdhg<gb::B200Backend<float, float>, gb::B200Backend<float, double>,
//                                       gb::B200Backend<double, double>>(lp, opt, "b200");
//
// Header-only; needs ganit::ScaledLP (src/scaling.hpp) and libganit_b200.so.
// Errors from the library become std::runtime_error, as CudaBackend's do.
#pragma once
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "ganit_b200.h"
#include "scaling.hpp"

namespace gb {

inline void check(int rc) {
    if (rc != GB_OK) throw std::runtime_error(std::string("libganit_b200: ") + gb_last_error());
}

template <class M, class V>
class B200Backend {
    static_assert(std::is_same<M, float>::value || std::is_same<M, double>::value, "M is float or double");
    static_assert(std::is_same<V, float>::value || std::is_same<V, double>::value, "V is float or double");

   public:
    // Move-only owning device vector (the concept's Vec; std::swap-able).
    class Vec {
       public:
        Vec() = default;
        explicit Vec(gb_vec* h) : h_(h) {}
        ~Vec() { if (h_) gb_vec_destroy(h_); }
        Vec(const Vec&) = delete;
        Vec& operator=(const Vec&) = delete;
        Vec(Vec&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
        Vec& operator=(Vec&& o) noexcept {
            std::swap(h_, o.h_);
            return *this;
        }
        gb_vec* get() const { return h_; }
        size_t size() const { return h_ ? static_cast<size_t>(gb_vec_size(h_)) : 0; }

       private:
        gb_vec* h_ = nullptr;
    };

    explicit B200Backend(const ganit::ScaledLP& s) {
        gb_scaled_lp g{};
        g.m = s.m;
        g.n = s.n;
        g.a_ptr = s.A.ptr.data();
        g.a_idx = s.A.idx.data();
        g.a_val = s.A.val.data();
        g.at_ptr = s.AT.ptr.data();
        g.at_idx = s.AT.idx.data();
        g.at_val = s.AT.val.data();
        if (s.has_q()) {
            g.q_ptr = s.Q.ptr.data();
            g.q_idx = s.Q.idx.data();
            g.q_val = s.Q.val.data();
        }
        g.c = s.c.data();
        g.l = s.l.data();
        g.u = s.u.data();
        g.lo = s.lo.data();
        g.hi = s.hi.data();
        g.rres = s.Rres.data();
        g.cres = s.Cres.data();
        check(gb_backend_create(&g, std::is_same<M, float>::value ? GB_F32 : GB_F64,
                                std::is_same<V, float>::value ? GB_F32 : GB_F64, &b_));
    }
    ~B200Backend() { gb_backend_destroy(b_); }
    B200Backend(const B200Backend&) = delete;
    B200Backend& operator=(const B200Backend&) = delete;

    Vec zeros(int k) {
        gb_vec* h = nullptr;
        check(gb_vec_zeros(b_, k, &h));
        return Vec(h);
    }
    Vec from_host(const std::vector<double>& v) {
        gb_vec* h = nullptr;
        check(gb_vec_from_host(b_, v.data(), static_cast<int>(v.size()), &h));
        return Vec(h);
    }
    std::vector<double> to_host(const Vec& v) {
        std::vector<double> out(v.size());
        check(gb_vec_to_host(b_, v.get(), out.data()));
        return out;
    }
    void copy(const Vec& src, Vec& dst) { check(gb_copy(b_, src.get(), dst.get())); }
    void fill(Vec& v, double a) { check(gb_fill(b_, v.get(), a)); }
    void spmv_A(const Vec& x, Vec& ax) { check(gb_spmv_A(b_, x.get(), ax.get())); }
    void spmv_AT(const Vec& y, Vec& aty) { check(gb_spmv_AT(b_, y.get(), aty.get())); }
    void spmv_Q(const Vec& x, Vec& qx) { check(gb_spmv_Q(b_, x.get(), qx.get())); }
    void primal_step(const Vec& x, const Vec& aty, const Vec* qx, double tau, Vec& xn, Vec& xbar, Vec& sumx) {
        check(gb_primal_step(b_, x.get(), aty.get(), qx ? qx->get() : nullptr, tau, xn.get(), xbar.get(),
                             sumx.get()));
    }
    void dual_step(const Vec& y, const Vec& axbar, double sigma, Vec& yn, Vec& sumy) {
        check(gb_dual_step(b_, y.get(), axbar.get(), sigma, yn.get(), sumy.get()));
    }
    void sub(const Vec& a, const Vec& c, Vec& d) { check(gb_sub(b_, a.get(), c.get(), d.get())); }
    void scale_into(const Vec& src, double a, Vec& dst) { check(gb_scale_into(b_, src.get(), a, dst.get())); }
    double primal_res2(const Vec& ax) {
        double r = 0;
        check(gb_primal_res2(b_, ax.get(), &r));
        return r;
    }
    void dual_res(const Vec& aty, const Vec* qx, double& rd2, double& vobj, bool with_c = true) {
        check(gb_dual_res(b_, aty.get(), qx ? qx->get() : nullptr, with_c ? 1 : 0, &rd2, &vobj));
    }
    double row_dual_obj(const Vec& y) {
        double r = 0;
        check(gb_row_dual_obj(b_, y.get(), &r));
        return r;
    }
    double dot(const Vec& a, const Vec& c) {
        double r = 0;
        check(gb_dot(b_, a.get(), c.get(), &r));
        return r;
    }
    double dot_c(const Vec& x) {
        double r = 0;
        check(gb_dot_c(b_, x.get(), &r));
        return r;
    }
    double diff2(const Vec& a, const Vec& c) {
        double r = 0;
        check(gb_diff2(b_, a.get(), c.get(), &r));
        return r;
    }

   private:
    gb_backend* b_ = nullptr;
};

}  // namespace gb

// MPS / QPS problem files into the engine's gb_lp (gb_read_mps).
//
// Same format rules as the reference reader (src/mps.cpp:69-272): free-form
// whitespace-separated fields; sections NAME, OBJSENSE (header argument or
// next line), ROWS, COLUMNS ('MARKER' INTORG/INTEND lines mark the columns
// between them integer; bound types UI, LI and BV do too),
// RHS, RANGES, BOUNDS, QUADOBJ (lower triangle, mirrored), QMATRIX/QSECTION
// (full), ENDATA; the first N row is the objective, further N rows are
// ignored; an objective RHS entry v gives obj_const = -v; RHS / RANGES lines
// may omit the set name; bounds UP/UI (a negative UP on a column whose lower
// bound was never set makes that lower bound -inf), LO/LI, FX, FR, MI, PL, BV;
// ranges: E rows widen to the side of the range's sign, L rows get
// lo = b - |r|, G rows hi = b + |r|.  Matrix entries are assembled row by
// row, sorted by column, duplicates summed, exact zeros dropped.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/ganit_b200.h"

namespace gb {
extern thread_local std::string g_last_error;
namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

struct Entry {
    int r, c;
    double v;
};

// CSR of rows x cols from triplets: per row sorted by column (stable, so
// duplicates are summed in file order), duplicates merged, zeros dropped.
void assemble(int rows, std::vector<Entry>& t, std::vector<int32_t>& ptr, std::vector<int32_t>& idx,
              std::vector<double>& val) {
    std::vector<int> cnt(rows + 1, 0);
    for (const Entry& e : t) ++cnt[e.r + 1];
    for (int i = 0; i < rows; ++i) cnt[i + 1] += cnt[i];
    std::vector<Entry> byrow(t.size());
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (const Entry& e : t) byrow[pos[e.r]++] = e;
    ptr.assign(rows + 1, 0);
    idx.clear();
    val.clear();
    for (int i = 0; i < rows; ++i) {
        auto b = byrow.begin() + cnt[i], e = byrow.begin() + cnt[i + 1];
        std::stable_sort(b, e, [](const Entry& x, const Entry& y) { return x.c < y.c; });
        for (auto it = b; it != e;) {
            const int c = it->c;
            double s = 0.0;
            for (; it != e && it->c == c; ++it) s += it->v;
            if (s != 0.0) {
                idx.push_back(c);
                val.push_back(s);
            }
        }
        ptr[i + 1] = static_cast<int32_t>(idx.size());
    }
}

class Parser {
   public:
    explicit Parser(const std::string& path) : path_(path) {}

    void run() {
        std::ifstream f(path_, std::ios::binary);
        if (!f) throw std::runtime_error("cannot open '" + path_ + "'");
        std::string line;
        while (std::getline(f, line)) {
            ++lineno_;
            if (!line.empty() && line.back() == '\r') line.pop_back();
            if (line.empty() || line[0] == '*') continue;
            fields(line);
            if (tok_.empty()) continue;
            if (!std::isspace(static_cast<unsigned char>(line[0]))) {
                if (header()) break;  // ENDATA
                continue;
            }
            body();
        }
        finish();
    }

    // outputs
    std::string name;
    int m = 0, n = 0;
    bool maximize = false;
    double obj_const = 0.0;
    std::vector<int32_t> a_ptr, a_idx, q_ptr, q_idx;
    std::vector<double> a_val, q_val, c, l, u, lo, hi;
    std::vector<unsigned char> is_int;

   private:
    enum Section { kNone, kName, kSense, kRows, kCols, kRhs, kRanges, kBounds, kQuadObj, kQMatrix };

    [[noreturn]] void fail(const std::string& what) const {
        throw std::runtime_error(path_ + ":" + std::to_string(lineno_) + ": " + what);
    }
    void fields(const std::string& line) {
        tok_.clear();
        size_t i = 0;
        while (i < line.size()) {
            while (i < line.size() && std::isspace(static_cast<unsigned char>(line[i]))) ++i;
            const size_t s = i;
            while (i < line.size() && !std::isspace(static_cast<unsigned char>(line[i]))) ++i;
            if (i > s) tok_.emplace_back(line, s, i - s);
        }
    }
    double number(const std::string& s) const {
        char* end = nullptr;
        const double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str()) fail("bad number '" + s + "'");
        return v;
    }
    int column(const std::string& s) const {
        auto it = cols_.find(s);
        if (it == cols_.end()) fail("unknown column '" + s + "'");
        return it->second;
    }
    static bool is_max(const std::string& s) { return s == "MAX" || s == "MAXIMIZE"; }

    bool header() {
        const std::string& h = tok_[0];
        if (h == "NAME") {
            sec_ = kName;
            if (tok_.size() > 1) name = tok_[1];
        } else if (h == "OBJSENSE" || h == "OBJSENCE") {
            sec_ = kSense;
            if (tok_.size() > 1) maximize = is_max(tok_[1]);
        } else if (h == "ROWS") sec_ = kRows;
        else if (h == "COLUMNS") sec_ = kCols;
        else if (h == "RHS") sec_ = kRhs;
        else if (h == "RANGES") sec_ = kRanges;
        else if (h == "BOUNDS") sec_ = kBounds;
        else if (h == "QUADOBJ") sec_ = kQuadObj;
        else if (h == "QMATRIX" || h == "QSECTION") sec_ = kQMatrix;
        else if (h == "ENDATA") return true;
        else fail("unknown section '" + h + "'");
        return false;
    }

    void body() {
        switch (sec_) {
            case kSense: maximize = is_max(tok_[0]); break;
            case kRows: row_line(); break;
            case kCols: column_line(); break;
            case kRhs:
            case kRanges: rhs_line(sec_ == kRhs); break;
            case kBounds: bound_line(); break;
            case kQuadObj:
            case kQMatrix: quad_line(sec_ == kQuadObj); break;
            default: break;
        }
    }

    void row_line() {
        if (tok_.size() < 2) fail("bad ROWS line");
        const char t = static_cast<char>(std::toupper(static_cast<unsigned char>(tok_[0][0])));
        if (t == 'N') {
            if (obj_.empty()) obj_ = tok_[1];
            else extra_n_.insert(tok_[1]);
            return;
        }
        rows_[tok_[1]] = m++;
        row_type_.push_back(t);
        rhs_.push_back(0.0);
        range_.push_back(std::nan(""));
    }

    void column_line() {
        if (tok_.size() >= 3 && tok_[1] == "'MARKER'") {
            if (tok_[2] == "'INTORG'") int_mode_ = true;
            else if (tok_[2] == "'INTEND'") int_mode_ = false;
            return;
        }
        if (tok_[0] != cur_name_) {
            cur_name_ = tok_[0];
            cur_ = n++;
            cols_[cur_name_] = cur_;
            c.push_back(0.0);
            l.push_back(0.0);
            u.push_back(kInf);
            is_int.push_back(int_mode_ ? 1 : 0);
            lower_given_.push_back(0);
        }
        for (size_t k = 1; k + 1 < tok_.size(); k += 2) {
            const double v = number(tok_[k + 1]);
            if (tok_[k] == obj_) {
                c[cur_] += v;
                continue;
            }
            auto it = rows_.find(tok_[k]);
            if (it == rows_.end()) {
                if (extra_n_.count(tok_[k])) continue;
                fail("unknown row '" + tok_[k] + "'");
            }
            a_.push_back({it->second, cur_, v});
        }
    }

    void rhs_line(bool rhs) {
        for (size_t k = tok_.size() % 2; k + 1 < tok_.size(); k += 2) {  // odd count: leading set name
            const double v = number(tok_[k + 1]);
            if (tok_[k] == obj_) {
                if (rhs) obj_const = -v;
                continue;
            }
            auto it = rows_.find(tok_[k]);
            if (it == rows_.end()) {
                if (extra_n_.count(tok_[k])) continue;
                fail("unknown row '" + tok_[k] + "'");
            }
            (rhs ? rhs_ : range_)[it->second] = v;
        }
    }

    void bound_line() {
        const std::string& t = tok_[0];
        const bool valued = t == "UP" || t == "LO" || t == "FX" || t == "LI" || t == "UI";
        std::string cname;
        double v = 0.0;
        if (valued) {
            if (tok_.size() >= 4) {
                cname = tok_[2];
                v = number(tok_[3]);
            } else if (tok_.size() == 3) {
                cname = tok_[1];
                v = number(tok_[2]);
            } else {
                fail("bad BOUNDS line");
            }
        } else {
            if (tok_.size() < 2) fail("bad BOUNDS line");
            cname = tok_.size() >= 3 ? tok_[2] : tok_[1];
        }
        const int j = column(cname);
        if (t == "UP" || t == "UI") {
            u[j] = v;
            if (v < 0 && l[j] == 0.0 && !lower_given_[j]) l[j] = -kInf;
            if (t == "UI") is_int[j] = 1;
        } else if (t == "LO" || t == "LI") {
            l[j] = v;
            lower_given_[j] = 1;
            if (t == "LI") is_int[j] = 1;
        } else if (t == "FX") {
            l[j] = u[j] = v;
            lower_given_[j] = 1;
        } else if (t == "FR") {
            l[j] = -kInf;
            u[j] = kInf;
            lower_given_[j] = 1;
        } else if (t == "MI") {
            l[j] = -kInf;
            lower_given_[j] = 1;
        } else if (t == "PL") {
            u[j] = kInf;
        } else if (t == "BV") {
            l[j] = 0.0;
            u[j] = 1.0;
            lower_given_[j] = 1;
            is_int[j] = 1;
        } else {
            fail("unknown bound type '" + t + "'");
        }
    }

    void quad_line(bool lower_triangle) {
        if (tok_.size() < 3) fail("bad quadratic line");
        const int a = column(tok_[0]), b = column(tok_[1]);
        const double v = number(tok_[2]);
        q_.push_back({a, b, v});
        if (lower_triangle && a != b) q_.push_back({b, a, v});
    }

    void finish() {
        lo.assign(m, 0.0);
        hi.assign(m, 0.0);
        for (int i = 0; i < m; ++i) {
            const double b = rhs_[i], r = range_[i];
            switch (row_type_[i]) {
                case 'E': lo[i] = hi[i] = b; break;
                case 'L': lo[i] = -kInf; hi[i] = b; break;
                case 'G': lo[i] = b; hi[i] = kInf; break;
                default: throw std::runtime_error(path_ + ": unknown row type '" + std::string(1, row_type_[i]) + "'");
            }
            if (std::isnan(r)) continue;
            if (row_type_[i] == 'E') (r > 0 ? hi[i] : lo[i]) = b + r;
            else if (row_type_[i] == 'L') lo[i] = b - std::fabs(r);
            else hi[i] = b + std::fabs(r);
        }
        assemble(m, a_, a_ptr, a_idx, a_val);
        if (!q_.empty()) assemble(n, q_, q_ptr, q_idx, q_val);
    }

    std::string path_;
    int lineno_ = 0;
    Section sec_ = kNone;
    std::vector<std::string> tok_;
    std::string obj_, cur_name_;
    int cur_ = -1;
    bool int_mode_ = false;
    std::unordered_map<std::string, int> rows_, cols_;
    std::unordered_set<std::string> extra_n_;
    std::vector<char> row_type_, lower_given_;
    std::vector<double> rhs_, range_;
    std::vector<Entry> a_, q_;
};

}  // namespace
}  // namespace gb

struct gb_model {
    gb::Parser p;
    gb_lp view;
    explicit gb_model(const std::string& path) : p(path) {}
};

extern "C" {

int gb_read_mps(const char* path, gb_model** out) {
    try {
        if (!path || !out) throw std::invalid_argument("null argument");
        *out = nullptr;
        auto mdl = std::make_unique<gb_model>(path);
        mdl->p.run();
        gb::Parser& p = mdl->p;
        gb_lp& v = mdl->view;
        std::memset(&v, 0, sizeof(v));
        v.m = p.m;
        v.n = p.n;
        v.a_ptr = p.a_ptr.data();
        v.a_idx = p.a_idx.data();
        v.a_val = p.a_val.data();
        v.c = p.c.data();
        v.l = p.l.data();
        v.u = p.u.data();
        v.lo = p.lo.data();
        v.hi = p.hi.data();
        v.obj_const = p.obj_const;
        v.maximize = p.maximize ? 1 : 0;
        if (!p.q_val.empty()) {
            v.q_ptr = p.q_ptr.data();
            v.q_idx = p.q_idx.data();
            v.q_val = p.q_val.data();
        }
        *out = mdl.release();
        return GB_OK;
    } catch (const std::bad_alloc&) {
        gb::g_last_error = "host allocation failed";
        return GB_ERR_NOMEM;
    } catch (const std::exception& e) {
        gb::g_last_error = e.what();
        return GB_ERR_INVALID;
    }
}

const gb_lp* gb_model_lp(const gb_model* mdl) { return mdl ? &mdl->view : nullptr; }

const char* gb_model_name(const gb_model* mdl) { return mdl ? mdl->p.name.c_str() : nullptr; }

const unsigned char* gb_model_is_int(const gb_model* mdl) { return mdl ? mdl->p.is_int.data() : nullptr; }

void gb_model_free(gb_model* mdl) { delete mdl; }

}  // extern "C"

// MPS reader feeding the C ABI (pdlpx_read_mps).
//
// Reads the free-format MPS files mipx reads (src/io/mps_reader.cpp), plain or
// gzip-compressed, with the same meaning of every section:
//   * lines starting with '*' or '$' are comments; " $" starts a trailing comment;
//   * ROWS (and LAZYCONS / USERCUTS, read as ordinary rows): N / L / G / E; an
//     N row is the objective (any N row's entries go to the objective);
//   * COLUMNS with 'MARKER' 'INTORG' / 'INTEND' integer blocks;
//   * RHS: a value on the objective row sets the objective offset to -value;
//   * RANGES: L rows get [rhs - |r|, rhs], G rows [rhs, rhs + |r|], E rows
//     [rhs, rhs + r] for r > 0 and [rhs + r, rhs] for r < 0;
//   * BOUNDS: LO, UP, FX, FR, MI, PL, BV (binary), LI / UI (integer), SC / SI
//     (semi-continuous: the LP relaxation keeps [0, upper]);
//   * columns default to [0, +inf); no OBJSENSE section (minimisation), as in mipx.
// Entries of a row are sorted by column, duplicates summed and exact zeros
// dropped, like mipx's CSR assembly.  The result is an owned pdlpx_gen_lp
// (released with pdlpx_free_lp); is_int marks integer and binary columns.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "pdlpx.h"

namespace pdlpx {
void setGlobalError(const std::string& msg);

namespace {

// Line source over gzread (reads plain files unchanged).
class GzLines {
public:
    explicit GzLines(const char* path) : f_(gzopen(path, "rb")) {
        if (f_) gzbuffer(f_, 1 << 20);
    }
    ~GzLines() {
        if (f_) gzclose(f_);
    }
    bool ok() const { return f_ != nullptr; }
    bool next(std::string& line) {
        line.clear();
        while (true) {
            if (pos_ >= len_) {
                if (eof_) return !line.empty();
                const int got = gzread(f_, buf_, sizeof(buf_));
                if (got <= 0) {
                    eof_ = true;
                    if (got < 0) err_ = true;
                    return !line.empty();
                }
                len_ = static_cast<size_t>(got);
                pos_ = 0;
            }
            const char* s = buf_ + pos_;
            const void* nl = std::memchr(s, '\n', len_ - pos_);
            if (nl) {
                const size_t k = static_cast<const char*>(nl) - s;
                line.append(s, k);
                pos_ += k + 1;
                if (!line.empty() && line.back() == '\r') line.pop_back();
                return true;
            }
            line.append(s, len_ - pos_);
            pos_ = len_;
        }
    }
    bool failed() const { return err_; }

private:
    gzFile f_;
    char buf_[1 << 16];
    size_t pos_ = 0, len_ = 0;
    bool eof_ = false, err_ = false;
};

int split(std::string_view s, std::string_view (&tok)[8]) {
    int n = 0;
    size_t i = 0;
    while (i < s.size() && n < 8) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
        if (i >= s.size()) break;
        const size_t b = i;
        while (i < s.size() && s[i] != ' ' && s[i] != '\t') ++i;
        tok[n++] = s.substr(b, i - b);
    }
    return n;
}

bool number(std::string_view s, double& v) {
    std::string t(s);
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end != t.c_str() && *end == '\0';
}

enum class Sec { None, Rows, Columns, Rhs, Ranges, Bounds, End };

template <class T>
T* own(const std::vector<T>& v) {
    T* p = static_cast<T*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
    if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

}  // namespace

int32_t readMps(const char* path, pdlpx_gen_lp* out, std::string& err) {
    std::memset(out, 0, sizeof(*out));
    GzLines in(path);
    if (!in.ok()) {
        err = std::string("cannot open ") + path;
        return PDLPX_E_INVALID;
    }
    const double inf = std::numeric_limits<double>::infinity();
    std::unordered_map<std::string, int32_t> rows, cols;  // row name -> index (-1: objective)
    std::vector<char> sense;
    std::vector<int32_t> er, ec;  // entries (row, column, value) in file order
    std::vector<double> ev, obj, lb, ub, rhs, rng;
    std::vector<int32_t> integer;
    double offset = 0.0;
    bool intblock = false;
    Sec sec = Sec::None;
    auto column = [&](std::string_view name) {
        auto it = cols.find(std::string(name));
        if (it != cols.end()) return it->second;
        const int32_t j = static_cast<int32_t>(obj.size());
        cols.emplace(std::string(name), j);
        obj.push_back(0.0);
        lb.push_back(0.0);
        ub.push_back(inf);
        integer.push_back(0);
        return j;
    };
    std::string line;
    std::string_view tok[8];
    int64_t lineno = 0;
    while (sec != Sec::End && in.next(line)) {
        ++lineno;
        if (line.empty() || line[0] == '*' || line[0] == '$') continue;
        for (size_t p = 1; p < line.size(); ++p)
            if (line[p] == '$' && (line[p - 1] == ' ' || line[p - 1] == '\t')) {
                line.resize(p);
                break;
            }
        const int n = split(line, tok);
        if (n == 0) continue;
        if (line[0] != ' ' && line[0] != '\t') {  // section header
            const std::string_view h = tok[0];
            if (h == "ROWS" || h == "LAZYCONS" || h == "USERCUTS")
                sec = Sec::Rows;
            else if (h == "COLUMNS")
                sec = Sec::Columns;
            else if (h == "RHS")
                sec = Sec::Rhs;
            else if (h == "RANGES")
                sec = Sec::Ranges;
            else if (h == "BOUNDS")
                sec = Sec::Bounds;
            else if (h == "ENDATA")
                sec = Sec::End;
            else
                sec = Sec::None;  // NAME, OBJSENSE and unknown sections: skipped
            continue;
        }
        switch (sec) {
            case Sec::Rows: {
                if (n < 2) break;
                const char t = tok[0][0];
                if (t == 'N') {
                    rows.emplace(std::string(tok[1]), -1);
                } else {
                    rows.emplace(std::string(tok[1]), static_cast<int32_t>(sense.size()));
                    sense.push_back(t);
                }
                break;
            }
            case Sec::Columns: {
                if (n >= 3 && tok[1] == "'MARKER'") {
                    if (tok[2] == "'INTORG'") intblock = true;
                    if (tok[2] == "'INTEND'") intblock = false;
                    break;
                }
                if (n < 3) break;
                const int32_t j = column(tok[0]);
                if (intblock) integer[j] = 1;
                for (int k = 1; k + 1 < n; k += 2) {
                    auto it = rows.find(std::string(tok[k]));
                    double v;
                    if (it == rows.end()) {
                        err = "MPS line " + std::to_string(lineno) + ": unknown row '" + std::string(tok[k]) + "'";
                        return PDLPX_E_INVALID;
                    }
                    if (!number(tok[k + 1], v)) {
                        err = "MPS line " + std::to_string(lineno) + ": bad number '" + std::string(tok[k + 1]) + "'";
                        return PDLPX_E_INVALID;
                    }
                    if (it->second < 0) {
                        obj[j] = v;
                    } else {
                        er.push_back(it->second);
                        ec.push_back(j);
                        ev.push_back(v);
                    }
                }
                break;
            }
            case Sec::Rhs:
            case Sec::Ranges: {
                if (n < 3) break;
                for (int k = 1; k + 1 < n; k += 2) {
                    auto it = rows.find(std::string(tok[k]));
                    double v;
                    if (it == rows.end() || !number(tok[k + 1], v)) continue;
                    if (it->second < 0) {
                        if (sec == Sec::Rhs) offset = -v;
                        continue;
                    }
                    std::vector<double>& dst = sec == Sec::Rhs ? rhs : rng;
                    if (static_cast<size_t>(it->second) >= dst.size()) dst.resize(it->second + 1, 0.0);
                    dst[it->second] = v;
                }
                break;
            }
            case Sec::Bounds: {
                if (n < 3) break;
                const std::string_view t = tok[0];
                const int32_t j = column(tok[2]);
                double v = 0.0;
                const bool val = n >= 4 && number(tok[3], v);
                if (t == "LO" && val) {
                    lb[j] = v;
                } else if (t == "UP" && val) {
                    ub[j] = v;
                } else if (t == "FX" && val) {
                    lb[j] = ub[j] = v;
                } else if (t == "FR") {
                    lb[j] = -inf;
                    ub[j] = inf;
                } else if (t == "MI") {
                    lb[j] = -inf;
                } else if (t == "PL") {
                    ub[j] = inf;
                } else if (t == "BV") {
                    lb[j] = 0.0;
                    ub[j] = 1.0;
                    integer[j] = 1;
                } else if (t == "LI" && val) {
                    lb[j] = v;
                    integer[j] = 1;
                } else if (t == "UI" && val) {
                    ub[j] = v;
                    integer[j] = 1;
                } else if (t == "SC" || t == "SI") {
                    lb[j] = 0.0;  // semi-continuous: the relaxation is [0, upper]
                }
                break;
            }
            default:
                break;
        }
    }
    if (in.failed()) {
        err = std::string("read error in ") + path;
        return PDLPX_E_INVALID;
    }
    const int32_t m = static_cast<int32_t>(sense.size()), ncol = static_cast<int32_t>(obj.size());
    // CSR: rows in order, columns sorted inside a row, duplicates summed, zeros dropped
    std::vector<int32_t> ptr(static_cast<size_t>(m) + 1, 0);
    for (int32_t r : er) ++ptr[r + 1];
    for (int32_t i = 0; i < m; ++i) ptr[i + 1] += ptr[i];
    std::vector<int32_t> ci(er.size());
    std::vector<double> cv(er.size());
    {
        std::vector<int32_t> at(ptr.begin(), ptr.end() - 1);
        for (size_t k = 0; k < er.size(); ++k) {
            const int32_t p = at[er[k]]++;
            ci[p] = ec[k];
            cv[p] = ev[k];
        }
    }
    std::vector<int32_t> rp(static_cast<size_t>(m) + 1, 0), idx;
    std::vector<double> val;
    idx.reserve(ci.size());
    val.reserve(ci.size());
    std::vector<std::pair<int32_t, double>> row;
    for (int32_t i = 0; i < m; ++i) {
        row.clear();
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) row.emplace_back(ci[k], cv[k]);
        std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < row.size();) {
            const int32_t c = row[k].first;
            double s = 0.0;
            for (; k < row.size() && row[k].first == c; ++k) s += row[k].second;
            if (s != 0.0) {
                idx.push_back(c);
                val.push_back(s);
            }
        }
        rp[i + 1] = static_cast<int32_t>(idx.size());
    }
    rhs.resize(m, 0.0);
    rng.resize(m, 0.0);
    std::vector<double> rl(m), ru(m);
    for (int32_t i = 0; i < m; ++i) {
        const double b = rhs[i], r = rng[i];
        switch (sense[i]) {
            case 'L':
                ru[i] = b;
                rl[i] = r != 0.0 ? b - std::fabs(r) : -inf;
                break;
            case 'G':
                rl[i] = b;
                ru[i] = r != 0.0 ? b + std::fabs(r) : inf;
                break;
            case 'E':
                rl[i] = r < 0.0 ? b + r : b;
                ru[i] = r > 0.0 ? b + r : b;
                break;
            default:
                rl[i] = -inf;
                ru[i] = inf;
                break;
        }
    }
    out->m = m;
    out->n = ncol;
    out->nnz = static_cast<int32_t>(idx.size());
    out->row_ptr = own(rp);
    out->col_idx = own(idx);
    out->val = own(val);
    out->obj = own(obj);
    out->col_lb = own(lb);
    out->col_ub = own(ub);
    out->row_lb = own(rl);
    out->row_ub = own(ru);
    out->x0 = nullptr;
    out->is_int = own(integer);
    out->obj_offset = offset;
    if (!out->row_ptr || !out->col_idx || !out->val || !out->obj || !out->col_lb || !out->col_ub || !out->row_lb ||
        !out->row_ub || !out->is_int) {
        pdlpx_free_lp(out);
        err = "host allocation failed";
        return PDLPX_E_NOMEM;
    }
    return PDLPX_OK;
}

}  // namespace pdlpx

extern "C" int32_t pdlpx_read_mps(const char* path, pdlpx_gen_lp* out) {
    if (path == nullptr || out == nullptr) {
        pdlpx::setGlobalError("null path or output");
        return PDLPX_E_INVALID;
    }
    std::string err;
    int32_t rc;
    try {
        rc = pdlpx::readMps(path, out, err);
    } catch (const std::bad_alloc&) {
        rc = PDLPX_E_NOMEM;
        err = "host allocation failed";
    }
    if (rc != PDLPX_OK) pdlpx::setGlobalError(err);
    return rc;
}

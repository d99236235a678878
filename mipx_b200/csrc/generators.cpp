// Seeded synthetic LP generators for the benchmark workloads (random sparse
// LP, transportation LP, power-law large LP).  Deterministic across hosts: a
// xoshiro256** stream seeded by splitmix64, uniforms from the top 53 bits,
// normals by Box-Muller.  The matrix is assembled in CSR with the semantics
// of mipx::SparseMatrix's triplet constructor (sparse_matrix.cpp:12-73):
// columns sorted within a row, duplicate draws summed, exact zeros dropped.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#include "pdlpx.h"

namespace pdlpx {
namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (auto& w : s) {
            z += 0x9e3779b97f4a7c15ULL;
            uint64_t t = z;
            t = (t ^ (t >> 30)) * 0xbf58476d1ce4e5b9ULL;
            t = (t ^ (t >> 27)) * 0x94d049bb133111ebULL;
            w = t ^ (t >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
    // Integer in [0, k).
    int64_t below(int64_t k) { return static_cast<int64_t>(uniform() * static_cast<double>(k)); }
    bool have_spare = false;
    double spare = 0.0;
    double normal() {
        if (have_spare) {
            have_spare = false;
            return spare;
        }
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        double r = std::sqrt(-2.0 * std::log(u1));
        double th = 6.283185307179586476925286766559 * u2;
        spare = r * std::sin(th);
        have_spare = true;
        return r * std::cos(th);
    }
};

template <class T>
T* dup(const std::vector<T>& v) {
    T* p = static_cast<T*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
    if (p != nullptr && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

// Column-major draws (col_ptr, rows, vals) -> canonical CSR.
void assemble(int m, int n, const std::vector<int64_t>& col_ptr, const std::vector<int>& rows,
              const std::vector<double>& vals, std::vector<int32_t>& rp, std::vector<int32_t>& ci,
              std::vector<double>& v) {
    std::vector<int64_t> cnt(static_cast<size_t>(m) + 1, 0);
    for (int r : rows) ++cnt[r + 1];
    for (int i = 0; i < m; ++i) cnt[i + 1] += cnt[i];
    std::vector<int32_t> tc(rows.size());
    std::vector<double> tv(rows.size());
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int j = 0; j < n; ++j)  // column order => each row's entries sorted by column
        for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
            int64_t p = pos[rows[k]]++;
            tc[p] = j;
            tv[p] = vals[k];
        }
    rp.assign(static_cast<size_t>(m) + 1, 0);
    ci.clear();
    v.clear();
    ci.reserve(rows.size());
    v.reserve(rows.size());
    for (int i = 0; i < m; ++i) {
        for (int64_t k = cnt[i]; k < cnt[i + 1];) {
            int c = tc[k];
            double s = 0.0;
            while (k < cnt[i + 1] && tc[k] == c) s += tv[k++];
            if (s != 0.0) {
                ci.push_back(c);
                v.push_back(s);
            }
        }
        rp[i + 1] = static_cast<int32_t>(ci.size());
    }
}

// Feasibility construction shared by the random and power-law generators:
// x0~U[0,10], rows alternate '=' (even) and '<=' (odd) with b = A x0, slack
// U[0,1] on '<='; bounds [0,10]; c~N(0,1).
void finishRandom(Rng& rng, int m, int n, const std::vector<int32_t>& rp,
                  const std::vector<int32_t>& ci, const std::vector<double>& v,
                  pdlpx_gen_lp* out) {
    const double inf = std::numeric_limits<double>::infinity();
    std::vector<double> x0(n), c(n), cl(n, 0.0), cu(n, 10.0), rl(m), ru(m);
    for (int j = 0; j < n; ++j) x0[j] = 10.0 * rng.uniform();
    for (int j = 0; j < n; ++j) c[j] = rng.normal();
    for (int i = 0; i < m; ++i) {
        double ax = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) ax += v[k] * x0[ci[k]];
        if (i % 2 == 0) {
            rl[i] = ax;
            ru[i] = ax;
        } else {
            rl[i] = -inf;
            ru[i] = ax + rng.uniform();
        }
    }
    out->m = m;
    out->n = n;
    out->nnz = static_cast<int32_t>(ci.size());
    out->row_ptr = dup(rp);
    out->col_idx = dup(ci);
    out->val = dup(v);
    out->obj = dup(c);
    out->col_lb = dup(cl);
    out->col_ub = dup(cu);
    out->row_lb = dup(rl);
    out->row_ub = dup(ru);
    out->x0 = dup(x0);
    out->is_int = nullptr;
}

}  // namespace
}  // namespace pdlpx

using pdlpx::Rng;

extern "C" {

int32_t pdlpx_gen_random(int32_t m, int32_t n, int32_t nnz_lo, int32_t nnz_hi, uint64_t seed,
                         pdlpx_gen_lp* out) {
    if (out == nullptr || m <= 0 || n <= 0 || nnz_lo < 1 || nnz_hi < nnz_lo) return PDLPX_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    Rng rng(seed);
    std::vector<int64_t> cp(static_cast<size_t>(n) + 1, 0);
    std::vector<int> rows;
    std::vector<double> vals;
    rows.reserve(static_cast<size_t>(n) * (nnz_lo + nnz_hi) / 2);
    vals.reserve(rows.capacity());
    for (int j = 0; j < n; ++j) {
        int k = nnz_lo + static_cast<int>(rng.below(nnz_hi - nnz_lo + 1));
        for (int t = 0; t < k; ++t) {
            rows.push_back(static_cast<int>(rng.below(m)));
            vals.push_back(rng.normal());
        }
        cp[j + 1] = static_cast<int64_t>(rows.size());
    }
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
    pdlpx::assemble(m, n, cp, rows, vals, rp, ci, v);
    pdlpx::finishRandom(rng, m, n, rp, ci, v, out);
    return PDLPX_OK;
}

int32_t pdlpx_gen_transport(int32_t s, int32_t d, uint64_t seed, pdlpx_gen_lp* out) {
    if (out == nullptr || s <= 0 || d <= 0) return PDLPX_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    const double inf = std::numeric_limits<double>::infinity();
    Rng rng(seed);
    const int64_t n64 = static_cast<int64_t>(s) * d;
    if (n64 > std::numeric_limits<int32_t>::max() / 2) return PDLPX_E_INVALID;
    const int n = static_cast<int>(n64), m = s + d;
    std::vector<double> supply(s), demand(d), c(n), cl(n, 0.0), cu(n, inf), rl(m), ru(m), x0(n);
    for (auto& v : supply) v = 50.0 + 100.0 * rng.uniform();
    for (auto& v : demand) v = 50.0 + 100.0 * rng.uniform();
    double ts = 0.0, td = 0.0;
    for (double v : supply) ts += v;
    for (double v : demand) td += v;
    for (auto& v : demand) v *= 0.95 * ts / td;
    for (auto& v : c) v = 1.0 + 99.0 * rng.uniform();
    // Rows 0..s-1: supply i, sum_j x_ij <= s_i.  Rows s..s+d-1: demand j, sum_i x_ij >= d_j.
    std::vector<int32_t> rp(static_cast<size_t>(m) + 1), ci(static_cast<size_t>(2) * n);
    std::vector<double> v(static_cast<size_t>(2) * n, 1.0);
    int64_t w = 0;
    for (int i = 0; i < s; ++i) {
        rp[i] = static_cast<int32_t>(w);
        for (int j = 0; j < d; ++j) ci[w++] = i * d + j;
        rl[i] = -inf;
        ru[i] = supply[i];
    }
    for (int j = 0; j < d; ++j) {
        rp[s + j] = static_cast<int32_t>(w);
        for (int i = 0; i < s; ++i) ci[w++] = i * d + j;
        rl[s + j] = demand[j];
        ru[s + j] = inf;
    }
    rp[m] = static_cast<int32_t>(w);
    double tdn = 0.0;
    for (double dv : demand) tdn += dv;
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < d; ++j) x0[static_cast<size_t>(i) * d + j] = supply[i] * demand[j] / ts;
    (void)tdn;
    out->m = m;
    out->n = n;
    out->nnz = static_cast<int32_t>(w);
    out->row_ptr = pdlpx::dup(rp);
    out->col_idx = pdlpx::dup(ci);
    out->val = pdlpx::dup(v);
    out->obj = pdlpx::dup(c);
    out->col_lb = pdlpx::dup(cl);
    out->col_ub = pdlpx::dup(cu);
    out->row_lb = pdlpx::dup(rl);
    out->row_ub = pdlpx::dup(ru);
    out->x0 = pdlpx::dup(x0);
    out->is_int = nullptr;
    return PDLPX_OK;
}

int32_t pdlpx_gen_powerlaw(int32_t m, int32_t n, int32_t kmin, int32_t kmax, double kmean,
                           double big_frac, double big_scale, uint64_t seed, pdlpx_gen_lp* out) {
    if (out == nullptr || m <= 0 || n <= 0 || kmin < 1 || kmax < kmin || kmean < kmin ||
        kmean > kmax)
        return PDLPX_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    Rng rng(seed);
    // Discrete power law p(k) ~ k^-alpha on [kmin, kmax]; alpha by bisection so the mean is kmean.
    const int K = kmax - kmin + 1;
    std::vector<double> cdf(K);
    auto meanFor = [&](double a) {
        double z = 0.0, mu = 0.0;
        for (int k = kmin; k <= kmax; ++k) {
            double p = std::pow(static_cast<double>(k), -a);
            z += p;
            mu += p * k;
        }
        return mu / z;
    };
    double lo = 0.0, hi = 6.0;
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (meanFor(mid) > kmean)
            lo = mid;
        else
            hi = mid;
    }
    const double alpha = 0.5 * (lo + hi);
    double z = 0.0;
    for (int k = kmin; k <= kmax; ++k) z += std::pow(static_cast<double>(k), -alpha);
    double acc = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
        acc += std::pow(static_cast<double>(k), -alpha) / z;
        cdf[k - kmin] = acc;
    }
    cdf[K - 1] = 1.0;
    std::vector<double> rowmul(m, 1.0);
    for (int i = 0; i < m; ++i)
        if (rng.uniform() < big_frac) rowmul[i] = big_scale;
    std::vector<int64_t> cp(static_cast<size_t>(n) + 1, 0);
    std::vector<int> rows;
    std::vector<double> vals;
    rows.reserve(static_cast<size_t>(static_cast<double>(n) * kmean * 1.05));
    vals.reserve(rows.capacity());
    for (int j = 0; j < n; ++j) {
        double u = rng.uniform();
        int k = kmin + static_cast<int>(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        k = std::min(k, std::min(kmax, m));
        for (int t = 0; t < k; ++t) {
            int r = static_cast<int>(rng.below(m));
            rows.push_back(r);
            vals.push_back(rng.normal() * rowmul[r]);
        }
        cp[j + 1] = static_cast<int64_t>(rows.size());
    }
    if (rows.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) return PDLPX_E_INVALID;
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
    pdlpx::assemble(m, n, cp, rows, vals, rp, ci, v);
    pdlpx::finishRandom(rng, m, n, rp, ci, v, out);
    return PDLPX_OK;
}

void pdlpx_free_lp(pdlpx_gen_lp* lp) {
    if (lp == nullptr) return;
    std::free(lp->row_ptr);
    std::free(lp->col_idx);
    std::free(lp->val);
    std::free(lp->obj);
    std::free(lp->col_lb);
    std::free(lp->col_ub);
    std::free(lp->row_lb);
    std::free(lp->row_ub);
    std::free(lp->x0);
    std::free(lp->is_int);
    std::memset(lp, 0, sizeof(*lp));
}

}  // extern "C"

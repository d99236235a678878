#include "problem.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <thread>

namespace pdlpx {

namespace {
inline bool fin(double v) { return std::isfinite(v); }
}  // namespace

bool canonicalCsr(int32_t m, int32_t n, int32_t nnz, const int32_t* rp, const int32_t* ci,
                  const double* v, Csr& out) {
    out.rows = m;
    out.cols = n;
    out.ptr.assign(static_cast<size_t>(m) + 1, 0);
    out.idx.clear();
    out.val.clear();
    if (m < 0 || n < 0 || nnz < 0) return false;
    if (m > 0 && (rp == nullptr || rp[0] != 0 || rp[m] != nnz)) return false;
    if (nnz > 0 && (ci == nullptr || v == nullptr)) return false;
    out.idx.reserve(static_cast<size_t>(nnz));
    out.val.reserve(static_cast<size_t>(nnz));
    std::vector<int32_t> order;
    for (int32_t i = 0; i < m; ++i) {
        const int32_t b = rp[i], e = rp[i + 1];
        if (e < b || e > nnz) return false;
        bool sorted = true;
        for (int32_t k = b; k < e; ++k) {
            if (ci[k] < 0 || ci[k] >= n) return false;
            if (k > b && ci[k] <= ci[k - 1]) sorted = false;
        }
        if (sorted) {
            for (int32_t k = b; k < e; ++k)
                if (v[k] != 0.0) {
                    out.idx.push_back(ci[k]);
                    out.val.push_back(v[k]);
                }
        } else {
            order.resize(static_cast<size_t>(e - b));
            std::iota(order.begin(), order.end(), b);
            std::stable_sort(order.begin(), order.end(),
                             [&](int32_t x, int32_t y) { return ci[x] < ci[y]; });
            for (size_t t = 0; t < order.size();) {
                const int32_t c = ci[order[t]];
                double sum = 0.0;
                while (t < order.size() && ci[order[t]] == c) sum += v[order[t++]];
                if (sum != 0.0) {
                    out.idx.push_back(c);
                    out.val.push_back(sum);
                }
            }
        }
        out.ptr[i + 1] = static_cast<int32_t>(out.idx.size());
    }
    return true;
}

namespace {

// Host threads for the O(nnz) passes of large LPs (1 below 1M entries).
int hostThreads(size_t work) {
    if (work < (1u << 20)) return 1;
    return static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
}

template <class F>
void forBlocks(int nt, int64_t count, F&& f) {  // f(t, begin, end) over nt contiguous blocks
    if (nt <= 1) {
        f(0, int64_t{0}, count);
        return;
    }
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; ++t)
        ts.emplace_back([&, t] { f(t, count * t / nt, count * (t + 1) / nt); });
    for (auto& th : ts) th.join();
}

}  // namespace

// Counting transpose.  With T threads each takes a contiguous block of rows,
// counts its entries per column, and scatters them after the entries of the
// blocks before it, so every A^T row keeps ascending row order -- the output
// does not depend on T.
void transposeCsr(const Csr& a, Csr& at) {
    at.rows = a.cols;
    at.cols = a.rows;
    const int32_t n = a.cols;
    at.ptr.assign(static_cast<size_t>(n) + 1, 0);
    at.idx.resize(a.idx.size());
    at.val.resize(a.val.size());
    const int nt = std::min<int64_t>(hostThreads(a.idx.size()), std::max<int32_t>(1, a.rows));
    if (nt <= 1) {
        for (int32_t c : a.idx) ++at.ptr[c + 1];
        for (int32_t j = 0; j < n; ++j) at.ptr[j + 1] += at.ptr[j];
        std::vector<int32_t> cur(at.ptr.begin(), at.ptr.end() - 1);
        for (int32_t i = 0; i < a.rows; ++i)
            for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                const int32_t p = cur[a.idx[k]]++;
                at.idx[p] = i;
                at.val[p] = a.val[k];
            }
        return;
    }
    std::vector<std::vector<int32_t>> cnt(nt, std::vector<int32_t>(static_cast<size_t>(n), 0));
    forBlocks(nt, a.rows, [&](int t, int64_t r0, int64_t r1) {
        std::vector<int32_t>& c = cnt[t];
        for (int64_t k = a.ptr[r0]; k < a.ptr[r1]; ++k) ++c[a.idx[k]];
    });
    // column starts, then each block's first slot inside every column
    for (int32_t j = 0; j < n; ++j) {
        int32_t tot = 0;
        for (int t = 0; t < nt; ++t) tot += cnt[t][j];
        at.ptr[j + 1] = at.ptr[j] + tot;
    }
    forBlocks(nt, n, [&](int, int64_t j0, int64_t j1) {
        for (int64_t j = j0; j < j1; ++j) {
            int32_t pos = at.ptr[j];
            for (int t = 0; t < nt; ++t) {
                const int32_t c = cnt[t][j];
                cnt[t][j] = pos;
                pos += c;
            }
        }
    });
    forBlocks(nt, a.rows, [&](int t, int64_t r0, int64_t r1) {
        std::vector<int32_t>& cur = cnt[t];
        for (int64_t i = r0; i < r1; ++i)
            for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                const int32_t p = cur[a.idx[k]]++;
                at.idx[p] = static_cast<int32_t>(i);
                at.val[p] = a.val[k];
            }
    });
}

void pockChambolle(const ScaledLp& s, std::vector<double>& sigma, std::vector<double>& tau) {
    // Row sums run along each row of A, column sums along each row of A^T; both
    // accumulate in ascending inner index, i.e. the order of the reference's
    // single row-major sweep (pdlp.cpp:590-597).
    const Csr& a = s.a;
    const Csr& at = s.at;
    sigma.assign(static_cast<size_t>(a.rows), 1.0);
    tau.assign(static_cast<size_t>(a.cols), 1.0);
    const int nt = hostThreads(a.idx.size());  // rows are independent: any split gives the same sums
    forBlocks(nt, a.rows, [&](int, int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            double acc = 0.0;
            for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) acc += a.val[k] * a.val[k];
            sigma[i] = 1.0 / std::max(std::sqrt(acc), 1e-8);
        }
    });
    forBlocks(nt, at.rows, [&](int, int64_t j0, int64_t j1) {
        for (int64_t j = j0; j < j1; ++j) {
            double acc = 0.0;
            for (int32_t k = at.ptr[j]; k < at.ptr[j + 1]; ++k) acc += at.val[k] * at.val[k];
            tau[j] = 1.0 / std::max(std::sqrt(acc), 1e-8);
        }
    });
}

void buildScaled(const HostLp& lp, const pdlpx_options& o, ScaledLp& s, const RuizFn& ruiz) {
    const int32_t m = lp.m, n = lp.n;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    s.obj_sign = lp.maximize ? -1.0 : 1.0;
    s.c.resize(static_cast<size_t>(n));
    for (int32_t j = 0; j < n; ++j) s.c[j] = s.obj_sign * lp.obj[j];
    s.cl = lp.cl;
    s.cu = lp.cu;
    s.rl = lp.rl;
    s.ru = lp.ru;
    s.row_scale.assign(static_cast<size_t>(m), 1.0);
    s.col_scale.assign(static_cast<size_t>(n), 1.0);

    Csr& a = s.a;
    a.rows = m;
    a.cols = n;
    if (o.matrix_zero_tol > 0.0 && lp.a.nnz() > 0) {
        a.ptr.assign(static_cast<size_t>(m) + 1, 0);
        a.idx.clear();
        a.val.clear();
        for (int32_t i = 0; i < m; ++i) {
            for (int32_t k = lp.a.ptr[i]; k < lp.a.ptr[i + 1]; ++k)
                if (std::abs(lp.a.val[k]) >= o.matrix_zero_tol) {
                    a.idx.push_back(lp.a.idx[k]);
                    a.val.push_back(lp.a.val[k]);
                }
            a.ptr[i + 1] = static_cast<int32_t>(a.idx.size());
        }
    } else {
        // the copy of a large matrix on host threads (blocks of entries)
        a.ptr = lp.a.ptr;
        a.idx.resize(lp.a.idx.size());
        a.val.resize(lp.a.val.size());
        const int64_t z = static_cast<int64_t>(lp.a.idx.size());
        forBlocks(hostThreads(static_cast<size_t>(z)), z, [&](int, int64_t k0, int64_t k1) {
            std::copy(lp.a.idx.begin() + k0, lp.a.idx.begin() + k1, a.idx.begin() + k0);
            std::copy(lp.a.val.begin() + k0, lp.a.val.begin() + k1, a.val.begin() + k0);
        });
    }

    const auto t1 = clk::now();
    // Ruiz: alternate row and column infinity-norm equilibration, scale 1/sqrt(max).
    bool ruiz_done = false;
    if (o.do_ruiz_scaling && m > 0 && n > 0 && a.nnz() > 0 && ruiz) {
        ruiz_done = ruiz(a, s.row_scale, s.col_scale, o.ruiz_iterations);
        if (!ruiz_done) {
            // the device path may have written part of its result before it
            // failed: the host loop starts again from the unscaled values
            const double tol = o.matrix_zero_tol;
            size_t q = 0;
            for (int32_t i = 0; i < m; ++i)
                for (int32_t k = lp.a.ptr[i]; k < lp.a.ptr[i + 1]; ++k)
                    if (!(tol > 0.0) || std::abs(lp.a.val[k]) >= tol) a.val[q++] = lp.a.val[k];
            std::fill(s.row_scale.begin(), s.row_scale.end(), 1.0);
            std::fill(s.col_scale.begin(), s.col_scale.end(), 1.0);
        }
    }
    if (o.do_ruiz_scaling && m > 0 && n > 0 && a.nnz() > 0 && !ruiz_done) {
        std::vector<double> cmax(static_cast<size_t>(n));
        for (int32_t pass = 0; pass < o.ruiz_iterations; ++pass) {
            for (int32_t i = 0; i < m; ++i) {
                double rmax = 0.0;
                for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) rmax = std::max(rmax, std::abs(a.val[k]));
                if (rmax <= 1e-12) continue;
                const double f = 1.0 / std::sqrt(rmax);
                s.row_scale[i] *= f;
                for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) a.val[k] *= f;
            }
            std::fill(cmax.begin(), cmax.end(), 0.0);
            for (size_t k = 0; k < a.val.size(); ++k) {
                double& cm = cmax[a.idx[k]];
                cm = std::max(cm, std::abs(a.val[k]));
            }
            for (int32_t j = 0; j < n; ++j)
                if (cmax[j] > 1e-12) s.col_scale[j] *= 1.0 / std::sqrt(cmax[j]);
            for (size_t k = 0; k < a.val.size(); ++k) {
                const double cm = cmax[a.idx[k]];
                if (cm > 1e-12) a.val[k] *= 1.0 / std::sqrt(cm);
            }
        }
    }
    for (int32_t j = 0; j < n; ++j) {
        s.c[j] *= s.col_scale[j];
        if (fin(s.cl[j])) s.cl[j] /= s.col_scale[j];
        if (fin(s.cu[j])) s.cu[j] /= s.col_scale[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        if (fin(s.rl[i])) s.rl[i] *= s.row_scale[i];
        if (fin(s.ru[i])) s.ru[i] *= s.row_scale[i];
    }
    const auto t2 = clk::now();
    transposeCsr(a, s.at);
    const auto t3 = clk::now();

    if (o.do_pock_chambolle_scaling && m > 0 && n > 0) {
        pockChambolle(s, s.sigma, s.tau);
    } else {
        s.sigma.assign(static_cast<size_t>(m), 1.0);
        s.tau.assign(static_cast<size_t>(n), 1.0);
    }
    const auto t4 = clk::now();

    s.obj_scale = 1.0;
    s.con_scale = 1.0;
    if (o.do_bound_obj_rescaling && m > 0 && n > 0) {
        double osq = 0.0;
        for (int32_t j = 0; j < n; ++j) osq += s.c[j] * s.c[j];
        s.obj_scale = 1.0 / (std::sqrt(osq) + 1.0);
        double bsq = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            if (fin(s.rl[i])) bsq += s.rl[i] * s.rl[i];
            if (fin(s.ru[i])) bsq += s.ru[i] * s.ru[i];
        }
        s.con_scale = 1.0 / (std::sqrt(bsq) + 1.0);
        for (int32_t j = 0; j < n; ++j) s.c[j] *= s.obj_scale;
        for (int32_t i = 0; i < m; ++i) {
            if (fin(s.rl[i])) s.rl[i] *= s.con_scale;
            if (fin(s.ru[i])) s.ru[i] *= s.con_scale;
        }
        for (int32_t j = 0; j < n; ++j) {
            if (fin(s.cl[j])) s.cl[j] *= s.con_scale;
            if (fin(s.cu[j])) s.cu[j] *= s.con_scale;
        }
    }

    s.row_type.resize(static_cast<size_t>(m));
    for (int32_t i = 0; i < m; ++i) {
        const double l = s.rl[i], u = s.ru[i];
        if (l == u)
            s.row_type[i] = kRowEq;
        else if (!fin(l))
            s.row_type[i] = kRowUpper;
        else if (!fin(u))
            s.row_type[i] = kRowLower;
        else
            s.row_type[i] = kRowRanged;
    }
    s.precond_pw = o.primal_weight;
    if (o.verbose) {
        auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
        std::printf("PDLP scaling: copy %.3fs, Ruiz %.3fs, transpose %.3fs, Pock-Chambolle %.3fs, rest %.3fs\n",
                    sec(t0, t1), sec(t1, t2), sec(t2, t3), sec(t3, t4), sec(t4, clk::now()));
        std::fflush(stdout);
    }
}

void terminationNorms(const HostLp& lp, int32_t norm, double& c_norm, double& b_norm) {
    c_norm = 0.0;
    b_norm = 0.0;
    if (norm == PDLPX_NORM_LINF) {
        for (double c : lp.obj) c_norm = std::max(c_norm, std::abs(c));
        for (int32_t i = 0; i < lp.m; ++i) {
            if (fin(lp.ru[i])) b_norm = std::max(b_norm, std::abs(lp.ru[i]));
            if (fin(lp.rl[i]) && lp.rl[i] != lp.ru[i]) b_norm = std::max(b_norm, std::abs(lp.rl[i]));
        }
        return;
    }
    double csq = 0.0;
    for (double c : lp.obj) csq += c * c;
    c_norm = std::sqrt(csq);
    double bsq = 0.0;
    for (int32_t i = 0; i < lp.m; ++i) {
        if (fin(lp.ru[i])) bsq += lp.ru[i] * lp.ru[i];
        if (fin(lp.rl[i]) && lp.rl[i] != lp.ru[i]) bsq += lp.rl[i] * lp.rl[i];
    }
    b_norm = std::sqrt(bsq);
}

void csrMultiplyTranspose(const Csr& a, const double* x, double* y) {
    std::fill(y, y + a.cols, 0.0);
    for (int32_t i = 0; i < a.rows; ++i) {
        if (x[i] == 0.0) continue;
        for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) y[a.idx[k]] += a.val[k] * x[i];
    }
}

}  // namespace pdlpx

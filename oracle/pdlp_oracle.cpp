// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A serial FP64 CPU restatement of mipx's PDLP path (spoorendonk/mipx,
// src/lp/pdlp.cpp, CPU branch of PdlpSolver::solve and helpers).  It is the
// checker for the CUDA engine: tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg call it, nothing in mipx_b200/ does.  Every function keeps
// the reference's floating-point operation order so that, built with the same
// flags, its results equal those of the reference compiled from source
// (oracle/_ref, see oracle/Makefile); tests/test_oracle_pin.py checks that.
//
// Where a piece follows the reference, the comment names the file:line.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "pdlpx.h"

namespace {

using Vec = std::vector<double>;
const double kInf = std::numeric_limits<double>::infinity();

bool fin(double v) { return std::isfinite(v); }

double l2norm(const Vec& v) {  // pdlp.cpp:27-32
    double s = 0.0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

double dotv(const Vec& a, const Vec& b) {  // pdlp.cpp:41-46
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// CSR matrix with the semantics of mipx::SparseMatrix (sparse_matrix.cpp).
struct Csr {
    int rows = 0, cols = 0;
    Vec val;
    std::vector<int> idx;
    std::vector<int> ptr;
    int nnz() const { return static_cast<int>(val.size()); }
};

// Canonicalise arbitrary CSR input like the triplet constructor
// (sparse_matrix.cpp:12-73): sort by column within each row, sum duplicates,
// drop exact zero sums.
Csr canonical(int m, int n, const int* rp, const int* ci, const double* v) {
    Csr a;
    a.rows = m;
    a.cols = n;
    a.ptr.assign(static_cast<size_t>(m) + 1, 0);
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < m; ++i) {
        row.clear();
        for (int k = rp[i]; k < rp[i + 1]; ++k) row.emplace_back(ci[k], v[k]);
        std::stable_sort(row.begin(), row.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t k = 0; k < row.size();) {
            int c = row[k].first;
            double s = 0.0;
            while (k < row.size() && row[k].first == c) {
                s += row[k].second;
                ++k;
            }
            if (s != 0.0) {
                a.val.push_back(s);
                a.idx.push_back(c);
                ++a.ptr[i + 1];
            }
        }
    }
    for (int i = 0; i < m; ++i) a.ptr[i + 1] += a.ptr[i];
    return a;
}

void mul(const Csr& a, const Vec& x, Vec& y) {  // sparse_matrix.cpp:181-193
    for (int i = 0; i < a.rows; ++i) {
        double s = 0.0;
        for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) s += a.val[k] * x[a.idx[k]];
        y[i] = s;
    }
}

void mulT(const Csr& a, const Vec& x, Vec& y) {  // sparse_matrix.cpp:195-208
    std::fill(y.begin(), y.end(), 0.0);
    for (int i = 0; i < a.rows; ++i) {
        if (x[i] == 0.0) continue;
        for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) y[a.idx[k]] += a.val[k] * x[i];
    }
}

struct Lp {
    int m = 0, n = 0;
    bool maximize = false;
    Csr a;
    Vec obj, cl, cu, rl, ru;
    double offset = 0.0;
};

// State produced by buildScaledProblem (pdlp.cpp:469-669).
struct Scaled {
    double obj_sign = 1.0;
    Csr a;
    Vec c, cl, cu, rl, ru;
    Vec row_scale, col_scale, sigma, tau;
    double obj_scale = 1.0, con_scale = 1.0;
    double precond_pw = 1.0;  // primal weight at the last preconditioning (pdlp.cpp:668, 741)
};

void pockChambolle(const Csr& a, Vec& sigma, Vec& tau) {  // pdlp.cpp:581-604, 713-742
    Vec row_sq(static_cast<size_t>(a.rows), 0.0), col_sq(static_cast<size_t>(a.cols), 0.0);
    for (int i = 0; i < a.rows; ++i)
        for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
            double v = a.val[k];
            row_sq[i] += v * v;
            col_sq[a.idx[k]] += v * v;
        }
    for (int i = 0; i < a.rows; ++i) sigma[i] = 1.0 / std::max(std::sqrt(row_sq[i]), 1e-8);
    for (int j = 0; j < a.cols; ++j) tau[j] = 1.0 / std::max(std::sqrt(col_sq[j]), 1e-8);
}

void buildScaled(const Lp& lp, const pdlpx_options& o, Scaled& s) {
    const int m = lp.m, n = lp.n;
    s.obj_sign = lp.maximize ? -1.0 : 1.0;
    s.c.resize(n);
    for (int j = 0; j < n; ++j) s.c[j] = s.obj_sign * lp.obj[j];
    s.cl = lp.cl;
    s.cu = lp.cu;
    s.rl = lp.rl;
    s.ru = lp.ru;
    s.row_scale.assign(m, 1.0);
    s.col_scale.assign(n, 1.0);
    Vec val = lp.a.val;
    std::vector<int> idx = lp.a.idx, ptr = lp.a.ptr;

    if (o.matrix_zero_tol > 0.0 && !val.empty()) {  // pdlp.cpp:499-518
        int w = 0;
        for (int i = 0; i < m; ++i) {
            int b = ptr[i], e = ptr[i + 1];
            ptr[i] = w;
            for (int k = b; k < e; ++k)
                if (std::abs(val[k]) >= o.matrix_zero_tol) {
                    val[w] = val[k];
                    idx[w] = idx[k];
                    ++w;
                }
        }
        ptr[m] = w;
        val.resize(w);
        idx.resize(w);
    }

    if (o.do_ruiz_scaling && m > 0 && n > 0 && !val.empty()) {  // pdlp.cpp:520-558
        Vec cn(static_cast<size_t>(n), 0.0);
        for (int it = 0; it < o.ruiz_iterations; ++it) {
            for (int i = 0; i < m; ++i) {
                double rmax = 0.0;
                for (int k = ptr[i]; k < ptr[i + 1]; ++k) rmax = std::max(rmax, std::abs(val[k]));
                if (rmax <= 1e-12) continue;
                double sc = 1.0 / std::sqrt(rmax);
                s.row_scale[i] *= sc;
                for (int k = ptr[i]; k < ptr[i + 1]; ++k) val[k] *= sc;
            }
            std::fill(cn.begin(), cn.end(), 0.0);
            for (size_t k = 0; k < val.size(); ++k) cn[idx[k]] = std::max(cn[idx[k]], std::abs(val[k]));
            for (int j = 0; j < n; ++j) {
                if (cn[j] <= 1e-12) continue;
                s.col_scale[j] *= 1.0 / std::sqrt(cn[j]);
            }
            for (size_t k = 0; k < val.size(); ++k) {
                int j = idx[k];
                if (cn[j] > 1e-12) val[k] *= 1.0 / std::sqrt(cn[j]);
            }
        }
    }
    for (int j = 0; j < n; ++j) {  // pdlp.cpp:561-567
        s.c[j] *= s.col_scale[j];
        if (fin(s.cl[j])) s.cl[j] /= s.col_scale[j];
        if (fin(s.cu[j])) s.cu[j] /= s.col_scale[j];
    }
    for (int i = 0; i < m; ++i) {  // pdlp.cpp:568-573
        if (fin(s.rl[i])) s.rl[i] *= s.row_scale[i];
        if (fin(s.ru[i])) s.ru[i] *= s.row_scale[i];
    }
    s.a.rows = m;
    s.a.cols = n;
    s.a.val = std::move(val);
    s.a.idx = std::move(idx);
    s.a.ptr = std::move(ptr);

    s.sigma.assign(m, 1.0);
    s.tau.assign(n, 1.0);
    if (o.do_pock_chambolle_scaling && m > 0 && n > 0) pockChambolle(s.a, s.sigma, s.tau);

    s.obj_scale = 1.0;
    s.con_scale = 1.0;
    if (o.do_bound_obj_rescaling && m > 0 && n > 0) {  // pdlp.cpp:606-640
        double osq = 0.0;
        for (int j = 0; j < n; ++j) osq += s.c[j] * s.c[j];
        s.obj_scale = 1.0 / (std::sqrt(osq) + 1.0);
        double bsq = 0.0;
        for (int i = 0; i < m; ++i) {
            if (fin(s.rl[i])) bsq += s.rl[i] * s.rl[i];
            if (fin(s.ru[i])) bsq += s.ru[i] * s.ru[i];
        }
        s.con_scale = 1.0 / (std::sqrt(bsq) + 1.0);
        for (int j = 0; j < n; ++j) s.c[j] *= s.obj_scale;
        for (int i = 0; i < m; ++i) {
            if (fin(s.rl[i])) s.rl[i] *= s.con_scale;
            if (fin(s.ru[i])) s.ru[i] *= s.con_scale;
        }
        for (int j = 0; j < n; ++j) {
            if (fin(s.cl[j])) s.cl[j] *= s.con_scale;
            if (fin(s.cu[j])) s.cu[j] *= s.con_scale;
        }
    }
}

// Power iteration on A^T A (pdlp.cpp:748-795).
double spectralNorm(const Csr& a, const pdlpx_options& o) {
    const int n = a.cols, m = a.rows;
    if (n == 0 || m == 0) return 1.0;
    std::mt19937 rng(42);
    std::normal_distribution<double> dist(0.0, 1.0);
    Vec x(n);
    for (auto& v : x) v = dist(rng);
    double xn = l2norm(x);
    if (xn < 1e-15) xn = 1.0;
    for (auto& v : x) v /= xn;
    Vec y(m), xnew(n);
    double s2 = 1.0;
    for (int it = 0; it < o.sv_max_iter; ++it) {
        mul(a, x, y);
        mulT(a, y, xnew);
        s2 = dotv(x, xnew);
        double r2 = 0.0;
        for (int j = 0; j < n; ++j) {
            double d = xnew[j] - s2 * x[j];
            r2 += d * d;
        }
        double r = std::sqrt(r2);
        x.swap(xnew);
        xn = l2norm(x);
        if (xn < 1e-15) break;
        for (auto& v : x) v /= xn;
        if (r < o.sv_tol * std::abs(s2)) break;
    }
    return std::sqrt(std::max(s2, 1e-12));
}

// Farkas certificate on the original problem (pdlp.cpp:119-211).
bool infeasCert(const Vec& y, const Lp& lp, double tol) {
    const int m = lp.m, n = lp.n;
    if (m == 0) return false;
    double yn = l2norm(y);
    if (yn < 1e-15) return false;
    Vec ray(y);
    for (auto& v : ray) v /= yn;
    for (int i = 0; i < m; ++i) {
        bool hl = fin(lp.rl[i]), hu = fin(lp.ru[i]);
        if (hu && !hl) {
            if (ray[i] < -tol) return false;
        } else if (hl && !hu) {
            if (ray[i] > tol) return false;
        }
    }
    Vec ar(static_cast<size_t>(n), 0.0);
    mulT(lp.a, ray, ar);
    for (int j = 0; j < n; ++j) {
        double r = ar[j];
        if (fin(lp.cl[j]) && r < -tol) return false;
        if (fin(lp.cu[j]) && r > tol) return false;
    }
    double robj = 0.0;
    for (int i = 0; i < m; ++i) {
        double l = lp.rl[i], u = lp.ru[i];
        if (l == u)
            robj += ray[i] * l;
        else if (ray[i] > 0.0 && fin(u))
            robj += ray[i] * u;
        else if (ray[i] < 0.0 && fin(l))
            robj += ray[i] * l;
    }
    double cs = 0.0;
    for (int j = 0; j < n; ++j) {
        double r = ar[j];
        if (r > 0.0 && fin(lp.cl[j]))
            cs += r * lp.cl[j];
        else if (r < 0.0 && fin(lp.cu[j]))
            cs += r * lp.cu[j];
    }
    return robj - cs < -tol;
}

// Primal ray certificate (pdlp.cpp:220-284).
bool unbddCert(const Vec& x, const Lp& lp, double tol) {
    const int m = lp.m, n = lp.n;
    if (n == 0) return false;
    double xn = l2norm(x);
    if (xn < 1e-15) return false;
    Vec ray(x);
    for (auto& v : ray) v /= xn;
    for (int j = 0; j < n; ++j) {
        if (fin(lp.cl[j]) && ray[j] < -tol) return false;
        if (fin(lp.cu[j]) && ray[j] > tol) return false;
    }
    Vec ar(static_cast<size_t>(m), 0.0);
    mul(lp.a, ray, ar);
    for (int i = 0; i < m; ++i) {
        double r = ar[i];
        bool hl = fin(lp.rl[i]), hu = fin(lp.ru[i]);
        if (hl && hu) {
            if (std::abs(r) > tol) return false;
        } else if (hu && !hl) {
            if (r > tol) return false;
        } else if (hl && !hu) {
            if (r < -tol) return false;
        }
    }
    double sg = lp.maximize ? -1.0 : 1.0;
    double cr = 0.0;
    for (int j = 0; j < n; ++j) cr += lp.obj[j] * ray[j];
    return sg * cr < -tol;
}

// Type-I Anderson acceleration with Tikhonov-regularised Cholesky (pdlp.cpp:293-437).
struct Anderson {
    int window = 0, dim = 0, count = 0;
    double reg = 1e-10;
    std::vector<Vec> xs, rs;
    void init(int w, int d, double r) {
        window = w;
        dim = d;
        reg = r;
        count = 0;
        xs.assign(w, Vec(d, 0.0));
        rs.assign(w, Vec(d, 0.0));
    }
    void store(const Vec& it, const Vec& res) {
        int slot = count % window;
        for (int k = 0; k < dim; ++k) {
            xs[slot][k] = it[k];
            rs[slot][k] = res[k];
        }
        ++count;
    }
    bool extrapolate(Vec& out) const {
        int d = std::min(count, window);
        if (d < 2) return false;
        auto slot = [&](int i) { return (count - d + i) % window; };
        Vec g(static_cast<size_t>(d * d), 0.0);
        for (int i = 0; i < d; ++i) {
            const Vec& ri = rs[slot(i)];
            for (int j = i; j < d; ++j) {
                const Vec& rj = rs[slot(j)];
                double s = 0.0;
                for (int k = 0; k < dim; ++k) s += ri[k] * rj[k];
                g[i * d + j] = s;
                g[j * d + i] = s;
            }
        }
        double tr = 0.0;
        for (int i = 0; i < d; ++i) tr += g[i * d + i];
        double mu = reg * tr / static_cast<double>(d);
        for (int i = 0; i < d; ++i) g[i * d + i] += mu;
        Vec L(static_cast<size_t>(d * d), 0.0);
        for (int i = 0; i < d; ++i)
            for (int j = 0; j <= i; ++j) {
                double s = g[i * d + j];
                for (int p = 0; p < j; ++p) s -= L[i * d + p] * L[j * d + p];
                if (i == j) {
                    if (s <= 0.0) return false;
                    L[i * d + j] = std::sqrt(s);
                } else {
                    L[i * d + j] = s / L[j * d + j];
                }
            }
        Vec z(d, 0.0), al(d, 0.0);
        for (int i = 0; i < d; ++i) {
            double s = 1.0;
            for (int p = 0; p < i; ++p) s -= L[i * d + p] * z[p];
            z[i] = s / L[i * d + i];
        }
        for (int i = d - 1; i >= 0; --i) {
            double s = z[i];
            for (int p = i + 1; p < d; ++p) s -= L[p * d + i] * al[p];
            al[i] = s / L[i * d + i];
        }
        double sa = 0.0;
        for (int i = 0; i < d; ++i) sa += al[i];
        if (std::abs(sa) < 1e-15) return false;
        for (int i = 0; i < d; ++i) al[i] /= sa;
        for (int k = 0; k < dim; ++k) out[k] = 0.0;
        for (int i = 0; i < d; ++i) {
            const Vec& xi = xs[slot(i)];
            for (int k = 0; k < dim; ++k) out[k] += al[i] * xi[k];
        }
        double aa = 0.0;
        for (int k = 0; k < dim; ++k) {
            double r = 0.0;
            for (int i = 0; i < d; ++i) r += al[i] * rs[slot(i)][k];
            aa += r * r;
        }
        const Vec& rl = rs[slot(d - 1)];
        double ll = 0.0;
        for (int k = 0; k < dim; ++k) ll += rl[k] * rl[k];
        return aa < ll;
    }
};

struct Outcome {
    int status = PDLPX_STATUS_ERROR;
    double objective = 0.0;
    int iterations = 0;
    double work = 0.0;
    Vec x, y;
    double rp = 0, rd = 0, gap = 0, pobj = 0, dobj = 0, step = 0, pw = 0;
    int restarts = 0;
};

// One PDHG batch of `batch` Halpern iterations (pdlp.cpp:980-1072).  Returns
// false when the time limit cut it short (iterations done in *done).
struct Iterates {
    Vec cx, cy, ix, iy, px, py, rx, ry, aty, axr, ax, dyv, atdy, atpy, prev_axr, prev_rx;
};

// Reduced relative residuals at (px, py) (pdlp.cpp:1106-1154).
struct Kkt {
    double rp2 = 0, rpmax = 0, rd2 = 0, rdmax = 0;
};

Kkt residuals(const Scaled& s, Iterates& v) {
    const int m = s.a.rows, n = s.a.cols;
    Kkt k;
    mul(s.a, v.px, v.ax);
    for (int i = 0; i < m; ++i) {
        double vs = v.ax[i] - std::clamp(v.ax[i], s.rl[i], s.ru[i]);
        double vv = vs / (s.con_scale * s.row_scale[i]);
        k.rp2 += vv * vv;
        k.rpmax = std::max(k.rpmax, std::abs(vv));
    }
    mulT(s.a, v.py, v.atpy);
    for (int j = 0; j < n; ++j) {
        double g = s.c[j] + v.atpy[j];
        double xj = v.px[j], lb = s.cl[j], ub = s.cu[j];
        double dr;
        if (xj <= lb + 1e-12 && fin(lb))
            dr = std::min(g, 0.0);
        else if (xj >= ub - 1e-12 && fin(ub))
            dr = std::max(g, 0.0);
        else
            dr = g;
        double d = dr / (s.obj_scale * s.col_scale[j]);
        k.rd2 += d * d;
        k.rdmax = std::max(k.rdmax, std::abs(d));
    }
    return k;
}

bool timeUp(std::chrono::steady_clock::time_point t0, double lim) {  // pdlp.cpp:83-90
    if (lim < 0.0) return false;
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= lim;
}

Outcome solve(const Lp& lp, const pdlpx_options& o, const Vec* wx, const Vec* wy) {
    Outcome out;
    auto t0 = std::chrono::steady_clock::now();
    Scaled s;
    buildScaled(lp, o, s);
    const int m = lp.m, n = lp.n;
    out.x.assign(n, 0.0);
    out.y.assign(m, 0.0);

    if (n == 0) {  // pdlp.cpp:813-820
        out.status = PDLPX_STATUS_OPTIMAL;
        out.objective = lp.offset;
        return out;
    }
    if (m == 0) {  // pdlp.cpp:823-860
        double ov = lp.offset;
        for (int j = 0; j < n; ++j) {
            double c = s.c[j], lb = s.cl[j], ub = s.cu[j], xj;
            if (c > 0.0) {
                if (!fin(lb)) {
                    out.status = PDLPX_STATUS_UNBOUNDED;
                    return out;
                }
                xj = lb;
            } else if (c < 0.0) {
                if (!fin(ub)) {
                    out.status = PDLPX_STATUS_UNBOUNDED;
                    return out;
                }
                xj = ub;
            } else {
                xj = fin(lb) ? lb : (fin(ub) ? ub : 0.0);
            }
            out.x[j] = xj * s.col_scale[j] / s.con_scale;
            ov += lp.obj[j] * out.x[j];
        }
        out.objective = ov;
        out.status = PDLPX_STATUS_OPTIMAL;
        return out;
    }

    double spectral = spectralNorm(s.a, o);
    double step = 0.998 / spectral;
    const bool adaptive = o.adaptive_step != 0;
    const double step_lb = step * o.adaptive_step_min, step_ub = step * o.adaptive_step_max;
    double pw = o.primal_weight;
    const int N = o.termination_eval_frequency;

    Iterates v;
    v.cx.assign(n, 0.0);
    v.cy.assign(m, 0.0);
    v.ix.assign(n, 0.0);
    v.iy.assign(m, 0.0);
    v.px.assign(n, 0.0);
    v.py.assign(m, 0.0);
    v.rx.assign(n, 0.0);
    v.ry.assign(m, 0.0);
    v.aty.assign(n, 0.0);
    v.atpy.assign(n, 0.0);
    v.axr.assign(m, 0.0);
    v.ax.assign(m, 0.0);
    v.dyv.assign(m, 0.0);
    v.atdy.assign(n, 0.0);
    if (adaptive) {
        v.prev_axr.assign(m, 0.0);
        v.prev_rx.assign(n, 0.0);
    }
    bool have_prev = false;
    if (wx != nullptr && wy != nullptr && static_cast<int>(wx->size()) == n &&
        static_cast<int>(wy->size()) == m) {  // pdlp.cpp:918-930
        for (int j = 0; j < n; ++j) {
            double xj = (*wx)[j] / s.col_scale[j] * s.con_scale;
            v.cx[j] = xj;
            v.ix[j] = xj;
        }
        for (int i = 0; i < m; ++i) {
            double yi = (*wy)[i] * s.obj_scale / (s.obj_sign * s.row_scale[i]);
            v.cy[i] = yi;
            v.iy[i] = yi;
        }
    }

    int inner = 0, total = 0;
    double fpe0 = -1.0, last_fpe = kInf;
    double esum = 0.0, elast = 0.0, best_pw = pw, best_score = kInf;

    // Termination norms on the original problem (pdlp.cpp:53-81).
    double c_norm = 0.0, b_norm = 0.0;
    if (o.optimality_norm == PDLPX_NORM_LINF) {
        for (double c : lp.obj) c_norm = std::max(c_norm, std::abs(c));
        for (int i = 0; i < m; ++i) {
            if (fin(lp.ru[i])) b_norm = std::max(b_norm, std::abs(lp.ru[i]));
            if (fin(lp.rl[i]) && lp.rl[i] != lp.ru[i]) b_norm = std::max(b_norm, std::abs(lp.rl[i]));
        }
    } else {
        c_norm = l2norm(lp.obj);
        double bsq = 0.0;
        for (int i = 0; i < m; ++i) {
            if (fin(lp.ru[i])) bsq += lp.ru[i] * lp.ru[i];
            if (fin(lp.rl[i]) && lp.rl[i] != lp.ru[i]) bsq += lp.rl[i] * lp.rl[i];
        }
        b_norm = std::sqrt(bsq);
    }
    const bool linf = o.optimality_norm == PDLPX_NORM_LINF;
    bool converged = false;

    Anderson aa;
    Vec aa_it, aa_res, aa_out;
    const bool use_aa = o.anderson_acceleration && o.anderson_window_size >= 2;
    if (use_aa) {
        aa.init(o.anderson_window_size, n + m, o.anderson_regularization);
        aa_it.resize(n + m);
        aa_res.resize(n + m);
        aa_out.resize(n + m);
    }
    const double work_per_iter =
        4.0 * static_cast<double>(s.a.nnz()) + 2.0 * static_cast<double>(m + n);

    // One Halpern iteration at weight lambda (pdlp.cpp:986-1071 and 1484-1522).
    auto primalStep = [&](double lambda) {
        mulT(s.a, v.cy, v.aty);
        for (int j = 0; j < n; ++j) {
            double tau = step * s.tau[j] / pw;
            double t = v.cx[j] - tau * (s.c[j] + v.aty[j]);
            v.px[j] = std::clamp(t, s.cl[j], s.cu[j]);
            v.rx[j] = 2.0 * v.px[j] - v.cx[j];
            v.cx[j] = lambda * v.rx[j] + (1.0 - lambda) * v.ix[j];
        }
        mul(s.a, v.rx, v.axr);
    };
    auto dualStep = [&](double lambda) {
        for (int i = 0; i < m; ++i) {
            double sg = step * s.sigma[i] * pw;
            double vv = v.cy[i] + sg * v.axr[i];
            double l = s.rl[i], u = s.ru[i], py;
            if (l == u)
                py = vv - sg * l;
            else if (!fin(l))
                py = std::max(0.0, vv - sg * u);
            else if (!fin(u))
                py = std::min(0.0, vv - sg * l);
            else if (vv >= sg * u)
                py = vv - sg * u;
            else if (vv <= sg * l)
                py = vv - sg * l;
            else
                py = 0.0;
            v.py[i] = py;
            v.ry[i] = 2.0 * py - v.cy[i];
            v.cy[i] = lambda * v.ry[i] + (1.0 - lambda) * v.iy[i];
        }
    };
    // Fixed-point error of the batch (pdlp.cpp:1076-1100).
    auto fixedPointError = [&]() {
        double dx2 = 0.0, dy2 = 0.0;
        for (int j = 0; j < n; ++j) {
            double d = v.px[j] - v.ix[j];
            dx2 += d * d;
        }
        for (int i = 0; i < m; ++i) {
            double d = v.py[i] - v.iy[i];
            dy2 += d * d;
        }
        double mov = dx2 * pw + dy2 / pw;
        for (int i = 0; i < m; ++i) v.dyv[i] = v.py[i] - v.iy[i];
        mulT(s.a, v.dyv, v.atdy);
        double inter = 0.0;
        for (int j = 0; j < n; ++j) inter += v.atdy[j] * (v.px[j] - v.ix[j]);
        inter *= 2.0 * step;
        return std::sqrt(std::max(mov + inter, 0.0));
    };
    auto dists = [&](double& pd, double& dd) {
        pd = 0.0;
        dd = 0.0;
        for (int j = 0; j < n; ++j) {
            double d = v.px[j] - v.ix[j];
            pd += d * d;
        }
        pd = std::sqrt(pd);
        for (int i = 0; i < m; ++i) {
            double d = v.py[i] - v.iy[i];
            dd += d * d;
        }
        dd = std::sqrt(dd);
    };
    auto restartCopy = [&]() {
        for (int j = 0; j < n; ++j) {
            v.ix[j] = v.px[j];
            v.cx[j] = v.px[j];
        }
        for (int i = 0; i < m; ++i) {
            v.iy[i] = v.py[i];
            v.cy[i] = v.py[i];
        }
    };

    while (total < o.max_iter) {  // pdlp.cpp:966-1395
        if (timeUp(t0, o.max_solve_seconds)) {
            out.status = PDLPX_STATUS_TIME_LIMIT;
            out.iterations = total;
            return out;
        }
        int batch = std::min(N, o.max_iter - total);
        for (int k = 1; k <= batch; ++k) {
            if (timeUp(t0, o.max_solve_seconds)) {
                out.status = PDLPX_STATUS_TIME_LIMIT;
                out.iterations = total + k - 1;
                return out;
            }
            double lambda = static_cast<double>(inner + k) / static_cast<double>(inner + k + 1);
            primalStep(lambda);
            if (adaptive && have_prev) {  // pdlp.cpp:1006-1035
                double ad = 0.0, xd = 0.0;
                for (int i = 0; i < m; ++i) {
                    double d = v.axr[i] - v.prev_axr[i];
                    ad += s.sigma[i] * d * d;
                }
                for (int j = 0; j < n; ++j) {
                    double d = v.rx[j] - v.prev_rx[j];
                    xd += d * d / s.tau[j];
                }
                if (xd > 1e-30) {
                    double lip2 = ad / xd;
                    double ls = 0.998 / std::sqrt(std::max(lip2, 1e-30));
                    double ns = step > ls ? step * o.adaptive_step_down : step * o.adaptive_step_up;
                    step = std::clamp(ns, step_lb, step_ub);
                }
            }
            if (adaptive) {
                v.prev_axr = v.axr;
                v.prev_rx = v.rx;
                have_prev = true;
            }
            dualStep(lambda);
        }
        inner += batch;
        total += batch;

        double fpe = fixedPointError();
        if (fpe0 < 0.0) fpe0 = fpe;

        Kkt k = residuals(s, v);
        double rel_p = std::sqrt(k.rp2) / (1.0 + b_norm);
        double rel_pi = k.rpmax / (1.0 + b_norm);
        double rel_d = std::sqrt(k.rd2) / (1.0 + c_norm);
        double rel_di = k.rdmax / (1.0 + c_norm);
        double pterm = linf ? rel_pi : rel_p;
        double dterm = linf ? rel_di : rel_d;

        double pobj_s = dotv(s.c, v.px);  // pdlp.cpp:1158-1202
        double unsc = 1.0 / (s.obj_scale * s.con_scale);
        double pobj = lp.offset + s.obj_sign * pobj_s * unsc;
        double dcol = 0.0;
        for (int j = 0; j < n; ++j) {
            double g = s.c[j] + v.atpy[j], lb = s.cl[j], ub = s.cu[j];
            if (!fin(lb)) g = std::min(g, 0.0);
            if (!fin(ub)) g = std::max(g, 0.0);
            if (g > 0.0 && fin(lb))
                dcol += g * lb;
            else if (g < 0.0 && fin(ub))
                dcol += g * ub;
        }
        double drow = 0.0;
        for (int i = 0; i < m; ++i) {
            double yi = v.py[i], l = s.rl[i], u = s.ru[i];
            if (!fin(u)) yi = std::min(yi, 0.0);
            if (!fin(l)) yi = std::max(yi, 0.0);
            if (yi > 0.0 && fin(u))
                drow -= yi * u;
            else if (yi < 0.0 && fin(l))
                drow -= yi * l;
        }
        double dobj = lp.offset + s.obj_sign * (dcol + drow) * unsc;
        double gap = std::abs(pobj - dobj) / (1.0 + std::abs(pobj) + std::abs(dobj));
        out.rp = pterm;
        out.rd = dterm;
        out.gap = gap;
        out.pobj = pobj;
        out.dobj = dobj;
        if (o.verbose && (total <= N || total % (10 * N) == 0))
            std::printf("ORACLE %7d  pobj=% .8e  pinf=% .2e  dinf=% .2e  gap=% .2e  fpe=% .2e  pw=% .2e\n",
                        total, pobj, pterm, dterm, gap, fpe, pw);
        if (pterm <= o.primal_tol && dterm <= o.dual_tol && gap <= o.optimality_tol) {
            converged = true;
            break;
        }

        if (total >= 10 * N && total % (10 * N) == 0) {  // pdlp.cpp:1224-1262
            Vec yo(m);
            double inv = 1.0 / s.obj_scale;
            for (int i = 0; i < m; ++i) yo[i] = s.obj_sign * v.py[i] * s.row_scale[i] * inv;
            if (infeasCert(yo, lp, 1e-6)) {
                out.status = PDLPX_STATUS_INFEASIBLE;
                out.iterations = total;
                out.y = yo;
                double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                out.work = static_cast<double>(total) * work_per_iter + secs * 1e-6;
                return out;
            }
            Vec xo(n);
            double invc = 1.0 / s.con_scale;
            for (int j = 0; j < n; ++j) xo[j] = v.px[j] * s.col_scale[j] * invc;
            if (unbddCert(xo, lp, 1e-6)) {
                out.status = PDLPX_STATUS_UNBOUNDED;
                out.iterations = total;
                out.x = xo;
                double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                out.work = static_cast<double>(total) * work_per_iter + secs * 1e-6;
                return out;
            }
        }

        bool restart = false;  // pdlp.cpp:1265-1279
        if (total == N)
            restart = true;
        else if (fpe0 > 0.0 && fpe <= o.restart_sufficient_decay * fpe0)
            restart = true;
        else if (fpe0 > 0.0 && fpe <= o.restart_necessary_decay * fpe0 && fpe > last_fpe)
            restart = true;
        else if (inner >= static_cast<int>(o.restart_artificial_fraction * static_cast<double>(total)))
            restart = true;
        last_fpe = fpe;

        if (restart) {
            ++out.restarts;
            if (o.update_primal_weight) {  // pdlp.cpp:1283-1323
                double pd, dd;
                dists(pd, dd);
                double ratio = rel_p > 1e-15 ? rel_d / rel_p : 0.0;
                if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
                    double e = std::log(dd) - std::log(pd) - std::log(pw);
                    esum = o.pid_i_smooth * esum + e;
                    double de = e - elast;
                    pw *= std::exp(o.pid_kp * e + o.pid_ki * esum + o.pid_kd * de);
                    pw = std::clamp(pw, 1e-4, 1e8);
                    elast = e;
                    double score = std::abs(std::log10(std::max(rel_d, 1e-15)) -
                                            std::log10(std::max(rel_p, 1e-15)));
                    if (score < best_score) {
                        best_score = score;
                        best_pw = pw;
                    }
                } else {
                    pw = best_pw;
                    esum = 0.0;
                    elast = 0.0;
                }
            }
            // Preconditioner refresh (pdlp.cpp:1326-1338).
            if (o.preconditioner_refresh && s.precond_pw > 0.0) {
                double drift = pw / s.precond_pw;
                if (drift > o.preconditioner_refresh_ratio || drift < 1.0 / o.preconditioner_refresh_ratio) {
                    pockChambolle(s.a, s.sigma, s.tau);
                    s.precond_pw = pw;
                }
            }
            bool used_aa = false;
            if (use_aa) {  // pdlp.cpp:1341-1378
                for (int j = 0; j < n; ++j) {
                    aa_it[j] = v.px[j];
                    aa_res[j] = v.px[j] - v.ix[j];
                }
                for (int i = 0; i < m; ++i) {
                    aa_it[n + i] = v.py[i];
                    aa_res[n + i] = v.py[i] - v.iy[i];
                }
                aa.store(aa_it, aa_res);
                if (aa.extrapolate(aa_out)) {
                    used_aa = true;
                    for (int j = 0; j < n; ++j) {
                        double xj = std::clamp(aa_out[j], s.cl[j], s.cu[j]);
                        v.ix[j] = xj;
                        v.cx[j] = xj;
                    }
                    for (int i = 0; i < m; ++i) {
                        v.iy[i] = aa_out[n + i];
                        v.cy[i] = aa_out[n + i];
                    }
                }
            }
            if (!used_aa) restartCopy();
            inner = 0;
            fpe0 = -1.0;
            last_fpe = kInf;
            have_prev = false;
        }
    }
    out.iterations = total;

    if (converged && o.enable_polishing) {  // pdlp.cpp:1407-1675
        Kkt k = residuals(s, v);
        double rp = linf ? k.rpmax / (1.0 + b_norm) : std::sqrt(k.rp2) / (1.0 + b_norm);
        double rd = linf ? k.rdmax / (1.0 + c_norm) : std::sqrt(k.rd2) / (1.0 + c_norm);
        bool needs = rp > o.polish_primal_tol || rd > o.polish_dual_tol;
        if (needs && !timeUp(t0, o.max_solve_seconds)) {
            restartCopy();
            inner = 0;
            fpe0 = -1.0;
            last_fpe = kInf;
            int pc = 0;
            while (pc < o.polish_max_iter) {
                if (timeUp(t0, o.max_solve_seconds)) break;
                int batch = std::min(N, o.polish_max_iter - pc);
                for (int kk = 1; kk <= batch; ++kk) {
                    if (timeUp(t0, o.max_solve_seconds)) break;
                    double lambda = static_cast<double>(inner + kk) / static_cast<double>(inner + kk + 1);
                    primalStep(lambda);
                    dualStep(lambda);
                }
                inner += batch;
                pc += batch;
                total += batch;
                double fpe = fixedPointError();
                if (fpe0 < 0.0) fpe0 = fpe;
                Kkt q = residuals(s, v);
                double rpn = linf ? q.rpmax / (1.0 + b_norm) : std::sqrt(q.rp2) / (1.0 + b_norm);
                double rdn = linf ? q.rdmax / (1.0 + c_norm) : std::sqrt(q.rd2) / (1.0 + c_norm);
                double rpp = std::sqrt(q.rp2) / (1.0 + b_norm);
                double rdp = std::sqrt(q.rd2) / (1.0 + c_norm);
                out.rp = rpn;
                out.rd = rdn;
                if (rpn <= o.polish_primal_tol && rdn <= o.polish_dual_tol) break;
                bool restart = false;
                if (pc == batch)
                    restart = true;
                else if (fpe0 > 0.0 && fpe <= o.restart_sufficient_decay * fpe0)
                    restart = true;
                else if (fpe0 > 0.0 && fpe <= o.restart_necessary_decay * fpe0 && fpe > last_fpe)
                    restart = true;
                else if (inner >= static_cast<int>(o.restart_artificial_fraction * static_cast<double>(pc)))
                    restart = true;
                last_fpe = fpe;
                if (restart) {
                    if (o.update_primal_weight) {
                        double pd, dd;
                        dists(pd, dd);
                        double ratio = rpp > 1e-15 ? rdp / rpp : 0.0;
                        if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
                            double e = std::log(dd) - std::log(pd) - std::log(pw);
                            esum = o.pid_i_smooth * esum + e;
                            double de = e - elast;
                            pw *= std::exp(o.pid_kp * e + o.pid_ki * esum + o.pid_kd * de);
                            pw = std::clamp(pw, 1e-4, 1e8);
                            elast = e;
                        }
                    }
                    restartCopy();
                    inner = 0;
                    fpe0 = -1.0;
                    last_fpe = kInf;
                }
            }
            out.iterations = total;
        }
    }

    out.step = step;
    out.pw = pw;
    if (converged) {  // pdlp.cpp:1677-1704
        double invc = 1.0 / s.con_scale;
        for (int j = 0; j < n; ++j) {
            double xj = v.px[j] * s.col_scale[j] * invc;
            if (fin(lp.cl[j])) xj = std::max(xj, lp.cl[j]);
            if (fin(lp.cu[j])) xj = std::min(xj, lp.cu[j]);
            out.x[j] = xj;
        }
        double invo = 1.0 / s.obj_scale;
        for (int i = 0; i < m; ++i) out.y[i] = s.obj_sign * v.py[i] * s.row_scale[i] * invo;
        double ov = lp.offset;
        for (int j = 0; j < n; ++j) ov += lp.obj[j] * out.x[j];
        out.objective = ov;
        out.status = PDLPX_STATUS_OPTIMAL;
    } else {
        out.status = timeUp(t0, o.max_solve_seconds) ? PDLPX_STATUS_TIME_LIMIT : PDLPX_STATUS_ITER_LIMIT;
        out.objective = 0.0;
    }
    out.work = static_cast<double>(total) * work_per_iter;
    return out;
}

Lp fromC(const pdlpx_lp* in) {
    Lp lp;
    lp.m = in->m;
    lp.n = in->n;
    lp.maximize = in->sense == PDLPX_MAXIMIZE;
    lp.a = canonical(in->m, in->n, in->row_ptr, in->col_idx, in->val);
    lp.obj.assign(in->obj, in->obj + in->n);
    lp.cl.assign(in->col_lb, in->col_lb + in->n);
    lp.cu.assign(in->col_ub, in->col_ub + in->n);
    lp.rl.assign(in->row_lb, in->row_lb + in->m);
    lp.ru.assign(in->row_ub, in->row_ub + in->m);
    lp.offset = in->obj_offset;
    return lp;
}

}  // namespace

extern "C" {

// Full CPU PDLP solve.  x[n], y[m] may be NULL.
int oracle_pdlp_solve(const pdlpx_lp* lp, const pdlpx_options* o, pdlpx_result* res, double* x,
                      double* y) {
    if (lp == nullptr || o == nullptr || res == nullptr) return PDLPX_E_INVALID;
    Lp p = fromC(lp);
    Vec wx, wy;
    bool warm = lp->warm_x != nullptr && lp->warm_y != nullptr;
    if (warm) {
        wx.assign(lp->warm_x, lp->warm_x + lp->n);
        wy.assign(lp->warm_y, lp->warm_y + lp->m);
    }
    auto t0 = std::chrono::steady_clock::now();
    Outcome r = solve(p, *o, warm ? &wx : nullptr, warm ? &wy : nullptr);
    std::memset(res, 0, sizeof(*res));
    res->status = r.status;
    res->objective = r.objective;
    res->iterations = r.iterations;
    res->work_units = r.work;
    res->rel_primal_resid = r.rp;
    res->rel_dual_resid = r.rd;
    res->rel_gap = r.gap;
    res->primal_objective = r.pobj;
    res->dual_objective = r.dobj;
    res->restarts = r.restarts;
    res->step_size = r.step;
    res->primal_weight = r.pw;
    res->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (x != nullptr)
        for (int j = 0; j < lp->n; ++j) x[j] = r.x[j];
    if (y != nullptr)
        for (int i = 0; i < lp->m; ++i) y[i] = r.y[i];
    return PDLPX_OK;
}

// Scaling pipeline outputs (pdlp.cpp:469-669), arrays sized like pdlpx_get_scaling.
int oracle_scaling(const pdlpx_lp* lp, const pdlpx_options* o, double* col_scale, double* cscaled,
                   double* cl, double* row_scale, double* rl, double* ru, double* tau, double* sigma,
                   double* cu, double* obj_scale, double* con_scale) {
    Lp p = fromC(lp);
    Scaled s;
    buildScaled(p, *o, s);
    for (int j = 0; j < p.n; ++j) {
        if (col_scale) col_scale[j] = s.col_scale[j];
        if (cscaled) cscaled[j] = s.c[j];
        if (cl) cl[j] = s.cl[j];
        if (cu) cu[j] = s.cu[j];
        if (tau) tau[j] = s.tau[j];
    }
    for (int i = 0; i < p.m; ++i) {
        if (row_scale) row_scale[i] = s.row_scale[i];
        if (rl) rl[i] = s.rl[i];
        if (ru) ru[i] = s.ru[i];
        if (sigma) sigma[i] = s.sigma[i];
    }
    if (obj_scale) *obj_scale = s.obj_scale;
    if (con_scale) *con_scale = s.con_scale;
    return 0;
}

// Spectral-norm estimate of the scaled matrix (pdlp.cpp:748-795).
double oracle_spectral_norm(const pdlpx_lp* lp, const pdlpx_options* o) {
    Lp p = fromC(lp);
    Scaled s;
    buildScaled(p, *o, s);
    return spectralNorm(s.a, *o);
}

// y = A x in FP64 with the reference's row order (sparse_matrix.cpp:181-193).
int oracle_csr_multiply(int rows, int cols, const int* rp, const int* ci, const double* v,
                        const double* x, double* y) {
    (void)cols;
    for (int i = 0; i < rows; ++i) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
    return 0;
}

// y = A^T x by row scatter (sparse_matrix.cpp:195-208).
int oracle_csr_multiply_transpose(int rows, int cols, const int* rp, const int* ci, const double* v,
                                  const double* x, double* y) {
    for (int j = 0; j < cols; ++j) y[j] = 0.0;
    for (int i = 0; i < rows; ++i) {
        if (x[i] == 0.0) continue;
        for (int k = rp[i]; k < rp[i + 1]; ++k) y[ci[k]] += v[k] * x[i];
    }
    return 0;
}

}  // extern "C"

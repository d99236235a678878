// Controller logic of one check, shared by the single-LP graph (engine.cu) and the
// packed batch (batch.cu, one warp per LP): restart / primal weight / polish /
// termination of PdlpSolver::solve (pdlp.cpp:2228-2469 main loop, 2592-2666
// polish), FP64, executed by one thread.
#pragma once

#include "kernels.cuh"
#include "pdlpx.h"

namespace pdlpx {

// Reduce [nb][NS] partials in fixed order into out[NS] (block of kBlock threads).
template <int NS>
__device__ inline void reducePartials(const double* part, int nb, const int (&ops)[NS], double* out) {
    double acc[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] = slotInit(ops[s]);
    for (int b = threadIdx.x; b < nb; b += kBlock) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double v = part[static_cast<size_t>(b) * NS + s];
            acc[s] = ops[s] == OP_SUM ? acc[s] + v : (ops[s] == OP_MIN ? fmin(acc[s], v) : fmax(acc[s], v));
        }
    }
    blockReduceSlots<NS>(acc, ops, out);
}

// Restart / primal weight / polish / termination logic of one check
// (pdlp.cpp:2228-2469 main loop, 2592-2666 polish), FP64, one thread.
__device__ inline void controlStep(DevState& s, const DevConst& c, const double* rows, const double* cols) {
    const int cur = s.phase == 0 ? s.total : s.polish_count;
    const int lim = s.phase == 0 ? c.max_iter : c.polish_max_iter;
    const int batch = min(c.N, lim - cur);
    s.total += batch;
    s.inner += batch;
    if (s.phase == 1) s.polish_count += batch;
    s.checks += 1;

    const double dx2 = cols[C_PDIST], dy2 = rows[R_DDIST];
    const double movement = dx2 * s.pw + dy2 / s.pw;
    const double interaction = cols[C_INTER] * (2.0 * s.step);
    const double fpe = sqrt(fmax(movement + interaction, 0.0));
    if (s.fpe0 < 0.0) s.fpe0 = fpe;

    const double rel_p = sqrt(rows[R_PRES_SQ]) / (1.0 + c.b_norm);
    const double rel_pi = rows[R_PRES_MAX] / (1.0 + c.b_norm);
    const double rel_d = sqrt(cols[C_DRES_SQ]) / (1.0 + c.c_norm);
    const double rel_di = cols[C_DRES_MAX] / (1.0 + c.c_norm);
    const double pterm = c.linf ? rel_pi : rel_p;
    const double dterm = c.linf ? rel_di : rel_d;
    const double unsc = 1.0 / (c.obj_scale * c.con_scale);
    const double pobj = c.offset + c.obj_sign * cols[C_POBJ] * unsc;
    const double dobj = c.offset + c.obj_sign * (cols[C_DOBJ_COL] + rows[R_DOBJ_ROW]) * unsc;
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    s.rel_p = rel_p;
    s.rel_d = rel_d;
    s.rel_pi = rel_pi;
    s.rel_di = rel_di;
    s.pterm = pterm;
    s.dterm = dterm;
    s.gap = gap;
    s.pobj = pobj;
    s.dobj = dobj;
    s.fpe = fpe;
    s.restart = 0;
    s.promote = 0;

    auto piUpdate = [&](double rp, double rd, bool track_best) {
        const double pd = sqrt(dx2), dd = sqrt(dy2);
        const double ratio = rp > 1e-15 ? rd / rp : 0.0;
        if (pd > 1e-16 && dd > 1e-16 && pd < 1e12 && dd < 1e12 && ratio > 1e-8 && ratio < 1e8) {
            const double e = log(dd) - log(pd) - log(s.pw);
            s.esum = c.ismooth * s.esum + e;
            const double de = e - s.elast;
            s.pw *= exp(c.kp * e + c.ki * s.esum + c.kd * de);
            s.pw = fmin(fmax(s.pw, 1e-4), 1e8);
            s.elast = e;
            if (track_best) {
                const double score = fabs(log10(fmax(rd, 1e-15)) - log10(fmax(rp, 1e-15)));
                if (score < s.best_score) {
                    s.best_score = score;
                    s.best_pw = s.pw;
                }
            }
        } else if (track_best) {
            s.pw = s.best_pw;
            s.esum = 0.0;
            s.elast = 0.0;
        }
    };
    auto resetCycle = [&]() {
        s.restart = 1;
        s.restarts += 1;
        s.inner = 0;
        s.fpe0 = -1.0;
        s.last_fpe = CUDART_INF;
        s.have_prev = 0;
    };

    if (s.phase == 0) {
        if (pterm <= c.primal_tol && dterm <= c.dual_tol && gap <= c.opt_tol) {
            s.converged = 1;
            if (c.enable_polish && (pterm > c.polish_ptol || dterm > c.polish_dtol)) {
                s.phase = 1;  // polish: restart from pdhg iterates (pdlp.cpp:2524-2529)
                s.polish_count = 0;
                s.restart = 1;
                s.inner = 0;
                s.fpe0 = -1.0;
                s.last_fpe = CUDART_INF;
            } else {
                s.done = 1;
                s.status = PDLPX_STATUS_OPTIMAL;
            }
        } else {
            if (c.adaptive) {  // GPU variant of the adaptive step (pdlp.cpp:2274-2307)
                if (s.have_prev) {
                    const double ad = rows[R_ADAPT], xd = cols[C_ADAPT];
                    if (xd > 1e-30) {
                        const double lip2 = ad / xd;
                        const double ls = 0.998 / sqrt(fmax(lip2, 1e-30));
                        const double ns = s.step > ls ? s.step * c.step_down : s.step * c.step_up;
                        s.step = fmin(fmax(ns, c.step_lb), c.step_ub);
                    }
                }
                s.have_prev = 1;
            }
            if (s.total >= 10 * c.N && s.total % (10 * c.N) == 0) {
                // Farkas dual ray (pdlp.cpp:119-211) from scaled-space reductions.
                const double yq = sqrt(rows[R_YNORM]);
                if (c.m > 0 && yq / c.obj_scale >= 1e-15) {
                    const double thr = 1e-6 * yq;
                    const bool signs = !(rows[R_MIN_LE] < -thr) && !(rows[R_MAX_GE] > thr) &&
                                       !(cols[C_MIN_GLB] < -thr) && !(cols[C_MAX_GUB] > thr);
                    if (signs) {
                        const double farkas = (rows[R_FARKAS_ROW] - cols[C_COLSUP]) / (c.con_scale * yq);
                        if (farkas < -1e-6) {
                            s.done = 1;
                            s.status = PDLPX_STATUS_INFEASIBLE;
                            s.cert_hit = 1;
                        }
                    }
                }
                // Primal ray (pdlp.cpp:220-284).
                const double xq = sqrt(cols[C_XNORM]);
                if (!s.done && c.n > 0 && xq / c.con_scale >= 1e-15) {
                    const double thr = 1e-6 * xq;
                    const bool ok = !(cols[C_MIN_XLB] < -thr) && !(cols[C_MAX_XUB] > thr) &&
                                    !(rows[R_UB_TWO] > thr) && !(rows[R_UB_LE] > thr) &&
                                    !(rows[R_UB_GE] < -thr);
                    if (ok && cols[C_POBJ] / (c.obj_scale * xq) < -1e-6) {
                        s.done = 1;
                        s.status = PDLPX_STATUS_UNBOUNDED;
                        s.cert_hit = 2;
                    }
                }
            }
            if (!s.done) {
                bool rs = false;
                if (s.total == c.N)
                    rs = true;
                else if (s.fpe0 > 0.0 && fpe <= c.suff * s.fpe0)
                    rs = true;
                else if (s.fpe0 > 0.0 && fpe <= c.nec * s.fpe0 && fpe > s.last_fpe)
                    rs = true;
                else if (s.inner >= static_cast<int>(c.art * static_cast<double>(s.total)))
                    rs = true;
                s.last_fpe = fpe;
                if (rs) {
                    if (c.update_pw) piUpdate(rel_p, rel_d, true);
                    // Preconditioner refresh recomputes sigma/tau from the unchanged scaled
                    // matrix (pdlp.cpp:713-742), which reproduces the same values; only the
                    // reference weight moves.
                    if (c.precond_refresh && s.precond_pw > 0.0) {
                        const double drift = s.pw / s.precond_pw;
                        if (drift > c.precond_ratio || drift < 1.0 / c.precond_ratio) s.precond_pw = s.pw;
                    }
                    resetCycle();
                }
                if (s.total >= c.max_iter) {
                    s.done = 1;
                    s.status = PDLPX_STATUS_ITER_LIMIT;
                }
            }
        }
    } else {
        if (pterm <= c.polish_ptol && dterm <= c.polish_dtol) {
            s.done = 1;
            s.status = PDLPX_STATUS_OPTIMAL;
        } else {
            bool rs = false;
            if (s.polish_count == batch)
                rs = true;
            else if (s.fpe0 > 0.0 && fpe <= c.suff * s.fpe0)
                rs = true;
            else if (s.fpe0 > 0.0 && fpe <= c.nec * s.fpe0 && fpe > s.last_fpe)
                rs = true;
            else if (s.inner >= static_cast<int>(c.art * static_cast<double>(s.polish_count)))
                rs = true;
            s.last_fpe = fpe;
            if (rs) {
                if (c.update_pw) piUpdate(rel_p, rel_d, false);
                resetCycle();
            }
            if (s.polish_count >= c.polish_max_iter) {
                s.done = 1;
                s.status = PDLPX_STATUS_OPTIMAL;
            }
        }
    }

    // Mixed precision: hand the iterates to FP64 when the FP32 phase stalls close
    // to the tolerance (score = worst KKT term / its tolerance <= switch_score)
    // while a residual that misses its tolerance sits near its FP32 noise floor:
    // the rounding of an FP32 product of row i is of order 2^-24 sum_j |a_ij x_j|,
    // so the primal (dual) residual cannot fall much below
    // 2^-24 || sum_j |a_ij x_j| || (the same with |a_ij y_i|), in the units of
    // the relative residual.  A plateau far
    // above that floor is ordinary PDHG behaviour and stays in FP32 (measured on
    // the 500k x 2M power-law LP: FP32 alone converges in the same iteration
    // count as the mixed solve that handed over at a quarter of it).
    if (c.mixed && c.fp64_switch && s.prec == 0 && !s.done) {
        const double pt = s.phase == 0 ? c.primal_tol : c.polish_ptol;
        const double dt = s.phase == 0 ? c.dual_tol : c.polish_dtol;
        double score = fmax(pterm / pt, dterm / dt);
        if (s.phase == 0) score = fmax(score, gap / c.opt_tol);
        constexpr double kU32 = 5.9604644775390625e-08;  // 2^-24
        const double noise_p = kU32 * sqrt(rows[R_NOISE_SQ]) / (1.0 + c.b_norm);
        const double noise_d = kU32 * sqrt(cols[C_NOISE_SQ]) / (1.0 + c.c_norm);
        // only a term that still misses its tolerance can be held up by the floor;
        // a gap-limited stall counts when either residual sits at its floor
        const bool p_floor = pterm <= c.noise_factor * noise_p;
        const bool d_floor = dterm <= c.noise_factor * noise_d;
        const bool gap_open = s.phase == 0 && gap > c.opt_tol;
        const bool near_floor = (pterm > pt && p_floor) || (dterm > dt && d_floor) ||
                                (gap_open && pterm <= pt && dterm <= dt && (p_floor || d_floor));
        if (score <= c.switch_score) {
            if (score < 0.7 * s.best_kkt) {
                s.best_kkt = score;
                s.stall = 0;
            } else if (near_floor) {
                s.stall += 1;
            }
            if (s.stall >= c.stall_limit) s.promote = 1;
        }
    }
    s.tau_fac = static_cast<float>(s.step / s.pw);
    s.sig_fac = static_cast<float>(s.step * s.pw);
}

}  // namespace pdlpx

// Family packs: node LPs that share the leading rows of one base matrix.
//
// Branch-and-bound node LPs of one base LP (bound changes on integer columns
// and a few appended cut rows) have the same constraint matrix in their first
// m_b rows.  A family pack stores those rows once and runs up to 32 node LPs
// over them in the same sweep: one lane per LP, a warp per group of adjacent
// rows or columns.  The warp loads a row's entries once
// (coalesced, broadcast by shuffle) and every lane gathers its own LP's value
// of each entry; per-LP vectors are interleaved [row or column][32 lanes], so
// each gather of the warp is one 256-byte request instead of 32 scattered
// sectors, and the matrix bytes of an iteration are shared by all its LPs.
//
// Each LP keeps its own scaling (Ruiz row / column factors, Pock-Chambolle
// step sizes, bound and objective rescaling, exactly as a separate solve
// computes them, pdlp.cpp:469-669): the shared values are the original ones and
// the scaled product is formed on the fly, (A_l x)_i = r_li sum_j a_ij (c_lj x_j).
// The primal step stores c .* x_refl and the dual step r .* y_cur next to the
// iterates, so the gathers need no scale factor.  Rows an LP appends after the
// base rows ("cut rows") are its own CSR rows, handled by a warp per row in the
// dual step and, for the primal step, by a per-column list of the appended
// entries of every LP.
//
// Iterates are FP64 throughout (the shared matrix is read once per iteration,
// so the per-LP vectors are the traffic); per-LP DevState / DevConst and the
// single-LP controlStep, restart, polish and termination rules as in the packed
// batch.  Lane l's arithmetic and reduction order depend on LP l alone, so a
// node LP's result is the same in a family of one and in any mix.

constexpr int kFam = 32;  // lanes (LPs) per family pack
// Consecutive columns / base rows one warp of a step kernel walks as one
// contiguous entry range (their CSR entries are adjacent), so a warp keeps
// several rows' loads and gathers in flight instead of one short row's.
constexpr int kFamColsPerWarp = 4;
constexpr int kFamRowsPerWarp = 2;
constexpr unsigned kFull = 0xffffffffu;

// Per-lane step parameters of the running cycle, structure of arrays so that a
// warp reads its 32 LPs' values with one coalesced load each (the solver state
// itself is an array of structures: 32 lanes would touch 32 cache lines per
// field).  Written at the end of every cycle (and before the first) from the
// controller's state; allow = iterations this cycle (0 when finished).
struct FamLane {
    double step[kFam];
    double pw[kFam];
    int inner[kFam];
    int allow[kFam];
};

struct FamArgs {
    const int* a_ptr;     // base rows (original values); the entry indices are
    const int* a_idx;     // stored times 32, the offset of the entry's slot of lane 0
    const double* a_val;
    const int* at_ptr;    // base rows transposed
    const int* at_idx;
    const double* at_val;
    const int* k_ptr;     // appended rows of all LPs
    const int* k_idx;
    const double* k_val;
    const int* k_lane;    // LP of each appended row
    const int* k_first;   // [33] first appended row of each lane
    const int* kt_ptr;    // appended entries by column: row, LP, value
    const int* kt_row;
    const int* kt_lane;
    const double* kt_val;
    const ColPack<double>* cp;  // [n][32]
    const double* cs;           // column scale [n][32]
    double *xc, *xi, *xh, *xs;  // [n][32]; xs = column scale * x_refl
    const RowPack<double>* rp;  // [m_b][32] then [K]
    const double* rs;           // row scale
    double *yc, *yi, *yh, *ys;  // ys = row scale * y_cur
    DevState* st;
    const DevConst* dc;
    PowerState* ps;
    int* flags;
    int* counters;
    const unsigned* live;  // bit l: LP l had not finished at the end of the last cycle
    FamLane* lanes;
    double* part_rows;  // [block][32][kRowSlots]
    double* part_cols;  // [block][32][kColSlots]
    double *pi_x, *pi_y, *pi_xn, *pi_part;
    int n, mb, K, L;
    int gb, gk;           // power blocks over base rows, appended rows (one row per warp)
    int gp, gd;           // step blocks: columns, base rows (kFamColsPerWarp / kFamRowsPerWarp per warp)
    int nbr, nbk, nbc;    // check blocks: base rows, appended rows (one per lane, or none), columns
    int max_iter, polish_max_iter, N, sv_max_iter;
    double sv_tol;
};

__device__ __forceinline__ size_t fIdx(int r, int l) { return static_cast<size_t>(r) * kFam + l; }
__device__ __forceinline__ size_t fCut(const FamArgs& a, int q) { return static_cast<size_t>(a.mb) * kFam + q; }

// Dot product of one shared row with lane l's vector get(entry index): the warp
// loads up to 32 entries with one coalesced load per array, broadcasts them by
// shuffle and every active lane gathers its own values, eight gathers in flight
// per round before the products wait on them.  The loop bounds are
// warp-uniform; the slots of a round past the row's end gather nothing.
template <class Get>
__device__ __forceinline__ double famDot(const int* __restrict__ idx, const double* __restrict__ val, int b, int e,
                                         int l, bool on, Get get) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int c0 = b; c0 < e; c0 += 32) {
        const int cnt = min(32, e - c0);
        int mc = 0;
        double mv = 0.0;
        if (l < cnt) {
            mc = __ldg(idx + c0 + l);
            mv = __ldg(val + c0 + l);
        }
        for (int k = 0; k < cnt; k += 8) {
            int q[8];
            double v[8], g[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                q[u] = __shfl_sync(kFull, mc, (k + u) & 31);
                v[u] = __shfl_sync(kFull, mv, (k + u) & 31);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) g[u] = (on && k + u < cnt) ? get(q[u]) : 0.0;
            s0 += v[0] * g[0];
            s1 += v[1] * g[1];
            s2 += v[2] * g[2];
            s3 += v[3] * g[3];
            s0 += v[4] * g[4];
            s1 += v[5] * g[5];
            s2 += v[6] * g[6];
            s3 += v[7] * g[7];
        }
    }
    return (s0 + s1) + (s2 + s3);
}

// famDot over R consecutive rows whose entries are adjacent: bnd[0..R] are
// their CSR bounds (rows past the last real one empty).  Entries are taken in
// order, eight gathers per round, into one running sum that is handed to the
// row's slot when the entry position crosses the row's end (a warp-uniform
// test; the next bound comes by shuffle from the lane that loaded it), so
// every row is summed in entry order with one multiply-add per entry.
template <int R, class Get>
__device__ __forceinline__ void famDotRows(const int* __restrict__ idx, const double* __restrict__ val,
                                           const int (&bnd)[R + 1], int pl, int l, bool on, Get get, double (&s)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) s[r] = 0.0;
    const int b = bnd[0], e = bnd[R];
    int cr = 0;
    int nextb = bnd[1];
    double acc = 0.0;
    auto flush = [&]() {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (r == cr) s[r] = acc;
        acc = 0.0;
        ++cr;
        nextb = __shfl_sync(kFull, pl, min(cr + 1, R));
    };
    for (int c0 = b; c0 < e; c0 += 32) {
        const int cnt = min(32, e - c0);
        int mc = 0;
        double mv = 0.0;
        if (l < cnt) {
            mc = __ldg(idx + c0 + l);
            mv = __ldg(val + c0 + l);
        }
        // full rounds of eight, then one masked round for the rest
        auto round = [&](int k, auto masked) {
            constexpr bool M = decltype(masked)::value;
            int q[8];
            double v[8], g[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                q[u] = __shfl_sync(kFull, mc, (k + u) & 31);
                v[u] = __shfl_sync(kFull, mv, (k + u) & 31);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) g[u] = (on && (!M || k + u < cnt)) ? get(q[u]) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (M && k + u >= cnt) break;
                const int pos = c0 + k + u;
                while (pos >= nextb) flush();
                acc += v[u] * g[u];
            }
        };
        int k = 0;
        for (; k + 8 <= cnt; k += 8) round(k, std::false_type{});
        if (k < cnt) round(k, std::true_type{});
    }
    while (cr < R) flush();
}

// CSR bounds of the rows first .. first + R - 1 (clipped to `rows`) from one
// coalesced load: bnd[r] = ptr[first + min(r, count)];
// pl is this lane's loaded bound (lane r holds bnd[r]; lanes past the last
// real row hold the last bound).
template <int R>
__device__ __forceinline__ int famBounds(const int* __restrict__ ptr, int first, int rows, int l, int (&bnd)[R + 1],
                                         int& pl) {
    const int count = min(R, rows - first);
    const int p = __ldg(ptr + first + min(l, count));
#pragma unroll
    for (int r = 0; r <= R; ++r) bnd[r] = __shfl_sync(kFull, p, min(r, count));
    pl = p;
    return count;
}

__device__ __forceinline__ void famPrefetch(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Sum of one appended row of LP lp against get(column): lanes stride over the
// entries, fixed-order butterfly; every lane returns the sum.
template <class Get>
__device__ __forceinline__ double famCutDot(const FamArgs& a, int q, int l, Get get) {
    double s = 0.0;
    for (int k = a.k_ptr[q] + l; k < a.k_ptr[q + 1]; k += 32) s += a.k_val[k] * get(a.k_idx[k]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(kFull, s, off);
    return s;
}

// Dual proximal step of one row (pdlp_kernels.cu:94-157, as dualUpdate) given
// s = (A_l x_refl)_i; returns the new current y, py the pdhg y.
__device__ __forceinline__ double famDualStep(const RowPack<double>& q, double yc, double yi, double s, double step,
                                              double pw, double lam, double& py) {
    const double sig = step * q.sigma * pw;
    const double v = yc + sig * s;
    const int type = static_cast<int>(q.type);
    if (type == 0) {
        py = v - sig * q.rl;
    } else if (type == 1) {
        py = v - sig * q.ru;
        if (py < 0.0) py = 0.0;
    } else if (type == 2) {
        py = v - sig * q.rl;
        if (py > 0.0) py = 0.0;
    } else {
        if (v >= sig * q.ru)
            py = v - sig * q.ru;
        else if (v <= sig * q.rl)
            py = v - sig * q.rl;
        else
            py = 0.0;
    }
    const double yr = 2.0 * py - yc;
    return lam * yr + (1.0 - lam) * yi;
}

// ---- PDHG step -----------------------------------------------------------------
// Primal: one warp per kFamColsPerWarp consecutive columns;
// (A_l^T y)_j = c_lj (sum_i a_ij ys_il + appended entries).  Lanes of LPs
// still running gather at once (the live mask of the last cycle); the solver
// state -- iteration limits inside the cycle, step, weight -- is read after
// the sums, and the per-lane column data is prefetched into L2 meanwhile.
__global__ void __launch_bounds__(kBlock, 4) famPrimal(FamArgs a, int koff) {
    constexpr int R = kFamColsPerWarp;
    const int j0 = (static_cast<int>(blockIdx.x) * kWarps + static_cast<int>(threadIdx.x >> 5)) * R;
    const int l = threadIdx.x & 31;
    if (j0 >= a.n) return;
    const bool live = (*a.live >> l) & 1u;
    if (__ballot_sync(kFull, live) == 0) return;
    int bnd[R + 1], kbd[R + 1], pl, pk;
    const int nr = famBounds<R>(a.at_ptr, j0, a.n, l, bnd, pl);
    famBounds<R>(a.kt_ptr, j0, a.n, l, kbd, pk);
    if (live)
        for (int r = 0; r < nr; ++r) {
            const size_t q = fIdx(j0 + r, l);
            famPrefetch(a.cp + q);
            famPrefetch(a.cs + q);
            famPrefetch(a.xc + q);
            famPrefetch(a.xi + q);
        }
    const double* ys = a.ys;
    double s[R];
    famDotRows<R>(a.at_idx, a.at_val, bnd, pl, l, live, [&](int i) { return __ldg(ys + (static_cast<size_t>(i) + l)); }, s);
#pragma unroll
    for (int r = 0; r < R; ++r)
        for (int k = kbd[r]; k < kbd[r + 1]; ++k)
            if (live && a.kt_lane[k] == l) s[r] += a.kt_val[k] * ys[fCut(a, a.kt_row[k])];
    const int allow = a.lanes->allow[l];
    if (!live || koff > allow) return;
    const bool last = koff == allow;
    const double step = a.lanes->step[l], pw = a.lanes->pw[l];
    const int kk = a.lanes->inner[l] + koff;
    const double lam = static_cast<double>(kk) / static_cast<double>(kk + 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (r >= nr) break;
        const size_t q = fIdx(j0 + r, l);
        const ColPack<double> c = a.cp[q];
        const double cs = a.cs[q], xc = a.xc[q], xi = a.xi[q];
        const double tau = step * c.tau / pw;
        double xh = xc - tau * (c.c + cs * s[r]);
        if (xh < c.lb) xh = c.lb;
        if (xh > c.ub) xh = c.ub;
        const double xr = 2.0 * xh - xc;
        a.xc[q] = lam * xr + (1.0 - lam) * xi;
        a.xs[q] = cs * xr;
        if (last) a.xh[q] = xh;
    }
}

// Dual: blocks [0, gd) one warp per kFamRowsPerWarp base rows, then one warp
// per appended row.
__global__ void __launch_bounds__(kBlock, 4) famDual(FamArgs a, int koff) {
    const int w = static_cast<int>(threadIdx.x >> 5);
    const int l = threadIdx.x & 31;
    const double* xs = a.xs;
    if (static_cast<int>(blockIdx.x) < a.gd) {
        constexpr int R = kFamRowsPerWarp;
        const int i0 = (static_cast<int>(blockIdx.x) * kWarps + w) * R;
        if (i0 >= a.mb) return;
        const bool live = (*a.live >> l) & 1u;
        if (__ballot_sync(kFull, live) == 0) return;
        int bnd[R + 1], pl;
        const int nr = famBounds<R>(a.a_ptr, i0, a.mb, l, bnd, pl);
        if (live)
            for (int r = 0; r < nr; ++r) {
                const size_t q = fIdx(i0 + r, l);
                famPrefetch(a.rp + q);
                famPrefetch(a.rs + q);
                famPrefetch(a.yc + q);
                famPrefetch(a.yi + q);
            }
        double s[R];
        famDotRows<R>(a.a_idx, a.a_val, bnd, pl, l, live, [&](int j) { return __ldg(xs + (static_cast<size_t>(j) + l)); }, s);
        const int allow = a.lanes->allow[l];
        if (!live || koff > allow) return;
        const bool last = koff == allow;
        const double step = a.lanes->step[l], pw = a.lanes->pw[l];
        const int kk = a.lanes->inner[l] + koff;
        const double lam = static_cast<double>(kk) / static_cast<double>(kk + 1);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r >= nr) break;
            const size_t q = fIdx(i0 + r, l);
            const double rs = a.rs[q], yc = a.yc[q];
            double py;
            const double yn = famDualStep(a.rp[q], yc, a.yi[q], rs * s[r], step, pw, lam, py);
            a.yc[q] = yn;
            a.ys[q] = rs * yn;
            if (last) a.yh[q] = py;
        }
        return;
    }
    const int qq = (static_cast<int>(blockIdx.x) - a.gd) * kWarps + w;
    if (qq >= a.K) return;
    const int lp = a.k_lane[qq];
    bool last = false;
    if (!active(a.st + lp, 1, koff, a.max_iter, a.polish_max_iter, last, a.N)) return;  // warp-uniform
    const double s = famCutDot(a, qq, l, [&](int j) { return __ldg(xs + fIdx(j, lp)); });
    if (l != 0) return;
    const size_t q = fCut(a, qq);
    const DevState* st = a.st + lp;
    const int kk = st->inner + koff;
    const double lam = static_cast<double>(kk) / static_cast<double>(kk + 1);
    const double rs = a.rs[q], yc = a.yc[q];
    double py;
    const double yn = famDualStep(a.rp[q], yc, a.yi[q], rs * s, st->step, st->pw, lam, py);
    a.yc[q] = yn;
    a.ys[q] = rs * yn;
    if (last) a.yh[q] = py;
}

// ---- FP64 check pass: per-lane block partials [block][32][NS] -----------------------
template <int NS>
__device__ __forceinline__ void famBlockReduce(const double (&acc)[NS], const int (&ops)[NS], double* out) {
    __shared__ double red[kWarps][kFam][NS];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < NS; ++s) red[w][l][s] = acc[s];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            double v = red[0][l][s];
            for (int k = 1; k < kWarps; ++k) v = combine(ops[s], v, red[k][l][s]);
            out[static_cast<size_t>(l) * NS + s] = v;
        }
    }
}

__device__ __forceinline__ bool famChecking(const FamArgs& a, int l) {
    return l < a.L && !a.st[l].done && a.st[l].prec == 1;
}

// Rows: blocks [0, nbr) stride over the base rows; block nbr + l takes the
// appended rows of lane l (their terms go to lane l's partial), so an LP's
// reduction order does not depend on the other LPs of the pack.
__global__ void __launch_bounds__(kBlock) famCheckRows(FamArgs a) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int ops[kRowSlots];
    double acc[kRowSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) {
        ops[s] = rowSlotOp(s);
        acc[s] = slotInit(ops[s]);
    }
    const double *xh = a.xh, *cs = a.cs;
    if (static_cast<int>(blockIdx.x) < a.nbr) {
        const bool on = famChecking(a, l);
        for (int i = static_cast<int>(blockIdx.x) * kWarps + w; i < a.mb; i += a.nbr * kWarps) {
            const double s = famDot(a.a_idx, a.a_val, a.a_ptr[i], a.a_ptr[i + 1], l, on, [&](int j) {
                const size_t c = static_cast<size_t>(j) + l;
                return cs[c] * xh[c];
            });
            if (on) {
                const size_t q = fIdx(i, l);
                const RowPack<double> r = a.rp[q];
                const double rsv = a.rs[q];
                accRowMetrics(acc, a.dc[l], rsv * s, r.rl, r.ru, rsv, a.yh[q], a.yi[q]);
            }
        }
    } else {
        const int lp = static_cast<int>(blockIdx.x) - a.nbr;
        const bool live = famChecking(a, lp);  // block-uniform
        const int q1 = a.k_first[lp + 1];
        for (int qq = a.k_first[lp] + w; live && qq < q1; qq += kWarps) {
            const double s = famCutDot(a, qq, l, [&](int j) {
                const size_t c = fIdx(j, lp);
                return cs[c] * xh[c];
            });
            if (l == lp) {
                const size_t q = fCut(a, qq);
                const RowPack<double> r = a.rp[q];
                const double rsv = a.rs[q];
                accRowMetrics(acc, a.dc[lp], rsv * s, r.rl, r.ru, rsv, a.yh[q], a.yi[q]);
            }
        }
    }
    famBlockReduce<kRowSlots>(acc, ops, a.part_rows + static_cast<size_t>(blockIdx.x) * kFam * kRowSlots);
}

// Columns: A_l^T y_hat and A_l^T (y_hat - y_init), column metrics.
__global__ void __launch_bounds__(kBlock) famCheckCols(FamArgs a) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int ops[kColSlots];
    double acc[kColSlots];
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) {
        ops[s] = colSlotOp(s);
        acc[s] = slotInit(ops[s]);
    }
    const bool on = famChecking(a, l);
    const double *yh = a.yh, *yi = a.yi, *rs = a.rs;
    for (int j = static_cast<int>(blockIdx.x) * kWarps + w; j < a.n; j += a.nbc * kWarps) {
        const int b = a.at_ptr[j], e = a.at_ptr[j + 1];
        double aty = famDot(a.at_idx, a.at_val, b, e, l, on, [&](int i) {
            const size_t q = static_cast<size_t>(i) + l;
            return rs[q] * yh[q];
        });
        double atdy = famDot(a.at_idx, a.at_val, b, e, l, on, [&](int i) {
            const size_t q = static_cast<size_t>(i) + l;
            return rs[q] * (yh[q] - yi[q]);
        });
        for (int k = a.kt_ptr[j]; k < a.kt_ptr[j + 1]; ++k) {
            if (!on || a.kt_lane[k] != l) continue;
            const size_t q = fCut(a, a.kt_row[k]);
            aty += a.kt_val[k] * (rs[q] * yh[q]);
            atdy += a.kt_val[k] * (rs[q] * (yh[q] - yi[q]));
        }
        if (on) {
            const size_t c = fIdx(j, l);
            const ColPack<double> p = a.cp[c];
            const double csv = a.cs[c];
            accColMetrics<double>(acc, a.dc[l], a.xh[c], a.xi[c], p.c, p.lb, p.ub, csv, csv * aty, csv * atdy);
        }
    }
    famBlockReduce<kColSlots>(acc, ops, a.part_cols + static_cast<size_t>(blockIdx.x) * kFam * kColSlots);
}

// Fixed-order reduction of LP l's partials over nb blocks across one warp.
template <int NS>
__device__ __forceinline__ void famLanes(const double* part, int nb, int l, int lane, const int (&ops)[NS],
                                         double (&out)[NS]) {
#pragma unroll
    for (int s = 0; s < NS; ++s) out[s] = slotInit(ops[s]);
    for (int b = lane; b < nb; b += 32) {
        const double* p = part + (static_cast<size_t>(b) * kFam + l) * NS;
#pragma unroll
        for (int s = 0; s < NS; ++s) out[s] = combine(ops[s], out[s], p[s]);
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) out[s] = combine(ops[s], out[s], __shfl_xor_sync(kFull, out[s], off));
}

// One warp per LP: reduce its partials, run the single-LP controller step.
__global__ void __launch_bounds__(32 * kCtlWarps) famController(FamArgs a) {
    const int l = static_cast<int>(blockIdx.x) * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L) return;
    DevState* st = a.st + l;
    if (st->done) return;
    int rops[kRowSlots], cops[kColSlots];
#pragma unroll
    for (int s = 0; s < kRowSlots; ++s) rops[s] = rowSlotOp(s);
#pragma unroll
    for (int s = 0; s < kColSlots; ++s) cops[s] = colSlotOp(s);
    double rows[kRowSlots], cols[kColSlots];
    famLanes<kRowSlots>(a.part_rows, a.nbr, l, lane, rops, rows);
    if (a.nbk > 0) {  // this LP's appended rows: the partial of lane l in block nbr + l
        const double* p = a.part_rows + (static_cast<size_t>(a.nbr + l) * kFam + l) * kRowSlots;
#pragma unroll
        for (int s = 0; s < kRowSlots; ++s) rows[s] = combine(rops[s], rows[s], p[s]);
    }
    famLanes<kColSlots>(a.part_cols, a.nbc, l, lane, cops, cols);
    if (lane == 0) {
        DevState s = *st;
        controlStep(s, a.dc[l], rows, cols);
        *st = s;
    }
}

// Restart copy (pdlp_kernels.cu:377-405) of the LPs whose controller restarted:
// anchor = current = pdhg; the scaled y gathered by the primal step follows y_cur.
__global__ void __launch_bounds__(kBlock) famRestart(FamArgs a) {
    const size_t ncol = static_cast<size_t>(a.n) * kFam, nrow = static_cast<size_t>(a.mb) * kFam;
    const size_t total = ncol + nrow + static_cast<size_t>(a.K);
    for (size_t t = static_cast<size_t>(blockIdx.x) * kBlock + threadIdx.x; t < total;
         t += static_cast<size_t>(gridDim.x) * kBlock) {
        int l;
        if (t < ncol + nrow)
            l = static_cast<int>(t % kFam);
        else
            l = a.k_lane[t - ncol - nrow];
        if (l >= a.L) continue;
        const DevState* st = a.st + l;
        if (st->done || !st->restart) continue;
        if (t < ncol) {
            const double v = a.xh[t];
            a.xi[t] = v;
            a.xc[t] = v;
        } else {
            const size_t r = t - ncol;
            const double v = a.yh[r];
            a.yi[r] = v;
            a.yc[r] = v;
            a.ys[r] = a.rs[r] * v;
        }
    }
}

// Lane parameters of the next cycle from the solver state (the iteration rule
// of `active`: the cycle runs min(N, limit - done so far) iterations).
__device__ __forceinline__ void famLaneParams(const FamArgs& a, int l, bool done) {
    FamLane& p = *a.lanes;
    if (done) {
        p.allow[l] = 0;
        return;
    }
    const DevState& s = a.st[l];
    const int cur = s.phase == 0 ? s.total : s.polish_count;
    const int lim = s.phase == 0 ? a.max_iter : a.polish_max_iter;
    p.allow[l] = max(0, min(a.N, lim - cur));
    p.step[l] = s.step;
    p.pw[l] = s.pw;
    p.inner[l] = s.inner;
}

__global__ void famFinish(FamArgs a) {
    const int l = threadIdx.x;
    const bool done = l >= a.L || a.st[l].done;
    const unsigned live = __ballot_sync(kFull, !done);
    if (l == 0) *const_cast<unsigned*>(a.live) = live;
    famLaneParams(a, l, done);
    if (l < a.L) a.flags[l] = (done ? 1 : 0) | 2;
}

// ---- power iteration on A_l^T A_l per lane (pdlp.cpp:748-795, 1985-2041) -------------
__global__ void __launch_bounds__(kBlock) famPowerA(FamArgs a) {
    const int w = static_cast<int>(threadIdx.x >> 5);
    const int l = threadIdx.x & 31;
    const double *px = a.pi_x, *cs = a.cs;
    if (static_cast<int>(blockIdx.x) < a.gb) {
        const int i = static_cast<int>(blockIdx.x) * kWarps + w;
        if (i >= a.mb) return;
        const bool on = l < a.L && !a.ps[l].done;
        if (__ballot_sync(kFull, on) == 0) return;
        const double s = famDot(a.a_idx, a.a_val, a.a_ptr[i], a.a_ptr[i + 1], l, on, [&](int j) {
            const size_t c = static_cast<size_t>(j) + l;
            return cs[c] * px[c];
        });
        if (on) a.pi_y[fIdx(i, l)] = a.rs[fIdx(i, l)] * s;
        return;
    }
    const int qq = (static_cast<int>(blockIdx.x) - a.gb) * kWarps + w;
    if (qq >= a.K) return;
    const int lp = a.k_lane[qq];
    if (a.ps[lp].done) return;
    const double s = famCutDot(a, qq, l, [&](int j) {
        const size_t c = fIdx(j, lp);
        return cs[c] * px[c];
    });
    if (l == 0) a.pi_y[fCut(a, qq)] = a.rs[fCut(a, qq)] * s;
}

__global__ void __launch_bounds__(kBlock) famPowerAt(FamArgs a) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const bool on = l < a.L && !a.ps[l].done;
    const double *py = a.pi_y, *rs = a.rs;
    double acc[2] = {0.0, 0.0};
    for (int j = static_cast<int>(blockIdx.x) * kWarps + w; j < a.n; j += a.nbc * kWarps) {
        double s = famDot(a.at_idx, a.at_val, a.at_ptr[j], a.at_ptr[j + 1], l, on, [&](int i) {
            const size_t q = static_cast<size_t>(i) + l;
            return rs[q] * py[q];
        });
        for (int k = a.kt_ptr[j]; k < a.kt_ptr[j + 1]; ++k)
            if (on && a.kt_lane[k] == l) {
                const size_t q = fCut(a, a.kt_row[k]);
                s += a.kt_val[k] * (rs[q] * py[q]);
            }
        if (on) {
            const size_t c = fIdx(j, l);
            const double xn = a.cs[c] * s;
            a.pi_xn[c] = xn;
            acc[0] += a.pi_x[c] * xn;
            acc[1] += xn * xn;
        }
    }
    const int ops[2] = {OP_SUM, OP_SUM};
    famBlockReduce<2>(acc, ops, a.pi_part + static_cast<size_t>(blockIdx.x) * kFam * 2);
}

__global__ void __launch_bounds__(32 * kCtlWarps) famPowerFinish1(FamArgs a) {
    const int l = static_cast<int>(blockIdx.x) * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L || a.ps[l].done) return;
    const int ops[2] = {OP_SUM, OP_SUM};
    double out[2];
    famLanes<2>(a.pi_part, a.nbc, l, lane, ops, out);
    if (lane == 0) {
        a.ps[l].s2 = out[0];
        a.ps[l].nrm = sqrt(out[1]);
    }
}

__global__ void __launch_bounds__(kBlock) famPowerNormalize(FamArgs a) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const bool on = l < a.L && !a.ps[l].done;
    double acc[2] = {0.0, 0.0};
    if (on) {
        const double s2 = a.ps[l].s2, nrm = a.ps[l].nrm;
        for (int j = static_cast<int>(blockIdx.x) * kWarps + w; j < a.n; j += a.nbc * kWarps) {
            const size_t c = fIdx(j, l);
            const double xn = a.pi_xn[c];
            const double d = xn - s2 * a.pi_x[c];
            acc[0] += d * d;
            if (nrm >= 1e-15) a.pi_x[c] = xn / nrm;
        }
    }
    const int ops[2] = {OP_SUM, OP_SUM};
    famBlockReduce<2>(acc, ops, a.pi_part + static_cast<size_t>(blockIdx.x) * kFam * 2);
}

__global__ void __launch_bounds__(32 * kCtlWarps) famPowerFinish2(FamArgs a) {
    const int l = static_cast<int>(blockIdx.x) * kCtlWarps + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (l >= a.L || a.ps[l].done) return;
    const int ops[2] = {OP_SUM, OP_SUM};
    double out[2];
    famLanes<2>(a.pi_part, a.nbc, l, lane, ops, out);
    if (lane == 0) {
        PowerState& p = a.ps[l];
        p.resid = sqrt(out[0]);
        p.iter += 1;
        if (p.nrm < 1e-15 || p.resid < a.sv_tol * fabs(p.s2) || p.iter >= a.sv_max_iter) {
            p.done = 1;
            atomicAdd(a.counters, 1);
        }
    }
}

// Step size from the spectral-norm estimate (0.998 / ||A_l||_2, pdlp.cpp:796-800).
__global__ void famInitStep(FamArgs a) {
    const int l = threadIdx.x;
    if (l < a.L) {
        DevState& s = a.st[l];
        const double step = 0.998 / sqrt(fmax(a.ps[l].s2, 1e-12));
        s.step = step;
        s.tau_fac = static_cast<float>(step / s.pw);
        s.sig_fac = static_cast<float>(step * s.pw);
    }
    famLaneParams(a, l, l >= a.L || a.st[l].done);
}

// ---------------------------------------------------------------------------
// Host side of a family pack
// ---------------------------------------------------------------------------
// Offered between restart cycles when a lane is free: return a prepared
// member of the family for which fits(item) holds (its appended rows fit the
// pack's reserved room) and the caller's id for it, or false when none is
// waiting.  The pack reports that member through `done(id, outcome)`.
using FamAdmit = std::function<bool(const std::function<bool(const Item&)>& fits, Item*& item, int& id)>;

struct FamPack {
    const FamilyBase* base = nullptr;
    std::vector<Item*> items;   // by lane (kFam entries; null for a lane never used)
    int L = 0, n = 0, mb = 0, K = 0;
    int Kcap = 0;               // appended rows the arrays hold (room for admitted members)
    int64_t Zb = 0, Zk = 0, Zkcap = 0;
    std::vector<int> qfirst;    // first appended row of each lane (kFam + 1 entries)
    size_t o_aptr, o_aidx, o_aval, o_atptr, o_atidx, o_atval, o_kptr, o_kidx, o_kval, o_klane, o_kfirst, o_live, o_lanes;
    size_t o_ktptr, o_ktrow, o_ktlane, o_ktval, o_cp, o_cs, o_rp, o_rs, o_st, o_dc, o_ps, o_pix;
    size_t image_end;
    size_t o_xc, o_xi, o_xh, o_xs, o_yc, o_yi, o_yh, o_ys;
    size_t iter_end;
    size_t o_piy, o_pixn, o_pipart, o_prows, o_pcols, o_flags, o_counters;
    size_t total;
    char* d = nullptr;
    cudaStream_t s = nullptr;
    cudaGraphExec_t cycle = nullptr, power = nullptr;
    int cycle_launches = 0, power_launches = 0;
    FamArgs args{};

    ~FamPack() {
        if (cycle) cudaGraphExecDestroy(cycle);
        if (power) cudaGraphExecDestroy(power);
        if (d) cudaFreeAsync(d, s);
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }

    size_t rowsAll() const { return static_cast<size_t>(mb) * kFam + static_cast<size_t>(Kcap); }
    size_t colsAll() const { return static_cast<size_t>(n) * kFam; }

    void layout(int nbr, int nbc) {
        size_t off = 0;
        auto take = [&](size_t bytes) {
            const size_t at = off;
            off += al256(bytes);
            return at;
        };
        const size_t R = rowsAll(), C = colsAll();
        o_aptr = take(4 * (static_cast<size_t>(mb) + 1));
        o_aidx = take(4 * static_cast<size_t>(Zb));
        o_aval = take(8 * static_cast<size_t>(Zb));
        o_atptr = take(4 * (static_cast<size_t>(n) + 1));
        o_atidx = take(4 * static_cast<size_t>(Zb));
        o_atval = take(8 * static_cast<size_t>(Zb));
        o_kptr = take(4 * (static_cast<size_t>(Kcap) + 1));
        o_kidx = take(4 * static_cast<size_t>(Zkcap));
        o_kval = take(8 * static_cast<size_t>(Zkcap));
        o_klane = take(4 * static_cast<size_t>(Kcap));
        o_kfirst = take(4 * (kFam + 1));
        o_live = take(4);
        o_lanes = take(sizeof(FamLane));
        o_ktptr = take(4 * (static_cast<size_t>(n) + 1));
        o_ktrow = take(4 * static_cast<size_t>(Zkcap));
        o_ktlane = take(4 * static_cast<size_t>(Zkcap));
        o_ktval = take(8 * static_cast<size_t>(Zkcap));
        o_cp = take(32 * C);
        o_cs = take(8 * C);
        o_rp = take(32 * R);
        o_rs = take(8 * R);
        o_st = take(sizeof(DevState) * kFam);
        o_dc = take(sizeof(DevConst) * kFam);
        o_ps = take(sizeof(PowerState) * kFam);
        o_pix = take(8 * C);
        image_end = off;
        o_xc = take(8 * C);
        o_xi = take(8 * C);
        o_xh = take(8 * C);
        o_xs = take(8 * C);
        o_yc = take(8 * R);
        o_yi = take(8 * R);
        o_yh = take(8 * R);
        o_ys = take(8 * R);
        iter_end = off;
        o_piy = take(8 * R);
        o_pixn = take(8 * C);
        o_pipart = take(8 * 2 * kFam * static_cast<size_t>(nbc));
        // appended rows are checked in one block per lane: room for every lane
        o_prows = take(8 * kRowSlots * kFam * static_cast<size_t>(nbr + kFam));
        o_pcols = take(8 * kColSlots * kFam * static_cast<size_t>(nbc));
        o_flags = take(4 * kFam);
        o_counters = take(16);
        total = off;
    }
};

// Device bytes of a family pack of L members with the given appended rows / entries.
size_t familyPackBytes(int64_t n, int64_t mb, int64_t zb, int64_t K, int64_t zk, int nbc, int nbrk) {
    const size_t C = static_cast<size_t>(n) * kFam, R = static_cast<size_t>(mb) * kFam + static_cast<size_t>(K);
    size_t b = 4 * static_cast<size_t>(mb + n + 2) + 24 * static_cast<size_t>(zb);
    b += 4 * static_cast<size_t>(K + n + 2) + 28 * static_cast<size_t>(zk) + 4 * static_cast<size_t>(K);
    b += C * (32 + 8 + 8 * 6) + R * (32 + 8 + 8 * 5);
    b += 8 * kFam * (2 * static_cast<size_t>(nbc) + kRowSlots * static_cast<size_t>(nbrk) + kColSlots * static_cast<size_t>(nbc));
    return b + 64 * 1024;
}

int famBlocks(int64_t rows) { return static_cast<int>(std::max<int64_t>(1, (rows + kWarps - 1) / kWarps)); }

// Appended rows a lane's member brings (rows after the base rows) and their entries.
int famCuts(const Item& it, int mb) { return it.lp.m - mb; }
int64_t famCutEntries(const Item& it, int mb) { return it.lp.a.ptr[it.lp.m] - it.lp.a.ptr[mb]; }

// Per-lane data of one member in its own (contiguous) order: the scaled
// column constants, column scales, starting x (warm start scaled like the
// reference, pdlp.cpp:1812-1827, else 0) and its column-scaled copy; the same
// for every row of the member (base rows, then its appended rows).
struct FamLaneData {
    std::vector<ColPack<double>> cp;
    std::vector<double> cs, x, xs;
    std::vector<RowPack<double>> rp;
    std::vector<double> rs, y, ys;
};

void famLaneData(const Item& it, int n, FamLaneData& q) {
    const ScaledLp& sc = it.sc;
    const int32_t m = it.lp.m;
    q.cp.resize(n);
    q.cs.resize(n);
    q.x.assign(n, 0.0);
    q.xs.resize(n);
    q.rp.resize(m);
    q.rs.resize(m);
    q.y.assign(m, 0.0);
    q.ys.resize(m);
    if (!it.warm_x.empty()) {
        for (int32_t j = 0; j < n; ++j) q.x[j] = it.warm_x[j] / sc.col_scale[j] * sc.con_scale;
        for (int32_t i = 0; i < m; ++i) q.y[i] = it.warm_y[i] * sc.obj_scale / (sc.obj_sign * sc.row_scale[i]);
    }
    for (int32_t j = 0; j < n; ++j) {
        q.cp[j] = ColPack<double>{sc.c[j], sc.cl[j], sc.cu[j], sc.tau[j]};
        q.cs[j] = sc.col_scale[j];
        q.xs[j] = sc.col_scale[j] * q.x[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        q.rp[i] = RowPack<double>{sc.sigma[i], sc.rl[i], sc.ru[i], static_cast<double>(sc.row_type[i])};
        q.rs[i] = sc.row_scale[i];
        q.ys[i] = sc.row_scale[i] * q.y[i];
    }
}

// The appended rows of the lanes in use (lane order; a lane without a member
// contributes none): row pointers, entries, lanes, per-lane first row, and the
// same entries by column (row order inside a column).
struct FamCuts {
    std::vector<int32_t> kp, ki, kl, kf, ktp, ktr, ktl;
    std::vector<double> kv, ktv;
    int K = 0;
    int64_t Zk = 0;
};

void famBuildCuts(const FamPack& fp, const std::vector<char>& in_use, FamCuts& c) {
    const int n = fp.n, mb = fp.mb;
    c.kp.clear();
    c.ki.clear();
    c.kv.clear();
    c.kl.clear();
    c.kf.assign(kFam + 1, 0);
    std::vector<int32_t> colcnt(static_cast<size_t>(n) + 1, 0);
    int q = 0;
    for (int l = 0; l < kFam; ++l) {
        c.kf[l] = q;
        if (!in_use[l] || fp.items[l] == nullptr) continue;
        const Csr& a = fp.items[l]->lp.a;
        for (int32_t i = mb; i < a.rows; ++i, ++q) {
            c.kp.push_back(static_cast<int32_t>(c.ki.size()));
            c.kl.push_back(l);
            for (int32_t k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                c.ki.push_back(a.idx[k]);
                c.kv.push_back(a.val[k]);
                ++colcnt[a.idx[k] + 1];
            }
        }
    }
    c.kf[kFam] = q;
    c.K = q;
    c.Zk = static_cast<int64_t>(c.ki.size());
    c.kp.push_back(static_cast<int32_t>(c.Zk));
    for (int32_t j = 0; j < n; ++j) colcnt[j + 1] += colcnt[j];
    c.ktp = colcnt;
    c.ktr.resize(static_cast<size_t>(c.Zk));
    c.ktl.resize(static_cast<size_t>(c.Zk));
    c.ktv.resize(static_cast<size_t>(c.Zk));
    for (int qq = 0; qq < c.K; ++qq)
        for (int32_t k = c.kp[qq]; k < c.kp[qq + 1]; ++k) {
            const int32_t at = colcnt[c.ki[k]]++;
            c.ktr[at] = qq;
            c.ktl[at] = c.kl[qq];
            c.ktv[at] = c.kv[k];
        }
}

// Build the image, run the power iteration and the restart cycles of one family
// pack; `done(id, outcome)` as for a regular pack, with id = the member's
// position in fp.items for the initial members and the id `admit` returned for
// members admitted later (admit may be empty: no admission).
int32_t solveFamilyPack(FamPack& fp, const pdlpx_options& o, std::chrono::steady_clock::time_point t0,
                        const std::atomic<int>* stop, const LpDone& done, std::string& err,
                        const FamAdmit& admit) {
    const int n = fp.n, mb = fp.mb;
    int L = fp.L;
    const FamilyBase& fb = *fp.base;
    int sms = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    fp.items.resize(kFam, nullptr);
    std::vector<char> in_use(kFam, 0);  // lane holds a member that is not yet reported
    std::vector<int> lane_id(kFam, -1);
    for (int l = 0; l < L; ++l) {
        in_use[l] = 1;
        lane_id[l] = l;
    }
    FamCuts cuts;
    famBuildCuts(fp, in_use, cuts);
    fp.K = cuts.K;
    fp.Zk = cuts.Zk;
    fp.qfirst.assign(cuts.kf.begin(), cuts.kf.end());
    // room for the appended rows of members admitted later: at least 64 rows of
    // 256 entries per lane, and twice what the first members bring
    fp.Kcap = std::max(2 * cuts.K, kFam * 64);
    fp.Zkcap = std::max<int64_t>(2 * cuts.Zk, static_cast<int64_t>(kFam) * 64 * 256);
    fp.Zb = fb.ptr[mb];
    const int gb = famBlocks(mb);
    const int gp = famBlocks((static_cast<int64_t>(n) + kFamColsPerWarp - 1) / kFamColsPerWarp);
    const int gd = famBlocks((static_cast<int64_t>(mb) + kFamRowsPerWarp - 1) / kFamRowsPerWarp);
    const int cap = 4 * sms;
    const int nbr = std::min(gb, cap), nbc = std::min(famBlocks(n), cap);
    fp.layout(nbr, nbc);

    // ---- host image
    std::unique_ptr<char[]> img(new char[fp.image_end]);
    std::unique_ptr<char[]> iters(new char[fp.iter_end - fp.image_end]);
    char* H = img.get();
    auto I = [&](size_t off) { return reinterpret_cast<int32_t*>(H + off); };
    auto D = [&](size_t off) { return reinterpret_cast<double*>(H + off); };
    auto ID = [&](size_t off) { return reinterpret_cast<double*>(iters.get() + (off - fp.image_end)); };
    std::memcpy(I(fp.o_aptr), fb.ptr.data(), 4 * (static_cast<size_t>(mb) + 1));
    for (int64_t k = 0; k < fp.Zb; ++k) I(fp.o_aidx)[k] = fb.idx[k] * kFam;
    std::memcpy(D(fp.o_aval), fb.val.data(), 8 * static_cast<size_t>(fp.Zb));
    {
        Csr a;
        a.rows = mb;
        a.cols = n;
        a.ptr = fb.ptr;
        a.idx = fb.idx;
        a.val = fb.val;
        Csr at;
        transposeCsr(a, at);
        std::memcpy(I(fp.o_atptr), at.ptr.data(), 4 * (static_cast<size_t>(n) + 1));
        for (int64_t k = 0; k < fp.Zb; ++k) I(fp.o_atidx)[k] = at.idx[k] * kFam;
        std::memcpy(D(fp.o_atval), at.val.data(), 8 * static_cast<size_t>(fp.Zb));
    }
    std::memcpy(I(fp.o_kptr), cuts.kp.data(), 4 * cuts.kp.size());
    std::memcpy(I(fp.o_kidx), cuts.ki.data(), 4 * cuts.ki.size());
    std::memcpy(D(fp.o_kval), cuts.kv.data(), 8 * cuts.kv.size());
    std::memcpy(I(fp.o_klane), cuts.kl.data(), 4 * cuts.kl.size());
    std::memcpy(I(fp.o_kfirst), cuts.kf.data(), 4 * cuts.kf.size());
    *reinterpret_cast<uint32_t*>(H + fp.o_live) = L >= kFam ? ~0u : ((1u << L) - 1u);
    std::memcpy(I(fp.o_ktptr), cuts.ktp.data(), 4 * cuts.ktp.size());
    std::memcpy(I(fp.o_ktrow), cuts.ktr.data(), 4 * cuts.ktr.size());
    std::memcpy(I(fp.o_ktlane), cuts.ktl.data(), 4 * cuts.ktl.size());
    std::memcpy(D(fp.o_ktval), cuts.ktv.data(), 8 * cuts.ktv.size());
    // per-lane constants, state, power start vector and iterates
    const double inf = std::numeric_limits<double>::infinity();
    std::vector<double> g(n);
    {
        std::mt19937 rng(42);
        std::normal_distribution<double> dist(0.0, 1.0);
        double xn = 0.0;
        for (int32_t j = 0; j < n; ++j) {
            g[j] = dist(rng);
            xn += g[j] * g[j];
        }
        xn = std::sqrt(xn);
        if (xn < 1e-15) xn = 1.0;
        for (auto& v : g) v /= xn;
    }
    ColPack<double>* cp = reinterpret_cast<ColPack<double>*>(H + fp.o_cp);
    RowPack<double>* rp = reinterpret_cast<RowPack<double>*>(H + fp.o_rp);
    double *cs = D(fp.o_cs), *pix = D(fp.o_pix);
    double* rs = D(fp.o_rs);
    double *xc = ID(fp.o_xc), *xi = ID(fp.o_xi), *xh = ID(fp.o_xh), *xsv = ID(fp.o_xs);
    double *yc = ID(fp.o_yc), *yi = ID(fp.o_yi), *yh = ID(fp.o_yh), *ysv = ID(fp.o_ys);
    const size_t Rb = static_cast<size_t>(mb) * kFam;
    // appended-row slots no member uses yet: empty, free rows
    for (size_t r = Rb; r < fp.rowsAll(); ++r) {
        rp[r] = RowPack<double>{1.0, -inf, inf, static_cast<double>(kRowRanged)};
        rs[r] = 1.0;
        yc[r] = yi[r] = yh[r] = ysv[r] = 0.0;
    }
    parallelFor(kFam, [&](int l) {
        if (l >= L) {
            for (int32_t j = 0; j < n; ++j) {
                const size_t c = static_cast<size_t>(j) * kFam + l;
                cp[c] = ColPack<double>{0.0, -inf, inf, 1.0};
                cs[c] = 1.0;
                pix[c] = xc[c] = xi[c] = xh[c] = xsv[c] = 0.0;
            }
            for (int32_t i = 0; i < mb; ++i) {
                const size_t r = static_cast<size_t>(i) * kFam + l;
                rp[r] = RowPack<double>{1.0, -inf, inf, static_cast<double>(kRowRanged)};
                rs[r] = 1.0;
                yc[r] = yi[r] = yh[r] = ysv[r] = 0.0;
            }
            return;
        }
        const Item& it = *fp.items[l];
        FamLaneData q;
        famLaneData(it, n, q);
        for (int32_t j = 0; j < n; ++j) {
            const size_t c = static_cast<size_t>(j) * kFam + l;
            cp[c] = q.cp[j];
            cs[c] = q.cs[j];
            pix[c] = g[j];
            xc[c] = xi[c] = xh[c] = q.x[j];
            xsv[c] = q.xs[j];
        }
        for (int32_t i = 0; i < it.lp.m; ++i) {
            const size_t r = i < mb ? static_cast<size_t>(i) * kFam + l : Rb + static_cast<size_t>(fp.qfirst[l] + i - mb);
            rp[r] = q.rp[i];
            rs[r] = q.rs[i];
            yc[r] = yi[r] = yh[r] = q.y[i];
            ysv[r] = q.ys[i];
        }
        DevConst dc{};
        DevState st{};
        lpState(it, o, false, nbr + L, nbc, dc, st);
        reinterpret_cast<DevConst*>(H + fp.o_dc)[l] = dc;
        reinterpret_cast<DevState*>(H + fp.o_st)[l] = st;
        reinterpret_cast<PowerState*>(H + fp.o_ps)[l] = PowerState{1.0, 0.0, 0.0, 0, o.sv_max_iter <= 0 ? 1 : 0};
    });
    for (int l = L; l < kFam; ++l) {
        reinterpret_cast<DevConst*>(H + fp.o_dc)[l] = DevConst{};
        DevState st{};
        st.done = 1;
        reinterpret_cast<DevState*>(H + fp.o_st)[l] = st;
        reinterpret_cast<PowerState*>(H + fp.o_ps)[l] = PowerState{1.0, 0.0, 0.0, 0, 1};
    }

    // ---- device image
    PDLPX_BCK(cudaStreamCreateWithFlags(&fp.s, cudaStreamNonBlocking));
    PDLPX_BCK(cudaMallocAsync(reinterpret_cast<void**>(&fp.d), fp.total, fp.s));
    cudaStream_t s = fp.s;
    PDLPX_BCK(cudaMemcpyAsync(fp.d, H, fp.image_end, cudaMemcpyHostToDevice, s));
    PDLPX_BCK(cudaMemcpyAsync(fp.d + fp.image_end, iters.get(), fp.iter_end - fp.image_end, cudaMemcpyHostToDevice, s));
    PDLPX_BCK(cudaMemsetAsync(fp.d + fp.iter_end, 0, fp.total - fp.iter_end, s));
    {
        FamArgs& a = fp.args;
        char* d = fp.d;
        auto Pi = [&](size_t off) { return reinterpret_cast<int*>(d + off); };
        auto Pd = [&](size_t off) { return reinterpret_cast<double*>(d + off); };
        a.a_ptr = Pi(fp.o_aptr);
        a.a_idx = Pi(fp.o_aidx);
        a.a_val = Pd(fp.o_aval);
        a.at_ptr = Pi(fp.o_atptr);
        a.at_idx = Pi(fp.o_atidx);
        a.at_val = Pd(fp.o_atval);
        a.k_ptr = Pi(fp.o_kptr);
        a.k_idx = Pi(fp.o_kidx);
        a.k_val = Pd(fp.o_kval);
        a.k_lane = Pi(fp.o_klane);
        a.k_first = Pi(fp.o_kfirst);
        a.live = reinterpret_cast<const unsigned*>(d + fp.o_live);
        a.lanes = reinterpret_cast<FamLane*>(d + fp.o_lanes);
        a.kt_ptr = Pi(fp.o_ktptr);
        a.kt_row = Pi(fp.o_ktrow);
        a.kt_lane = Pi(fp.o_ktlane);
        a.kt_val = Pd(fp.o_ktval);
        a.cp = reinterpret_cast<const ColPack<double>*>(d + fp.o_cp);
        a.cs = Pd(fp.o_cs);
        a.xc = Pd(fp.o_xc);
        a.xi = Pd(fp.o_xi);
        a.xh = Pd(fp.o_xh);
        a.xs = Pd(fp.o_xs);
        a.rp = reinterpret_cast<const RowPack<double>*>(d + fp.o_rp);
        a.rs = Pd(fp.o_rs);
        a.yc = Pd(fp.o_yc);
        a.yi = Pd(fp.o_yi);
        a.yh = Pd(fp.o_yh);
        a.ys = Pd(fp.o_ys);
        a.st = reinterpret_cast<DevState*>(d + fp.o_st);
        a.dc = reinterpret_cast<const DevConst*>(d + fp.o_dc);
        a.ps = reinterpret_cast<PowerState*>(d + fp.o_ps);
        a.flags = Pi(fp.o_flags);
        a.counters = Pi(fp.o_counters);
        a.part_rows = Pd(fp.o_prows);
        a.part_cols = Pd(fp.o_pcols);
        a.pi_x = Pd(fp.o_pix);
        a.pi_y = Pd(fp.o_piy);
        a.pi_xn = Pd(fp.o_pixn);
        a.pi_part = Pd(fp.o_pipart);
        a.n = n;
        a.mb = mb;
        a.gb = gb;
        a.gp = gp;
        a.gd = gd;
        a.nbr = nbr;
        a.nbc = nbc;
        a.max_iter = o.max_iter;
        a.polish_max_iter = o.polish_max_iter;
        a.N = o.termination_eval_frequency;
        a.sv_max_iter = o.sv_max_iter;
        a.sv_tol = o.sv_tol;
    }
    // the parts of the arguments that admission changes
    auto setShape = [&](FamArgs& a) {
        a.K = fp.K;
        a.L = L;
        a.gk = fp.K > 0 ? famBlocks(fp.K) : 0;
        a.nbk = L;  // one check block per lane for its appended rows (identity partials when it has none)
    };
    setShape(fp.args);

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    PDLPX_BCK(cudaEventCreate(&ev0));
    PDLPX_BCK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev_guard{ev0, ev1};
    PDLPX_BCK(cudaEventRecord(ev0, s));
    int launches = 0;
    auto deviceSeconds = [&]() -> double {
        float ms = 0.0f;
        if (cudaEventRecord(ev1, s) == cudaSuccess && cudaEventSynchronize(ev1) == cudaSuccess)
            cudaEventElapsedTime(&ms, ev0, ev1);
        return 1e-3 * ms;
    };
    auto hostSeconds = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    auto stopped = [&]() { return stop != nullptr && stop->load(std::memory_order_relaxed) != 0; };
    std::vector<int> h_flags(kFam);
    auto capture = [&](cudaGraphExec_t& gx, int& count, bool power) -> int32_t {
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
        const FamArgs args = fp.args;
        const int stepRows = args.gb + args.gk;
        const int ctl = (args.L + kCtlWarps - 1) / kCtlWarps;
        const int nrs = std::max(1, std::min<int>(static_cast<int>((fp.colsAll() + fp.rowsAll() + kBlock - 1) / kBlock),
                                                  8 * sms));
        cudaGraph_t graph = nullptr;
        PDLPX_BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        count = 0;
        if (power) {
            for (int r = 0; r < 8; ++r) {
                famPowerA<<<stepRows, kBlock, 0, s>>>(args);
                famPowerAt<<<args.nbc, kBlock, 0, s>>>(args);
                famPowerFinish1<<<ctl, 32 * kCtlWarps, 0, s>>>(args);
                famPowerNormalize<<<args.nbc, kBlock, 0, s>>>(args);
                famPowerFinish2<<<ctl, 32 * kCtlWarps, 0, s>>>(args);
                count += 5;
            }
        } else {
            for (int k = 1; k <= o.termination_eval_frequency; ++k) {
                famPrimal<<<args.gp, kBlock, 0, s>>>(args, k);
                famDual<<<args.gd + args.gk, kBlock, 0, s>>>(args, k);
                count += 2;
            }
            famCheckRows<<<args.nbr + args.nbk, kBlock, 0, s>>>(args);
            famCheckCols<<<args.nbc, kBlock, 0, s>>>(args);
            famController<<<ctl, 32 * kCtlWarps, 0, s>>>(args);
            famRestart<<<nrs, kBlock, 0, s>>>(args);
            famFinish<<<1, kFam, 0, s>>>(args);
            count += 5;
        }
        PDLPX_BCK(cudaStreamEndCapture(s, &graph));
        const cudaError_t ie = cudaGraphInstantiate(&gx, graph, 0);
        cudaGraphDestroy(graph);
        PDLPX_BCK(ie);
        return PDLPX_OK;
    };
    // power iteration of every lane whose PowerState is not done, then the step sizes
    auto powerPhase = [&]() -> int32_t {
        if (o.sv_max_iter > 0) {
            int32_t rc = capture(fp.power, fp.power_launches, true);
            if (rc != PDLPX_OK) return rc;
            for (int guard = 0; guard < 2 + o.sv_max_iter / 8; ++guard) {
                PDLPX_BCK(cudaGraphLaunch(fp.power, s));
                launches += fp.power_launches;
                PDLPX_BCK(cudaMemcpyAsync(h_flags.data(), fp.args.counters, 4, cudaMemcpyDeviceToHost, s));
                PDLPX_BCK(cudaStreamSynchronize(s));
                if (h_flags[0] >= L || stopped()) break;
            }
        }
        // the step of every lane from its power result; a lane already iterating
        // gets the value it has (its power state is unchanged) and its lane
        // parameters as the end of a cycle writes them
        famInitStep<<<1, kFam, 0, s>>>(fp.args);
        ++launches;
        PDLPX_BCK(cudaGetLastError());
        return PDLPX_OK;
    };
    {
        int32_t rc = powerPhase();
        if (rc != PDLPX_OK) return rc;
        rc = capture(fp.cycle, fp.cycle_launches, false);
        if (rc != PDLPX_OK) return rc;
    }

    // ---- admission: members that arrive while the pack runs take free lanes
    // between cycles.  The appended rows of all lanes are rebuilt (the members
    // still running keep their appended rows' iterates), the new member's
    // columns and base rows are written into its lane, its state starts fresh,
    // its power iteration runs (the others' power state is done, so the power
    // kernels skip them) and the graphs are captured again for the new shape.
    std::vector<double> lane_dev0(kFam, 0.0), lane_t0(kFam, 0.0);
    auto admitMembers = [&](std::vector<int>& fresh_lanes) -> int32_t {
        fresh_lanes.clear();
        if (!admit) return PDLPX_OK;
        int K_run = 0;
        int64_t Z_run = 0;
        for (int l = 0; l < kFam; ++l)
            if (in_use[l] && fp.items[l]) {
                K_run += famCuts(*fp.items[l], mb);
                Z_run += famCutEntries(*fp.items[l], mb);
            }
        for (int l = 0; l < kFam; ++l) {
            if (in_use[l]) continue;
            Item* it = nullptr;
            int id = -1;
            auto fits = [&](const Item& c) {
                return K_run + famCuts(c, mb) <= fp.Kcap && Z_run + famCutEntries(c, mb) <= fp.Zkcap;
            };
            if (!admit(fits, it, id) || it == nullptr) break;
            K_run += famCuts(*it, mb);
            Z_run += famCutEntries(*it, mb);
            fp.items[l] = it;
            in_use[l] = 1;
            lane_id[l] = id;
            fresh_lanes.push_back(l);
        }
        if (fresh_lanes.empty()) return PDLPX_OK;
        const int L_new = std::max(L, fresh_lanes.back() + 1);
        // appended rows: keep the running members' iterates of their rows
        const size_t Kold = static_cast<size_t>(fp.K);
        std::vector<double> ov[4];
        double* const drow[4] = {fp.args.yc, fp.args.yi, fp.args.yh, fp.args.ys};
        for (int k = 0; k < 4; ++k) {
            ov[k].resize(Kold);
            if (Kold > 0)
                PDLPX_BCK(cudaMemcpyAsync(ov[k].data(), drow[k] + Rb, 8 * Kold, cudaMemcpyDeviceToHost, s));
        }
        PDLPX_BCK(cudaStreamSynchronize(s));
        const std::vector<int> old_first = fp.qfirst;
        FamCuts c;
        famBuildCuts(fp, in_use, c);
        const size_t Kn = static_cast<size_t>(c.K);
        std::vector<RowPack<double>> krp(Kn);
        std::vector<double> krs(Kn), kv[4];
        for (auto& v : kv) v.assign(Kn, 0.0);
        std::vector<FamLaneData> fresh(fresh_lanes.size());
        for (size_t f = 0; f < fresh_lanes.size(); ++f) famLaneData(*fp.items[fresh_lanes[f]], n, fresh[f]);
        for (int l = 0; l < kFam; ++l) {
            if (!in_use[l]) continue;
            const Item& it = *fp.items[l];
            const auto fi = std::find(fresh_lanes.begin(), fresh_lanes.end(), l);
            const bool is_new = fi != fresh_lanes.end();
            const ScaledLp& sc = it.sc;
            for (int i = mb; i < it.lp.m; ++i) {
                const size_t r = static_cast<size_t>(c.kf[l] + i - mb);
                krp[r] = RowPack<double>{sc.sigma[i], sc.rl[i], sc.ru[i], static_cast<double>(sc.row_type[i])};
                krs[r] = sc.row_scale[i];
                if (is_new) {
                    const FamLaneData& q = fresh[static_cast<size_t>(fi - fresh_lanes.begin())];
                    kv[0][r] = kv[1][r] = kv[2][r] = q.y[i];
                    kv[3][r] = q.ys[i];
                } else {
                    const size_t o_r = static_cast<size_t>(old_first[l] + i - mb);
                    for (int k = 0; k < 4; ++k) kv[k][r] = ov[k][o_r];
                }
            }
        }
        auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
            return bytes == 0 ? cudaSuccess : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        char* d = fp.d;
        PDLPX_BCK(up(d + fp.o_kptr, c.kp.data(), 4 * c.kp.size()));
        PDLPX_BCK(up(d + fp.o_kidx, c.ki.data(), 4 * c.ki.size()));
        PDLPX_BCK(up(d + fp.o_kval, c.kv.data(), 8 * c.kv.size()));
        PDLPX_BCK(up(d + fp.o_klane, c.kl.data(), 4 * c.kl.size()));
        PDLPX_BCK(up(d + fp.o_kfirst, c.kf.data(), 4 * c.kf.size()));
        PDLPX_BCK(up(d + fp.o_ktptr, c.ktp.data(), 4 * c.ktp.size()));
        PDLPX_BCK(up(d + fp.o_ktrow, c.ktr.data(), 4 * c.ktr.size()));
        PDLPX_BCK(up(d + fp.o_ktlane, c.ktl.data(), 4 * c.ktl.size()));
        PDLPX_BCK(up(d + fp.o_ktval, c.ktv.data(), 8 * c.ktv.size()));
        PDLPX_BCK(up(d + fp.o_rp + 32 * Rb, krp.data(), 32 * Kn));
        PDLPX_BCK(up(d + fp.o_rs + 8 * Rb, krs.data(), 8 * Kn));
        for (int k = 0; k < 4; ++k) PDLPX_BCK(up(drow[k] + Rb, kv[k].data(), 8 * Kn));
        // the new members' lanes: columns and base rows are interleaved by lane
        auto lane2d = [&](size_t base_off, int l, const void* src, size_t elem, size_t rows) -> cudaError_t {
            if (rows == 0) return cudaSuccess;
            return cudaMemcpy2DAsync(d + base_off + elem * static_cast<size_t>(l), elem * kFam, src, elem, elem, rows,
                                     cudaMemcpyHostToDevice, s);
        };
        std::vector<DevConst> hdc(fresh_lanes.size());
        std::vector<DevState> hst(fresh_lanes.size());
        std::vector<PowerState> hps(fresh_lanes.size());
        const double now_dev = deviceSeconds(), now_host = hostSeconds();
        for (size_t f = 0; f < fresh_lanes.size(); ++f) {
            const int l = fresh_lanes[f];
            const FamLaneData& q = fresh[f];
            const size_t nn = static_cast<size_t>(n), mm = static_cast<size_t>(mb);
            PDLPX_BCK(lane2d(fp.o_cp, l, q.cp.data(), sizeof(ColPack<double>), nn));
            PDLPX_BCK(lane2d(fp.o_cs, l, q.cs.data(), 8, nn));
            PDLPX_BCK(lane2d(fp.o_pix, l, g.data(), 8, nn));
            for (size_t off : {fp.o_xc, fp.o_xi, fp.o_xh}) PDLPX_BCK(lane2d(off, l, q.x.data(), 8, nn));
            PDLPX_BCK(lane2d(fp.o_xs, l, q.xs.data(), 8, nn));
            PDLPX_BCK(lane2d(fp.o_rp, l, q.rp.data(), sizeof(RowPack<double>), mm));
            PDLPX_BCK(lane2d(fp.o_rs, l, q.rs.data(), 8, mm));
            for (size_t off : {fp.o_yc, fp.o_yi, fp.o_yh}) PDLPX_BCK(lane2d(off, l, q.y.data(), 8, mm));
            PDLPX_BCK(lane2d(fp.o_ys, l, q.ys.data(), 8, mm));
            lpState(*fp.items[l], o, false, nbr + L_new, nbc, hdc[f], hst[f]);
            hps[f] = PowerState{1.0, 0.0, 0.0, 0, o.sv_max_iter <= 0 ? 1 : 0};
            PDLPX_BCK(up(d + fp.o_dc + sizeof(DevConst) * l, &hdc[f], sizeof(DevConst)));
            PDLPX_BCK(up(d + fp.o_st + sizeof(DevState) * l, &hst[f], sizeof(DevState)));
            PDLPX_BCK(up(d + fp.o_ps + sizeof(PowerState) * l, &hps[f], sizeof(PowerState)));
            PDLPX_BCK(cudaMemsetAsync(d + fp.o_flags + 4 * static_cast<size_t>(l), 0, 4, s));
            lane_dev0[l] = now_dev;
            lane_t0[l] = now_host;
        }
        uint32_t live = 0;
        for (int l = 0; l < kFam; ++l)
            if (in_use[l]) live |= 1u << l;
        int32_t powered = L_new - static_cast<int32_t>(o.sv_max_iter > 0 ? fresh_lanes.size() : 0);
        PDLPX_BCK(up(d + fp.o_live, &live, 4));
        PDLPX_BCK(up(d + fp.o_counters, &powered, 4));
        PDLPX_BCK(cudaStreamSynchronize(s));  // the host buffers above go out of scope
        fp.K = c.K;
        fp.Zk = c.Zk;
        fp.qfirst = c.kf;
        L = L_new;
        setShape(fp.args);
        int32_t rc = powerPhase();
        if (rc != PDLPX_OK) return rc;
        return capture(fp.cycle, fp.cycle_launches, false);
    };

    // ---- restart cycles
    SleepWait sleeper;
    std::vector<char> collected(kFam, 0);
    int cycles = 0;
    auto collect = [&](int l, bool out_of_time, double secs, double dev_s) -> int32_t {
        const Item& it = *fp.items[l];
        const int32_t m = it.lp.m;
        DevState f{};
        std::vector<double> xv(n), yv(m);
        PDLPX_BCK(cudaMemcpyAsync(&f, fp.args.st + l, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaMemcpy2DAsync(xv.data(), 8, fp.args.xh + l, 8 * kFam, 8, n, cudaMemcpyDeviceToHost, s));
        if (mb > 0)
            PDLPX_BCK(cudaMemcpy2DAsync(yv.data(), 8, fp.args.yh + l, 8 * kFam, 8, mb, cudaMemcpyDeviceToHost, s));
        if (m > mb)
            PDLPX_BCK(cudaMemcpyAsync(yv.data() + mb, fp.args.yh + Rb + fp.qfirst[l], 8 * static_cast<size_t>(m - mb),
                                      cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaStreamSynchronize(s));
        LpOutcome out;
        finishOutcome(it, f, xv, yv, false, out_of_time, secs - lane_t0[l], dev_s - lane_dev0[l], launches, out);
        collected[l] = 1;
        in_use[l] = 0;
        done(lane_id[l], std::move(out));
        return PDLPX_OK;
    };
    auto running = [&]() {
        int k = 0;
        for (int l = 0; l < kFam; ++l) k += in_use[l];
        return k;
    };
    std::vector<int> fresh_lanes;
    while (running() > 0) {
        if (timeUp(t0, o.max_solve_seconds) || stopped()) break;
        PDLPX_BCK(cudaGraphLaunch(fp.cycle, s));
        launches += fp.cycle_launches;
        ++cycles;
        PDLPX_BCK(sleeper.wait(s));
        PDLPX_BCK(cudaMemcpyAsync(h_flags.data(), fp.args.flags, 4 * static_cast<size_t>(L), cudaMemcpyDeviceToHost, s));
        PDLPX_BCK(cudaStreamSynchronize(s));
        bool fresh = false;
        for (int l = 0; l < L; ++l) fresh |= in_use[l] && (h_flags[l] & 1);
        if (fresh) {
            const double dev_s = deviceSeconds(), secs = hostSeconds();
            for (int l = 0; l < L; ++l) {
                if (!in_use[l] || !(h_flags[l] & 1)) continue;
                const int32_t rc = collect(l, false, secs, dev_s);
                if (rc != PDLPX_OK) return rc;
            }
        }
        if (o.verbose && cycles % 10 == 0) {
            std::printf("PDLP family %7d cycles  %d LPs running  %d shared rows  %d appended rows  %.3fs  [B200]\n",
                        cycles, running(), mb, fp.K, hostSeconds());
            std::fflush(stdout);
        }
        if (!stopped() && running() < kFam) {
            const int32_t rc = admitMembers(fresh_lanes);
            if (rc != PDLPX_OK) return rc;
        }
    }
    if (running() > 0) {
        const double dev_s = deviceSeconds(), secs = hostSeconds();
        const bool out_of_time = timeUp(t0, o.max_solve_seconds);
        for (int l = 0; l < L; ++l) {
            if (!in_use[l]) continue;
            const int32_t rc = collect(l, out_of_time, secs, dev_s);
            if (rc != PDLPX_OK) return rc;
        }
    }
    return PDLPX_OK;
}

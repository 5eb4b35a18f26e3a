// blk_plan.cpp -- host side of the BLKTRI-order FP64 mode solve: COMPB's
// root table, PRDCT programs and BLKTR1's stage table (see blk.h).
//
// Compiled with -ffp-contract=off: every root and every shift difference
// rounds exactly as the reference's FP64 arithmetic does.
#include "blk.h"

#include <cmath>

#include "plan.h"

namespace chy {

namespace {

// TQLRAT (pot/blktri.f:348-423): eigenvalues of the symmetric tridiagonal
// matrix with diagonal d[1..n] and couplings e2[2..n] (e2[i] joins i-1 and
// i), by the rational QL method; 1-based arrays, eigenvalues returned in d in
// order of increasing magnitude.  Returns 0, or the index l whose eigenvalue
// needed more than 30 iterations.
int tqlrat(int n, double machep, double *d, double *e2)
{
    if (n == 1) return 0;
    for (int i = 2; i <= n; i++) e2[i - 1] = e2[i] * e2[i];
    double f = 0.0, b = 0.0, c = 0.0;
    e2[n] = 0.0;
    for (int l = 1; l <= n; l++) {
        double h = machep * (std::fabs(d[l]) + std::sqrt(e2[l]));
        if (!(b > h)) {
            b = h;
            c = b * b;
        }
        int m = l;
        for (; m <= n; m++)
            if (e2[m] <= c) break;
        if (m != l) {
            for (int iter = 0;; iter++) {
                if (iter == 30) return l;
                const int l1 = l + 1;
                double s = std::sqrt(e2[l]);
                double g = d[l];
                double p = (d[l1] - g) / (2.0 * s);
                double r = std::sqrt(p * p + 1.0);
                d[l] = s / (p + std::copysign(r, p));
                h = g - d[l];
                for (int i = l1; i <= n; i++) d[i] = d[i] - h;
                f = f + h;
                // rational QL transformation
                g = d[m];
                if (g == 0.0) g = b;
                h = g;
                s = 0.0;
                for (int i = m - 1; i >= l; i--) {
                    p = g * h;
                    r = p + e2[i];
                    e2[i + 1] = s * r;
                    s = e2[i] / r;
                    d[i + 1] = h + s * (h + d[i]);
                    g = d[i] - e2[i] / g;
                    if (g == 0.0) g = b;
                    h = g * p / r;
                }
                e2[l] = s * g;
                d[l] = h;
                // converged when the coupling is negligible
                if (h == 0.0) break;
                if (std::fabs(e2[l]) <= std::fabs(c / h)) break;
                e2[l] = h * e2[l];
                if (e2[l] == 0.0) break;
            }
        }
        const double p = d[l] + f;
        // insert p among d[1..l-1], kept in increasing magnitude
        int i = l;
        if (l > 1) {
            const double absp = std::fabs(p);
            for (; i >= 2; i--) {
                if (absp >= std::fabs(d[i - 1])) break;
                d[i] = d[i - 1];
            }
        } else {
            i = 1;
        }
        d[i] = p;
    }
    return 0;
}

// Walks PRDCT's control flow (pot/blktri.f:177-260) for one call and
// appends its program.  Root arrays are given by their 1-based start index
// into COMPB's table (BD(i) = B(bd + i - 1)); aa is AN or the shifted CN with
// AA(i) = aa[aa_off + i - 1].
struct Recorder {
    BlkSchedule &s;
    bool bad = false;   // a root index fell outside COMPB's table
    double root(int start, int i)
    {
        const long long q = (long long)start + i - 2;
        if (q < 0 || q >= (long long)s.roots.size()) {
            bad = true;
            return 0.0;
        }
        return s.roots[(size_t)q];
    }

    int prdct(int nd, int bd, int nm1, int bm1, int nm2, int bm2, int na, const double *aa, int aa_off, int is)
    {
        BlkProg pg{};
        pg.first = (int)s.steps.size();
        pg.neg = (nd > 0 && is <= 0) ? 1 : 0;
        int id = nd, ibr = 0, m1 = nm1, m2 = nm2, ia = na;
        auto BD = [&](int i) { return root(bd, i); };
        auto BM1 = [&](int i) { return root(bm1, i); };
        auto BM2 = [&](int i) { return root(bm2, i); };
        for (;;) {
            // label 35: Y = AA(IA) * W
            if (ia > 0) {
                const double c = aa[aa_off + ia - 1];
                ia--;
                if ((int)s.steps.size() == pg.first) {
                    pg.pre = 1;
                    pg.pre_coef = c;
                } else {
                    s.steps.back().post = BLK_SCALE;
                    s.steps.back().coef = c;
                }
            }
            // label 50: the next pass
            if (id <= 0) break;
            double rt = BD(id);
            id--;
            if (id == 0) ibr = 1;
            s.steps.push_back(BlkStep{rt, 0.0, BLK_NONE, 0});
            if (na > 0) continue;
            // label 90: which BM root shifts the right-hand side next
            int use = 0;   // 0: label 80 (Y = W), 1: BM1, 2: BM2
            if (m1 > 0) {
                if (m2 > 0 && std::fabs(BM1(m1)) <= std::fabs(BM2(m2))) use = 2;
                else use = 1;
            } else {
                use = (m2 <= 0) ? 0 : 2;
            }
            if (use == 1 && ibr <= 0 && std::fabs(BM1(m1) - BD(id)) < std::fabs(BM1(m1) - rt)) use = 0;
            if (use == 2 && ibr <= 0 && std::fabs(BM2(m2) - BD(id)) < std::fabs(BM2(m2) - rt)) use = 0;
            if (use == 0) {
                s.steps.back().post = BLK_COPY;
                ibr = 1;
            } else {
                rt = (use == 1) ? rt - BM1(m1) : rt - BM2(m2);
                if (use == 1) m1--;
                else m2--;
                s.steps.back().post = BLK_AXPY;
                s.steps.back().coef = rt;
            }
        }
        pg.nsteps = (int)s.steps.size() - pg.first;
        if (pg.nsteps > s.max_steps) s.max_steps = pg.nsteps;
        s.progs.push_back(pg);
        return (int)s.progs.size() - 1;
    }
};

}  // namespace

int build_blk_schedule(const std::vector<double> &an, const std::vector<double> &bn, const std::vector<double> &cn,
                       int m, BlkSchedule &s, std::string &err)
{
    s = BlkSchedule{};
    const int n = (int)an.size();
    // BLKTRI(IFLG=0) checks (pot/blktri.f:13-34), NP = 1
    if (m < 2) { err = "BLKTRI: M < 2"; return 1; }
    int kx = 0;
    for (int ik = 2, nh = n + 1;;) {
        ik += ik;
        kx++;
        if (nh / ik <= 0) break;
    }
    if (kx < 2 || n != (1 << kx) - 1) { err = "BLKTRI: N is not 2**k - 1"; return 2; }
    s.n = n;
    s.m = m;
    s.kx = kx;
    const int H = (n + 1) / 2;
    s.nvec = n + 3 * H;

    // CN as BLKTR1 sees it: W(IWCN) = CN(N), W(IWCN+J-1) = CN(J-1) (pot/blktri.f:40-45)
    s.cns.assign(n, 0.0);
    s.cns[0] = cn[n - 1];
    for (int j = 2; j <= n; j++) s.cns[j - 1] = cn[j - 2];

    // COMPB (pot/blktri.f:264-344), NP = 1
    const int iwcn = 2 * (n + 1) * (kx - 1) - n + 3;
    s.roots.assign((size_t)iwcn - 1, 0.0);
    double *B = s.roots.data() - 1;   // 1-based view
    const double *AN = an.data() - 1, *BN = bn.data() - 1, *CN = s.cns.data() - 1;
    volatile double epslon = 1.0;
    for (;;) {
        epslon = epslon / 10.0;
        volatile double dif = 1.0 + epslon;
        if (!(dif > 1.0)) break;
    }
    epslon = 100.0 * epslon;
    for (int j = 2; j <= n; j++) {   // J = 1 is skipped for NP != 0
        const double arg = AN[j] * CN[j];
        if (arg < 0) { err = "COMPB: AN*CN < 0"; return 4; }
        const double chld = std::sqrt(arg);
        B[j] = (CN[j] < 0) ? -chld : chld;
    }
    {
        const int ifull = 1 << kx;
        int lh = ifull, i1 = 1;
        std::vector<double> ah(n + 1), bh(n + 1);
        for (int lx = 1; lx <= kx; lx++) {
            i1 += i1;
            const int nn = i1 + i1 - 1, ifl = ifull - i1 + 1;
            for (int i = 1; i <= ifl; i += i1) {
                if (i >= ifl) {   // the periodic wrap block: NP != 0 leaves it out
                    lh += nn;
                    continue;
                }
                for (int ls = 1, j = i; j <= i + nn - 1; j++, ls++) {
                    bh[ls] = BN[j];
                    ah[ls] = B[j];
                }
                if (tqlrat(nn, epslon, bh.data(), ah.data()) != 0) { err = "COMPB: TQLRAT did not converge"; return 4; }
                for (int j = 1; j <= nn; j++) {
                    lh++;
                    if (lh > iwcn - 1) { err = "COMPB: root table overflow"; return 4; }
                    B[lh] = -bh[j];
                }
            }
        }
    }
    for (int j = 1; j <= n; j++) B[j] = -BN[j];

    // BLKTR1 (pot/blktri.f:60-173) as stages of independent tasks, NP = 1
    Recorder rec{s};
    const int nh = 1 << kx, ih1 = nh + nh;
    auto Y = [](int col) { return col - 1; };          // Y(:,col), col 1-based
    auto V = [&](int q) { return n + q; };
    auto W1 = [&](int q) { return n + H + q; };
    auto W2 = [&](int q) { return n + 2 * H + q; };
    auto stage = [&](int kind) {
        s.stages.push_back(BlkStage{kind, (int)s.tasks.size(), 0, 0});
    };
    auto task = [&](int prog, int a, int b, int c, int out) {
        s.tasks.push_back(BlkTask{prog, a, b, c, out, 0});
        s.stages.back().ntasks++;
    };
    // reduction levels (pot/blktri.f:76-110)
    for (int lx = 1; lx <= kx - 1; lx++) {
        const int ir = lx - 1, iz = 1 << ir, isgn = (ir % 2 == 0) ? 1 : -1, msgn = -isgn;
        const int ih2 = 1 << (kx - ir + 1);
        const int lm = (ir - 2) * ih1 + ih2 + ih2 + 1, lz = (ir - 1) * ih1 + ih2 + 1;
        const int iim = iz - 1, iiz = iim + iim + 1, i1 = iz + iz, nif = 1 << (kx - ir - 1);
        // the products of the odd positions: the first W3 (:88-89) and the
        // W3 of every loop pass (:102-103)
        stage(BLK_TASK_PRDCT);
        for (int t = 0; t < nif; t++) {
            const int p = rec.prdct(iiz, lz + 2 * t * iiz, iim, lm + 4 * t * iim, iim, lm + (4 * t + 2) * iim, 0,
                                    nullptr, 0, isgn);
            task(p, Y((2 * t + 1) * iz), -1, -1, V(t));
        }
        // both neighbour products of each even position (:100-101, :104-105)
        stage(BLK_TASK_PRDCT);
        for (int jj = 1; jj < nif; jj++) {
            const int i = jj * i1, jm1 = (4 * jj - 2) * iim + lm, jp1 = 4 * jj * iim + lm;
            task(rec.prdct(iim, jm1, 0, 0, 0, 0, iz, an.data(), i - iz, msgn), V(jj - 1), -1, -1, W1(jj - 1));
            task(rec.prdct(iim, jp1, 0, 0, 0, 0, iz, s.cns.data(), i, msgn), V(jj), -1, -1, W2(jj - 1));
        }
        // Y(:,I) = W1 + W2 - Y(:,I) (:106-108)
        stage(BLK_TASK_SUMSUB);
        for (int jj = 1; jj < nif; jj++) task(-1, W1(jj - 1), W2(jj - 1), Y(jj * i1), Y(jj * i1));
    }
    // back-substitution levels (pot/blktri.f:112-170)
    for (int ll = 1; ll <= kx; ll++) {
        const int lx = kx - ll + 1, ir = lx - 1, isgn = (ir % 2 == 0) ? 1 : -1, msgn = -isgn;
        const int iz = 1 << ir, iim = iz - 1, iiz = iim + iim + 1, ih2 = 1 << (kx - ir + 1);
        const int lm = (ir - 2) * ih1 + ih2 + ih2 + 1, lz = (ir - 1) * ih1 + ih2 + 1;
        const int nif = (1 << (kx - ir)) - 1;
        // neighbour products (:145-146, :151-152); the edge ones are zero (:148-149, :155-156)
        stage(BLK_TASK_PRDCT);
        for (int jj = 1; jj <= nif; jj += 2) {
            const int i = jj * iz, q = (jj - 1) / 2, j2 = jj + jj;
            const int jm1 = (j2 - 2) * iim + lm, jp1 = j2 * iim + lm;
            if (jj > 1) task(rec.prdct(iim, jm1, 0, 0, 0, 0, iz, an.data(), i - iz, msgn), Y(i - iz), -1, -1, W1(q));
            if (jj < nif) task(rec.prdct(iim, jp1, 0, 0, 0, 0, iz, s.cns.data(), i, msgn), Y(i + iz), -1, -1, W2(q));
        }
        // W1 = Y(:,I) - W1 - W2 (:157-159)
        stage(BLK_TASK_SUBSUB);
        for (int jj = 1; jj <= nif; jj += 2) {
            const int i = jj * iz, q = (jj - 1) / 2;
            task(-1, Y(i), jj > 1 ? W1(q) : -1, jj < nif ? W2(q) : -1, V(q));
        }
        // Y(:,I) = the centre product of W1 (:160-161)
        stage(BLK_TASK_PRDCT);
        for (int jj = 1; jj <= nif; jj += 2) {
            const int i = jj * iz, q = (jj - 1) / 2, j2 = jj + jj;
            const int jm1 = (j2 - 2) * iim + lm, jz = (jj - 1) * iiz + lz, jp1 = j2 * iim + lm;
            task(rec.prdct(iiz, jz, iim, jm1, iim, jp1, 0, nullptr, 0, isgn), V(q), -1, -1, Y(i));
        }
    }
    if (rec.bad) { err = "BLKTR1: root index outside COMPB's table"; return 4; }
    // drop empty stages (the top reduction level has no even positions)
    std::vector<BlkStage> kept;
    for (const BlkStage &st : s.stages)
        if (st.ntasks > 0) kept.push_back(st);
    s.stages.swap(kept);
    return 0;
}

void blk_mode_bm(const HostPlan &hp, int l, double *bm)
{
    const int M = hp.M, n = hp.N;
    const int m = l <= n ? l : l - n;
    const double powrm = (m % 2 == 0) ? 1.0 : -1.0;
    const double xl = hp.xlamm[m];
    // BM(1) = -CM(1) + (POWRM-1) AMMIN + 2 (XLAMM-1) C(1); BM(J) = -CM(J) -
    // AM(J) + 2 (XLAMM-1) C(J); BM(M) with CMMAX for CM(M).  bm0 holds the
    // first two terms of each, formed as POT3 forms them.
    bm[0] = hp.bm0[0] + (powrm - 1.0) * hp.ammin + 2.0 * (xl - 1.0) * hp.cc[0];
    for (int j = 1; j < M; j++) bm[j] = hp.bm0[j] + 2.0 * (xl - 1.0) * hp.cc[j];
}

std::vector<double> blk_bm_table(const HostPlan &hp)
{
    const int M = hp.M, L = hp.L, nblk = L >= 32 ? L / 32 : 1;
    std::vector<double> t((size_t)nblk * M * 32), bm(M);
    for (int b = 0; b < nblk; b++)
        for (int lane = 0; lane < 32; lane++) {
            blk_mode_bm(hp, (32 * b + lane) % L, bm.data());
            for (int j = 0; j < M; j++) t[((size_t)b * M + j) * 32 + lane] = bm[j];
        }
    return t;
}

void blk_solve_host(const BlkSchedule &s, const double *am, const double *bm, const double *cm, double *y)
{
    const int m = s.m, n = s.n;
    std::vector<double> vec((size_t)s.nvec * m, 0.0), Wv(m), Dv(m);
    const std::vector<double> zero(m, 0.0);
    for (size_t i = 0; i < (size_t)n * m; i++) vec[i] = y[i];
    auto V = [&](int id) -> double * { return id < 0 ? const_cast<double *>(zero.data()) : vec.data() + (size_t)id * m; };
    for (const BlkStage &st : s.stages) {
        for (int t = st.first; t < st.first + st.ntasks; t++) {
            const BlkTask &tk = s.tasks[t];
            double *out = V(tk.out);
            if (st.kind == BLK_TASK_SUMSUB) {
                const double *a = V(tk.a), *b = V(tk.b), *c = V(tk.c);
                for (int j = 0; j < m; j++) out[j] = (a[j] + b[j]) - c[j];
                continue;
            }
            if (st.kind == BLK_TASK_SUBSUB) {
                const double *a = V(tk.a), *b = V(tk.b), *c = V(tk.c);
                for (int j = 0; j < m; j++) out[j] = (a[j] - b[j]) - c[j];
                continue;
            }
            const BlkProg &pg = s.progs[tk.prog];
            const double *x = V(tk.a);
            double *Y = out;
            for (int j = 0; j < m; j++) {
                const double w = pg.neg ? -x[j] : x[j];
                Y[j] = pg.pre ? pg.pre_coef * w : w;
            }
            for (int q = pg.first; q < pg.first + pg.nsteps; q++) {
                const BlkStep &sp = s.steps[q];
                const double rt = sp.rt;
                // elimination from the last row (pot/blktri.f:214-227)
                double dn = am[m - 1] / (bm[m - 1] - rt);
                double wn = Y[m - 1] / (bm[m - 1] - rt);
                Dv[m - 1] = dn;
                Wv[m - 1] = wn;
                for (int i = m - 2; i >= 1; i--) {
                    const double den = bm[i] - rt - cm[i] * dn;
                    dn = am[i] / den;
                    wn = (Y[i] - cm[i] * wn) / den;
                    Dv[i] = dn;
                    Wv[i] = wn;
                }
                const double den = bm[0] - rt - cm[0] * dn;
                double w = (den == 0) ? 1. : (Y[0] - cm[0] * wn) / den;
                // substitution (:229-231) and the right-hand-side update
                for (int j = 0; j < m; j++) {
                    if (j > 0) w = Wv[j] - Dv[j] * w;
                    switch (sp.post) {
                    case BLK_COPY: Y[j] = w; break;
                    case BLK_AXPY: Y[j] = Y[j] + sp.coef * w; break;
                    case BLK_SCALE: Y[j] = sp.coef * w; break;
                    default: break;
                    }
                }
            }
        }
    }
    for (size_t i = 0; i < (size_t)n * m; i++) y[i] = vec[i];
}

}  // namespace chy

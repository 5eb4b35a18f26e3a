// plan.cpp -- host tables of one pot3 grid.  Compiled with -ffp-contract=off
// (no FMA) so every table value equals the value the reference's own FP64
// arithmetic produces.
#include "plan.h"
#include "legendre.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>

namespace chy {

// pi/4 as the gcc build's REAL(4) ATAN(1.0) and as the -r8 builds' REAL(8).
static const float kQuarterPiF32 = 0x1.921fb6p-1f;
static const double kQuarterPiF64 = 0x1.921fb54442d18p-1;

// ---------------------------------------------------------------------------
// Azimuthal transform schedule.
//
// pot/fft.f:73-629 computes the LMAX/2-point complex transform in place by a
// sequence of radix-4 / radix-2 decimation stages (factor order from
// fft.f:147-187), rotates each butterfly output by a twiddle generated with a
// renormalised recurrence (fft.f:225-232, 296-307), and finally permutes the
// result (fft.f:800-840).  Its GCC build builds the twiddle angle from a
// REAL(4) pi (fft.f:129), so the transform differs from an exact DFT by ~1e-7
// and the only way to reproduce it is to use the very twiddles it generates.
// This walker follows the same loop control and records, for every butterfly,
// the rotation it applies; it records the permutation by applying the same
// swaps to an index array.  Only factors 2 and 4 occur for power-of-two N.
// ---------------------------------------------------------------------------
int build_fft_schedule(int n, int isn, int r8, FftSchedule &s)
{
    if (n < 2 || (n & (n - 1)) != 0 || n > 4096) return CHY_ERR_DIMS;
    s = FftSchedule();
    s.n = n;
    s.isn = isn;

    // factors of n, in the order fft.f:147-187 produces them
    int fac[32] = {0};
    int m = 0, kt = 0;
    {
        int k = n;
        while (k % 16 == 0) { fac[++m] = 4; k /= 16; }
        // no odd factors for powers of two
        if (k <= 4) {
            kt = m;
            fac[m + 1] = k;
            if (k != 1) m++;
        } else {
            if (k % 4 == 0) { fac[++m] = 2; k /= 4; }
            kt = m;
            for (int j = 2; j <= k;) {
                if (k % j == 0) { fac[++m] = j; k /= j; }
                j = ((j + 1) / 2) * 2 + 1;
            }
        }
        for (int j = kt; j >= 1; j--) fac[++m] = fac[j];
    }
    for (int i = 1; i <= m; i++)
        if (fac[i] != 2 && fac[i] != 4) return CHY_ERR_DIMS;
    if (2 * kt + 1 < m) return CHY_ERR_DIMS;  // square-free permutation never needed for 2^k
    s.nstage = m;
    s.tw.assign((size_t)m * n * 6, 0.0);
    s.twon.assign((size_t)m * n, 0);
    std::vector<int> seen((size_t)m * n, 0);

    double rad = r8 ? 8.0 * kQuarterPiF64 : (double)(8.0f * kQuarterPiF32);
    int inc = isn;
    if (isn < 0) { rad = -rad; inc = -inc; }
    const int nt = inc * n, ks = inc * n, nn = nt - inc;
    int jc = ks / n;
    int kspan = ks;
    const double radf = rad * (double)jc * 0.5;

    auto put = [&](int st, int kk, int on, double c1, double s1, double c2, double s2, double c3,
                   double s3) {
        size_t o = (size_t)st * n + (kk - 1);
        seen[o]++;
        s.twon[o] = (uint8_t)on;
        double *t = &s.tw[o * 6];
        t[0] = c1; t[1] = s1; t[2] = c2; t[3] = s2; t[4] = c3; t[5] = s3;
    };

    for (int i = 1; i <= m; i++) {
        const int st = i - 1;
        double sd = radf / (double)kspan;
        double tt = std::sin(sd);
        const double cd = 2.0 * (tt * tt);
        sd = std::sin(sd + sd);
        int kk = 1;
        if (fac[i] == 2) {
            kspan /= 2;
            s.radix[st] = 2;
            s.span[st] = kspan;
            int k1 = kspan + 2, k2;
            double c1, s1, ak;
            // j = 0 butterflies: no rotation
            for (;;) {
                k2 = kk + kspan;
                put(st, kk, 0, 1, 0, 1, 0, 1, 0);
                kk = k2 + kspan;
                if (kk <= nn) continue;
                kk = kk - nn;
                if (kk <= jc) continue;
                break;
            }
            if (kk > kspan) continue;  // stage done
            for (;;) {                  // pairs j, span-j share one recurrence step
                c1 = 1.0 - cd;
                s1 = sd;
                for (;;) {
                    k2 = kk + kspan;
                    put(st, kk, 1, c1, s1, 0, 0, 0, 0);
                    kk = k2 + kspan;
                    if (kk < nt) continue;
                    k2 = kk - nt;
                    c1 = -c1;
                    kk = k1 - k2;
                    if (kk > k2) continue;
                    ak = c1 - (cd * c1 + sd * s1);
                    s1 = (sd * c1 - cd * s1) + s1;
                    c1 = 0.5 / (ak * ak + s1 * s1) + 0.5;
                    s1 = c1 * s1;
                    c1 = c1 * ak;
                    kk = kk + jc;
                    if (kk < k2) continue;
                    break;
                }
                k1 = k1 + inc + inc;
                kk = (k1 - kspan) / 2 + jc;
                if (kk <= jc + jc) continue;
                break;
            }
        } else {
            kspan /= 4;
            s.radix[st] = 4;
            s.span[st] = kspan;
            double c1, s1, c2 = 0, s2 = 0, c3 = 0, s3 = 0;
            bool done = false;
            for (;;) {
                c1 = 1.0;
                s1 = 0.0;
                for (;;) {
                    // one butterfly at kk per block, then the recurrence step
                    for (;;) {
                        int k3 = kk + 3 * kspan;
                        if (s1 == 0.0) put(st, kk, 0, 1, 0, 1, 0, 1, 0);
                        else put(st, kk, 1, c1, s1, c2, s2, c3, s3);
                        kk = k3 + kspan;
                        if (kk <= nt) continue;
                        break;
                    }
                    c2 = c1 - (cd * c1 + sd * s1);
                    s1 = (sd * c1 - cd * s1) + s1;
                    c1 = 0.5 / (c2 * c2 + s1 * s1) + 0.5;
                    s1 = c1 * s1;
                    c1 = c1 * c2;
                    c2 = c1 * c1 - s1 * s1;
                    s2 = 2.0 * c1 * s1;
                    c3 = c2 * c1 - s2 * s1;
                    s3 = c2 * s1 + s2 * c1;
                    kk = kk - nt + jc;
                    if (kk <= kspan) continue;
                    break;
                }
                kk = kk - kspan + inc;
                if (kk <= jc) continue;
                if (kspan == jc) done = true;
                break;
            }
            (void)done;
        }
    }
    // every butterfly of every stage recorded exactly once, at the positions
    // b*radix*span + j (j < span) the device code assumes, and with a rotation
    // that depends on j only (the same for every block b)
    s.ncompact = 0;
    for (int st = 0; st < m; st++) {
        const int r = s.radix[st], h = s.span[st];
        for (int kk = 0; kk < n; kk++) {
            const bool first = (kk % (r * h)) < h;
            if (seen[(size_t)st * n + kk] != (first ? 1 : 0)) return CHY_ERR_DIMS;
            if (first) {
                const int j = kk % (r * h);
                const size_t a = (size_t)st * n + kk, b0 = (size_t)st * n + j;
                if (s.twon[a] != s.twon[b0] || std::memcmp(&s.tw[a * 6], &s.tw[b0 * 6], 6 * sizeof(double)) != 0)
                    return CHY_ERR_DIMS;
            }
        }
        s.off[st] = s.ncompact;
        s.ncompact += h;
    }
    s.twc.assign((size_t)s.ncompact * 6, 0.0);
    s.onc.assign(s.ncompact, 0);
    for (int st = 0; st < m; st++)
        for (int j = 0; j < s.span[st]; j++) {
            const size_t a = (size_t)st * n + j, o = (size_t)s.off[st] + j;
            s.onc[o] = s.twon[a];
            std::memcpy(&s.twc[o * 6], &s.tw[a * 6], 6 * sizeof(double));
        }

    // square-factor permutation (fft.f:800-840), applied to an index array
    {
        std::vector<int> idx(n + 1);
        for (int p = 0; p <= n; p++) idx[p] = p;
        int np_[64] = {0};
        int k, j, k2, k3;
        np_[1] = ks;
        if (kt != 0) {
            k = kt + kt + 1;
            if (m < k) k = k - 1;
            j = 1;
            np_[k + 1] = jc;
            do {
                np_[j + 1] = np_[j] / fac[j];
                np_[k] = np_[k + 1] * fac[j];
                j = j + 1;
                k = k - 1;
            } while (j < k);
            k3 = np_[k + 1];
            int span = np_[2];
            int kk = jc + 1;
            k2 = span + 1;
            j = 1;
            // single-variate transform: goto structure of fft.f:820-840
            int state = 820;
            for (;;) {
                if (state == 820) {
                    std::swap(idx[kk], idx[k2]);
                    kk = kk + inc;
                    k2 = span + k2;
                    if (k2 < ks) continue;
                    state = 830;
                } else if (state == 830) {
                    k2 = k2 - np_[j];
                    j = j + 1;
                    k2 = np_[j + 1] + k2;
                    if (k2 > np_[j]) continue;
                    j = 1;
                    state = 840;
                } else {  // 840
                    if (kk < k2) { state = 820; continue; }
                    kk = kk + inc;
                    k2 = span + k2;
                    if (k2 < ks) continue;
                    if (kk < ks) { state = 830; continue; }
                    break;
                }
            }
            jc = k3;
        }
        s.perm.resize(n);
        for (int p = 1; p <= n; p++) s.perm[p - 1] = idx[p] - 1;
    }

    // REALTR (fft.f:35-65): the (CN, SN) pair used at each of the N/2+1 steps
    {
        const int nk = n + 2;
        s.nh = nk / 2;
        s.rt.assign((size_t)s.nh * 2, 0.0);
        double sd = r8 ? 2.0 * kQuarterPiF64 / (double)n : (double)(2.0f * kQuarterPiF32 / (float)n);
        double tt = std::sin(sd);
        const double cd = 2.0 * (tt * tt);
        sd = std::sin(sd + sd);
        double sn = 0.0, cn, aa;
        if (isn < 0) { cn = -1.0; sd = -sd; }
        else cn = 1.0;
        for (int j = 1; j <= s.nh; j++) {
            s.rt[2 * (j - 1)] = cn;
            s.rt[2 * (j - 1) + 1] = sn;
            aa = cn - (cd * cn + sd * sn);
            sn = (sd * cn - cd * sn) + sn;
            cn = 0.5 / (aa * aa + sn * sn) + 0.5;
            sn = cn * sn;
            cn = cn * aa;
        }
    }
    return CHY_OK;
}

void fft_apply_host(const FftSchedule &s, double *a, double *b)
{
    const int n = s.n;
    for (int st = 0; st < s.nstage; st++) {
        const int r = s.radix[st], h = s.span[st];
        for (int base = 0; base < n; base += r * h)
            for (int j = 0; j < h; j++) {
                const int kk = base + j;
                const double *t = &s.tw[((size_t)st * n + kk) * 6];
                const bool on = s.twon[(size_t)st * n + kk] != 0;
                if (r == 2) {
                    const int k2 = kk + h;
                    if (!on) {
                        double ak = a[k2], bk = b[k2];
                        a[k2] = a[kk] - ak; b[k2] = b[kk] - bk;
                        a[kk] = a[kk] + ak; b[kk] = b[kk] + bk;
                    } else {
                        double ak = a[kk] - a[k2], bk = b[kk] - b[k2];
                        a[kk] = a[kk] + a[k2]; b[kk] = b[kk] + b[k2];
                        a[k2] = t[0] * ak - t[1] * bk;
                        b[k2] = t[1] * ak + t[0] * bk;
                    }
                } else {
                    const int k1 = kk + h, k2 = k1 + h, k3 = k2 + h;
                    double akp = a[kk] + a[k2], akm = a[kk] - a[k2];
                    double ajp = a[k1] + a[k3], ajm = a[k1] - a[k3];
                    a[kk] = akp + ajp;
                    ajp = akp - ajp;
                    double bkp = b[kk] + b[k2], bkm = b[kk] - b[k2];
                    double bjp = b[k1] + b[k3], bjm = b[k1] - b[k3];
                    b[kk] = bkp + bjp;
                    bjp = bkp - bjp;
                    if (s.isn >= 0) {
                        akp = akm - bjm; akm = akm + bjm; bkp = bkm + ajm; bkm = bkm - ajm;
                    } else {
                        akp = akm + bjm; akm = akm - bjm; bkp = bkm - ajm; bkm = bkm + ajm;
                    }
                    if (on) {
                        a[k1] = akp * t[0] - bkp * t[1]; b[k1] = akp * t[1] + bkp * t[0];
                        a[k2] = ajp * t[2] - bjp * t[3]; b[k2] = ajp * t[3] + bjp * t[2];
                        a[k3] = akm * t[4] - bkm * t[5]; b[k3] = akm * t[5] + bkm * t[4];
                    } else {
                        a[k1] = akp; b[k1] = bkp; a[k2] = ajp; b[k2] = bjp; a[k3] = akm; b[k3] = bkm;
                    }
                }
            }
    }
    std::vector<double> ta(a, a + n), tb(b, b + n);
    for (int p = 0; p < n; p++) { a[p] = ta[s.perm[p]]; b[p] = tb[s.perm[p]]; }
}

void realtr_apply_host(const FftSchedule &s, double *a, double *b)
{
    const int n = s.n;
    if (s.isn >= 0) { a[n] = a[0]; b[n] = b[0]; }
    for (int j = 0; j < s.nh; j++) {
        const int k = n - j;
        const double cn = s.rt[2 * j], sn = s.rt[2 * j + 1];
        double aa = a[j] + a[k], ab = a[j] - a[k], ba = b[j] + b[k], bb = b[j] - b[k];
        double re = cn * ba + sn * ab, im = sn * ba - cn * ab;
        b[k] = im - bb;
        b[j] = im + bb;
        a[k] = aa - re;
        a[j] = aa + re;
    }
}

// ---------------------------------------------------------------------------
// Symmetric tridiagonal eigen decomposition (implicit QL, Wilkinson shift).
// ---------------------------------------------------------------------------
int tridiag_eigen(int n, double *d, double *e, double *z)
{
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) z[i + (size_t)n * k] = (i == k) ? 1.0 : 0.0;
    if (n > 0) e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        for (;;) {
            for (m = l; m < n - 1; m++) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) + dd == dd) break;
            }
            if (m == l) break;
            if (iter++ == 100) return l + 1;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
            double sn = 1.0, c = 1.0, p = 0.0;
            int i;
            bool underflow = false;
            for (i = m - 1; i >= l; i--) {
                double f = sn * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    underflow = true;
                    break;
                }
                sn = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * sn + 2.0 * c * b;
                p = sn * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; k++) {
                    double zi1 = z[k + (size_t)n * (i + 1)], zi = z[k + (size_t)n * i];
                    z[k + (size_t)n * (i + 1)] = sn * zi + c * zi1;
                    z[k + (size_t)n * i] = c * zi - sn * zi1;
                }
            }
            if (underflow) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Legendre factors of BDYGEN.
//
// The reference expands in terms TERM(I), I = L(L+1)/2 + M + 1, built from
// the polynomial factors BLM(cos theta) of its statement functions
// (pot/boundary.f:204-253): BLM = [C1 *] P(C2) [* S^M], where P is a
// polynomial in C2 = cos^2 theta with the integer coefficients below
// (highest power first), C1 = cos theta is present when L-M is odd, and
// S = sin theta.  The ring pass multiplies BLM by r^L (and F1 for odd-L,
// M = 0 terms, pot/boundary.f:412-502); the boundary pass multiplies by the
// normalisation DLM = a * 2^-n (pot/boundary.f:694-772, written there as
// a*TWn with TW5..TW18 = 2^-5..2^-18).  Which terms exist depends on ISYM
// (pot/boundary.f:417-490).  Evaluation order follows the reference's
// expressions so the tables reproduce its values bit for bit.
// ---------------------------------------------------------------------------
static const LegTerm kLeg[66] = CHY_LEG_TABLE;

// TWn as the reference's PARAMETER statement defines it (pot/boundary.f:181-185):
// REAL(4) decimal literals (exact 2^-n) in the gcc build, REAL(8) decimals under -r8.
static double tw_value(int nexp, bool r8)
{
    static const char *dec[19] = {nullptr, nullptr, nullptr, nullptr, nullptr, "0.03125", "0.015625",
                                  "7.8125E-3", "3.90625E-3", "1.953125E-3", "9.765625E-04",
                                  "4.8828125E-4", "2.44140625E-4", "1.220703125E-4",
                                  "6.103515625E-5", "3.051757813E-5", "1.525878907E-5",
                                  "7.629394535E-6", "3.814697266E-6"};
    if (nexp < 5 || nexp > 18) return 1.0;
    if (r8) return std::strtod(dec[nexp], nullptr);
    return (double)std::strtof(dec[nexp], nullptr);
}

// ring pass TERM(I) (pot/boundary.f:385-502)
static void ring_terms(double *term, double C1, double S1, double rsph, int maxtrm, int isyma,
                       double F1)
{
    Powers p = make_powers(C1, S1, maxtrm);
    double q[11];
    for (int l = 1; l <= 10; l++) q[l] = ipow(rsph, l);
    for (int i = 0; i < 66; i++) term[i] = ring_term(kLeg[i], i, p, q, maxtrm, isyma, F1);
}

// boundary pass TERM(I) = DLM * BLM (pot/boundary.f:670-772)
static void bdy_terms(double *term, double C1, double S1, int maxtrm, int isyma, double F1,
                      bool r8)
{
    Powers p = make_powers(C1, S1, maxtrm);
    for (int i = 0; i < 66; i++) {
        const LegTerm &t = kLeg[i];
        term[i] = 0.0;
        if (t.l > maxtrm || !term_present(t.l, t.m, isyma)) continue;
        if (i == 0) { term[i] = 1.0; continue; }
        double dlm = t.tw ? t.dlm_a * tw_value(t.tw, r8) : t.dlm_a;
        double v;
        const bool odd = ((t.l - t.m) % 2) != 0;
        if (t.npoly == 0 && t.m > 0 && odd) {
            v = (dlm * p.c1) * p.s[t.m];   // written a*TWn*C1*S^m in the reference
        } else if (t.l == 1 && t.m == 0) {
            v = p.c1;                      // TERM(2) = C1*F1
        } else {
            v = dlm * blm_value(t, p);
        }
        if (t.m == 0 && (t.l % 2) == 1) v = v * F1;
        term[i] = v;
    }
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
static bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

int build_host_plan(const chy_grid &g, HostPlan &hp, std::string &err)
{
    hp = HostPlan();
    hp.g = g;
    const int J = g.jmax, K = g.kmax, L = g.lmax;
    if (J - 1 < 2) { err = "JMAX-1 < 2"; return CHY_ERR_M_LT_2; }
    if (!is_pow2(K) || K < 4) { err = "KMAX must be a power of 2 (BLKTRI needs KMAX-1 = 2**k-1)"; return CHY_ERR_N_NOT_POW2; }
    if (!is_pow2(L) || L < 32 || L > 1024) { err = "LMAX must be a power of 2 in [32, 1024]"; return CHY_ERR_DIMS; }
    if (J > 4096 || K > 128) { err = "JMAX <= 4096 and KMAX <= 128 are supported"; return CHY_ERR_DIMS; }
    const int isyma = std::abs(g.isym);
    if (!(isyma == 1 || isyma == 2 || isyma == 3)) { err = "ISYM must be +-1, +-2 or +-3"; return CHY_ERR_UNSUPPORTED; }
    if (g.maxtrm < 0 || g.maxtrm > 10) { err = "MAXTRM must be 0..10"; return CHY_ERR_UNSUPPORTED; }
    if (g.npoint < 2 || g.npoint > 10) { err = "NPOINT must be 2..10"; return CHY_ERR_UNSUPPORTED; }
    if (g.npoint / 2 + 2 > J + 1) { err = "NPOINT too large for JMAX"; return CHY_ERR_UNSUPPORTED; }
    const bool r8 = g.literal_kind == CHY_LITERAL_R8;

    hp.J = J; hp.K = K; hp.L = L; hp.N = L / 2; hp.M = J - 1; hp.NZ = K - 1;
    hp.dtheta = 2.0 * g.pi / (double)L;
    hp.sf1 = r8 ? 0.5 / (double)hp.N : (double)(0.5f / (float)hp.N);
    hp.pig4 = 4.0 * g.pi * g.grav;

    // /GRID/ arrays (radhydro/io.f:194-203 when not supplied)
    hp.r.resize(J + 2); hp.rhf.resize(J + 2); hp.z.resize(K + 2); hp.zhf.resize(K + 2);
    for (int j = 1; j <= J + 2; j++) {
        hp.r[j - 1] = g.r ? g.r[j - 1] : (double)(j - 2) * g.rof3n;
        hp.rhf[j - 1] = g.rhf ? g.rhf[j - 1] : hp.r[j - 1] + g.rof3n / 2.0;
    }
    for (int k = 1; k <= K + 2; k++) {
        hp.z[k - 1] = g.z ? g.z[k - 1] : (double)(k - 2) * g.zof3n;
        hp.zhf[k - 1] = g.zhf ? g.zhf[k - 1] : hp.z[k - 1] + g.zof3n / 2.0;
    }
    auto R = [&](int j) { return hp.r[j - 1]; };
    auto Z = [&](int k) { return hp.z[k - 1]; };
    auto RHF = [&](int j) { return hp.rhf[j - 1]; };
    auto ZHF = [&](int k) { return hp.zhf[k - 1]; };

    int st = build_fft_schedule(hp.N, 1, r8, hp.fwd);
    if (st == CHY_OK) st = build_fft_schedule(hp.N, -1, r8, hp.inv);
    if (st != CHY_OK) { err = "unsupported azimuthal transform length"; return st; }

    // COSM/SINM (pot/boundary.f:29-38)
    hp.cosm.assign((size_t)10 * L, 0.0);
    hp.sinm.assign((size_t)10 * L, 0.0);
    for (int l = 1; l <= L; l++) {
        double psi = (double)((float)l - 0.5f) * hp.dtheta;
        for (int m = 1; m <= 10; m++) {
            hp.cosm[(size_t)(m - 1) * L + (l - 1)] = std::cos((double)m * psi);
            hp.sinm[(size_t)(m - 1) * L + (l - 1)] = std::sin((double)m * psi);
        }
    }
    // COS(THETA - PI), THETA = (L - 1/2) DTHETA: the BINARY companion's
    // angle (pot/ExternalPot.f:56-62)
    hp.bcos.resize(L);
    for (int l = 1; l <= L; l++) hp.bcos[l - 1] = std::cos(((double)l - 0.5) * hp.dtheta - g.pi);

    // transforms of the boundary potential's azimuthal basis: the boundary
    // columns POT3 transforms (pot/pot3.f:93-140) are combinations of these
    // 21 columns (pot/boundary.f:814-830), and the transform is linear
    {
        const int N = hp.N;
        hp.fbasis.assign((size_t)21 * L, 0.0);
        std::vector<double> col(L), a(N + 2), b(N + 2);
        for (int q = 0; q < 21; q++) {
            for (int l = 0; l < L; l++)
                col[l] = q == 0 ? 1.0 : (q <= 10 ? hp.cosm[(size_t)(q - 1) * L + l] : hp.sinm[(size_t)(q - 11) * L + l]);
            std::fill(a.begin(), a.end(), 0.0);
            std::fill(b.begin(), b.end(), 0.0);
            for (int n = 0; n < N; n++) { a[n] = col[2 * n]; b[n] = col[2 * n + 1]; }
            fft_apply_host(hp.fwd, a.data(), b.data());
            realtr_apply_host(hp.fwd, a.data(), b.data());
            for (int l = 0; l < L; l++)
                hp.fbasis[(size_t)q * L + l] = (l <= N ? a[l] : b[l - N]) * hp.sf1;
        }
    }

    // BDYGEN constants (pot/boundary.f:344-358)
    double F1, F2;
    if (isyma == 2 || isyma == 9) { F1 = 0.0; F2 = 2.0; }
    else if (isyma == 3) { F1 = 0.0; F2 = 4.0; }
    else { F1 = 1.0; F2 = 1.0; }
    hp.ntrm = 0;
    for (int l = 0; l <= g.maxtrm; l++) hp.ntrm += l + 1;

    // rings
    const int M = hp.M, NZ = hp.NZ;
    hp.nring = M * NZ;
    hp.ring_rsph.assign(hp.nring, 0.0);
    hp.ring_dv.assign(hp.nring, 0.0);
    hp.ring_term.assign((size_t)hp.nring * 66, 0.0);
    hp.ring_qh.assign((size_t)hp.nring * 11, 0.0);
    std::vector<int> keep;
    for (int k = 0; k < NZ; k++) {
        const int kk = k + 2;
        const double ZZ = ZHF(kk), Z2 = ZZ * ZZ, ZDEL = Z(kk + 1) - Z(kk);
        for (int j = 0; j < M; j++) {
            const int jj = j + 2, ring = k * M + j;
            const double RR = RHF(jj), R2 = RR * RR, RSPH = std::sqrt(R2 + Z2);
            hp.ring_rsph[ring] = RSPH;
            if (g.redge > 0.0 && RSPH > g.redge) continue;
            keep.push_back(ring);
            ring_terms(&hp.ring_term[(size_t)ring * 66], ZZ / RSPH, RR / RSPH, RSPH, g.maxtrm, isyma, F1);
            hp.ring_dv[ring] = 0.5 * hp.dtheta * ZDEL * (R(jj + 1) * R(jj + 1) - R(jj) * R(jj)) * F2;
            for (int l = 0; l <= 10; l++) hp.ring_qh[(size_t)ring * 11 + l] = ipow(RSPH, -(2 * l + 1));
        }
    }
    hp.nkeep = (int)keep.size();
    hp.ring_sorted = keep;
    std::stable_sort(hp.ring_sorted.begin(), hp.ring_sorted.end(),
                     [&](int a, int b) { return hp.ring_rsph[a] < hp.ring_rsph[b]; });

    // active MRING columns: part 0 = TERM*mass-or-cos moment, part 1 = TERM*sin moment
    for (int i = 0; i < hp.ntrm; i++) {
        const LegTerm &t = kLeg[i];
        if (!term_present(t.l, t.m, isyma)) continue;
        if (t.m == 0 && (t.l % 2) == 1 && F1 == 0.0) continue;  // TERM * F1 = 0
        hp.col_term.push_back(i); hp.col_part.push_back(0); hp.col_m.push_back(t.m); hp.col_l.push_back(t.l);
        if (t.m > 0) {
            hp.col_term.push_back(i); hp.col_part.push_back(1); hp.col_m.push_back(t.m); hp.col_l.push_back(t.l);
        }
    }
    hp.ncol = (int)hp.col_term.size();

    // boundary points: top edge then outer edge (pot/boundary.f:50-79)
    {
        const double zk2 = ZHF(K + 1) * ZHF(K + 1);
        for (int j = 2; j <= J + 1; j++) {
            hp.jk_j.push_back(j - 2); hp.jk_k.push_back(K - 1);
            hp.jk_rbdy.push_back(std::sqrt(zk2 + RHF(j) * RHF(j)));
        }
        const double rj2 = RHF(J + 1) * RHF(J + 1);
        for (int k = 2; k <= K; k++) {
            hp.jk_j.push_back(J - 1); hp.jk_k.push_back(k - 2);
            hp.jk_rbdy.push_back(std::sqrt(rj2 + ZHF(k) * ZHF(k)));
        }
    }
    hp.njk = (int)hp.jk_j.size();
    hp.jk_split.resize(hp.njk);
    hp.jk_bin.assign((size_t)hp.njk * 66, 0.0);
    hp.jk_hout.assign((size_t)hp.njk * 66, 0.0);
    for (int q = 0; q < hp.njk; q++) {
        const double rb = hp.jk_rbdy[q];
        if (g.isym < 0) {
            hp.jk_split[q] = hp.nkeep;   // all mass inside (pot/boundary.f:607-614)
        } else {
            // rings with RSPHER <= RBDY(JK) (pot/boundary.f:561)
            auto it = std::upper_bound(hp.ring_sorted.begin(), hp.ring_sorted.end(), rb,
                                       [&](double v, int ring) { return v < hp.ring_rsph[ring]; });
            hp.jk_split[q] = (int)(it - hp.ring_sorted.begin());
        }
        const int jj = hp.jk_j[q] + 2, kk = hp.jk_k[q] + 2;
        double term[66];
        bdy_terms(term, ZHF(kk) / rb, RHF(jj) / rb, g.maxtrm, isyma, F1, r8);
        for (int i = 0; i < 66; i++) {
            const int l = kLeg[i].l;
            if (l > g.maxtrm) continue;
            const double rin = 1.0 / ipow(rb, l + 1), rout = ipow(rb, l);
            hp.jk_bin[(size_t)q * 66 + i] = term[i] * rin;
            hp.jk_hout[(size_t)q * 66 + i] = g.isym >= 0 ? term[i] * rout : 0.0;
        }
    }

    // sub-chunks of the sorted ring sequence: at most 64 rings, cut at every
    // boundary point's split so a prefix/suffix at a split is a sum of whole
    // sub-chunks
    {
        std::vector<int> cuts;
        for (int s0 = 0; s0 < hp.nkeep; s0 += 64) cuts.push_back(s0);
        cuts.push_back(hp.nkeep);
        for (int q = 0; q < hp.njk; q++) cuts.push_back(hp.jk_split[q]);
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
        hp.sub_start = cuts;   // starts at 0, ends at nkeep
        hp.jk_sub.resize(hp.njk);
        for (int q = 0; q < hp.njk; q++)
            hp.jk_sub[q] = (int)(std::lower_bound(cuts.begin(), cuts.end(), hp.jk_split[q]) - cuts.begin());
        hp.sring.resize((size_t)hp.nkeep * 4);
        for (int s0 = 0; s0 < hp.nkeep; s0++) {
            const int ring = hp.ring_sorted[s0], j = ring % M, k = ring / M;
            const double rsph = hp.ring_rsph[ring];
            hp.sring[(size_t)s0 * 4 + 0] = rsph;
            hp.sring[(size_t)s0 * 4 + 1] = ZHF(k + 2) / rsph;
            hp.sring[(size_t)s0 * 4 + 2] = RHF(j + 2) / rsph;
            hp.sring[(size_t)s0 * 4 + 3] = hp.ring_dv[ring];
        }
        // per sorted ring: TERM(1..NTRM), r^-(2l+1) for l = 0..10, DV
        hp.srow = hp.ntrm + 12;
        hp.sterm.assign((size_t)hp.nkeep * hp.srow, 0.0);
        for (int s0 = 0; s0 < hp.nkeep; s0++) {
            const int ring = hp.ring_sorted[s0];
            double *row = &hp.sterm[(size_t)s0 * hp.srow];
            for (int i = 0; i < hp.ntrm; i++) row[i] = hp.ring_term[(size_t)ring * 66 + i];
            for (int l = 0; l <= 10; l++) row[hp.ntrm + l] = hp.ring_qh[(size_t)ring * 11 + l];
            row[hp.ntrm + 11] = hp.ring_dv[ring];
        }
    }

    // POT3 stencil (pot/pot3.f:158-194)
    {
        const double dthet2 = 1.0 / (hp.dtheta * hp.dtheta);
        std::vector<double> denomr(J + 1), rd2(J + 1), rd3(J + 1), denomz(K + 1), zd2(K + 1);
        rd2[1] = 0.5 / RHF(2);
        rd3[1] = 1.0 / RHF(1);
        for (int j = 2; j <= J; j++) {
            denomr[j] = 1.0 / (RHF(j + 1) - RHF(j - 1));
            rd2[j] = 1.0 / (RHF(j + 1) - RHF(j));
            rd3[j] = 1.0 / RHF(j);
        }
        zd2[1] = 0.5 / ZHF(2);
        for (int k = 2; k <= K; k++) {
            denomz[k] = 1.0 / (ZHF(k + 1) - ZHF(k - 1));
            zd2[k] = 1.0 / (ZHF(k + 1) - ZHF(k));
        }
        hp.am.assign(M, 0.0); hp.cm.assign(M, 0.0); hp.cc.assign(M, 0.0); hp.bm0.assign(M, 0.0);
        hp.an.assign(NZ, 0.0); hp.bn.assign(NZ, 0.0); hp.cn.assign(NZ, 0.0);
        for (int j = 2; j <= J; j++) {
            hp.cm[j - 2] = 2. * (rd2[j] + 0.5 * rd3[j]) * denomr[j];
            hp.am[j - 2] = 2. * (rd2[j - 1] - 0.5 * rd3[j]) * denomr[j];
            hp.cc[j - 2] = rd3[j] * rd3[j] * dthet2;
        }
        for (int k = 2; k <= K; k++) {
            hp.cn[k - 2] = 2. * zd2[k] * denomz[k];
            hp.an[k - 2] = 2. * zd2[k - 1] * denomz[k];
            hp.bn[k - 2] = -hp.cn[k - 2] - hp.an[k - 2];
        }
        hp.cmmax = hp.cm[M - 1];
        hp.cm[M - 1] = 0.0;
        hp.ammin = hp.am[0];
        hp.am[0] = 0.0;
        hp.cnmax = hp.cn[NZ - 1];
        hp.cn[NZ - 1] = 0.0;
        hp.bn[0] = -hp.cn[0];
        hp.an[0] = 0.0;
        hp.xlamm.resize(hp.N + 1);
        for (int m = 0; m <= hp.N; m++) hp.xlamm[m] = std::cos((double)m * hp.dtheta);
        // m-independent part of BM (pot/pot3.f:226-230); row 0 adds the axis term
        for (int j = 0; j < M; j++) hp.bm0[j] = -hp.cm[j] - hp.am[j];
        hp.bm0[0] = -hp.cm[0];
        hp.bm0[M - 1] = -hp.cmmax - hp.am[M - 1];
    }

    // vertical eigenbasis: T_z = V diag(lam) U with T_z(k,k-1) = AN, (k,k) = BN,
    // (k,k+1) = CN.  Symmetrised by D = diag(d), d(k+1)/d(k) = sqrt(CN(k)/AN(k+1)).
    {
        std::vector<double> dsc(NZ), dd(NZ), ee(NZ, 0.0), zz((size_t)NZ * NZ);
        dsc[0] = 1.0;
        for (int k = 0; k + 1 < NZ; k++) {
            if (!(hp.cn[k] > 0.0 && hp.an[k + 1] > 0.0)) { err = "vertical operator not symmetrisable"; return CHY_ERR_EIGEN; }
            dsc[k + 1] = dsc[k] * std::sqrt(hp.cn[k] / hp.an[k + 1]);
            ee[k] = std::sqrt(hp.cn[k] * hp.an[k + 1]);
        }
        for (int k = 0; k < NZ; k++) dd[k] = hp.bn[k];
        if (tridiag_eigen(NZ, dd.data(), ee.data(), zz.data()) != 0) { err = "vertical eigen solve did not converge"; return CHY_ERR_EIGEN; }
        // order eigenpairs by eigenvalue (most negative first)
        std::vector<int> ord(NZ);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int a, int b) { return dd[a] < dd[b]; });
        hp.lam.resize(NZ);
        hp.U.assign((size_t)NZ * NZ, 0.0);
        hp.V.assign((size_t)NZ * NZ, 0.0);
        hp.Qt.assign((size_t)NZ * NZ, 0.0);
        hp.dsc = dsc;
        for (int p = 0; p < NZ; p++) {
            const int q = ord[p];
            hp.lam[p] = dd[q];
            for (int k = 0; k < NZ; k++) {
                const double qk = zz[k + (size_t)NZ * q];
                hp.V[(size_t)k * NZ + p] = qk / dsc[k];   // V(k,p)
                hp.U[(size_t)p * NZ + k] = qk * dsc[k];   // U(p,k)
                hp.Qt[(size_t)p * NZ + k] = qk;           // Q(k,p)
            }
        }
    }

    // ZAXPHI abscissae (pot/pot3.f:334-348)
    {
        int np = g.npoint;
        hp.npoint = np;
        int ichk = np % 2, n = np - ichk, num = n / 2;
        for (int j = 2; j <= num + 1; j++) {
            hp.zx[num + (j - 1)] = RHF(j);
            hp.zx[num - (j - 2)] = -RHF(j);
        }
        if (ichk == 1) hp.zx[num + num + 1] = RHF(num + 2);
    }
    return CHY_OK;
}

}  // namespace chy

/*
 * pot3_oracle.c -- TEST INFRASTRUCTURE ONLY (checker + CPU baseline).
 *
 * A line-faithful C restatement of CHYMERA's pot3 path:
 *   pot/fft.f       FFT (Singleton 1968 mixed radix), REALTR
 *   pot/blktri.f    BLKTRI, BLKTR1, PRDCT, COMPB, TQLRAT (FISHPACK)
 *   pot/pot3.f      POT3, ZAXPHI
 *   pot/boundary.f  SETBDY, BDYGEN
 * Loop orders, recurrences and GOTO control flow follow the Fortran; each
 * routine cites the lines it restates.  Build with -O2 -ffp-contract=off and
 * no -march (x86-64 SSE2, no FMA), which is the arithmetic gfortran -O3 uses.
 *
 * Parity status: UNPINNED (no Fortran compiler, no reference fixtures exist).
 *
 * Documented deviations from the reference binary:
 *  - With nthreads > 1 the BDYGEN thread partials are merged in thread-id
 *    order; the reference merges in CRITICAL-section arrival order
 *    (pot/boundary.f:636-645), which is not reproducible run to run.
 *  - BDYTRM is zeroed for every JK on every call (the reference zeroes only
 *    JK=1 when ISYM<0, pot/boundary.f:325-339, leaving stale values that
 *    never reach PHI).
 *  - REAL**INTEGER uses square-and-multiply (the libgcc __powidf2 order that
 *    an unoptimised gfortran build of boundary.f calls, bin/Makefile:114-116).
 *  - Unit-3 printing (IPRINT=1) is not performed; PHAC is kept for readers.
 */
#include "pot3_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* pi/4: the single-precision value gfortran folds ATAN(1.0) to in the gcc
 * build, and the double value of ATAN(1.0D0) in the -r8 builds. */
static const float  ATAN1_F32 = 0x1.921fb6p-1f;
static const double ATAN1_F64 = 0x1.921fb54442d18p-1;

/* Fortran REAL**INTEGER (square-and-multiply, negative exponents by 1/y). */
static double ipow(double x, int m)
{
    unsigned int n = m < 0 ? -(unsigned int)m : (unsigned int)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

/* ------------------------------------------------------------------------ */
/* REALTR  pot/fft.f:2-70                                                     */
/* ------------------------------------------------------------------------ */
void ora_realtr(double *a0, double *b0, int n, int isn, int r8)
{
    double *A = a0 - 1, *B = b0 - 1;
    int inc, nk, nh, j, k;
    double sd, cd, sn, cn, aa, ab, ba, bb, re, im, t;

    inc = abs(isn);
    nk = n * inc + 2;
    nh = nk / 2;
    /* SD=2.0*ATAN(1.0)/FLOAT(N) (fft.f:38): REAL(4) in the gcc build */
    if (r8) sd = 2.0 * ATAN1_F64 / (double)n;
    else    sd = (double)(2.0f * ATAN1_F32 / (float)n);
    t = sin(sd);
    cd = 2.0 * (t * t);
    sd = sin(sd + sd);
    sn = 0.0;
    if (isn < 0) goto L30;
    cn = 1.0;
    A[nk - 1] = A[1];
    B[nk - 1] = B[1];
L10:
    for (j = 1; j <= nh; j += inc) {
        k = nk - j;
        aa = A[j] + A[k];
        ab = A[j] - A[k];
        ba = B[j] + B[k];
        bb = B[j] - B[k];
        re = cn * ba + sn * ab;
        im = sn * ba - cn * ab;
        B[k] = im - bb;
        B[j] = im + bb;
        A[k] = aa - re;
        A[j] = aa + re;
        aa = cn - (cd * cn + sd * sn);
        sn = (sd * cn - cd * sn) + sn;
        cn = 0.5 / (aa * aa + sn * sn) + 0.5;
        sn = cn * sn;
        cn = cn * aa;
    }
    return;
L30:
    cn = -1.0;
    sd = -sd;
    goto L10;
}

/* ------------------------------------------------------------------------ */
/* FFT  pot/fft.f:73-629 (Singleton 1968)                                     */
/* ------------------------------------------------------------------------ */
void ora_fft(double *a0, double *b0, int ntot, int n, int nspan, int isn, int r8)
{
    double *A = a0 - 1, *B = b0 - 1;
    int nfac[12];
    int np[210];
    double at[24], ck[24], bt[24], sk[24];
    int maxf, maxp, inc, nt, ks, kspan, nn, jc, i, jf, m, k, j, jj, kt, kk, k1, k2, k3 = 0, k4, kspnn = 0;
    double rad, s72, c72, s120, radf, sd, cd, ak, bk, c1, s1, c2 = 0, s2 = 0, c3 = 0, s3 = 0;
    double akp, akm, ajp, ajm, bkp, bkm, bjp, bjm, aa, bb, aj, bj, t;
    /* EQUIVALENCE (I,II): ii is i */
#define II i

    maxf = 23;
    maxp = 209;
    if (n < 2) return;
    inc = isn;
    /* RAD=8.0*ATAN(1.0), S120=SQRT(0.75) (fft.f:129,133): REAL(4) in the gcc build */
    if (r8) { rad = 8.0 * ATAN1_F64; s120 = sqrt(0.75); }
    else    { rad = (double)(8.0f * ATAN1_F32); s120 = (double)sqrtf(0.75f); }
    s72 = rad / 5.0;
    c72 = cos(s72);
    s72 = sin(s72);
    if (isn >= 0) goto L10;
    s72 = -s72;
    s120 = -s120;
    rad = -rad;
    inc = -inc;
L10:
    nt = inc * ntot;
    ks = inc * nspan;
    kspan = ks;
    nn = nt - inc;
    jc = ks / n;
    radf = rad * (double)jc * 0.5;
    i = 0;
    jf = 0;
    /* determine the factors of n */
    m = 0;
    k = n;
    goto L20;
L15:
    m = m + 1;
    nfac[m] = 4;
    k = k / 16;
L20:
    if (k - (k / 16) * 16 == 0) goto L15;
    j = 3;
    jj = 9;
    goto L30;
L25:
    m = m + 1;
    nfac[m] = j;
    k = k / jj;
L30:
    if (k % jj == 0) goto L25;
    j = j + 2;
    jj = j * j;
    if (jj <= k) goto L30;
    if (k > 4) goto L40;
    kt = m;
    nfac[m + 1] = k;
    if (k != 1) m = m + 1;
    goto L80;
L40:
    if (k - (k / 4) * 4 != 0) goto L50;
    m = m + 1;
    nfac[m] = 2;
    k = k / 4;
L50:
    kt = m;
    j = 2;
L60:
    if (k % j != 0) goto L70;
    m = m + 1;
    nfac[m] = j;
    k = k / j;
L70:
    j = ((j + 1) / 2) * 2 + 1;
    if (j <= k) goto L60;
L80:
    if (kt == 0) goto L100;
    j = kt;
L90:
    m = m + 1;
    nfac[m] = nfac[j];
    j = j - 1;
    if (j != 0) goto L90;
    /* compute fourier transform */
L100:
    sd = radf / (double)kspan;
    t = sin(sd);
    cd = 2.0 * (t * t);
    sd = sin(sd + sd);
    kk = 1;
    i = i + 1;
    if (nfac[i] != 2) goto L400;
    /* factor of 2 (including rotation factor) */
    kspan = kspan / 2;
    k1 = kspan + 2;
L210:
    k2 = kk + kspan;
    ak = A[k2];
    bk = B[k2];
    A[k2] = A[kk] - ak;
    B[k2] = B[kk] - bk;
    A[kk] = A[kk] + ak;
    B[kk] = B[kk] + bk;
    kk = k2 + kspan;
    if (kk <= nn) goto L210;
    kk = kk - nn;
    if (kk <= jc) goto L210;
    if (kk > kspan) goto L800;
L220:
    c1 = 1.0 - cd;
    s1 = sd;
L230:
    k2 = kk + kspan;
    ak = A[kk] - A[k2];
    bk = B[kk] - B[k2];
    A[kk] = A[kk] + A[k2];
    B[kk] = B[kk] + B[k2];
    A[k2] = c1 * ak - s1 * bk;
    B[k2] = s1 * ak + c1 * bk;
    kk = k2 + kspan;
    if (kk < nt) goto L230;
    k2 = kk - nt;
    c1 = -c1;
    kk = k1 - k2;
    if (kk > k2) goto L230;
    ak = c1 - (cd * c1 + sd * s1);
    s1 = (sd * c1 - cd * s1) + s1;
    c1 = 0.5 / (ak * ak + s1 * s1) + 0.5;
    s1 = c1 * s1;
    c1 = c1 * ak;
    kk = kk + jc;
    if (kk < k2) goto L230;
    k1 = k1 + inc + inc;
    kk = (k1 - kspan) / 2 + jc;
    if (kk <= jc + jc) goto L220;
    goto L100;
    /* factor of 3 */
L320:
    k1 = kk + kspan;
    k2 = k1 + kspan;
    ak = A[kk];
    bk = B[kk];
    aj = A[k1] + A[k2];
    bj = B[k1] + B[k2];
    A[kk] = ak + aj;
    B[kk] = bk + bj;
    ak = -0.5 * aj + ak;
    bk = -0.5 * bj + bk;
    aj = (A[k1] - A[k2]) * s120;
    bj = (B[k1] - B[k2]) * s120;
    A[k1] = ak - bj;
    B[k1] = bk + aj;
    A[k2] = ak + bj;
    B[k2] = bk - aj;
    kk = k2 + kspan;
    if (kk < nn) goto L320;
    kk = kk - nn;
    if (kk <= kspan) goto L320;
    goto L700;
    /* factor of 4 */
L400:
    if (nfac[i] != 4) goto L600;
    kspnn = kspan;
    kspan = kspan / 4;
L410:
    c1 = 1.0;
    s1 = 0;
L420:
    k1 = kk + kspan;
    k2 = k1 + kspan;
    k3 = k2 + kspan;
    akp = A[kk] + A[k2];
    akm = A[kk] - A[k2];
    ajp = A[k1] + A[k3];
    ajm = A[k1] - A[k3];
    A[kk] = akp + ajp;
    ajp = akp - ajp;
    bkp = B[kk] + B[k2];
    bkm = B[kk] - B[k2];
    bjp = B[k1] + B[k3];
    bjm = B[k1] - B[k3];
    B[kk] = bkp + bjp;
    bjp = bkp - bjp;
    if (isn < 0) goto L450;
    akp = akm - bjm;
    akm = akm + bjm;
    bkp = bkm + ajm;
    bkm = bkm - ajm;
    if (s1 == 0.0) goto L460;
L430:
    A[k1] = akp * c1 - bkp * s1;
    B[k1] = akp * s1 + bkp * c1;
    A[k2] = ajp * c2 - bjp * s2;
    B[k2] = ajp * s2 + bjp * c2;
    A[k3] = akm * c3 - bkm * s3;
    B[k3] = akm * s3 + bkm * c3;
    kk = k3 + kspan;
    if (kk <= nt) goto L420;
L440:
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
    if (kk <= kspan) goto L420;
    kk = kk - kspan + inc;
    if (kk <= jc) goto L410;
    if (kspan == jc) goto L800;
    goto L100;
L450:
    akp = akm + bjm;
    akm = akm - bjm;
    bkp = bkm - ajm;
    bkm = bkm + ajm;
    if (s1 != 0.0) goto L430;
L460:
    A[k1] = akp;
    B[k1] = bkp;
    A[k2] = ajp;
    B[k2] = bjp;
    A[k3] = akm;
    B[k3] = bkm;
    kk = k3 + kspan;
    if (kk <= nt) goto L420;
    goto L440;
    /* factor of 5 */
L510:
    c2 = c72 * c72 - s72 * s72;
    s2 = 2.0 * c72 * s72;
L520:
    k1 = kk + kspan;
    k2 = k1 + kspan;
    k3 = k2 + kspan;
    k4 = k3 + kspan;
    akp = A[k1] + A[k4];
    akm = A[k1] - A[k4];
    bkp = B[k1] + B[k4];
    bkm = B[k1] - B[k4];
    ajp = A[k2] + A[k3];
    ajm = A[k2] - A[k3];
    bjp = B[k2] + B[k3];
    bjm = B[k2] - B[k3];
    aa = A[kk];
    bb = B[kk];
    A[kk] = aa + akp + ajp;
    B[kk] = bb + bkp + bjp;
    ak = akp * c72 + ajp * c2 + aa;
    bk = bkp * c72 + bjp * c2 + bb;
    aj = akm * s72 + ajm * s2;
    bj = bkm * s72 + bjm * s2;
    A[k1] = ak - bj;
    A[k4] = ak + bj;
    B[k1] = bk + aj;
    B[k4] = bk - aj;
    ak = akp * c2 + ajp * c72 + aa;
    bk = bkp * c2 + bjp * c72 + bb;
    aj = akm * s2 - ajm * s72;
    bj = bkm * s2 - bjm * s72;
    A[k2] = ak - bj;
    A[k3] = ak + bj;
    B[k2] = bk + aj;
    B[k3] = bk - aj;
    kk = k4 + kspan;
    if (kk < nn) goto L520;
    kk = kk - nn;
    if (kk <= kspan) goto L520;
    goto L700;
    /* odd factors */
L600:
    k = nfac[i];
    kspnn = kspan;
    kspan = kspan / k;
    if (k == 3) goto L320;
    if (k == 5) goto L510;
    if (k == jf) goto L640;
    jf = k;
    s1 = rad / (double)k;
    c1 = cos(s1);
    s1 = sin(s1);
    if (jf > maxf) goto L998;
    ck[jf] = 1.0;
    sk[jf] = 0.0;
    j = 1;
L630:
    ck[j] = ck[k] * c1 + sk[k] * s1;
    sk[j] = ck[k] * s1 - sk[k] * c1;
    k = k - 1;
    ck[k] = ck[j];
    sk[k] = -sk[j];
    j = j + 1;
    if (j < k) goto L630;
L640:
    k1 = kk;
    k2 = kk + kspnn;
    aa = A[kk];
    bb = B[kk];
    ak = aa;
    bk = bb;
    j = 1;
    k1 = k1 + kspan;
L650:
    k2 = k2 - kspan;
    j = j + 1;
    at[j] = A[k1] + A[k2];
    ak = at[j] + ak;
    bt[j] = B[k1] + B[k2];
    bk = bt[j] + bk;
    j = j + 1;
    at[j] = A[k1] - A[k2];
    bt[j] = B[k1] - B[k2];
    k1 = k1 + kspan;
    if (k1 < k2) goto L650;
    A[kk] = ak;
    B[kk] = bk;
    k1 = kk;
    k2 = kk + kspnn;
    j = 1;
L660:
    k1 = k1 + kspan;
    k2 = k2 - kspan;
    jj = j;
    ak = aa;
    bk = bb;
    aj = 0.0;
    bj = 0.0;
    k = 1;
L670:
    k = k + 1;
    ak = at[k] * ck[jj] + ak;
    bk = bt[k] * ck[jj] + bk;
    k = k + 1;
    aj = at[k] * sk[jj] + aj;
    bj = bt[k] * sk[jj] + bj;
    jj = jj + j;
    if (jj > jf) jj = jj - jf;
    if (k < jf) goto L670;
    k = jf - j;
    A[k1] = ak - bj;
    B[k1] = bk + aj;
    A[k2] = ak + bj;
    B[k2] = bk - aj;
    j = j + 1;
    if (j < k) goto L660;
    kk = kk + kspnn;
    if (kk <= nn) goto L640;
    kk = kk - nn;
    if (kk <= kspan) goto L640;
    /* multiply by rotation factor (except for factors of 2 and 4) */
L700:
    if (i == m) goto L800;
    kk = jc + 1;
L710:
    c2 = 1.0 - cd;
    s1 = sd;
L720:
    c1 = c2;
    s2 = s1;
    kk = kk + kspan;
L730:
    ak = A[kk];
    A[kk] = c2 * ak - s2 * B[kk];
    B[kk] = s2 * ak + c2 * B[kk];
    kk = kk + kspnn;
    if (kk <= nt) goto L730;
    ak = s1 * s2;
    s2 = s1 * c2 + c1 * s2;
    c2 = c1 * c2 - ak;
    kk = kk - nt + kspan;
    if (kk <= kspnn) goto L730;
    c2 = c1 - (cd * c1 + sd * s1);
    s1 = s1 + (sd * c1 - cd * s1);
    c1 = 0.5 / (c2 * c2 + s1 * s1) + 0.5;
    s1 = c1 * s1;
    c2 = c1 * c2;
    kk = kk - kspnn + jc;
    if (kk <= kspan) goto L720;
    kk = kk - kspan + jc + inc;
    if (kk <= jc + jc) goto L710;
    goto L100;
    /* permute the results to normal order -- square factors */
L800:
    np[1] = ks;
    if (kt == 0) goto L890;
    k = kt + kt + 1;
    if (m < k) k = k - 1;
    j = 1;
    np[k + 1] = jc;
L810:
    np[j + 1] = np[j] / nfac[j];
    np[k] = np[k + 1] * nfac[j];
    j = j + 1;
    k = k - 1;
    if (j < k) goto L810;
    k3 = np[k + 1];
    kspan = np[2];
    kk = jc + 1;
    k2 = kspan + 1;
    j = 1;
    if (n != ntot) goto L850;
    /* single-variate transform */
L820:
    ak = A[kk];
    A[kk] = A[k2];
    A[k2] = ak;
    bk = B[kk];
    B[kk] = B[k2];
    B[k2] = bk;
    kk = kk + inc;
    k2 = kspan + k2;
    if (k2 < ks) goto L820;
L830:
    k2 = k2 - np[j];
    j = j + 1;
    k2 = np[j + 1] + k2;
    if (k2 > np[j]) goto L830;
    j = 1;
L840:
    if (kk < k2) goto L820;
    kk = kk + inc;
    k2 = kspan + k2;
    if (k2 < ks) goto L840;
    if (kk < ks) goto L830;
    jc = k3;
    goto L890;
    /* multivariate transform */
L850:
    k = kk + jc;
L860:
    ak = A[kk];
    A[kk] = A[k2];
    A[k2] = ak;
    bk = B[kk];
    B[kk] = B[k2];
    B[k2] = bk;
    kk = kk + inc;
    k2 = k2 + inc;
    if (kk < k) goto L860;
    kk = kk + ks - jc;
    k2 = k2 + ks - jc;
    if (kk < nt) goto L850;
    k2 = k2 - nt + kspan;
    kk = kk - nt + jc;
    if (k2 < ks) goto L850;
L870:
    k2 = k2 - np[j];
    j = j + 1;
    k2 = np[j + 1] + k2;
    if (k2 > np[j]) goto L870;
    j = 1;
L880:
    if (kk < k2) goto L850;
    kk = kk + jc;
    k2 = kspan + k2;
    if (k2 < ks) goto L880;
    if (kk < ks) goto L870;
    jc = k3;
L890:
    if (2 * kt + 1 >= m) return;
    kspnn = np[kt + 1];
    /* permutation for square-free factors */
    j = m - kt;
    nfac[j + 1] = 1;
L900:
    nfac[j] = nfac[j] * nfac[j + 1];
    j = j - 1;
    if (j != kt) goto L900;
    kt = kt + 1;
    nn = nfac[kt] - 1;
    if (nn > maxp) goto L998;
    jj = 0;
    j = 0;
    goto L906;
L902:
    jj = jj - k2;
    k2 = kk;
    k = k + 1;
    kk = nfac[k];
L904:
    jj = kk + jj;
    if (jj >= k2) goto L902;
    np[j] = jj;
L906:
    k2 = nfac[kt];
    k = kt + 1;
    kk = nfac[k];
    j = j + 1;
    if (j <= nn) goto L904;
    /* permutation cycles of length greater than 1 */
    j = 0;
    goto L914;
L910:
    k = kk;
    kk = np[k];
    np[k] = -kk;
    if (kk != j) goto L910;
    k3 = kk;
L914:
    j = j + 1;
    kk = np[j];
    if (kk < 0) goto L914;
    if (kk != j) goto L910;
    np[j] = -j;
    if (j != nn) goto L914;
    maxf = inc * maxf;
    goto L950;
L924:
    j = j - 1;
    if (np[j] < 0) goto L924;
    jj = jc;
L926:
    kspan = jj;
    if (jj > maxf) kspan = maxf;
    jj = jj - kspan;
    k = np[j];
    kk = jc * k + II + jj;
    k1 = kk + kspan;
    k2 = 0;
L928:
    k2 = k2 + 1;
    at[k2] = A[k1];
    bt[k2] = B[k1];
    k1 = k1 - inc;
    if (k1 != kk) goto L928;
L932:
    k1 = kk + kspan;
    k2 = k1 - jc * (k + np[k]);
    k = -np[k];
L936:
    A[k1] = A[k2];
    B[k1] = B[k2];
    k1 = k1 - inc;
    k2 = k2 - inc;
    if (k1 != kk) goto L936;
    kk = k2;
    if (k != j) goto L932;
    k1 = kk + kspan;
    k2 = 0;
L940:
    k2 = k2 + 1;
    A[k1] = at[k2];
    B[k1] = bt[k2];
    k1 = k1 - inc;
    if (k1 != kk) goto L940;
    if (jj != 0) goto L926;
    if (j != 1) goto L924;
L950:
    j = k3 + 1;
    nt = nt - kspnn;
    II = nt - inc + 1;
    if (nt >= 0) goto L924;
    return;
L998:
    /* ISN=0; STOP (fft.f:625-628): array storage exceeded */
    abort();
#undef II
}

/* ------------------------------------------------------------------------ */
/* BLKTRI family  pot/blktri.f                                                */
/* ------------------------------------------------------------------------ */
typedef struct {
    /* COMMON /CBLKT/ NPP,Kx,EPSLON,CNV,Lx,NCMPLX,IK,IZ,DUM(1) (blktri.f:8) */
    int npp, kx;
    double epslon, cnv;
    int lx, ncmplx, ik, iz;
    double dum[1];
    /* COMMON /BLOKJ1/ IWCN,IW1,IW2,IW3,IWD,IWW,IWU (blktri.f:9) */
    int iwcn, iw1, iw2, iw3, iwd, iww, iwu;
} cblkt_t;

int ora_blktri_state_size(void) { return (int)sizeof(cblkt_t); }

/* PRDCT  pot/blktri.f:177-260.  All array arguments are 1-based views. */
static void prdct(int nd, const double *BD, int nm1, const double *BM1, int nm2,
                  const double *BM2, int na, const double *AA, const double *X, double *Y,
                  int m, const double *A, const double *B, const double *C, double *D,
                  double *W, double *U, int is)
{
    int j, k, mm, id, ibr, m1, m2, ia;
    double rt, den;
    (void)U;
    if (nd <= 0) goto L10;
    if (is <= 0) goto L20;
L10:
    for (j = 1; j <= m; j++) {
        W[j] = X[j];
        Y[j] = X[j];
    }
    goto L30;
L20:
    for (j = 1; j <= m; j++) {
        W[j] = -X[j];
        Y[j] = W[j];
    }
L30:
    mm = m - 1;
    id = nd;
    ibr = 0;
    m1 = nm1;
    m2 = nm2;
    ia = na;
L35:
    if (ia > 0) {
        rt = AA[ia];
        ia = ia - 1;
        for (j = 1; j <= m; j++) Y[j] = rt * W[j];
    }
    if (id <= 0) goto L150;
    rt = BD[id];
    id = id - 1;
    if (id == 0) ibr = 1;
    D[m] = A[m] / (B[m] - rt);
    W[m] = Y[m] / (B[m] - rt);
    for (j = 2; j <= mm; j++) {
        k = m - j;
        den = B[k + 1] - rt - C[k + 1] * D[k + 2];
        D[k + 1] = A[k + 1] / den;
        W[k + 1] = (Y[k + 1] - C[k + 1] * W[k + 2]) / den;
    }
    den = B[1] - rt - C[1] * D[2];
    if (den == 0) {
        W[1] = 1.;
    } else {
        W[1] = (Y[1] - C[1] * W[2]) / den;
    }
    for (j = 2; j <= m; j++) W[j] = W[j] - D[j] * W[j - 1];
    if (na <= 0) goto L90;
    goto L35;
L80:
    for (j = 1; j <= m; j++) Y[j] = W[j];
    ibr = 1;
    goto L35;
L90:
    if (m1 > 0) goto L100;
    if (m2 <= 0) goto L80;
    goto L125;
L100:
    if (m2 <= 0) goto L110;
    if (fabs(BM1[m1]) <= fabs(BM2[m2])) goto L125;
L110:
    if (ibr > 0) goto L120;
    if (fabs(BM1[m1] - BD[id]) < fabs(BM1[m1] - rt)) goto L80;
L120:
    rt = rt - BM1[m1];
    m1 = m1 - 1;
    goto L140;
L125:
    if (ibr > 0) goto L135;
    if (fabs(BM2[m2] - BD[id]) < fabs(BM2[m2] - rt)) goto L80;
L135:
    rt = rt - BM2[m2];
    m2 = m2 - 1;
L140:
    for (j = 1; j <= m; j++) Y[j] = Y[j] + rt * W[j];
    goto L35;
L150:
    return;
}

/* TQLRAT  pot/blktri.f:348-423 (D, E2 1-based; MACHEP = /CBLKT/ EPSLON) */
static void tqlrat(cblkt_t *st, int n, double *D, double *E2, int *ierr)
{
    int i, j, l, m, l1, ii, mml;
    double b, c = 0.0, f, g, h, p, r, s, absp, machep = st->epslon;

    *ierr = 0;
    if (n == 1) goto L70;
    for (i = 2; i <= n; i++) E2[i - 1] = E2[i] * E2[i];
    f = 0.0;
    b = 0.0;
    E2[n] = 0.0;
    for (l = 1; l <= n; l++) {
        j = 0;
        h = machep * (fabs(D[l]) + sqrt(E2[l]));
        if (b > h) goto L10;
        b = h;
        c = b * b;
    L10:
        for (m = l; m <= n; m++) {
            if (E2[m] <= c) goto L20;
        }
    L20:
        if (m == l) goto L40;
    L25:
        if (j == 30) goto L65;
        j = j + 1;
        l1 = l + 1;
        s = sqrt(E2[l]);
        g = D[l];
        p = (D[l1] - g) / (2.0 * s);
        r = sqrt(p * p + 1.0);
        D[l] = s / (p + copysign(r, p));
        h = g - D[l];
        for (i = l1; i <= n; i++) D[i] = D[i] - h;
        f = f + h;
        g = D[m];
        if (g == 0.0) g = b;
        h = g;
        s = 0.0;
        mml = m - l;
        for (ii = 1; ii <= mml; ii++) {
            i = m - ii;
            p = g * h;
            r = p + E2[i];
            E2[i + 1] = s * r;
            s = E2[i] / r;
            D[i + 1] = h + s * (h + D[i]);
            g = D[i] - E2[i] / g;
            if (g == 0.0) g = b;
            h = g * p / r;
        }
        E2[l] = s * g;
        D[l] = h;
        if (h == 0.0) goto L40;
        if (fabs(E2[l]) <= fabs(c / h)) goto L40;
        E2[l] = h * E2[l];
        if (E2[l] != 0.0) goto L25;
    L40:
        p = D[l] + f;
        if (l == 1) goto L50;
        absp = fabs(p);
        for (ii = 2; ii <= l; ii++) {
            i = l + 2 - ii;
            if (absp >= fabs(D[i - 1])) goto L55;
            D[i] = D[i - 1];
        }
    L50:
        i = 1;
    L55:
        D[i] = p;
    }
    goto L70;
L65:
    *ierr = l;
L70:
    return;
}

/* COMPB  pot/blktri.f:264-344 (all arrays 1-based) */
static void compb(cblkt_t *st, int n, int *ierror, const double *AN, const double *BN,
                  const double *CN, double *B, double *AH, double *BH)
{
    int j, if_, lh, lh1, i1, nn, ifl, i, ls, i1m, jfl;
    double dif, difh, bnorm, arg, chld;
    volatile double vdif;

    st->epslon = 1.;
L5:
    st->epslon = st->epslon / 10.;
    dif = 1. + st->epslon;
    vdif = dif;
    difh = vdif;
    if (difh > 1.) goto L5;
    st->epslon = 100. * st->epslon;
    bnorm = fabs(BN[1]);
    for (j = 2; j <= n; j++) bnorm = fmax(bnorm, fabs(BN[j]));
    st->cnv = st->epslon * bnorm;
    for (j = 1; j <= n; j++) {
        if (j != 1) goto L25;
        if (st->npp != 0) continue;
    L25:
        arg = AN[j] * CN[j];
        if (arg < 0) goto L140;
        chld = sqrt(arg);
        if (CN[j] < 0) goto L40;
        B[j] = chld;
        continue;
    L40:
        B[j] = -chld;
    }
    if_ = 1 << st->kx;
    lh = if_;
    lh1 = if_ + 1;
    i1 = 1;
    for (st->lx = 1; st->lx <= st->kx; st->lx++) {
        i1 = i1 + i1;
        nn = i1 + i1 - 1;
        ifl = if_ - i1 + 1;
        for (i = 1; i <= ifl; i += i1) {
            if (i < ifl) goto L75;
            if (st->npp == 0) goto L60;
            lh = lh + nn;
            continue;
        L60:
            ls = 0;
            for (j = i; j <= if_; j++) {
                ls = ls + 1;
                BH[ls] = BN[j];
                AH[ls] = B[j];
            }
            i1m = i1 - 1;
            for (j = 1; j <= i1m; j++) {
                ls = ls + 1;
                BH[ls] = BN[j];
                AH[ls] = B[j];
            }
            goto L85;
        L75:
            ls = 0;
            jfl = i + nn - 1;
            for (j = i; j <= jfl; j++) {
                ls = ls + 1;
                BH[ls] = BN[j];
                AH[ls] = B[j];
            }
        L85:
            tqlrat(st, nn, BH, AH, ierror);
            if (*ierror != 0) goto L140;
            for (j = 1; j <= nn; j++) {
                lh = lh + 1;
                B[lh] = -BH[j];
            }
        }
        lh1 = lh + 1;
    }
    (void)lh1;
    for (j = 1; j <= n; j++) B[j] = -BN[j];
    return;
L140:
    *ierror = 4;
}

/* BLKTR1  pot/blktri.f:60-173 (all arrays 1-based; Y(IDIMY,*)) */
static void blktr1(cblkt_t *st, int n, const double *AN, const double *BN, const double *CN,
                   int m, const double *AM, const double *BM, const double *CM, int idimy,
                   double *Y, const double *B, double *W1, double *W2, double *W3, double *WD,
                   double *WW, double *WU)
{
    int nh, ih1, kdo, ir, isgn, msgn, ih2, lm, lz, iim, iiz, jm1, i1, if_, jj, i, i6, i7, i9;
    int j2, j4, jp1, jp2, jp3, ll, i5, jz, j;
    const double *DUM = st->dum - 1;
#define YC(col) (Y + (size_t)((col) - 1) * idimy)

    nh = 1 << st->kx;
    ih1 = nh + nh;
    if (st->npp == 0) kdo = st->kx;
    else kdo = st->kx - 1;
    for (st->lx = 1; st->lx <= kdo; st->lx++) {
        ir = st->lx - 1;
        st->iz = 1 << ir;
        isgn = (ir % 2 == 0) ? 1 : -1;
        msgn = -isgn;
        ih2 = 1 << (st->kx - ir + 1);
        lm = (ir - 2) * ih1 + ih2 + ih2 + 1;
        lz = (ir - 1) * ih1 + ih2 + 1;
        iim = st->iz - 1;
        iiz = iim + iim + 1;
        jm1 = iim + iim + lm;
        i1 = st->iz + st->iz;
        prdct(iiz, B + lz - 1, iim, B + lm - 1, iim, B + jm1 - 1, 0, DUM, YC(st->iz), W3, m,
              AM, BM, CM, WD, WW, WU, isgn);
        if_ = 1 << (st->kx - ir - 1);
        for (jj = 1; jj <= if_; jj++) {
            i = jj * i1;
            i6 = i;
            i7 = i - st->iz;
            i9 = i + st->iz;
            j2 = jj + jj;
            j4 = j2 + j2;
            jm1 = (j4 - 2) * iim + lm;
            jp1 = j4 * iim + lm;
            jp2 = j2 * iiz + lz;
            jp3 = (j4 + 2) * iim + lm;
            if (jj < if_) goto L25;
            if (st->npp != 0) continue;
            jp1 = lm;
            jp2 = lz;
            jp3 = iim + iim + lm;
            i6 = 0;
            i9 = st->iz;
        L25:
            prdct(iim, B + jm1 - 1, 0, DUM, 0, DUM, st->iz, AN + i7, W3, W1, m, AM, BM, CM,
                  WD, WW, WU, msgn);
            prdct(iiz, B + jp2 - 1, iim, B + jp1 - 1, iim, B + jp3 - 1, 0, DUM, YC(i9), W3,
                  m, AM, BM, CM, WD, WW, WU, isgn);
            prdct(iim, B + jp1 - 1, 0, DUM, 0, DUM, st->iz, CN + i6, W3, W2, m, AM, BM, CM,
                  WD, WW, WU, msgn);
            for (j = 1; j <= m; j++) YC(i)[j] = W1[j] + W2[j] - YC(i)[j];
        }
    }

    for (ll = 1; ll <= st->kx; ll++) {
        st->lx = st->kx - ll + 1;
        ir = st->lx - 1;
        isgn = (ir % 2 == 0) ? 1 : -1;
        msgn = -isgn;
        st->iz = 1 << ir;
        iim = st->iz - 1;
        iiz = iim + iim + 1;
        ih2 = 1 << (st->kx - ir + 1);
        lm = (ir - 2) * ih1 + ih2 + ih2 + 1;
        lz = (ir - 1) * ih1 + ih2 + 1;
        if_ = (1 << (st->kx - ir)) - 1;
        for (jj = 1; jj <= if_; jj += 2) {
            i = jj * st->iz;
            i5 = i - st->iz;
            i6 = i + st->iz;
            i7 = i5;
            j2 = jj + jj;
            jm1 = (j2 - 2) * iim + lm;
            jz = (jj - 1) * iiz + lz;
            jp1 = j2 * iim + lm;
            if (jj > 1) goto L85;
            if (st->npp != 0) goto L75;
            i7 = n;
            goto L85;
        L75:
            for (j = 1; j <= m; j++) W1[j] = 0.;
            goto L90;
        L85:
            prdct(iim, B + jm1 - 1, 0, DUM, 0, DUM, st->iz, AN + i5, YC(i7), W1, m, AM, BM,
                  CM, WD, WW, WU, msgn);
        L90:
            if (jj < if_ || st->npp == 0) goto L110;
            for (j = 1; j <= m; j++) W2[j] = 0.;
            goto L115;
        L110:
            prdct(iim, B + jp1 - 1, 0, DUM, 0, DUM, st->iz, CN + i, YC(i6), W2, m, AM, BM,
                  CM, WD, WW, WU, msgn);
        L115:
            for (j = 1; j <= m; j++) W1[j] = YC(i)[j] - W1[j] - W2[j];
            prdct(iiz, B + jz - 1, iim, B + jm1 - 1, iim, B + jp1 - 1, 0, DUM, W1, YC(i), m,
                  AM, BM, CM, WD, WW, WU, isgn);
        }
    }
#undef YC
}

/* BLKTRI  pot/blktri.f:3-56.  0-based pointers in; converted to 1-based. */
void ora_blktri(void *state, int iflg, int np, int n, const double *an0, const double *bn0,
                const double *cn0, int mp, int m, const double *am0, const double *bm0,
                const double *cm0, int idimy, double *y0, int *ierror, double *w0)
{
    cblkt_t *st = (cblkt_t *)state;
    const double *AN = an0 - 1, *BN = bn0 - 1, *CN = cn0 - 1;
    const double *AM = am0 - 1, *BM = bm0 - 1, *CM = cm0 - 1;
    double *Y = y0 - 1, *W = w0 - 1;
    int nh, nck, i, j, iwah, iwbh;
    (void)mp;

    if (iflg == 0) {
        *ierror = 1;
        if (m < 2) return;
        nh = n;
        st->npp = np;
        if (st->npp != 0) nh = nh + 1;
        st->ik = 2;
        st->kx = 0;
        do {
            st->ik = st->ik + st->ik;
            st->kx = st->kx + 1;
        } while (nh / st->ik > 0);
        *ierror = 2;
        st->iwcn = 2 * (n + 1) * (st->kx - 1) - n + 3;
        st->iw1 = st->iwcn + n;
        iwah = st->iw1;
        iwbh = iwah + n;
        if (st->kx < 2) return;
        nck = (1 << st->kx) - 1;
        if (n != nck) return;
        *ierror = 5;
        if (idimy < m) return;
        *ierror = 0;
        st->iw2 = st->iw1 + m;
        st->iw3 = st->iw2 + m;
        st->iwd = st->iw3 + m;
        st->iww = st->iwd + m;
        st->iwu = st->iww + m;
        W[st->iwcn] = CN[n];
        i = st->iwcn;
        for (j = 2; j <= n; j++) {
            i = i + 1;
            W[i] = CN[j - 1];
        }
        compb(st, n, ierror, AN, BN, W + st->iwcn - 1, W, W + iwah - 1, W + iwbh - 1);
    } else {
        blktr1(st, n, AN, BN, W + st->iwcn - 1, m, AM, BM, CM, idimy, Y,
               W, W + st->iw1 - 1, W + st->iw2 - 1, W + st->iw3 - 1, W + st->iwd - 1,
               W + st->iww - 1, W + st->iwu - 1);
    }
}

int ora_blktri_wsize(int jmax, int kmax)
{
    /* WFW(2*(KMAX3+2)*KWFW+6*JMAX3+2), KWFW = log2(KMAX)-1 (pot/pot3.f:30,
     * radhydro/3dhyd-main.f:175); padded so IWU+M-1 always fits. */
    int kwfw = 0, k = kmax;
    while (k > 1) { k >>= 1; kwfw++; }
    kwfw -= 1;
    int need = 2 * (kmax - 1 + 2) * (kwfw + 1) + 6 * (jmax - 1) + 64;
    int ref = 2 * (kmax - 1 + 2) * kwfw + 6 * (jmax - 1) + 2;
    return need > ref ? need : ref;
}

/* ------------------------------------------------------------------------ */
/* Context (COMMON-block stand-ins)                                          */
/* ------------------------------------------------------------------------ */
struct ora_ctx {
    int jmax, kmax, lmax, r8, nthreads;
    double *phi, *rho, *r, *z, *rhf, *zhf, *coef;
    double rof3n, zof3n, dtheta, pi, grav;
    /* /BDY/ /BDY1/ */
    double *cosm, *sinm, *rbdy, bdychk;
    int *jpos, *kpos, jkmax, jkm1;
    /* /BDYGENSHARED/ */
    double *massin, *massout;
    /* /INSIDE/ */
    double tmass, enew, elost, edif, phichk;
    int klocat;
    double *phac;
};

ora_ctx *ora_new(int jmax, int kmax, int lmax, int r8, int nthreads, int want_coef)
{
    ora_ctx *c = (ora_ctx *)calloc(1, sizeof(ora_ctx));
    size_t nvol = (size_t)(jmax + 2) * (kmax + 2) * lmax;
    c->jmax = jmax; c->kmax = kmax; c->lmax = lmax; c->r8 = r8;
    c->nthreads = nthreads < 1 ? 1 : nthreads;
    c->phi = (double *)calloc(nvol, sizeof(double));
    c->rho = (double *)calloc(nvol, sizeof(double));
    c->r = (double *)calloc(jmax + 2, sizeof(double));
    c->rhf = (double *)calloc(jmax + 2, sizeof(double));
    c->z = (double *)calloc(kmax + 2, sizeof(double));
    c->zhf = (double *)calloc(kmax + 2, sizeof(double));
    if (want_coef)
        c->coef = (double *)calloc((size_t)(jmax + 2) * (kmax + 2) * (lmax / 2) * 2, sizeof(double));
    c->jkm1 = 2 * jmax + kmax - 1;       /* JKM1 (pot/boundary.f:22) */
    c->cosm = (double *)calloc((size_t)lmax * 10, sizeof(double));
    c->sinm = (double *)calloc((size_t)lmax * 10, sizeof(double));
    c->rbdy = (double *)calloc(c->jkm1, sizeof(double));
    c->jpos = (int *)calloc(c->jkm1, sizeof(int));
    c->kpos = (int *)calloc(c->jkm1, sizeof(int));
    c->massin = (double *)calloc((size_t)2 * 66 * c->jkm1, sizeof(double));
    c->massout = (double *)calloc((size_t)2 * 66 * c->jkm1, sizeof(double));
    c->phac = (double *)calloc(kmax + 2, sizeof(double));
    c->pi = 3.1415926535897932;
    c->grav = 1.0;
    c->dtheta = 2.0 * c->pi / (double)lmax;
    return c;
}

void ora_free(ora_ctx *c)
{
    if (!c) return;
    free(c->phi); free(c->rho); free(c->r); free(c->rhf); free(c->z); free(c->zhf);
    free(c->coef); free(c->cosm); free(c->sinm); free(c->rbdy); free(c->jpos); free(c->kpos);
    free(c->massin); free(c->massout); free(c->phac);
    free(c);
}

double *ora_phi(ora_ctx *c) { return c->phi; }
double *ora_rho(ora_ctx *c) { return c->rho; }
double *ora_r(ora_ctx *c) { return c->r; }
double *ora_z(ora_ctx *c) { return c->z; }
double *ora_rhf(ora_ctx *c) { return c->rhf; }
double *ora_zhf(ora_ctx *c) { return c->zhf; }
double *ora_coef(ora_ctx *c) { return c->coef; }
double *ora_massin(ora_ctx *c) { return c->massin; }
double *ora_massout(ora_ctx *c) { return c->massout; }
double *ora_rbdy(ora_ctx *c) { return c->rbdy; }
int ora_jkmax(ora_ctx *c) { return c->jkmax; }
double *ora_phac(ora_ctx *c) { return c->phac; }

void ora_set_scalars(ora_ctx *c, double rof3n, double zof3n, double dtheta, double pi, double grav)
{
    c->rof3n = rof3n; c->zof3n = zof3n; c->dtheta = dtheta; c->pi = pi; c->grav = grav;
}

/* radhydro/io.f:194-203: R(J)=(J-2)*DELR, RHF(J)=R(J)+DELR/2.0, same for Z. */
void ora_make_grid(ora_ctx *c, double delr, double delz)
{
    int j, k;
    for (j = 1; j <= c->jmax + 2; j++) {
        c->r[j - 1] = (double)(j - 2) * delr;
        c->rhf[j - 1] = c->r[j - 1] + delr / 2.0;
    }
    for (k = 1; k <= c->kmax + 2; k++) {
        c->z[k - 1] = (double)(k - 2) * delz;
        c->zhf[k - 1] = c->z[k - 1] + delz / 2.0;
    }
    c->rof3n = delr;
    c->zof3n = delz;
}

void ora_inside(ora_ctx *c, double *out3)
{
    out3[0] = c->tmass;
    out3[1] = c->phichk;
    out3[2] = (double)c->klocat;
}

/* ------------------------------------------------------------------------ */
/* SETBDY  pot/boundary.f:2-82                                                */
/* ------------------------------------------------------------------------ */
void ora_setbdy(ora_ctx *c, int ncall, int isym)
{
    const int lmax = c->lmax, jm1 = c->jmax + 1, km1 = c->kmax + 1;
    int isyma = abs(isym), l, m, jk, i, j, k;
    double psi, zk2, rj2;
    const double *RHF = c->rhf - 1, *ZHF = c->zhf - 1;

    if (ncall == 0) {
        c->bdychk = 1.0;
        for (l = 1; l <= lmax; l++) {
            psi = (double)((float)l - 0.5f) * c->dtheta;
            for (m = 1; m <= 10; m++) {
                c->cosm[(l - 1) + (size_t)lmax * (m - 1)] = cos((double)m * psi);
                c->sinm[(l - 1) + (size_t)lmax * (m - 1)] = sin((double)m * psi);
            }
        }
    }
    for (jk = 0; jk < c->jkm1; jk++) {
        c->rbdy[jk] = 0.0;
        c->jpos[jk] = 0;
        c->kpos[jk] = 0;
    }
    i = 0;
    zk2 = ZHF[km1] * ZHF[km1];
    for (j = 2; j <= jm1; j++) {
        i = i + 1;
        c->rbdy[i - 1] = sqrt(zk2 + RHF[j] * RHF[j]);
        c->jpos[i - 1] = j;
        c->kpos[i - 1] = km1;
    }
    if (isyma == 1 || isyma == 8) {
        zk2 = ZHF[1] * ZHF[1];
        for (j = 2; j <= jm1; j++) {
            i = i + 1;
            c->rbdy[i - 1] = sqrt(zk2 + RHF[j] * RHF[j]);
            c->jpos[i - 1] = j;
            c->kpos[i - 1] = 1;
        }
    }
    rj2 = RHF[jm1] * RHF[jm1];
    for (k = 2; k <= c->kmax; k++) {
        i = i + 1;
        c->rbdy[i - 1] = sqrt(rj2 + ZHF[k] * ZHF[k]);
        c->jpos[i - 1] = jm1;
        c->kpos[i - 1] = k;
    }
    c->jkmax = i;
}

/* ------------------------------------------------------------------------ */
/* BDYGEN  pot/boundary.f:88-908                                              */
/* ------------------------------------------------------------------------ */
/* Statement functions BLM, pot/boundary.f:204-253 */
static inline double B20(double AA) { return 3.0 * AA - 1.0; }
static inline double B30(double AA, double D) { return D * (5.0 * AA - 3.0); }
static inline double B31(double AA, double D) { return (5.0 * AA - 1.0) * D; }
static inline double B40(double AA, double D) { return 35.0 * AA - 30.0 * D + 3.0; }
static inline double B41(double AA, double D, double E) { return D * (7.0 * AA - 3.0) * E; }
static inline double B42(double AA, double D) { return (7.0 * AA - 1.0) * D; }
static inline double B50(double AA, double D, double E) { return E * (63.0 * AA - 70.0 * D + 15.0); }
static inline double B51(double AA, double D, double E) { return (21.0 * AA - 14.0 * D + 1.0) * E; }
static inline double B52(double AA, double D, double E) { return D * (3.0 * AA - 1.0) * E; }
static inline double B53(double AA, double D) { return (9.0 * AA - 1.0) * D; }
static inline double B60(double AA, double D, double E) { return 231.0 * AA - 315.0 * D + 105.0 * E - 5.0; }
static inline double B61(double AA, double D, double E, double F) { return E * (33.0 * AA - 30.0 * D + 5.0) * F; }
static inline double B62(double AA, double D, double E) { return (33.0 * AA - 18.0 * D + 1.0) * E; }
static inline double B63(double AA, double D, double E) { return D * (11.0 * AA - 3.0) * E; }
static inline double B64(double AA, double D) { return (11.0 * AA - 1.0) * D; }
static inline double B70(double AA, double D, double E, double F) { return F * (429.0 * AA - 693.0 * D + 315.0 * E - 35.0); }
static inline double B71(double AA, double D, double E, double F) { return (429.0 * AA - 495.0 * D + 135.0 * E - 5.0) * F; }
static inline double B72(double AA, double D, double E, double F) { return E * (143.0 * AA - 110.0 * D + 15.0) * F; }
static inline double B73(double AA, double D, double E) { return (143.0 * AA - 66.0 * D + 3.0) * E; }
static inline double B74(double AA, double D, double E) { return D * (13.0 * AA - 3.0) * E; }
static inline double B75(double AA, double D) { return (13.0 * AA - 1.0) * D; }
static inline double B80(double AA, double D, double E, double F) { return 6435.0 * AA - 12012.0 * D + 6930.0 * E - 1260.0 * F + 35.0; }
static inline double B81(double AA, double D, double E, double F, double GG) { return F * (715.0 * AA - 1001.0 * D + 385.0 * E - 35.0) * GG; }
static inline double B82(double AA, double D, double E, double F) { return (143.0 * AA - 143.0 * D + 33.0 * E - 1.0) * F; }
static inline double B83(double AA, double D, double E, double F) { return E * (39.0 * AA - 26.0 * D + 3.0) * F; }
static inline double B84(double AA, double D, double E) { return (65.0 * AA - 26.0 * D + 1.0) * E; }
static inline double B85(double AA, double D, double E) { return D * (5.0 * AA - 1.0) * E; }
static inline double B86(double AA, double D) { return (15.0 * AA - 1.0) * D; }
static inline double B90(double AA, double D, double E, double F, double GG) { return GG * (12155.0 * AA - 25740.0 * D + 18018.0 * E - 4620.0 * F + 315.0); }
static inline double B91(double AA, double D, double E, double F, double GG) { return (2431.0 * AA - 4004.0 * D + 2002.0 * E - 308.0 * F + 7.0) * GG; }
static inline double B92(double AA, double D, double E, double F, double GG) { return F * (221.0 * AA - 273.0 * D + 91.0 * E - 7.0) * GG; }
static inline double B93(double AA, double D, double E, double F) { return (221.0 * AA - 195.0 * D + 39.0 * E - 1.0) * F; }
static inline double B94(double AA, double D, double E, double F) { return E * (17.0 * AA - 10.0 * D + 1.0) * F; }
static inline double B95(double AA, double D, double E) { return (85.0 * AA - 30.0 * D + 1.0) * E; }
static inline double B96(double AA, double D, double E) { return D * (17.0 * AA - 3.0) * E; }
static inline double B97(double AA, double D) { return (17.0 * AA - 1.0) * D; }
static inline double B100(double AA, double D, double E, double F, double GG) { return 46189.0 * AA - 109395.0 * D + 90090.0 * E - 30030.0 * F + 3465.0 * GG - 63.0; }
static inline double B101(double AA, double D, double E, double F, double GG, double X) { return GG * (4199.0 * AA - 7956.0 * D + 4914.0 * E - 1092.0 * F + 63.0) * X; }
static inline double B102(double AA, double D, double E, double F, double GG) { return (4199.0 * AA - 6188.0 * D + 2730.0 * E - 364.0 * F + 7.0) * GG; }
static inline double B103(double AA, double D, double E, double F, double GG) { return F * (323.0 * AA - 357.0 * D + 105.0 * E - 7.0) * GG; }
static inline double B104(double AA, double D, double E, double F) { return (323.0 * AA - 255.0 * D + 45.0 * E - 1.0) * F; }
static inline double B105(double AA, double D, double E, double F) { return E * (323.0 * AA - 170.0 * D + 15.0) * F; }
static inline double B106(double AA, double D, double E) { return (323.0 * AA - 102.0 * D + 3.0) * E; }
static inline double B107(double AA, double D, double E) { return D * (19.0 * AA - 3.0) * E; }
static inline double B108(double AA, double D) { return (19.0 * AA - 1.0) * D; }

/* TW5..TW18 (pot/boundary.f:181-185): REAL(4) literals in the gcc build round
 * to exact powers of two; under -r8 they are the decimal doubles. */
typedef struct { double tw5, tw6, tw7, tw8, tw9, tw10, tw11, tw12, tw13, tw14, tw15, tw16, tw17, tw18; } tw_t;
static tw_t make_tw(int r8)
{
    tw_t t;
    if (r8) {
        t.tw5 = 0.03125; t.tw6 = 0.015625; t.tw7 = 7.8125E-3; t.tw8 = 3.90625E-3;
        t.tw9 = 1.953125E-3; t.tw10 = 9.765625E-04; t.tw11 = 4.8828125E-4;
        t.tw12 = 2.44140625E-4; t.tw13 = 1.220703125E-4; t.tw14 = 6.103515625E-5;
        t.tw15 = 3.051757813E-5; t.tw16 = 1.525878907E-5; t.tw17 = 7.629394535E-6;
        t.tw18 = 3.814697266E-6;
    } else {
        t.tw5 = 0.03125f; t.tw6 = 0.015625f; t.tw7 = 7.8125E-3f; t.tw8 = 3.90625E-3f;
        t.tw9 = 1.953125E-3f; t.tw10 = 9.765625E-04f; t.tw11 = 4.8828125E-4f;
        t.tw12 = 2.44140625E-4f; t.tw13 = 1.220703125E-4f; t.tw14 = 6.103515625E-5f;
        t.tw15 = 3.051757813E-5f; t.tw16 = 1.525878907E-5f; t.tw17 = 7.629394535E-6f;
        t.tw18 = 3.814697266E-6f;
    }
    return t;
}

/* Ring terms BLM(theta)*r^l (pot/boundary.f:385-502).  TERM is 1-based(66). */
static void ring_terms(double *TERM, int ntrm, int maxtrm, int isyma, double F1,
                       double C1, double S1, double rspher)
{
    double C2, C4, S2, S3, S4, C6 = 0, C8 = 0, S5 = 0, S6 = 0, S7 = 0, S8 = 0, C10 = 0, S9 = 0, S10 = 0, QH;
    double Q[11];
    int i, l;
    C2 = C1 * C1;
    C4 = C2 * C2;
    S2 = S1 * S1;
    S3 = S1 * S2;
    S4 = S2 * S2;
    if (maxtrm <= 4) goto L602;
    C6 = C2 * C4;
    C8 = C4 * C4;
    S5 = S1 * S4;
    S6 = S2 * S4;
    S7 = S1 * S6;
    S8 = S4 * S4;
    if (maxtrm <= 8) goto L602;
    C10 = C2 * C8;
    S9 = S1 * S8;
    S10 = S2 * S8;
L602:
    for (i = 1; i <= ntrm; i++) TERM[i] = 0.0;
    for (l = 1; l <= maxtrm; l++) Q[l] = ipow(rspher, l);
    TERM[1] = 1.0;
    TERM[2] = C1 * Q[1] * F1;
    TERM[4] = B20(C2) * Q[2];
    TERM[7] = B30(C2, C1) * Q[3] * F1;
    TERM[11] = B40(C4, C2) * Q[4];
    if (isyma >= 8) goto L611;
    TERM[6] = S2 * Q[2];
    TERM[13] = B42(C2, S2) * Q[4];
    TERM[15] = S4 * Q[4];
    if (isyma == 3) goto L611;
    TERM[3] = S1 * Q[1];
    TERM[8] = B31(C2, S1) * Q[3];
    TERM[10] = S3 * Q[3];
    if (isyma == 2) goto L611;
    TERM[5] = C1 * S1 * Q[2];
    TERM[9] = C1 * S2 * Q[3];
    TERM[12] = B41(C2, C1, S1) * Q[4];
    TERM[14] = C1 * S3 * Q[4];
L611:
    if (maxtrm <= 4) goto L620;
    TERM[16] = B50(C4, C2, C1) * Q[5] * F1;
    TERM[22] = B60(C6, C4, C2) * Q[6];
    TERM[29] = B70(C6, C4, C2, C1) * Q[7] * F1;
    TERM[37] = B80(C8, C6, C4, C2) * Q[8];
    if (isyma >= 8) goto L613;
    QH = Q[6];
    TERM[24] = B62(C4, C2, S2) * QH;
    TERM[26] = B64(C2, S4) * QH;
    TERM[28] = S6 * QH;
    QH = Q[8];
    TERM[39] = B82(C6, C4, C2, S2) * QH;
    TERM[41] = B84(C4, C2, S4) * QH;
    TERM[43] = B86(C2, S6) * QH;
    TERM[45] = S8 * QH;
    if (isyma == 3) goto L613;
    QH = Q[5];
    TERM[17] = B51(C4, C2, S1) * QH;
    TERM[19] = B53(C2, S3) * QH;
    TERM[21] = S5 * QH;
    QH = Q[7];
    TERM[30] = B71(C6, C4, C2, S1) * QH;
    TERM[32] = B73(C4, C2, S3) * QH;
    TERM[34] = B75(C2, S5) * QH;
    TERM[36] = S7 * QH;
    if (isyma == 2) goto L613;
    TERM[18] = B52(C2, C1, S2) * Q[5];
    TERM[20] = C1 * S4 * Q[5];
    QH = Q[6];
    TERM[23] = B61(C4, C2, C1, S1) * QH;
    TERM[25] = B63(C2, C1, S3) * QH;
    TERM[27] = C1 * S5 * QH;
    QH = Q[7];
    TERM[31] = B72(C4, C2, C1, S2) * QH;
    TERM[33] = B74(C2, C1, S4) * QH;
    TERM[35] = C1 * S6 * QH;
    QH = Q[8];
    TERM[38] = B81(C6, C4, C2, C1, S1) * QH;
    TERM[40] = B83(C4, C2, C1, S3) * QH;
    TERM[42] = B85(C2, C1, S5) * QH;
    TERM[44] = C1 * S7 * QH;
L613:
    if (maxtrm <= 8) goto L620;
    TERM[46] = B90(C8, C6, C4, C2, C1) * Q[9] * F1;
    TERM[56] = B100(C10, C8, C6, C4, C2) * Q[10];
    if (isyma >= 8) goto L617;
    QH = Q[10];
    TERM[58] = B102(C8, C6, C4, C2, S2) * QH;
    TERM[60] = B104(C6, C4, C2, S4) * QH;
    TERM[62] = B106(C4, C2, S6) * QH;
    TERM[64] = B108(C2, S8) * QH;
    TERM[66] = S10 * QH;
    if (isyma == 3) goto L617;
    QH = Q[9];
    TERM[47] = B91(C8, C6, C4, C2, S1) * QH;
    TERM[49] = B93(C6, C4, C2, S3) * QH;
    TERM[51] = B95(C4, C2, S5) * QH;
    TERM[53] = B97(C2, S7) * QH;
    TERM[55] = S9 * QH;
    if (isyma == 2) goto L617;
    TERM[48] = B92(C6, C4, C2, C1, S2) * QH;
    TERM[50] = B94(C4, C2, C1, S4) * QH;
    TERM[52] = B96(C2, C1, S6) * QH;
    TERM[54] = C1 * S8 * QH;
    QH = Q[10];
    TERM[57] = B101(C8, C6, C4, C2, C1, S1) * QH;
    TERM[59] = B103(C6, C4, C2, C1, S3) * QH;
    TERM[61] = B105(C4, C2, C1, S5) * QH;
    TERM[63] = B107(C2, C1, S7) * QH;
    TERM[65] = C1 * S9 * QH;
L617:
L620:
    return;
}

/* Boundary terms DLM*BLM(theta) (pot/boundary.f:670-772).  TERM 1-based(66). */
static void bdy_terms(double *TERM, int maxtrm, int isyma, double F1, double C1, double S1,
                      const tw_t *tw)
{
    double C2, C4, S2, S3, S4, C6 = 0, C8 = 0, S5 = 0, S6 = 0, S7 = 0, S8 = 0, C10 = 0, S9 = 0, S10 = 0;
    int i;
    C2 = C1 * C1;
    C4 = C2 * C2;
    S2 = S1 * S1;
    S3 = S1 * S2;
    S4 = S2 * S2;
    if (maxtrm <= 4) goto L304;
    C6 = C2 * C4;
    C8 = C4 * C4;
    S5 = S1 * S4;
    S6 = S2 * S4;
    S7 = S1 * S6;
    S8 = S4 * S4;
    if (maxtrm <= 8) goto L304;
    C10 = C2 * C8;
    S9 = S1 * S8;
    S10 = S2 * S8;
L304:
    for (i = 1; i <= 66; i++) TERM[i] = 0.0;
    TERM[1] = 1.0;
    TERM[2] = C1 * F1;
    TERM[4] = 0.25 * B20(C2);
    TERM[7] = 0.25 * B30(C2, C1) * F1;
    TERM[11] = tw->tw6 * B40(C4, C2);
    if (isyma >= 8) goto L307;
    TERM[6] = 0.375 * S2;
    TERM[13] = 5.0 * tw->tw5 * B42(C2, S2);
    TERM[15] = 35.0 * tw->tw7 * S4;
    if (isyma == 3) goto L307;
    TERM[3] = 0.5 * S1;
    TERM[8] = 0.1875 * B31(C2, S1);
    TERM[10] = 0.3125 * S3;
    if (isyma == 2) goto L307;
    TERM[5] = 1.5 * C1 * S1;
    TERM[9] = 1.875 * C1 * S2;
    TERM[12] = 0.3125 * B41(C2, C1, S1);
    TERM[14] = 2.1875 * C1 * S3;
L307:
    if (maxtrm <= 4) goto L310;
    TERM[16] = tw->tw6 * B50(C4, C2, C1) * F1;
    TERM[22] = tw->tw8 * B60(C6, C4, C2);
    TERM[29] = tw->tw8 * B70(C6, C4, C2, C1) * F1;
    TERM[37] = tw->tw14 * B80(C8, C6, C4, C2);
    if (isyma >= 8) goto L308;
    TERM[24] = 105.0 * tw->tw10 * B62(C4, C2, S2);
    TERM[26] = 63.0 * tw->tw9 * B64(C2, S4);
    TERM[28] = 231.0 * tw->tw10 * S6;
    TERM[39] = 315.0 * tw->tw12 * B82(C6, C4, C2, S2);
    TERM[41] = 693.0 * tw->tw13 * B84(C4, C2, S4);
    TERM[43] = 429.0 * tw->tw12 * B86(C2, S6);
    TERM[45] = 6435.0 * tw->tw15 * S8;
    if (isyma == 3) goto L308;
    TERM[17] = 15.0 * tw->tw7 * B51(C4, C2, S1);
    TERM[19] = 35.0 * tw->tw8 * B53(C2, S3);
    TERM[21] = 63.0 * tw->tw8 * S5;
    TERM[30] = 7.0 * tw->tw11 * B71(C6, C4, C2, S1);
    TERM[32] = 21.0 * tw->tw11 * B73(C4, C2, S3);
    TERM[34] = 231.0 * tw->tw11 * B75(C2, S5);
    TERM[36] = 429.0 * tw->tw11 * S7;
    if (isyma == 2) goto L308;
    TERM[18] = 105.0 * tw->tw5 * B52(C2, C1, S2);
    TERM[20] = 315.0 * tw->tw7 * C1 * S4;
    TERM[23] = 21.0 * tw->tw7 * B61(C4, C2, C1, S1);
    TERM[25] = 105.0 * tw->tw8 * B63(C2, C1, S3);
    TERM[27] = 693.0 * tw->tw8 * C1 * S5;
    TERM[31] = 21.0 * tw->tw10 * B72(C4, C2, C1, S2);
    TERM[33] = 231.0 * tw->tw9 * B74(C2, C1, S4);
    TERM[35] = 3003.0 * tw->tw10 * C1 * S6;
    TERM[38] = 9.0 * tw->tw11 * B81(C6, C4, C2, C1, S1);
    TERM[40] = 1155.0 * tw->tw11 * B83(C4, C2, C1, S3);
    TERM[42] = 9009.0 * tw->tw11 * B85(C2, C1, S5);
    TERM[44] = 6435.0 * tw->tw11 * C1 * S7;
L308:
    if (maxtrm <= 8) goto L310;
    TERM[46] = tw->tw14 * B90(C8, C6, C4, C2, C1) * F1;
    TERM[56] = tw->tw16 * B100(C10, C8, C6, C4, C2);
    if (isyma >= 8) goto L309;
    TERM[58] = 165.0 * tw->tw17 * B102(C8, C6, C4, C2, S2);
    TERM[60] = 2145.0 * tw->tw15 * B104(C6, C4, C2, S4);
    TERM[62] = 2145.0 * tw->tw18 * B106(C4, C2, S6);
    TERM[64] = 12155.0 * tw->tw17 * B108(C2, S8);
    TERM[66] = 46189.0 * tw->tw18 * S10;
    if (isyma == 3) goto L309;
    TERM[47] = 45.0 * tw->tw15 * B91(C8, C6, C4, C2, S1);
    TERM[49] = 1155.0 * tw->tw14 * B93(C6, C4, C2, S3);
    TERM[51] = 1287.0 * tw->tw14 * B95(C4, C2, S5);
    TERM[53] = 6435.0 * tw->tw16 * B97(C2, S7);
    TERM[55] = 12155.0 * tw->tw16 * S9;
    if (isyma == 2) goto L309;
    TERM[48] = 495.0 * tw->tw12 * B92(C6, C4, C2, C1, S2);
    TERM[50] = 45045.0 * tw->tw13 * B94(C4, C2, C1, S4);
    TERM[52] = 2145.0 * tw->tw12 * B96(C2, C1, S6);
    TERM[54] = 109395.0 * tw->tw15 * C1 * S8;
    TERM[57] = 55.0 * tw->tw15 * B101(C8, C6, C4, C2, C1, S1);
    TERM[59] = 2145.0 * tw->tw14 * B103(C6, C4, C2, C1, S3);
    TERM[61] = 429.0 * tw->tw14 * B105(C4, C2, C1, S5);
    TERM[63] = 36465.0 * tw->tw16 * B107(C2, C1, S7);
    TERM[65] = 230945.0 * tw->tw16 * C1 * S9;
L309:
L310:
    return;
}

#define PHI_(c, j, k, l) (c)->phi[((size_t)(j) - 1) + (size_t)((c)->jmax + 2) * (((size_t)(k) - 1) + (size_t)((c)->kmax + 2) * ((size_t)(l) - 1))]
#define RHO_(c, j, k, l) (c)->rho[((size_t)(j) - 1) + (size_t)((c)->jmax + 2) * (((size_t)(k) - 1) + (size_t)((c)->kmax + 2) * ((size_t)(l) - 1))]

/* Returns 0, or -1 if SETBDY was never called (pot/boundary.f:311,901-907). */
int ora_bdygen(ora_ctx *c, int maxtrm, int isym, double redge)
{
    const int lmax = c->lmax, jmax = c->jmax, kmax = c->kmax, jkm1 = c->jkm1;
    const int jkmax = c->jkmax;
    const double *RHF = c->rhf - 1, *ZHF = c->zhf - 1, *R = c->r - 1, *Z = c->z - 1;
    const double dtheta = c->dtheta, grav = c->grav;
    int isyma, ntrm, l, nth, t;
    double F1, F2, tmass_total;
    tw_t tw = make_tw(c->r8);
    double *bdytrm_all;

    if (c->bdychk != 1.0) return -1;

    isyma = abs(isym);
    if (isyma == 2 || isyma == 9) { F1 = 0.0; F2 = 2.0; }
    else if (isyma == 3) { F1 = 0.0; F2 = 4.0; }
    else { F1 = 1.0; F2 = 1.0; }
    ntrm = 0;
    for (l = 0; l <= maxtrm; l++) ntrm = ntrm + (l + 1);

    nth = c->nthreads;
    /* thread-private BDYTRM(2,2,66,JKM1) and TMASS partials */
    bdytrm_all = (double *)calloc((size_t)nth * 4 * 66 * jkm1, sizeof(double));
    double *tmass_part = (double *)calloc((size_t)nth, sizeof(double));

#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *bdytrm = bdytrm_all + (size_t)tid * 4 * 66 * jkm1;
#define BDYTRM(a, b, i, jk) bdytrm[((a) - 1) + 2 * (((b) - 1) + 2 * (((i) - 1) + 66 * ((size_t)(jk) - 1)))]
        double TERM[67], CM[11], SM[11], MRING1[67], MRING2[67];
        double tm = 0.0;
        int kk;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (kk = 2; kk <= kmax; kk++) {
            double ZZ = ZHF[kk], Z2 = ZZ * ZZ, ZDEL = Z[kk + 1] - Z[kk];
            int jj;
            for (jj = 2; jj <= jmax; jj++) {
                double RR = RHF[jj], R2 = RR * RR, RSPHER = sqrt(R2 + Z2);
                double C1, S1, DV, SUMASS, H, QH;
                int m, ll, i, ichk, jk;
                if (redge > 0.0 && RSPHER > redge) continue;
                C1 = ZZ / RSPHER;
                S1 = RR / RSPHER;
                ring_terms(TERM, ntrm, maxtrm, isyma, F1, C1, S1, RSPHER);
                DV = 0.5 * dtheta * ZDEL * (R[jj + 1] * R[jj + 1] - R[jj] * R[jj]) * F2;
                for (m = 1; m <= maxtrm; m++) { CM[m] = 0.0; SM[m] = 0.0; }
                SUMASS = 0.0;
                for (ll = 1; ll <= lmax; ll++) {
                    H = RHO_(c, jj, kk, ll) * DV;
                    SUMASS = SUMASS + H;
                    for (m = 1; m <= maxtrm; m++) {
                        CM[m] = CM[m] + c->cosm[(ll - 1) + (size_t)lmax * (m - 1)] * H;
                        SM[m] = SM[m] + c->sinm[(ll - 1) + (size_t)lmax * (m - 1)] * H;
                    }
                }
                i = 0;
                for (l = 0; l <= maxtrm; l++) {
                    i = i + 1;
                    MRING1[i] = TERM[i] * SUMASS;
                    MRING2[i] = 0.0;
                    for (m = 1; m <= l; m++) {
                        i = i + 1;
                        MRING1[i] = TERM[i] * CM[m];
                        MRING2[i] = TERM[i] * SM[m];
                    }
                }
                tm = tm + MRING1[1];
                if (isym < 0) {
                    for (i = 1; i <= ntrm; i++) {
                        BDYTRM(1, 1, i, 1) = BDYTRM(1, 1, i, 1) + MRING1[i];
                        BDYTRM(1, 2, i, 1) = BDYTRM(1, 2, i, 1) + MRING2[i];
                    }
                    continue;
                }
                ichk = 0;
                for (jk = 1; jk <= jkmax; jk++) {
                    if (RSPHER <= c->rbdy[jk - 1]) {
                        for (i = 1; i <= ntrm; i++) {
                            BDYTRM(1, 1, i, jk) = BDYTRM(1, 1, i, jk) + MRING1[i];
                            BDYTRM(1, 2, i, jk) = BDYTRM(1, 2, i, jk) + MRING2[i];
                        }
                    } else {
                        ichk = ichk + 1;
                    }
                }
                if (ichk == 0) continue;
                i = 0;
                for (l = 0; l <= maxtrm; l++) {
                    QH = ipow(RSPHER, -(2 * l + 1));
                    for (m = 0; m <= l; m++) {
                        i = i + 1;
                        MRING1[i] = MRING1[i] * QH;
                        MRING2[i] = MRING2[i] * QH;
                    }
                }
                for (jk = 1; jk <= jkmax; jk++) {
                    if (RSPHER > c->rbdy[jk - 1]) {
                        for (i = 1; i <= ntrm; i++) {
                            BDYTRM(2, 1, i, jk) = BDYTRM(2, 1, i, jk) + MRING1[i];
                            BDYTRM(2, 2, i, jk) = BDYTRM(2, 2, i, jk) + MRING2[i];
                        }
                    }
                }
            }
        }
        tmass_part[tid] = tm;
#undef BDYTRM
    }

    /* merge the thread partials in thread-id order (pot/boundary.f:624-645) */
    {
        int jk, i;
        for (jk = 0; jk < jkm1; jk++)
            for (i = 0; i < 2 * 66; i++) {
                c->massin[i + 132 * (size_t)jk] = 0.0;
                c->massout[i + 132 * (size_t)jk] = 0.0;
            }
        tmass_total = 0.0;
        for (t = 0; t < nth; t++) {
            double *bdytrm = bdytrm_all + (size_t)t * 4 * 66 * jkm1;
            for (jk = 1; jk <= jkmax; jk++)
                for (i = 1; i <= ntrm; i++) {
                    size_t o = 4 * ((i - 1) + 66 * ((size_t)jk - 1));
                    size_t q = 2 * ((i - 1) + 66 * ((size_t)jk - 1));
                    c->massin[q + 0] = c->massin[q + 0] + bdytrm[o + 0];   /* (1,1) */
                    c->massin[q + 1] = c->massin[q + 1] + bdytrm[o + 2];   /* (1,2) */
                    c->massout[q + 0] = c->massout[q + 0] + bdytrm[o + 1]; /* (2,1) */
                    c->massout[q + 1] = c->massout[q + 1] + bdytrm[o + 3]; /* (2,2) */
                }
            tmass_total = tmass_total + tmass_part[t];
        }
        c->tmass = tmass_total;
    }
    free(bdytrm_all);
    free(tmass_part);

    /* potential on each boundary cell (pot/boundary.f:659-833) */
#ifdef _OPENMP
#pragma omp parallel for num_threads(nth) schedule(static)
#endif
    for (int jk = 1; jk <= jkmax; jk++) {
        int jj = c->jpos[jk - 1], kk = c->kpos[jk - 1];
        double RSPHER = c->rbdy[jk - 1];
        double TERM[67], TRM1[67], TRM2[67], CM[11], SM[11];
        double C1 = ZHF[kk] / RSPHER, S1 = RHF[jj] / RSPHER, RIN, ROUT, B, H, SUM;
        int l2, m, i, ll;
        bdy_terms(TERM, maxtrm, isyma, F1, C1, S1, &tw);
        if (isym >= 0) {
            i = 0;
            for (l2 = 0; l2 <= maxtrm; l2++) {
                RIN = 1.0 / ipow(RSPHER, l2 + 1);
                ROUT = ipow(RSPHER, l2);
                for (m = 0; m <= l2; m++) {
                    i = i + 1;
                    B = TERM[i] * RIN;
                    H = TERM[i] * ROUT;
                    size_t q = 2 * ((i - 1) + 66 * ((size_t)jk - 1));
                    TRM1[i] = B * c->massin[q + 0] + H * c->massout[q + 0];
                    TRM2[i] = B * c->massin[q + 1] + H * c->massout[q + 1];
                }
            }
        } else {
            i = 0;
            for (l2 = 0; l2 <= maxtrm; l2++) {
                RIN = 1.0 / ipow(RSPHER, l2 + 1);
                for (m = 0; m <= l2; m++) {
                    i = i + 1;
                    B = TERM[i] * RIN;
                    size_t q = 2 * (i - 1);
                    TRM1[i] = B * c->massin[q + 0];
                    TRM2[i] = B * c->massin[q + 1];
                }
            }
        }
        for (ll = 1; ll <= lmax; ll++) {
            for (m = 1; m <= maxtrm; m++) {
                CM[m] = c->cosm[(ll - 1) + (size_t)lmax * (m - 1)];
                SM[m] = c->sinm[(ll - 1) + (size_t)lmax * (m - 1)];
            }
            i = 0;
            SUM = 0.0;
            for (l2 = 0; l2 <= maxtrm; l2++) {
                i = i + 1;
                SUM = SUM + TRM1[i];
                for (m = 1; m <= l2; m++) {
                    i = i + 1;
                    SUM = SUM + 2.0 * (CM[m] * TRM1[i] + SM[m] * TRM2[i]);
                }
            }
            PHI_(c, jj, kk, ll) = -grav * SUM;
        }
    }

    /* tidy boundary symmetries (pot/boundary.f:862-894) */
    {
        int ll, lhaf, lp;
        isyma = abs(isym);
        if (isyma == 1) goto L550;
        if (isyma != 3 && isyma != 8 && isyma != 9) goto L525;
        for (ll = 1; ll <= lmax; ll++) PHI_(c, 1, kmax + 1, ll) = PHI_(c, 2, kmax + 1, ll);
        if (isyma != 8) goto L525;
        for (ll = 1; ll <= lmax; ll++) PHI_(c, 1, 1, ll) = PHI_(c, 2, 1, ll);
        goto L580;
    L525:
        if (isyma != 2 && isyma != 3 && isyma != 9) goto L550;
        for (ll = 1; ll <= lmax; ll++) PHI_(c, jmax + 1, 1, ll) = PHI_(c, jmax + 1, 2, ll);
        if (isyma != 2) goto L580;
    L550:
        lhaf = lmax / 2;
        for (ll = 1; ll <= lhaf; ll++) {
            lp = ll + lhaf;
            PHI_(c, 1, kmax + 1, ll) = PHI_(c, 2, kmax + 1, lp);
            PHI_(c, 1, kmax + 1, lp) = PHI_(c, 2, kmax + 1, ll);
            if (isyma == 1) {
                PHI_(c, 1, 1, ll) = PHI_(c, 2, 1, lp);
                PHI_(c, 1, 1, lp) = PHI_(c, 2, 1, ll);
            }
        }
    L580:;
    }
    (void)grav;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* ZAXPHI  pot/pot3.f:311-423                                                 */
/* ------------------------------------------------------------------------ */
static void zaxphi(ora_ctx *c, int npoint, int iprint)
{
    const int lmax = c->lmax, kmax = c->kmax, jmax = c->jmax;
    const double *RHF = c->rhf - 1;
    double X[11], PHI2[11], *PH, *PHAC = c->phac - 1;
    double xpoint, phmax, xinv, xr, xratio, p1, p2, err, er, xx;
    int lm, n, ichk, num, ispecl, jsp, j, i1, i2, k, l, lp, im, i, ist;
    (void)iprint;

    PH = (double *)calloc(lmax + 1, sizeof(double));
    if (npoint > 10) npoint = 10;
    xpoint = 0.0;
    lm = lmax / 2;
    n = npoint;
    ichk = n % 2;
    n = n - ichk;
    num = n / 2;
    ispecl = num + num + 1;
    jsp = num + 1;
    for (j = 2; j <= jsp; j++) {
        i1 = num + (j - 1);
        i2 = num - (j - 2);
        X[i1] = RHF[j];
        X[i2] = -RHF[j];
    }
    if (ichk == 1) X[ispecl] = RHF[num + 2];

    for (k = 2; k <= kmax + 1; k++) {
        phmax = 0.0;
        for (l = 1; l <= lm; l++) {
            lp = l + lm;
            for (j = 2; j <= jsp; j++) {
                i1 = num + (j - 1);
                i2 = num - (j - 2);
                PHI2[i1] = PHI_(c, j, k, l);
                PHI2[i2] = PHI_(c, j, k, lp);
            }
            if (ichk == 1) PHI2[ispecl] = PHI_(c, num + 2, k, l);
            im = npoint - 1;
            for (i = 1; i <= im; i++) {
                p1 = PHI2[i];
                xinv = 1.0 / X[i];
                xr = xpoint * xinv;
                ist = i + 1;
                for (j = ist; j <= npoint; j++) {
                    xratio = X[j] * xinv;
                    p2 = PHI2[j];
                    PHI2[j] = (p1 * (xratio - xr) + p2 * (xr - 1.0)) / (xratio - 1.0);
                }
            }
            PH[l] = PHI2[npoint];
            if (fabs(PH[l]) > fabs(phmax)) phmax = PH[l];
            PHI_(c, jmax + 2, k, l) = PH[l];
            PHI_(c, jmax + 2, k, lp) = PH[l];
        }
        err = 0.0;
        for (l = 1; l <= lm; l++) {
            er = 1.0 - PH[l] / phmax;
            if (fabs(er) > fabs(err)) err = er;
        }
        PHAC[k] = err;
    }
    err = 0.0;
    for (k = 2; k <= kmax + 1; k++) {
        xx = fabs(PHAC[k]);
        if (xx > fabs(err)) {
            err = PHAC[k];
            c->klocat = k;
        }
    }
    c->phichk = err;
    free(PH);
}

/* ------------------------------------------------------------------------ */
/* POT3  pot/pot3.f:15-306                                                    */
/* ------------------------------------------------------------------------ */
void ora_pot3(ora_ctx *c, int npoint, int iprint)
{
    const int jmax = c->jmax, kmax = c->kmax, lmax = c->lmax, r8 = c->r8;
    const int jm3 = jmax - 1, km3 = kmax - 1;
    const double *RHF = c->rhf - 1, *ZHF = c->zhf - 1;
    const int nth = c->nthreads;
    const int wsize = ora_blktri_wsize(jmax, kmax);
    int n;
    double sf1, sf2;
    /* m-independent coefficients (shared, computed serially below) */
    double *AN = (double *)calloc(km3 + 1, sizeof(double)) - 1;
    double *BN = (double *)calloc(km3 + 1, sizeof(double)) - 1;
    double *CN = (double *)calloc(km3 + 1, sizeof(double)) - 1;
    double *AM = (double *)calloc(jm3 + 1, sizeof(double)) - 1;
    double *CMc = (double *)calloc(jm3 + 1, sizeof(double)) - 1;
    double *Cc = (double *)calloc(jm3 + 1, sizeof(double)) - 1;
    double *DENOMR = (double *)calloc(jmax + 1, sizeof(double)) - 1;
    double *RD2 = (double *)calloc(jmax + 1, sizeof(double)) - 1;
    double *RD3 = (double *)calloc(jmax + 1, sizeof(double)) - 1;
    double *DENOMZ = (double *)calloc(kmax + 1, sizeof(double)) - 1;
    double *ZD2 = (double *)calloc(kmax + 1, sizeof(double)) - 1;
    double *XLAMM = (double *)calloc(lmax / 2 + 2, sizeof(double)) - 1;
    double dthet2, pig4, cmmax, ammin, cnmax;

    n = lmax / 2;
    if (lmax == 1) n = 1;
    sf1 = r8 ? 0.5 / (double)n : (double)(0.5f / (float)n);
    sf2 = 0.5;

    /* rho -> phi for J=2..JMAX, K=2..KMAX (pot3.f:70-82) */
#ifdef _OPENMP
#pragma omp parallel for num_threads(nth) schedule(static)
#endif
    for (int l = 1; l <= lmax; l++)
        for (int k = 2; k <= kmax; k++)
            for (int j = 2; j <= jmax; j++) PHI_(c, j, k, l) = RHO_(c, j, k, l);

    /* forward real FFT of every (J,K) column (pot3.f:90-149) */
    if (lmax > 1) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
        {
            double *A1 = (double *)calloc(lmax + 2, sizeof(double)) - 1;
            double *B1 = (double *)calloc(lmax + 2, sizeof(double)) - 1;
            int k;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (k = 2; k <= kmax + 1; k++) {
                for (int j = 2; j <= jmax + 1; j++) {
                    int l;
                    double x1, philag;
                    for (l = 1; l <= n; l++) {
                        A1[l] = PHI_(c, j, k, 2 * l - 1);
                        B1[l] = PHI_(c, j, k, 2 * l);
                    }
                    ora_fft(A1 + 1, B1 + 1, n, n, n, 1, r8);
                    ora_realtr(A1 + 1, B1 + 1, n, 1, r8);
                    if (c->coef) {
#define COEF_(jj, kk, ll, ii) c->coef[((jj) - 1) + (size_t)(jmax + 2) * (((kk) - 1) + (size_t)(kmax + 2) * (((ll) - 1) + (size_t)(lmax / 2) * ((ii) - 1)))]
                        x1 = fabs(A1[1]);
                        if (x1 != 0.0) {
                            for (l = 2; l <= n; l++)
                                COEF_(j, k, l - 1, 1) = 2.0 * sqrt(A1[l] * A1[l] + B1[l] * B1[l]) / x1;
                            COEF_(j, k, n, 1) = fabs(A1[n + 1]) / x1;
                        }
                        for (l = 2; l <= n; l++) {
                            if (A1[l] > 0.0) philag = atan(B1[l] / A1[l]);
                            else if (A1[l] < 0.0) philag = atan(B1[l] / A1[l]) + c->pi;
                            else {
                                if (B1[l] > 0.0) philag = 0.5 * c->pi;
                                else if (B1[l] < 0.0) philag = -0.5 * c->pi;
                                else philag = 4.0 * c->pi;
                            }
                            COEF_(j, k, l - 1, 2) = philag * 180. / c->pi;
                        }
                        COEF_(j, k, n, 2) = A1[1];
#undef COEF_
                    }
                    for (l = 1; l <= n + 1; l++) {
                        PHI_(c, j, k, l) = A1[l] * sf1;
                        if (l < n) PHI_(c, j, k, l + n + 1) = B1[l + 1] * sf1;
                    }
                    for (l = n + 1; l <= lmax; l++) {
                        A1[l] = 0.0;
                        B1[l] = 0.0;
                    }
                }
            }
            free(A1 + 1);
            free(B1 + 1);
        }
    }

    /* coefficients (pot3.f:158-194) */
    dthet2 = 1.0 / (c->dtheta * c->dtheta);
    pig4 = 4.0 * c->pi * c->grav;
    RD2[1] = 0.5 / RHF[2];
    RD3[1] = 1.0 / RHF[1];
    for (int j = 2; j <= jmax; j++) {
        DENOMR[j] = 1.0 / (RHF[j + 1] - RHF[j - 1]);
        RD2[j] = 1.0 / (RHF[j + 1] - RHF[j]);
        RD3[j] = 1.0 / RHF[j];
    }
    ZD2[1] = 0.5 / ZHF[2];
    for (int k = 2; k <= kmax; k++) {
        DENOMZ[k] = 1.0 / (ZHF[k + 1] - ZHF[k - 1]);
        ZD2[k] = 1.0 / (ZHF[k + 1] - ZHF[k]);
    }
    for (int j = 2; j <= jmax; j++) {
        CMc[j - 1] = 2. * (RD2[j] + 0.5 * RD3[j]) * DENOMR[j];
        AM[j - 1] = 2. * (RD2[j - 1] - 0.5 * RD3[j]) * DENOMR[j];
        Cc[j - 1] = RD3[j] * RD3[j] * dthet2;
    }
    for (int k = 2; k <= kmax; k++) {
        CN[k - 1] = 2. * ZD2[k] * DENOMZ[k];
        AN[k - 1] = 2. * ZD2[k - 1] * DENOMZ[k];
        BN[k - 1] = -CN[k - 1] - AN[k - 1];
    }
    cmmax = CMc[jmax - 1];
    CMc[jmax - 1] = 0.0;
    ammin = AM[1];
    AM[1] = 0.0;
    cnmax = CN[kmax - 1];
    CN[kmax - 1] = 0.0;
    BN[1] = -CN[1];
    AN[1] = 0.0;
    for (int m = 1; m <= n + 1; m++) XLAMM[m] = cos((double)(m - 1) * c->dtheta);

    /* per-mode solves (pot3.f:201-248) */
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
    {
        double *Y = (double *)calloc((size_t)jm3 * km3, sizeof(double));
        double *BM = (double *)calloc(jm3 + 1, sizeof(double)) - 1;
        double *W = (double *)calloc(wsize, sizeof(double));
        double state[32]; /* holds a cblkt_t */
        int init_blktri = 1, ierror = 0, l;
        memset(state, 0, sizeof(state));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (l = 1; l <= lmax; l++) {
            int m = (l <= n + 1) ? l - 1 : l - (n + 1);
            double powrm = (m % 2 == 0) ? 1.0 : -1.0;
#define Y_(jj, kk) Y[((jj) - 1) + (size_t)jm3 * ((kk) - 1)]
            for (int k = 2; k <= kmax; k++)
                for (int j = 2; j <= jmax; j++) Y_(j - 1, k - 1) = pig4 * PHI_(c, j, k, l);
            for (int j = 2; j <= jmax; j++)
                Y_(j - 1, kmax - 1) = Y_(j - 1, kmax - 1) - cnmax * PHI_(c, j, kmax + 1, l);
            for (int k = 2; k <= kmax; k++)
                Y_(jmax - 1, k - 1) = Y_(jmax - 1, k - 1) - cmmax * PHI_(c, jmax + 1, k, l);
            BM[1] = -CMc[1] + (powrm - 1.0) * ammin + 2.0 * (XLAMM[m + 1] - 1.0) * Cc[1];
            for (int j = 2; j <= jmax - 2; j++)
                BM[j] = -CMc[j] - AM[j] + 2.0 * (XLAMM[m + 1] - 1.0) * Cc[j];
            BM[jmax - 1] = -cmmax - AM[jmax - 1] + 2.0 * (XLAMM[m + 1] - 1.0) * Cc[jmax - 1];
            if (init_blktri) {
                ora_blktri(state, 0, 1, kmax - 1, AN + 1, BN + 1, CN + 1, 1, jmax - 1, AM + 1,
                           BM + 1, CMc + 1, jmax - 1, Y, &ierror, W);
                init_blktri = 0;
            }
            ora_blktri(state, 1, 1, kmax - 1, AN + 1, BN + 1, CN + 1, 1, jmax - 1, AM + 1,
                       BM + 1, CMc + 1, jmax - 1, Y, &ierror, W);
            for (int k = 2; k <= kmax; k++)
                for (int j = 2; j <= jmax; j++) PHI_(c, j, k, l) = Y_(j - 1, k - 1);
#undef Y_
        }
        free(Y);
        free(BM + 1);
        free(W);
    }

    /* inverse real FFT (pot3.f:256-283) */
    if (lmax != 1) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nth)
#endif
        {
            double *A1 = (double *)calloc(lmax + 2, sizeof(double)) - 1;
            double *B1 = (double *)calloc(lmax + 2, sizeof(double)) - 1;
            int k;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (k = 2; k <= kmax + 1; k++) {
                for (int j = 2; j <= jmax + 1; j++) {
                    int l;
                    for (l = 1; l <= lmax; l++) {
                        A1[l] = 0.0;
                        B1[l] = 0.0;
                    }
                    for (l = 1; l <= n + 1; l++) {
                        A1[l] = PHI_(c, j, k, l);
                        if (l < n) B1[l + 1] = PHI_(c, j, k, l + n + 1);
                    }
                    ora_realtr(A1 + 1, B1 + 1, n, -1, r8);
                    ora_fft(A1 + 1, B1 + 1, n, n, n, -1, r8);
                    for (l = 1; l <= n; l++) {
                        PHI_(c, j, k, 2 * l - 1) = sf2 * A1[l];
                        PHI_(c, j, k, 2 * l) = sf2 * B1[l];
                    }
                }
            }
            free(A1 + 1);
            free(B1 + 1);
        }
    }

    /* axis and midplane ghosts (pot3.f:287-298) */
    for (int l = 1; l <= n; l++) {
        for (int k = 2; k <= kmax + 1; k++) {
            PHI_(c, 1, k, l) = PHI_(c, 2, k, n + l);
            PHI_(c, 1, k, n + l) = PHI_(c, 2, k, l);
        }
        for (int j = 1; j <= jmax + 1; j++) {
            PHI_(c, j, 1, l) = PHI_(c, j, 2, l);
            PHI_(c, j, 1, n + l) = PHI_(c, j, 2, n + l);
        }
    }

    zaxphi(c, npoint, iprint);

    free(AN + 1); free(BN + 1); free(CN + 1); free(AM + 1); free(CMc + 1); free(Cc + 1);
    free(DENOMR + 1); free(RD2 + 1); free(RD3 + 1); free(DENOMZ + 1); free(ZD2 + 1);
    free(XLAMM + 1);
}

/* ------------------------------------------------------------------------ */
/* ExternalPot (pot/ExternalPot.f:1-80): the central star's potential added  */
/* to PHI after POT3 (radhydro/3dhyd-main.f:510-512, EXTERNAL_POT builds).   */
/* ------------------------------------------------------------------------ */
/* INDIRECTX/Y start at RPSTAR*COS/SIN(PHI_STAR) (ExternalPot.f:18-19).  With
 * indirect != 0 (INDIRECT builds, ExternalPot.f:21-40) the disk's mass
 * moment over L, K = 2..KMAX1, J = JMIN..JMAX1 is summed in the reference's
 * serial loop order, added as an OpenMP reduction adds it to the start value,
 * and divided by -MASS_STAR.  STARPHI over the whole grid (ExternalPot.f:42-54)
 * is added to PHI and, if starphi is not NULL, stored there.  ixy (if not
 * NULL) receives INDIRECTX, INDIRECTY. */
/* ExternalPot (pot/ExternalPot.f:1-80), with the BINARY build's companion
 * term when binary != 0: getBinaryPosition's circular orbit
 * (radhydro/ExternalRoutines.f:91-105: muBin = massBin + mass_star,
 * omegaBin = sqrt(muBin/aBin**3), rBin = aBin), rcom (ExternalPot.f:15) and
 * PHI = PHI - massBin/rdist - half*omegaBin**2*((x+rcom)**2+y**2) per cell
 * (ExternalPot.f:57-69). */
void ora_external_pot_binary(ora_ctx *c, double mass_star, double tmassacc, double rpstar, double phi_star,
                             int indirect, int jmin, int binary, double mass_bin, double a_bin, double *starphi,
                             double *ixy)
{
    const int jmax = c->jmax, kmax = c->kmax, lmax = c->lmax;
    const double dtheta = c->dtheta, half = 0.5, two = 2.0;
    double ix = rpstar * cos(phi_star), iy = rpstar * sin(phi_star);
    if (indirect) {
        double sx = 0.0, sy = 0.0;
        for (int l = 1; l <= lmax; l++)
            for (int k = 2; k <= kmax + 1; k++)
                for (int j = jmin; j <= jmax + 1; j++) {
                    const double rhf = c->rhf[j - 1];
                    const double m = RHO_(c, j, k, l) * rhf * c->rof3n * c->zof3n * two * dtheta;
                    sx = sx + m * cos(((double)(l - 1) + half) * dtheta) * rhf;
                    sy = sy + m * sin(((double)(l - 1) + half) * dtheta) * rhf;
                }
        ix = -(ix + sx) / mass_star;
        iy = -(iy + sy) / mass_star;
    }
    const double mass = mass_star + tmassacc;
    double rbin = 0.0, omega2 = 0.0, rcom = 0.0;
    if (binary) {
        const double mu = mass_bin + mass_star;
        const double omega = sqrt((mu) / (a_bin * a_bin * a_bin));
        rbin = a_bin;
        omega2 = omega * omega;
        rcom = rbin - rbin * mass_star / mu;
    }
    for (int l = 1; l <= lmax; l++) {
        const double cl = cos(((double)(l - 1) + half) * dtheta), sl = sin(((double)(l - 1) + half) * dtheta);
        const double theta = ((double)l - half) * dtheta;
        const double cb = cos(theta - c->pi), ct = cos(theta), st = sin(theta);
        for (int k = 1; k <= kmax + 2; k++)
            for (int j = 1; j <= jmax + 2; j++) {
                const double rhf = c->rhf[j - 1], zhf = c->zhf[k - 1];
                const double sp = -mass / sqrt(rhf * rhf + zhf * zhf + ix * ix + iy * iy -
                                               two * rhf * (cl * ix + sl * iy));
                PHI_(c, j, k, l) = PHI_(c, j, k, l) + sp;
                if (starphi)
                    starphi[((size_t)j - 1) + (size_t)(jmax + 2) * (((size_t)k - 1) + (size_t)(kmax + 2) * ((size_t)l - 1))] = sp;
                if (binary) {
                    const double rdist = sqrt(rbin * rbin + rhf * rhf - two * rbin * rhf * cb + zhf * zhf);
                    const double x = rhf * ct, y = rhf * st;
                    PHI_(c, j, k, l) = PHI_(c, j, k, l) - mass_bin / rdist - half * omega2 * ((x + rcom) * (x + rcom) + y * y);
                }
            }
    }
    if (ixy) { ixy[0] = ix; ixy[1] = iy; }
}

void ora_external_pot(ora_ctx *c, double mass_star, double tmassacc, double rpstar, double phi_star,
                      int indirect, int jmin, double *starphi, double *ixy)
{
    ora_external_pot_binary(c, mass_star, tmassacc, rpstar, phi_star, indirect, jmin, 0, 0.0, 0.0, starphi, ixy);
}

/* ------------------------------------------------------------------------ */
/* SOURCE's first loop nest (radhydro/source.f:45-81): the potential,        */
/* pressure and rotation terms of the S, T, A momenta, with the BINARY       */
/* build's terms when binary != 0.                                           */
/* ------------------------------------------------------------------------ */
/* Hydro arrays omega, p, s, t, a, u are (jmax+2, kmax+2, lmax); rho and phi
 * are the potential grid's (j2p, k2p, lmax); r and rhf are R(j2p), RHF(j2p).
 * Column-major.  With binary != 0, omegaBin comes from getBinaryPosition's
 * circular orbit (massBin, aBin, mass_star) and each statement takes its
 * BINARY term after the DELT term, as the reference's single statements
 * evaluate left to right. */
void ora_source_binary(int jmax, int kmax, int lmax, int j2p, int k2p, int jmin, double delt, double dr, double dz,
                       double dtheta, const double *r, const double *rho, const double *phi, const double *omega,
                       const double *p, double *s, double *t, double *a, int binary, double mass_star,
                       double mass_bin, double a_bin, const double *rhf, const double *u)
{
    const double quarter = 0.25, half = 0.5, two = 2.0;
    const size_t j2 = (size_t)jmax + 2, k2 = (size_t)kmax + 2;
#define H_(x, j, k, l) (x)[((size_t)(j) - 1) + j2 * (((size_t)(k) - 1) + k2 * ((size_t)(l) - 1))]
#define P_(x, j, k, l) (x)[((size_t)(j) - 1) + (size_t)j2p * (((size_t)(k) - 1) + (size_t)k2p * ((size_t)(l) - 1))]
    const int jstart = jmin > 2 ? jmin : 2;   /* radhydro/source.f:33-37 */
    /* getBinaryPosition's circular orbit (radhydro/ExternalRoutines.f:101-102) */
    double omega_bin = 0.0;
    if (binary) {
        const double mu = mass_bin + mass_star;
        omega_bin = sqrt((mu) / (a_bin * a_bin * a_bin));
    }
    for (int l = 1; l <= lmax; l++) {
        int lm = l - 1, lp = l + 1;
        if (l == 1) lm = lmax;
        if (l == lmax) lp = 1;
        for (int k = 2; k <= kmax + 1; k++) {
            for (int j = jstart + 1; j <= jmax + 1; j++) {
                const double om = H_(omega, j, k, l) + H_(omega, j - 1, k, l);
                H_(s, j, k, l) = H_(s, j, k, l) +
                    delt * (r[j - 1] * (P_(rho, j, k, l) + P_(rho, j - 1, k, l)) * (om * om) * quarter * half -
                            (P_(rho, j, k, l) + P_(rho, j - 1, k, l)) * (P_(phi, j, k, l) - P_(phi, j - 1, k, l)) /
                                (two * dr) -
                            (H_(p, j, k, l) - H_(p, j - 1, k, l)) / dr);
                if (binary) /* source.f:61-62 */
                    H_(s, j, k, l) = H_(s, j, k, l) +
                        omega_bin * H_(omega, j, k, l) * rhf[j - 1] * two * P_(rho, j, k, l) * delt;
            }
            for (int j = jstart; j <= jmax + 1; j++)
                H_(t, j, k, l) = H_(t, j, k, l) -
                    delt * (half * (P_(rho, j, k, l) + P_(rho, j, k - 1, l)) * (P_(phi, j, k, l) - P_(phi, j, k - 1, l)) / dz +
                            (H_(p, j, k, l) - H_(p, j, k - 1, l)) / dz);
            for (int j = jstart; j <= jmax + 1; j++) {
                H_(a, j, k, l) = H_(a, j, k, l) -
                    delt * (P_(rho, j, k, l) * (P_(phi, j, k, lp) - P_(phi, j, k, lm)) + H_(p, j, k, lp) - H_(p, j, k, lm)) /
                        (two * dtheta);
                if (binary) /* source.f:76-77 */
                    H_(a, j, k, l) = H_(a, j, k, l) -
                        P_(rho, j, k, l) * omega_bin * (H_(u, j + 1, k, l) + H_(u, j, k, l)) * delt * rhf[j - 1];
            }
        }
    }
#undef H_
#undef P_
}

void ora_source(int jmax, int kmax, int lmax, int j2p, int k2p, int jmin, double delt, double dr, double dz,
                double dtheta, const double *r, const double *rho, const double *phi, const double *omega,
                const double *p, double *s, double *t, double *a)
{
    ora_source_binary(jmax, kmax, lmax, j2p, k2p, jmin, delt, dr, dz, dtheta, r, rho, phi, omega, p, s, t, a, 0, 0.0,
                      0.0, 0.0, NULL, NULL);
}

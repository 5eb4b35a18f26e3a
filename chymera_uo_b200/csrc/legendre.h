// legendre.h -- Legendre factors of the boundary-potential expansion, usable on
// host and device.  Device code that includes this must be compiled with
// --fmad=false so the values match the host tables bit for bit.
//
// The reference expands the exterior potential in terms TERM(I),
// I = L(L+1)/2 + M + 1, built from the polynomial factors BLM(cos theta) of its
// statement functions (pot/boundary.f:204-253): BLM = [C1 *] P(C2) [* S^M],
// where P is a polynomial in C2 = cos^2 theta with the integer coefficients
// below (highest power first), C1 = cos theta is a factor when L-M is odd, and
// S = sin theta.  The ring pass multiplies BLM by r^L (and by F1 for odd-L,
// M = 0 terms, pot/boundary.f:412-502); the boundary pass multiplies by the
// normalisation DLM = a * 2^-n (pot/boundary.f:694-772, written there as
// a*TWn with TWn = 2^-n).  Which terms exist depends on ISYM
// (pot/boundary.f:417-490).  The evaluation order follows the reference's
// expressions.
#pragma once

#ifdef __CUDACC__
#define CHY_HD __host__ __device__
#else
#define CHY_HD
#endif

namespace chy {

struct LegTerm {
    int l, m;
    int npoly;       // number of polynomial coefficients (0: no polynomial)
    double poly[6];  // highest power of C2 first
    double dlm_a;    // DLM = dlm_a * TWn (or dlm_a when tw == 0)
    int tw;          // n of TWn, or 0
};

// clang-format off
#define CHY_LEG_TABLE { \
    {0, 0, 0, {0}, 1.0, 0}, \
    {1, 0, 0, {0}, 1.0, 0}, \
    {1, 1, 0, {0}, 0.5, 0}, \
    {2, 0, 2, {3, -1}, 0.25, 0}, \
    {2, 1, 0, {0}, 1.5, 0}, \
    {2, 2, 0, {0}, 0.375, 0}, \
    {3, 0, 2, {5, -3}, 0.25, 0}, \
    {3, 1, 2, {5, -1}, 0.1875, 0}, \
    {3, 2, 0, {0}, 1.875, 0}, \
    {3, 3, 0, {0}, 0.3125, 0}, \
    {4, 0, 3, {35, -30, 3}, 1.0, 6}, \
    {4, 1, 2, {7, -3}, 0.3125, 0}, \
    {4, 2, 2, {7, -1}, 5.0, 5}, \
    {4, 3, 0, {0}, 2.1875, 0}, \
    {4, 4, 0, {0}, 35.0, 7}, \
    {5, 0, 3, {63, -70, 15}, 1.0, 6}, \
    {5, 1, 3, {21, -14, 1}, 15.0, 7}, \
    {5, 2, 2, {3, -1}, 105.0, 5}, \
    {5, 3, 2, {9, -1}, 35.0, 8}, \
    {5, 4, 0, {0}, 315.0, 7}, \
    {5, 5, 0, {0}, 63.0, 8}, \
    {6, 0, 4, {231, -315, 105, -5}, 1.0, 8}, \
    {6, 1, 3, {33, -30, 5}, 21.0, 7}, \
    {6, 2, 3, {33, -18, 1}, 105.0, 10}, \
    {6, 3, 2, {11, -3}, 105.0, 8}, \
    {6, 4, 2, {11, -1}, 63.0, 9}, \
    {6, 5, 0, {0}, 693.0, 8}, \
    {6, 6, 0, {0}, 231.0, 10}, \
    {7, 0, 4, {429, -693, 315, -35}, 1.0, 8}, \
    {7, 1, 4, {429, -495, 135, -5}, 7.0, 11}, \
    {7, 2, 3, {143, -110, 15}, 21.0, 10}, \
    {7, 3, 3, {143, -66, 3}, 21.0, 11}, \
    {7, 4, 2, {13, -3}, 231.0, 9}, \
    {7, 5, 2, {13, -1}, 231.0, 11}, \
    {7, 6, 0, {0}, 3003.0, 10}, \
    {7, 7, 0, {0}, 429.0, 11}, \
    {8, 0, 5, {6435, -12012, 6930, -1260, 35}, 1.0, 14}, \
    {8, 1, 4, {715, -1001, 385, -35}, 9.0, 11}, \
    {8, 2, 4, {143, -143, 33, -1}, 315.0, 12}, \
    {8, 3, 3, {39, -26, 3}, 1155.0, 11}, \
    {8, 4, 3, {65, -26, 1}, 693.0, 13}, \
    {8, 5, 2, {5, -1}, 9009.0, 11}, \
    {8, 6, 2, {15, -1}, 429.0, 12}, \
    {8, 7, 0, {0}, 6435.0, 11}, \
    {8, 8, 0, {0}, 6435.0, 15}, \
    {9, 0, 5, {12155, -25740, 18018, -4620, 315}, 1.0, 14}, \
    {9, 1, 5, {2431, -4004, 2002, -308, 7}, 45.0, 15}, \
    {9, 2, 4, {221, -273, 91, -7}, 495.0, 12}, \
    {9, 3, 4, {221, -195, 39, -1}, 1155.0, 14}, \
    {9, 4, 3, {17, -10, 1}, 45045.0, 13}, \
    {9, 5, 3, {85, -30, 1}, 1287.0, 14}, \
    {9, 6, 2, {17, -3}, 2145.0, 12}, \
    {9, 7, 2, {17, -1}, 6435.0, 16}, \
    {9, 8, 0, {0}, 109395.0, 15}, \
    {9, 9, 0, {0}, 12155.0, 16}, \
    {10, 0, 6, {46189, -109395, 90090, -30030, 3465, -63}, 1.0, 16}, \
    {10, 1, 5, {4199, -7956, 4914, -1092, 63}, 55.0, 15}, \
    {10, 2, 5, {4199, -6188, 2730, -364, 7}, 165.0, 17}, \
    {10, 3, 4, {323, -357, 105, -7}, 2145.0, 14}, \
    {10, 4, 4, {323, -255, 45, -1}, 2145.0, 15}, \
    {10, 5, 3, {323, -170, 15}, 429.0, 14}, \
    {10, 6, 3, {323, -102, 3}, 2145.0, 18}, \
    {10, 7, 2, {19, -3}, 36465.0, 16}, \
    {10, 8, 2, {19, -1}, 12155.0, 17}, \
    {10, 9, 0, {0}, 230945.0, 16}, \
    {10, 10, 0, {0}, 46189.0, 18}, \
}
// clang-format on

// Is term (l, m) present for this |ISYM| (pot/boundary.f:417-490)?
CHY_HD inline bool term_present(int l, int m, int isyma)
{
    if (m == 0) return true;
    if (isyma >= 8) return false;
    if ((l + m) % 2 == 0 && m % 2 == 0) return true;  // ISYM 1, 2, 3
    if ((l + m) % 2 == 0) return isyma != 3;          // odd m: ISYM 1, 2
    return isyma != 2 && isyma != 3;                  // l+m odd: ISYM 1
}

struct Powers {
    double c1, c2, c4, c6, c8, c10, s[11];
};

// cos/sin powers in the order pot/boundary.f:385-402 forms them
CHY_HD inline Powers make_powers(double C1, double S1, int maxtrm)
{
    Powers p{};
    p.c1 = C1;
    p.c2 = C1 * C1;
    p.c4 = p.c2 * p.c2;
    const double S2 = S1 * S1, S3 = S1 * S2, S4 = S2 * S2;
    p.s[0] = 1.0;
    p.s[1] = S1;
    p.s[2] = S2;
    p.s[3] = S3;
    p.s[4] = S4;
    if (maxtrm > 4) {
        p.c6 = p.c2 * p.c4;
        p.c8 = p.c4 * p.c4;
        p.s[5] = S1 * S4;
        p.s[6] = S2 * S4;
        p.s[7] = S1 * p.s[6];
        p.s[8] = S4 * S4;
        if (maxtrm > 8) {
            p.c10 = p.c2 * p.c8;
            p.s[9] = S1 * p.s[8];
            p.s[10] = S2 * p.s[8];
        }
    }
    return p;
}

CHY_HD inline double poly_value(const LegTerm &t, const Powers &p)
{
    const double cp[6] = {1.0, p.c2, p.c4, p.c6, p.c8, p.c10};
    const int d = t.npoly - 1;
    double acc = t.poly[0] * cp[d];
    for (int e = 1; e < t.npoly; e++) acc = acc + t.poly[e] * cp[d - e];
    return acc;
}

// BLM(theta) as the statement functions compute it
CHY_HD inline double blm_value(const LegTerm &t, const Powers &p)
{
    const bool odd = ((t.l - t.m) % 2) != 0;
    if (t.npoly == 0) {
        if (t.m == 0) return odd ? p.c1 : 1.0;
        return odd ? p.c1 * p.s[t.m] : p.s[t.m];
    }
    double v = poly_value(t, p);
    if (odd) v = p.c1 * v;
    if (t.m > 0) v = v * p.s[t.m];
    return v;
}

// Fortran REAL**INTEGER by square-and-multiply (negative powers as 1/y)
CHY_HD inline double ipow(double x, int m)
{
    unsigned int n = m < 0 ? 0u - (unsigned int)m : (unsigned int)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

// Ring-pass term i (0-based) for a ring at spherical radius rsph with
// cos/sin of its polar angle C1/S1 (pot/boundary.f:385-502).
CHY_HD inline double ring_term(const LegTerm &t, int i, const Powers &p, const double *q, int maxtrm,
                               int isyma, double F1)
{
    if (t.l > maxtrm || !term_present(t.l, t.m, isyma)) return 0.0;
    if (i == 0) return 1.0;
    double v = blm_value(t, p) * q[t.l];
    if (t.m == 0 && (t.l % 2) == 1) v = v * F1;
    return v;
}

}  // namespace chy

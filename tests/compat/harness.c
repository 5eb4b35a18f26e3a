/* Test harness for chymera_uo_b200/csrc/compat/pot3_common.cpp: a C program
 * that lays out the reference's COMMON blocks (headers/globals.h) the way a
 * gfortran executable does, then issues the ITYPE=71 call sequence of
 * radhydro/io.f:212-218 through the gfortran-mangled entry points.
 *
 *   harness <rho.bin> <out prefix> [mode]
 * rho.bin: RHO(JMAX+2, KMAX+2, LMAX) float64, column-major.
 * Writes <prefix>.phi (PHI), <prefix>.coef (COEF), <prefix>.inside
 * (TMASS, PHICHK, KLOCAT as float64) and prints the status.
 * mode "nosetup": calls BDYGEN and POT3 without SETBDY (expects status 13).
 * Sizes come from -DCHY_JMAX/-DCHY_KMAX/-DCHY_LMAX. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define J2 (CHY_JMAX + 2)
#define K2 (CHY_KMAX + 2)
#define L (CHY_LMAX)
#define VOL ((size_t)J2 * K2 * L)

struct { double indirectx, indirecty; double phi[VOL], rho[VOL], rhotot[VOL]; } pois_;
struct { int jreq, kzpol; double r[J2], z[K2], rhf[J2], zhf[K2]; double rof3n, zof3n; } grid_;
struct { double dtheta, pi, grav, bgden, gsoft; int kwfw; } blok6_;
struct { double tmass, enew, elost, edif, phichk; int klocat; } inside_;
struct { double coef[(size_t)J2 * K2 * (L / 2) * 2]; } coefs_;

void setbdy_(const int *, const int *);
void bdygen_(const int *, const int *, const double *);
void pot3_(const int *, const int *);
int chy_compat_status_(void);
void chy_compat_finalize_(void);

static int dump(const char *prefix, const char *ext, const double *a, size_t n)
{
    char path[1024];
    snprintf(path, sizeof path, "%s.%s", prefix, ext);
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    size_t w = fwrite(a, sizeof(double), n, f);
    fclose(f);
    return w != n;
}

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    FILE *f = fopen(argv[1], "rb");
    if (!f || fread(pois_.rho, sizeof(double), VOL, f) != VOL) return 3;
    fclose(f);
    /* grid of radhydro/io.f:194-203 with ROF3N = 1/JMAX, ZOF3N = 0.5/KMAX */
    grid_.rof3n = 1.0 / CHY_JMAX;
    grid_.zof3n = 0.5 / CHY_KMAX;
    for (int j = 0; j < J2; j++) {
        grid_.r[j] = (j - 1) * grid_.rof3n;
        grid_.rhf[j] = grid_.r[j] + grid_.rof3n / 2.0;
    }
    for (int k = 0; k < K2; k++) {
        grid_.z[k] = (k - 1) * grid_.zof3n;
        grid_.zhf[k] = grid_.z[k] + grid_.zof3n / 2.0;
    }
    blok6_.pi = 3.1415926535897932;
    blok6_.grav = 1.0;
    blok6_.dtheta = 2.0 * blok6_.pi / L;
    memset(pois_.phi, 0, sizeof pois_.phi);
    int ncall = 0, isym = 2, maxtrm = 10, npoint = 8, iprint = 1;
    double redge = 0.0;
    if (argc > 3 && strcmp(argv[3], "nosetup") == 0) {
        bdygen_(&maxtrm, &isym, &redge);
        int s1 = chy_compat_status_();
        pot3_(&npoint, &iprint);
        int s2 = chy_compat_status_();
        printf("status %d %d\n", s1, s2);
        return 0;
    }
    setbdy_(&ncall, &isym);
    bdygen_(&maxtrm, &isym, &redge);
    pot3_(&npoint, &iprint);
    int st = chy_compat_status_();
    printf("status %d\n", st);
    double inside[3] = {inside_.tmass, inside_.phichk, (double)inside_.klocat};
    int bad = dump(argv[2], "phi", pois_.phi, VOL) || dump(argv[2], "inside", inside, 3) ||
              dump(argv[2], "coef", coefs_.coef, (size_t)J2 * K2 * (L / 2) * 2);
    chy_compat_finalize_();
    return bad ? 4 : 0;
}

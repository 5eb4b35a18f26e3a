// report.cpp -- the text POT3 writes to unit 3 with IPRINT = 1
// (pot/pot3.f:402-418): PHAC(2:KMAX1) under FORMAT(1P11E11.3), then for
// LMAX > 8 the Fourier amplitudes and phases of row K = 2 under
// FORMAT(20X,I5,' COEFS=',1P8E12.3,/,25X,' PHASE=',0P8F12.2).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "chy_pot3.h"
#include "planimpl.h"

namespace {

void right(std::string &o, const std::string &s, int w)
{
    if ((int)s.size() > w) {
        o.append((size_t)w, '*');   // the field does not fit: asterisks, as Fortran prints
        return;
    }
    o.append((size_t)(w - (int)s.size()), ' ');
    o += s;
}

std::string special(double v)
{
    if (std::isnan(v)) return "NaN";
    return v < 0 ? "-Infinity" : "Infinity";
}

// 1PEw.3: one digit before the point, three after, exponent E+dd, or +ddd
// without the E for |exponent| > 99
void edit_e(std::string &o, double v, int w)
{
    if (!std::isfinite(v)) return right(o, special(v), w);
    char b[64];
    std::snprintf(b, sizeof b, "%.3E", v);
    std::string s(b);
    const size_t e = s.find('E');
    if (e != std::string::npos && s.size() - e - 2 > 2) s.erase(e, 1);
    right(o, s, w);
}

// 0PFw.2
void edit_f(std::string &o, double v, int w)
{
    if (!std::isfinite(v)) return right(o, special(v), w);
    char b[64];
    std::snprintf(b, sizeof b, "%.2f", v);
    right(o, b, w);
}

}  // namespace

extern "C" long long chy_plan_report(chy_plan *p, char *buf, long long cap)
{
    if (!p || (!buf && cap > 0) || cap < 0) return -CHY_ERR_ARG;
    const chy::HostPlan &hp = p->hp;
    const int J = hp.J, K = hp.K, L = hp.L, N = L / 2;
    const double *coef = p->w.coef;
    if (!coef) return -CHY_ERR_NOT_SETUP;   // COEF is not being written
    std::vector<double> phac((size_t)K + 2), cf(2 * 8 * ((size_t)J + 2), 0.0);
    const size_t J2 = (size_t)J + 2, plane = J2 * ((size_t)K + 2) * sizeof(double);
    const int nm = N < 8 ? N : 8;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(phac.data(), p->w.phac, phac.size() * sizeof(double), cudaMemcpyDeviceToHost);
    // COEF(1:J+2, 2, M, I), M = 1..8: one row of each (M, I) plane
    for (int i = 0; i < 2 && e == cudaSuccess; i++)
        e = cudaMemcpy2D(cf.data() + (size_t)i * 8 * J2, J2 * sizeof(double),
                         coef + J2 * 1 + (size_t)i * N * (plane / sizeof(double)), plane, J2 * sizeof(double), nm,
                         cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return -CHY_ERR_CUDA;
    std::string o = "PHAC(1:KMAX1):\n";
    int cnt = 0;
    for (int k = 2; k <= K + 1; k++) {
        edit_e(o, phac[k], 11);
        if (++cnt % 11 == 0) o += '\n';
    }
    if (cnt % 11 != 0) o += '\n';
    o += "Fourier amplitudes and phases:\n";
    if (L > 8) {
        char jb[16];
        for (int j = 2; j <= J; j++) {
            o.append(20, ' ');
            std::snprintf(jb, sizeof jb, "%5d", j);
            o += jb;
            o += " COEFS=";
            for (int m = 0; m < 8; m++) edit_e(o, cf[(size_t)m * J2 + (j - 1)], 12);
            o += '\n';
            o.append(25, ' ');
            o += " PHASE=";
            for (int m = 0; m < 8; m++) edit_f(o, cf[(size_t)(8 + m) * J2 + (j - 1)], 12);
            o += '\n';
        }
    }
    if (cap > 0) {
        const size_t n = o.size() < (size_t)cap - 1 ? o.size() : (size_t)cap - 1;
        std::memcpy(buf, o.data(), n);
        buf[n] = '\0';
    }
    return (long long)o.size();
}

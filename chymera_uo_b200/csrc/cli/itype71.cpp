// itype71.cpp -- the ITYPE=71 potential-only run (radhydro/io.f:151-229)
// on libchy_pot3.
//
//   chy_itype71 [--dir D] [--jmax J --kmax K --lmax L] [--hj HJ --hk HK]
//               [--precision blktri|fp64|mixed] [--literal gcc|r8] [--check-input]
//
// Reads D/fort.5 (radhydro/io.f:100-119: ITYPE must be 71; ITSTOP names the
// output) and D/fort.2 (io.f:157-166, list-directed: PINDEX, CON2, RRR2,
// OMCEN, DENCEN, TOVERW, ROF3N, ZOF3N, A1NEWZ, JREQ, KZPOL, then
// DENNY(HJ+2, HK+2) of the hscf model, column-major).  Builds the
// axisymmetric RHO(J,K,L) = max(DENNY(J,K), GRIDLIM*DENCEN) on J = 2..JMAX+1,
// K = 2..KMAX+1 (io.f:170-183, GRIDLIM = 1e-10 from headers/units.h:22), the
// grid of io.f:186-203, PI and GRAV = 1 (io.f:136-138), and runs
// SETBDY(0,2), BDYGEN(10,2,0), POT3(8,1) (io.f:212-218, MAXTRM and ISYM of
// radhydro/3dhyd-main.f:166-167).  Writes D/phi3d.<ITSTOP, 6 digits> as two
// unformatted sequential records, PHI then TIME (io.f:221-226; TIME is 0 in
// this run), with 4-byte record markers as gfortran writes them.  The
// reference's grid sizes are compile-time parameters (headers/hydroparam.h);
// here they are options with the same defaults (256, 128, 256; HJ = HK = 256).
// --check-input parses the inputs and prints a summary without a GPU.
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "chy_pot3.h"

namespace {

constexpr double kGridLim = 1.0e-10;   // headers/units.h:22

int die(const std::string &msg, int code = 2)
{
    std::fprintf(stderr, "chy_itype71: %s\n", msg.c_str());
    return code;
}

// Fortran list-directed values: separators are blanks, commas and line ends;
// "r*c" repeats c r times; D exponents are accepted.
class ListReader {
  public:
    explicit ListReader(std::istream &in) : in_(in) {}
    bool next(std::string *tok)
    {
        if (repeat_ > 0) {
            --repeat_;
            *tok = rep_val_;
            return true;
        }
        std::string t;
        int ch;
        while ((ch = in_.get()) != EOF && (std::isspace(ch) || ch == ',')) {}
        if (ch == EOF) return false;
        do {
            t.push_back((char)ch);
        } while ((ch = in_.get()) != EOF && !std::isspace(ch) && ch != ',');
        const size_t star = t.find('*');
        if (star != std::string::npos) {
            repeat_ = std::atol(t.substr(0, star).c_str()) - 1;
            rep_val_ = t.substr(star + 1);
            t = rep_val_;
        }
        *tok = t;
        return true;
    }
    bool real(double *v)
    {
        std::string t;
        if (!next(&t)) return false;
        for (char &c : t)
            if (c == 'D' || c == 'd') c = 'E';
        char *end = nullptr;
        *v = std::strtod(t.c_str(), &end);
        return end && *end == '\0';
    }
    bool integer(long *v)
    {
        double d;
        if (!real(&d)) return false;
        *v = std::lround(d);
        return true;
    }

  private:
    std::istream &in_;
    long repeat_ = 0;
    std::string rep_val_;
};

// One gfortran unformatted sequential record.
bool write_record(std::FILE *f, const void *data, size_t bytes)
{
    if (bytes > 0x7fffffffu) return false;
    const int32_t n = (int32_t)bytes;
    return std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(data, 1, bytes, f) == bytes && std::fwrite(&n, 4, 1, f) == 1;
}

}  // namespace

int main(int argc, char **argv)
{
    std::string dir = ".";
    int J = 256, K = 128, L = 256, HJ = 256, HK = 256, precision = CHY_PREC_FP64_BLKTRI, literal = CHY_LITERAL_GCC;
    bool check = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](const char *name) -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "chy_itype71: %s needs a value\n", name);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--dir") dir = val("--dir");
        else if (a == "--jmax") J = std::atoi(val("--jmax"));
        else if (a == "--kmax") K = std::atoi(val("--kmax"));
        else if (a == "--lmax") L = std::atoi(val("--lmax"));
        else if (a == "--hj") HJ = std::atoi(val("--hj"));
        else if (a == "--hk") HK = std::atoi(val("--hk"));
        else if (a == "--precision") {
            const std::string v = val("--precision");
            precision = v == "mixed" ? CHY_PREC_MIXED : v == "fp64" ? CHY_PREC_FP64 : CHY_PREC_FP64_BLKTRI;
        }
        else if (a == "--literal") literal = std::string(val("--literal")) == "r8" ? CHY_LITERAL_R8 : CHY_LITERAL_GCC;
        else if (a == "--check-input") check = true;
        else {
            std::fprintf(stderr, "chy_itype71: unknown option %s\n", a.c_str());
            return 2;
        }
    }
    if (J + 1 > HJ + 2 || K + 1 > HK + 2) return die("JMAX+1 / KMAX+1 exceed the hscf grid (HJ+2, HK+2)");

    // ---- fort.5 (radhydro/io.f:100-119): the run parameters
    std::ifstream f5(dir + "/fort.5");
    if (!f5) return die("cannot open fort.5");
    std::string line1, line2, line3;
    std::getline(f5, line1);
    std::getline(f5, line2);
    std::getline(f5, line3);
    long it[8] = {0};
    {
        // FORMAT(9(I6,1X)): fields of width 6 separated by one column
        for (int q = 0; q < 8; ++q) {
            const size_t at = (size_t)q * 7;
            if (at >= line3.size()) return die("fort.5 line 3: too few integers");
            it[q] = std::atol(line3.substr(at, 6).c_str());
        }
    }
    const long itstop = it[1], itype = it[4];
    if (itype != 71) return die("fort.5: ITYPE is " + std::to_string(itype) + ", this driver runs ITYPE=71");

    // ---- fort.2 (radhydro/io.f:157-166)
    std::ifstream f2(dir + "/fort.2");
    if (!f2) return die("cannot open fort.2");
    ListReader rd(f2);
    double hdr[9];
    long jreq = 0, kzpol = 0;
    for (double &h : hdr)
        if (!rd.real(&h)) return die("fort.2: bad header");
    if (!rd.integer(&jreq) || !rd.integer(&kzpol)) return die("fort.2: bad JREQ/KZPOL");
    const double dencen = hdr[4], rof3n = hdr[6], zof3n = hdr[7];
    const size_t hj2 = (size_t)HJ + 2, hk2 = (size_t)HK + 2;
    std::vector<double> denny(hj2 * hk2);
    for (double &d : denny)
        if (!rd.real(&d)) return die("fort.2: fewer than (HJ+2)(HK+2) density values");

    // ---- RHO (io.f:170-183) and the grid (io.f:186-203)
    const size_t J2 = (size_t)J + 2, K2 = (size_t)K + 2;
    std::vector<double> rho(J2 * K2 * L, 0.0), phi(J2 * K2 * L, 0.0);
    const double floor_ = kGridLim * dencen;
    for (int l = 0; l < L; ++l)
        for (size_t k = 1; k <= (size_t)K; ++k)
            for (size_t j = 1; j <= (size_t)J; ++j) {
                const double v = denny[j + hj2 * k];
                rho[j + J2 * (k + K2 * l)] = v < floor_ ? floor_ : v;
            }
    std::vector<double> r(J2), z(K2), rhf(J2), zhf(K2);
    for (size_t j = 0; j < J2; ++j) {
        r[j] = ((double)j - 1.0) * rof3n;
        rhf[j] = r[j] + rof3n / 2.0;
    }
    for (size_t k = 0; k < K2; ++k) {
        z[k] = ((double)k - 1.0) * zof3n;
        zhf[k] = z[k] + zof3n / 2.0;
    }
    if (check) {
        double mass = 0.0;
        for (double v : rho) mass += v;
        std::printf("ITYPE=71 ITSTOP=%ld JMAX=%d KMAX=%d LMAX=%d ROF3N=%.17g ZOF3N=%.17g DENCEN=%.17g "
                    "JREQ=%ld KZPOL=%ld sum(RHO)=%.17g\n",
                    itstop, J, K, L, rof3n, zof3n, dencen, jreq, kzpol, mass);
        return 0;
    }

    // ---- SETBDY(0,2), BDYGEN(10,2,0), POT3(8,1)
    chy_grid g;
    chy_grid_defaults(&g, J, K, L);
    g.rof3n = rof3n;
    g.zof3n = zof3n;
    g.r = r.data();
    g.z = z.data();
    g.rhf = rhf.data();
    g.zhf = zhf.data();
    g.pi = 3.1415926535897932;
    g.grav = 1.0;
    g.isym = 2;
    g.maxtrm = 10;
    g.redge = 0.0;
    g.npoint = 8;
    g.literal_kind = literal;
    chy_plan *plan = nullptr;
    int st = chy_plan_create(&g, precision, 1, &plan);
    chy_diag d{};
    // POT3(8, IPRINT=1): /COEFS/ for the unit-3 report (pot/pot3.f:402-418)
    std::vector<double> coef((size_t)(J + 2) * (K + 2) * (L / 2) * 2, 0.0);
    if (st == CHY_OK) st = chy_plan_set_coef_host(plan, coef.data());
    if (st == CHY_OK) st = chy_solve(plan, rho.data(), phi.data(), &d, CHY_PTR_HOST, nullptr);
    std::string report;
    if (st == CHY_OK) {
        const long long n = chy_plan_report(plan, nullptr, 0);
        if (n < 0) {
            st = (int)-n;
        } else {
            report.resize((size_t)n + 1);
            chy_plan_report(plan, &report[0], n + 1);
            report.resize((size_t)n);
        }
    }
    if (st != CHY_OK) {
        std::fprintf(stderr, "chy_itype71: %s: %s\n", chy_status_string(st), chy_last_error());
        chy_plan_destroy(plan);
        return 1;
    }
    chy_plan_destroy(plan);
    // unit 3 is not open yet in the reference's ITYPE=71 branch: gfortran's
    // default connection writes the report to fort.3
    {
        const std::string p3 = dir + "/fort.3";
        std::FILE *f3 = std::fopen(p3.c_str(), "w");
        if (!f3 || std::fwrite(report.data(), 1, report.size(), f3) != report.size()) {
            if (f3) std::fclose(f3);
            return die("cannot write " + p3, 1);
        }
        std::fclose(f3);
    }
    std::printf("TMASS=%.17g PHICHK=%.17g KLOCAT=%d\n", d.tmass, d.phichk, d.klocat);

    // ---- phi3d.NNNNNN (io.f:221-226)
    char name[32];
    std::snprintf(name, sizeof name, "phi3d.%06ld", itstop);
    const std::string path = dir + "/" + name;
    std::FILE *out = std::fopen(path.c_str(), "wb");
    const double time = 0.0;
    const bool ok = out && write_record(out, phi.data(), phi.size() * sizeof(double)) &&
                    write_record(out, &time, sizeof time);
    if (out) std::fclose(out);
    if (!ok) return die("cannot write " + path, 1);
    std::printf("wrote %s\n", path.c_str());
    return 0;
}

// pot3_common.cpp -- gfortran-callable SETBDY / BDYGEN / POT3 that run
// libchy_pot3 on the reference's COMMON blocks.
//
// A CHYMERA build links this object (compiled for its grid size) and
// -lchy_pot3 instead of pot/boundary.f, pot/pot3.f, pot/fft.f and
// pot/blktri.f; the call sites (radhydro/io.f:215-218, :1212-1215,
// :1359-1363, radhydro/3dhyd-main.f:475-477) stay as they are.  The COMMON
// layouts follow headers/globals.h with POT3JMAX = JMAX, POT3KMAX = KMAX:
//   /POIS/   indirectx, indirecty, PHI, RHO, RHOTOT (POT3JMAX2, POT3KMAX2, LMAX)
//   /GRID/   JREQ, KZPOL, R(POT3JMAX2), Z(POT3KMAX2), RHF, ZHF, ROF3N, ZOF3N
//   /BLOK6/  DTHETA, PI, GRAV, BGDEN, GSOFT, KWFW
//   /INSIDE/ TMASS, ENEW, ELOST, EDIF, PHICHK, KLOCAT   (pot/boundary.f:112)
//   /COEFS/  COEF(POT3JMAX2, POT3KMAX2, LMAX2, 2)       (pot/pot3.f:20)
//
// Compile-time sizes (required): -DCHY_JMAX=.. -DCHY_KMAX=.. -DCHY_LMAX=..
// Options: -DCHY_PARTICLE=1 solves for RHOTOT (pot/pot3.f:74-78);
//          -DCHY_PRECISION selects the mode solve: 2 (default) BLKTRI in the
//          reference's order, 0 the FP64 eigenbasis solver, 1 the
//          mixed-precision tensor-core path;
//          -DCHY_LITERAL_KIND=1 for -r8 / -fdefault-real-8 builds.
//
// Semantics.  SETBDY records that the boundary tables may be built (the
// reference fills /BDY/; here the tables live in a per-parameter plan that
// the first POT3 builds).  BDYGEN records MAXTRM, ISYM and REDGE; POT3 runs
// BDYGEN's and POT3's work in one solve, so the boundary cells of PHI are
// written by POT3 rather than between the two calls -- no reference caller
// reads PHI there.  /INSIDE/ TMASS, PHICHK, KLOCAT and /COEFS/ are filled as
// the reference fills them.  IPRINT's unit-3 report is not written.
// Failures do not stop the program (the reference STOPs, pot/boundary.f:990):
// they are reported on stderr and by CHY_COMPAT_STATUS(), and PHI is left as
// it was.  SETBDY may be called from every thread of a parallel region, as
// radhydro/io.f:212-216 does; the calls are serialised.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "chy_pot3.h"

#if !defined(CHY_JMAX) || !defined(CHY_KMAX) || !defined(CHY_LMAX)
#error "define CHY_JMAX, CHY_KMAX and CHY_LMAX (the reference's POT3JMAX, POT3KMAX, LMAX)"
#endif
#ifndef CHY_PARTICLE
#define CHY_PARTICLE 0
#endif
#ifndef CHY_PRECISION
#define CHY_PRECISION CHY_PREC_FP64_BLKTRI
#endif
#ifndef CHY_LITERAL_KIND
#define CHY_LITERAL_KIND CHY_LITERAL_GCC
#endif

namespace {
constexpr int kJ2 = CHY_JMAX + 2, kK2 = CHY_KMAX + 2, kL = CHY_LMAX;
constexpr size_t kVol = (size_t)kJ2 * kK2 * kL;
}  // namespace

extern "C" {
struct chy_common_pois {
    double indirectx, indirecty;
    double phi[kVol], rho[kVol], rhotot[kVol];
};
struct chy_common_grid {
    int jreq, kzpol;
    double r[kJ2], z[kK2], rhf[kJ2], zhf[kK2];
    double rof3n, zof3n;
};
struct chy_common_blok6 {
    double dtheta, pi, grav, bgden, gsoft;   // KWFW follows; not used here
};
struct chy_common_inside {
    double tmass, enew, elost, edif, phichk;
    int klocat;
};
struct chy_common_coefs {
    double coef[(size_t)kJ2 * kK2 * (kL / 2) * 2];
};
extern chy_common_pois pois_;
extern chy_common_grid grid_;
extern chy_common_blok6 blok6_;
extern chy_common_inside inside_;
extern chy_common_coefs coefs_;
}

namespace {

struct State {
    std::mutex mu;
    bool setbdy = false;
    int isym = 2, maxtrm = 10;
    double redge = 0.0;
    int status = CHY_OK;
    // one plan per (ISYM, MAXTRM, REDGE, NPOINT): the grid is fixed for a run
    std::map<std::tuple<int, int, double, int>, chy_plan *> plans;
};

State &state()
{
    static State s;
    return s;
}

void report(State &s, int status, const char *where)
{
    s.status = status;
    std::fprintf(stderr, "chy pot3 %s: %s: %s\n", where, chy_status_string(status), chy_last_error());
}

void drop_plans(State &s)
{
    for (auto &kv : s.plans) chy_plan_destroy(kv.second);
    s.plans.clear();
}

}  // namespace

extern "C" {

// SUBROUTINE SETBDY(NCALL, ISYM) -- pot/boundary.f:2
void setbdy_(const int *ncall, const int *isym)
{
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    (void)ncall;   // NCALL = 0 (first call) or IGRID (regrid): tables are rebuilt
    drop_plans(s);
    s.setbdy = true;
    s.isym = *isym;
    s.status = CHY_OK;
}

// SUBROUTINE BDYGEN(MAXTRM, ISYM, REDGE) -- pot/boundary.f:88
void bdygen_(const int *maxtrm, const int *isym, const double *redge)
{
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    if (!s.setbdy) {   // the reference stops here (BDYCHK, pot/boundary.f:311)
        s.status = CHY_ERR_NOT_SETUP;
        std::fprintf(stderr, "chy pot3 BDYGEN: SETBDY has not been called\n");
        return;
    }
    s.maxtrm = *maxtrm;
    s.isym = *isym;
    s.redge = *redge;
    s.status = CHY_OK;
}

// SUBROUTINE POT3(NPOINT, IPRINT) -- pot/pot3.f:15
void pot3_(const int *npoint, const int *iprint)
{
    (void)iprint;
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    if (!s.setbdy) {
        s.status = CHY_ERR_NOT_SETUP;
        std::fprintf(stderr, "chy pot3 POT3: SETBDY has not been called\n");
        return;
    }
    const auto key = std::make_tuple(s.isym, s.maxtrm, s.redge, *npoint);
    chy_plan *plan = nullptr;
    auto it = s.plans.find(key);
    if (it != s.plans.end()) {
        plan = it->second;
    } else {
        chy_grid g;
        chy_grid_defaults(&g, CHY_JMAX, CHY_KMAX, CHY_LMAX);
        g.rof3n = grid_.rof3n;
        g.zof3n = grid_.zof3n;
        g.r = grid_.r;
        g.z = grid_.z;
        g.rhf = grid_.rhf;
        g.zhf = grid_.zhf;
        g.pi = blok6_.pi;
        g.grav = blok6_.grav;
        g.isym = s.isym;
        g.maxtrm = s.maxtrm;
        g.redge = s.redge;
        g.npoint = *npoint;
        g.literal_kind = CHY_LITERAL_KIND;
        int st = chy_plan_create(&g, CHY_PRECISION, 1, &plan);
        if (st == CHY_OK) st = chy_plan_set_coef_host(plan, coefs_.coef);
        if (st != CHY_OK) {
            if (plan) chy_plan_destroy(plan);
            report(s, st, "POT3 setup");
            return;
        }
        s.plans[key] = plan;
    }
    chy_diag d;
    const double *rho = CHY_PARTICLE ? pois_.rhotot : pois_.rho;
    const int st = chy_solve(plan, rho, pois_.phi, &d, CHY_PTR_HOST, nullptr);
    if (st != CHY_OK) {
        report(s, st, "POT3");
        return;
    }
    inside_.tmass = d.tmass;
    inside_.phichk = d.phichk;
    inside_.klocat = d.klocat;
    s.status = CHY_OK;
}

// INTEGER FUNCTION CHY_COMPAT_STATUS() -- status of the last SETBDY / BDYGEN /
// POT3 call (0 = ok; the CHY_* codes of chy_pot3.h otherwise).  No reference
// counterpart: the reference stops instead.
int chy_compat_status_(void)
{
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    return s.status;
}

// SUBROUTINE CHY_COMPAT_FINALIZE() -- releases the device plans (no reference
// counterpart; optional at program end).
void chy_compat_finalize_(void)
{
    State &s = state();
    std::lock_guard<std::mutex> lk(s.mu);
    drop_plans(s);
    s.setbdy = false;
}

}  // extern "C"

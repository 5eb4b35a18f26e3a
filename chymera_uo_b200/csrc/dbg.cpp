// dbg.cpp -- host-only test hooks (include/chy_pot3_testing.h).
#include <cstring>
#include <string>
#include <vector>

#include "blk.h"
#include "chy_pot3_testing.h"
#include "plan.h"

using namespace chy;

extern "C" int chy_dbg_fft(int n, int isn, int literal_kind, double *a, double *b)
{
    FftSchedule s;
    int st = build_fft_schedule(n, isn, literal_kind == CHY_LITERAL_R8, s);
    if (st != CHY_OK) return st;
    fft_apply_host(s, a, b);
    return CHY_OK;
}

extern "C" int chy_dbg_realtr(int n, int isn, int literal_kind, double *a, double *b)
{
    FftSchedule s;
    int st = build_fft_schedule(n, isn, literal_kind == CHY_LITERAL_R8, s);
    if (st != CHY_OK) return st;
    realtr_apply_host(s, a, b);
    return CHY_OK;
}

template <class T>
static long long put(const std::vector<T> &v, double *out, long long cap)
{
    long long n = (long long)v.size();
    for (long long i = 0; i < n && i < cap; i++) out[i] = (double)v[i];
    return n;
}

extern "C" long long chy_dbg_table(const chy_grid *g, const char *name, double *out, long long cap)
{
    if (!g || !name || !out) return -CHY_ERR_ARG;
    HostPlan hp;
    std::string err;
    int st = build_host_plan(*g, hp, err);
    if (st != CHY_OK) return -st;
    const std::string n(name);
    if (n == "U") return put(hp.U, out, cap);
    if (n == "V") return put(hp.V, out, cap);
    if (n == "Qt") return put(hp.Qt, out, cap);
    if (n == "dsc") return put(hp.dsc, out, cap);
    if (n == "row_scales") return put(mixed_row_scales(hp), out, cap);
    if (n == "lam") return put(hp.lam, out, cap);
    if (n == "an") return put(hp.an, out, cap);
    if (n == "bn") return put(hp.bn, out, cap);
    if (n == "cn") return put(hp.cn, out, cap);
    if (n == "am") return put(hp.am, out, cap);
    if (n == "cm") return put(hp.cm, out, cap);
    if (n == "cc") return put(hp.cc, out, cap);
    if (n == "bm0") return put(hp.bm0, out, cap);
    if (n == "xlamm") return put(hp.xlamm, out, cap);
    if (n == "ring_term") return put(hp.ring_term, out, cap);
    if (n == "ring_dv") return put(hp.ring_dv, out, cap);
    if (n == "ring_rsph") return put(hp.ring_rsph, out, cap);
    if (n == "jk_split") return put(hp.jk_split, out, cap);
    if (n == "jk_bin") return put(hp.jk_bin, out, cap);
    if (n == "jk_hout") return put(hp.jk_hout, out, cap);
    if (n == "sub_start") return put(hp.sub_start, out, cap);
    if (n == "jk_sub") return put(hp.jk_sub, out, cap);
    if (n == "sweep") return put(mixed_sweep_table(hp), out, cap);
    if (n == "blk_roots" || n == "blk_cns") {
        BlkSchedule bs;
        if (build_blk_schedule(hp.an, hp.bn, hp.cn, hp.M, bs, err) != 0) return -CHY_ERR_EIGEN;
        return put(n == "blk_roots" ? bs.roots : bs.cns, out, cap);
    }
    if (n == "blk_bm") {
        std::vector<double> v((size_t)hp.L * hp.M);
        for (int l = 0; l < hp.L; l++) blk_mode_bm(hp, l, v.data() + (size_t)l * hp.M);
        return put(v, out, cap);
    }
    if (n == "blk_bm_table") return put(blk_bm_table(hp), out, cap);
    if (n == "umma_tiles") return put(mixed_operand_tiles(hp), out, cap);
    if (n == "scalars") {
        std::vector<double> v = {hp.sf1, hp.pig4, hp.cmmax, hp.ammin, hp.cnmax, (double)hp.nkeep,
                                 (double)hp.ncol, (double)(hp.sub_start.size() - 1)};
        return put(v, out, cap);
    }
    return -CHY_ERR_ARG;
}

extern "C" int chy_dbg_blktri(const chy_grid *g, int l, double *y)
{
    if (!g || !y) return CHY_ERR_ARG;
    HostPlan hp;
    std::string err;
    int st = build_host_plan(*g, hp, err);
    if (st != CHY_OK) return st;
    if (l < 0 || l >= hp.L) return CHY_ERR_ARG;
    BlkSchedule bs;
    st = build_blk_schedule(hp.an, hp.bn, hp.cn, hp.M, bs, err);
    if (st != 0) return st == 1 ? CHY_ERR_M_LT_2 : st == 2 ? CHY_ERR_N_NOT_POW2 : CHY_ERR_EIGEN;
    std::vector<double> bm(hp.M);
    blk_mode_bm(hp, l, bm.data());
    blk_solve_host(bs, hp.am.data(), bm.data(), hp.cm.data(), y);
    return CHY_OK;
}

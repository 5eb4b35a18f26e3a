// api.cu -- the C ABI of libchy_pot3 (include/chy_pot3.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "chy_pot3.h"
#include "chy_pot3_testing.h"
#include "planimpl.h"

using namespace chy;

namespace {

thread_local std::string g_last_error;
thread_local int g_last_cuda = 0;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where)
{
    g_last_cuda = (int)e;
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return CHY_ERR_CUDA;
}

#define CHY_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Packs host vectors into one device allocation (256-byte aligned pieces).
struct Packer {
    std::vector<char> host;
    size_t add(const void *p, size_t bytes)
    {
        size_t off = (host.size() + 255) & ~(size_t)255;
        host.resize(off + bytes);
        if (bytes) std::memcpy(host.data() + off, p, bytes);
        return off;
    }
    template <class T>
    size_t vec(const std::vector<T> &v) { return add(v.data(), v.size() * sizeof(T)); }
};

}  // namespace

// The calling thread's last-error message, for the other translation units
// (serve.cu); returns code.
int chy_internal_fail(int code, const char *msg) { return fail(code, msg); }

static int ensure_host_staging(chy_plan *p);

// getBinaryPosition's circular orbit (radhydro/ExternalRoutines.f:91-105):
// MUBIN = MASSBIN + MASS_STAR, OMEGABIN = SQRT(MUBIN/ABIN**3), RBIN = ABIN,
// and RCOM = RBIN - RBIN*MASS_STAR/MUBIN (pot/ExternalPot.f:15).
static int set_binary_orbit(chy_plan *p)
{
    StarDev &x = p->star;
    if (!x.binary) return CHY_OK;
    const double mu = x.mass_bin + x.mass_star, a = p->bin_a;
    const double omega = std::sqrt((mu) / (a * a * a));
    x.rbin = a;
    x.omega2 = omega * omega;
    x.rcom = x.rbin - x.rbin * x.mass_star / mu;
    return CHY_OK;
}


// The plan's arrays live on the device that was current at chy_plan_create;
// launching with another device current would hand them to the wrong GPU.
static int check_device(const chy_plan *p)
{
    int dev = -1;
    CHY_CUDA(cudaGetDevice(&dev));
    if (dev != p->device)
        return fail(CHY_ERR_ARG, "plan was created on device " + std::to_string(p->device) + ", device " +
                                     std::to_string(dev) + " is current");
    return CHY_OK;
}

extern "C" {

void chy_grid_defaults(chy_grid *g, int jmax, int kmax, int lmax)
{
    std::memset(g, 0, sizeof(*g));
    g->jmax = jmax;
    g->kmax = kmax;
    g->lmax = lmax;
    g->rof3n = 1.0 / jmax;
    g->zof3n = 0.5 / kmax;
    g->pi = 3.1415926535897932;
    g->grav = 1.0;
    g->isym = 2;
    g->maxtrm = 10;
    g->redge = 0.0;
    g->npoint = 8;
    g->literal_kind = CHY_LITERAL_GCC;
}

const char *chy_status_string(int s)
{
    switch (s) {
    case CHY_OK: return "ok";
    case CHY_ERR_M_LT_2: return "JMAX-1 < 2 (BLKTRI IERROR=1)";
    case CHY_ERR_N_NOT_POW2: return "KMAX-1 is not 2**k-1 (BLKTRI IERROR=2)";
    case CHY_ERR_EIGEN: return "vertical operator eigen decomposition failed (BLKTRI IERROR=4)";
    case CHY_ERR_IDIMY: return "leading dimension too small (BLKTRI IERROR=5)";
    case CHY_ERR_ARG: return "invalid argument";
    case CHY_ERR_DIMS: return "unsupported grid dimensions";
    case CHY_ERR_UNSUPPORTED: return "unsupported ISYM/MAXTRM/NPOINT";
    case CHY_ERR_NOT_SETUP: return "BDYGEN called before SETBDY";
    case CHY_ERR_CUDA: return "CUDA runtime error";
    case CHY_ERR_NOMEM: return "device allocation failed";
    case CHY_ERR_NOCONV: return "refinement did not converge";
    case CHY_ERR_TIMEOUT: return "a device-side bounded wait expired";
    case CHY_ERR_CAPACITY: return "batch larger than plan capacity";
    default: return "unknown status";
    }
}

const char *chy_last_error(void) { return g_last_error.c_str(); }
int chy_last_cuda_error(void) { return g_last_cuda; }

void chy_plan_destroy(chy_plan *p)
{
    if (!p) return;
    for (auto &set : p->ev)
        for (auto &e : set)
            if (e) cudaEventDestroy(e);
    cudaFree(p->d_tables);
    cudaFree(p->d_work);
    cudaFree(p->stage);
    cudaFree(p->coef_dev);
    for (int i = 0; i < chy_plan::kStageSlots; i++) {
        if (p->ev_in[i]) cudaEventDestroy(p->ev_in[i]);
        if (p->ev_done[i]) cudaEventDestroy(p->ev_done[i]);
        if (p->ev_out[i]) cudaEventDestroy(p->ev_out[i]);
    }
    if (p->ev_start) cudaEventDestroy(p->ev_start);
    if (p->s_h2d) cudaStreamDestroy(p->s_h2d);
    if (p->s_d2h) cudaStreamDestroy(p->s_d2h);
    cudaFreeHost(p->h_diag);
    chy_mixed_release(p);
    delete p;
}

int chy_plan_create(const chy_grid *g, int precision, int max_batch, chy_plan **out)
{
    if (!g || !out || max_batch < 1) return fail(CHY_ERR_ARG, "null descriptor/output or max_batch < 1");
    if (precision != CHY_PREC_FP64 && precision != CHY_PREC_MIXED && precision != CHY_PREC_FP64_BLKTRI)
        return fail(CHY_ERR_ARG, "unknown precision");
    *out = nullptr;
    chy_plan *p = new (std::nothrow) chy_plan();
    if (!p) return fail(CHY_ERR_NOMEM, "host allocation");
    std::string err;
    int st = build_host_plan(*g, p->hp, err);
    if (st != CHY_OK) {
        delete p;
        return fail(st, err);
    }
    if (precision == CHY_PREC_MIXED && !chy_mixed_supported(&p->hp)) {
        delete p;
        return fail(CHY_ERR_UNSUPPORTED, "mixed precision needs KMAX <= 128 and JMAX in 64..1024 (or a multiple of 16 up to 256)");
    }
    p->precision = precision;
    p->max_batch = max_batch;
    const HostPlan &hp = p->hp;
    BlkSchedule bs;
    if (precision == CHY_PREC_FP64_BLKTRI) {
        // BLKTRI(IFLG=0) (pot/blktri.f:13-46): COMPB's roots and the recorded
        // cyclic-reduction schedule
        st = build_blk_schedule(hp.an, hp.bn, hp.cn, hp.M, bs, err);
        if (st != 0) {
            delete p;
            return fail(st == 1 ? CHY_ERR_M_LT_2 : st == 2 ? CHY_ERR_N_NOT_POW2 : CHY_ERR_EIGEN, err);
        }
    }

    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (ce != cudaSuccess) {
        delete p;
        return cuda_fail(ce, "cudaGetDevice");
    }
    p->device = dev;

    // ---- tables
    Packer pk;
    size_t o_twf = pk.vec(hp.fwd.twc), o_twonf = pk.vec(hp.fwd.onc), o_permf = pk.vec(hp.fwd.perm), o_rtf = pk.vec(hp.fwd.rt);
    size_t o_twi = pk.vec(hp.inv.twc), o_twoni = pk.vec(hp.inv.onc), o_permi = pk.vec(hp.inv.perm), o_rti = pk.vec(hp.inv.rt);
    size_t o_cosm = pk.vec(hp.cosm), o_sinm = pk.vec(hp.sinm), o_fb = pk.vec(hp.fbasis), o_bcos = pk.vec(hp.bcos);
    size_t o_rhf = pk.vec(hp.rhf), o_zhf = pk.vec(hp.zhf), o_r = pk.vec(hp.r);
    size_t o_rs = pk.vec(hp.ring_sorted), o_sring = pk.vec(hp.sring), o_sub = pk.vec(hp.sub_start);
    size_t o_sterm = pk.vec(hp.sterm);
    size_t o_ct = pk.vec(hp.col_term), o_cp = pk.vec(hp.col_part), o_cm_ = pk.vec(hp.col_m), o_cl = pk.vec(hp.col_l);
    size_t o_jkj = pk.vec(hp.jk_j), o_jkk = pk.vec(hp.jk_k), o_jks = pk.vec(hp.jk_sub);
    size_t o_bin = pk.vec(hp.jk_bin), o_hout = pk.vec(hp.jk_hout);
    size_t o_am = pk.vec(hp.am), o_cmv = pk.vec(hp.cm), o_cc = pk.vec(hp.cc), o_bm0 = pk.vec(hp.bm0), o_xl = pk.vec(hp.xlamm);
    size_t o_an = pk.vec(hp.an), o_bn = pk.vec(hp.bn), o_cn = pk.vec(hp.cn);
    size_t o_U = pk.vec(hp.U), o_V = pk.vec(hp.V), o_lam = pk.vec(hp.lam);
    size_t o_bst = 0, o_bpg = 0, o_btk = 0, o_bsg = 0, o_bmt = 0;
    if (precision == CHY_PREC_FP64_BLKTRI) {
        o_bst = pk.vec(bs.steps);
        o_bpg = pk.vec(bs.progs);
        o_btk = pk.vec(bs.tasks);
        o_bsg = pk.vec(bs.stages);
        o_bmt = pk.vec(blk_bm_table(hp));
    }
    size_t o_ext = chy_mixed_pack_tables(&hp, &pk.host, precision == CHY_PREC_MIXED);
    p->table_bytes = pk.host.size();
    ce = cudaMalloc(&p->d_tables, p->table_bytes);
    if (ce == cudaSuccess) ce = cudaMemcpy(p->d_tables, pk.host.data(), p->table_bytes, cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) {
        chy_plan_destroy(p);
        return ce == cudaErrorMemoryAllocation ? fail(CHY_ERR_NOMEM, "tables") : cuda_fail(ce, "tables");
    }
    char *D = p->d_tables;
    DevTables &t = p->t;
    t.J = hp.J; t.K = hp.K; t.L = hp.L; t.N = hp.N; t.M = hp.M; t.NZ = hp.NZ;
    t.nring = hp.nring; t.nkeep = hp.nkeep; t.njk = hp.njk; t.ncol = hp.ncol;
    t.nsub = (int)hp.sub_start.size() - 1; t.ntrm = hp.ntrm; t.maxtrm = g->maxtrm;
    t.isyma = g->isym < 0 ? -g->isym : g->isym; t.npoint = hp.npoint;
    t.sf1 = hp.sf1; t.pig4 = hp.pig4; t.grav = g->grav;
    t.F1 = (t.isyma == 1) ? 1.0 : 0.0;
    t.cmmax = hp.cmmax; t.ammin = hp.ammin; t.cnmax = hp.cnmax;
    auto setfft = [&](FftDev &f, const FftSchedule &s, size_t otw, size_t oon, size_t operm, size_t ort) {
        f.n = s.n; f.isn = s.isn; f.nst = s.nstage; f.nh = s.nh; f.ncompact = s.ncompact;
        for (int i = 0; i < s.nstage; i++) { f.radix[i] = s.radix[i]; f.span[i] = s.span[i]; f.off[i] = s.off[i]; }
        f.twc = (const double *)(D + otw); f.onc = (const uint8_t *)(D + oon);
        f.perm = (const int *)(D + operm); f.rt = (const double *)(D + ort);
    };
    setfft(t.fwd, hp.fwd, o_twf, o_twonf, o_permf, o_rtf);
    setfft(t.inv, hp.inv, o_twi, o_twoni, o_permi, o_rti);
    if (!fft_shape_supported(t.fwd, hp.L) || !fft_shape_supported(t.inv, hp.L)) {
        chy_plan_destroy(p);
        return fail(CHY_ERR_DIMS, "no device transform for this LMAX");
    }
    t.cosm = (const double *)(D + o_cosm); t.sinm = (const double *)(D + o_sinm);
    t.bcos = (const double *)(D + o_bcos);
    t.fbasis = (const double *)(D + o_fb);
    t.rhf = (const double *)(D + o_rhf); t.zhf = (const double *)(D + o_zhf); t.r = (const double *)(D + o_r);
    t.ring_sorted = (const int *)(D + o_rs); t.sring = (const double *)(D + o_sring);
    t.sterm = (const double *)(D + o_sterm); t.srow = hp.srow;
    t.sub_start = (const int *)(D + o_sub);
    t.col_term = (const int *)(D + o_ct); t.col_part = (const int *)(D + o_cp);
    t.col_m = (const int *)(D + o_cm_); t.col_l = (const int *)(D + o_cl);
    t.jk_j = (const int *)(D + o_jkj); t.jk_k = (const int *)(D + o_jkk); t.jk_sub = (const int *)(D + o_jks);
    t.jk_bin = (const double *)(D + o_bin); t.jk_hout = (const double *)(D + o_hout);
    t.am = (const double *)(D + o_am); t.cm = (const double *)(D + o_cmv); t.cc = (const double *)(D + o_cc);
    t.bm0 = (const double *)(D + o_bm0); t.xlamm = (const double *)(D + o_xl);
    t.an = (const double *)(D + o_an); t.bn = (const double *)(D + o_bn); t.cn = (const double *)(D + o_cn);
    t.U = (const double *)(D + o_U); t.V = (const double *)(D + o_V); t.lam = (const double *)(D + o_lam);
    for (int i = 0; i < 11; i++) t.zx[i] = hp.zx[i];
    if (precision == CHY_PREC_FP64_BLKTRI) {
        t.blk.nvec = bs.nvec;
        t.blk.nstage = (int)bs.stages.size();
        t.blk.nblk = hp.L >= 32 ? hp.L / 32 : 1;
        t.blk.steps = (const BlkStep *)(D + o_bst);
        t.blk.progs = (const BlkProg *)(D + o_bpg);
        t.blk.tasks = (const BlkTask *)(D + o_btk);
        t.blk.stages = (const BlkStage *)(D + o_bsg);
        t.blk.bmt = (const double *)(D + o_bmt);
    }
    chy_mixed_bind_tables(p, D + o_ext);

    // ---- work space
    const size_t nX = (size_t)hp.L * hp.K * hp.J;
    const size_t nsub = hp.sub_start.size() - 1;
    Work &w = p->w;
    w.sX = nX;
    w.sW = precision == CHY_PREC_FP64 ? nX : 0;
    w.sC = precision == CHY_PREC_FP64 ? nX : 0;
    w.smom = (size_t)21 * hp.nring;
    w.ssub = nsub * 2 * hp.ncol;
    w.sscan = (nsub + 1) * 2 * hp.ncol;
    w.sphac = (size_t)hp.K + 2;
    w.sdiag = (size_t)kDiagPart + 2 * (size_t)hp.L;
    // every array starts on a 256-byte boundary (16-byte async copies read them)
    auto al = [](size_t n) { return (n + 31) & ~(size_t)31; };
    const bool blk = precision == CHY_PREC_FP64_BLKTRI;
    const size_t nbvec = blk ? al(blk_vector_doubles(t, max_batch)) : 0;
    const size_t nbscr = blk ? al(blk_scratch_doubles(t, max_batch, p->num_sms)) : 0;
    const size_t per = al(w.sX * max_batch) + al(w.sW * max_batch) + al(w.sC * max_batch) +
                       al(w.smom * max_batch) + al(w.ssub * max_batch) + al(w.sscan * max_batch) +
                       al(w.sphac * max_batch) + al(w.sdiag * max_batch) + nbvec + nbscr;
    size_t ext = chy_mixed_work_doubles(p);
    p->work_bytes = (per + ext) * sizeof(double) + 4096;
    ce = cudaMalloc(&p->d_work, p->work_bytes);
    if (ce != cudaSuccess) {
        chy_plan_destroy(p);
        return fail(CHY_ERR_NOMEM, "work space");
    }
    double *q = (double *)p->d_work;
    w.X = q; q += al(w.sX * max_batch);
    w.W = q; q += al(w.sW * max_batch);
    w.C = q; q += al(w.sC * max_batch);
    w.mom = q; q += al(w.smom * max_batch);
    w.sub = q; q += al(w.ssub * max_batch);
    w.scan = q; q += al(w.sscan * max_batch);
    w.phac = q; q += al(w.sphac * max_batch);
    w.diag = q; q += al(w.sdiag * max_batch);
    w.bvec = blk ? q : nullptr; q += nbvec;
    w.bscr = blk ? q : nullptr; q += nbscr;
    w.coef = nullptr;
    chy_mixed_bind_work(p, q);
    CHY_CUDA(cudaMemset(p->d_work, 0, p->work_bytes));
    p->nvol = (size_t)(hp.J + 2) * (hp.K + 2) * hp.L;
    CHY_CUDA(cudaMallocHost(&p->h_diag, sizeof(double) * kDiagPart * max_batch));
    *out = p;
    return CHY_OK;
}

int chy_plan_set_coef(chy_plan *p, double *coef_dev)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    p->w.coef = coef_dev;
    p->coef_host = nullptr;
    return CHY_OK;
}

int chy_plan_set_coef_host(chy_plan *p, double *coef_host)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    if (!coef_host) {
        p->coef_host = nullptr;
        p->w.coef = nullptr;
        return CHY_OK;
    }
    if (!p->coef_dev) {
        const HostPlan &hp = p->hp;
        const size_t n = (size_t)(hp.J + 2) * (hp.K + 2) * (hp.L / 2) * 2;
        if (cudaMalloc(&p->coef_dev, n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            p->coef_dev = nullptr;
            return fail(CHY_ERR_NOMEM, "COEF device buffer");
        }
        p->coef_bytes = n * sizeof(double);
    }
    p->coef_host = coef_host;
    p->w.coef = p->coef_dev;
    return CHY_OK;
}

int chy_plan_set_refine(chy_plan *p, int corrections)
{
    if (!p || corrections < 0 || corrections > 7) return fail(CHY_ERR_ARG, "corrections must be 0..7");
    if (corrections >= 2) {
        const int st = chy_mixed_ensure_iterate(p);
        if (st != CHY_OK) return fail(st, "FP64 iterate for two or more corrections");
    }
    p->refine = corrections;
    return CHY_OK;
}

int chy_plan_set_external(chy_plan *p, const chy_external *e)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    StarDev x{};
    if (e) {
        if (e->indirect && e->jmin < 1) return fail(CHY_ERR_ARG, "JMIN must be >= 1");
        const HostPlan &hp = p->hp;
        x.on = 1;
        x.indirect = e->indirect ? 1 : 0;
        x.jmin = e->jmin;
        x.mass = e->mass_star + e->tmassacc;
        x.mass_star = e->mass_star;
        // INDIRECTX/Y = RPSTAR*COS/SIN(PHI_STAR) (pot/ExternalPot.f:18-19)
        x.ix = e->rpstar * std::cos(e->phi_star);
        x.iy = e->rpstar * std::sin(e->phi_star);
        x.rof3n = hp.g.rof3n;
        x.zof3n = hp.g.zof3n;
        x.dtheta = hp.dtheta;
    }
    // the BINARY companion, if set, stays with the plan
    x.binary = p->star.binary;
    x.mass_bin = p->star.mass_bin;
    x.rbin = p->star.rbin;
    x.omega2 = p->star.omega2;
    x.rcom = p->star.rcom;
    x.mass_star = e ? e->mass_star : p->star.mass_star;
    p->star = x;
    return e ? set_binary_orbit(p) : CHY_OK;
}

int chy_plan_set_binary(chy_plan *p, const chy_binary *b)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    if (!b) {
        p->star.binary = 0;
        return CHY_OK;
    }
    if (!(b->a_bin > 0.0)) return fail(CHY_ERR_ARG, "binary separation must be positive");
    p->star.binary = 1;
    p->star.mass_bin = b->mass_bin;
    p->bin_a = b->a_bin;
    return set_binary_orbit(p);
}

int chy_plan_star_potential(chy_plan *p, double *starphi, int ptr_kind, void *stream)
{
    if (!p || !starphi) return fail(CHY_ERR_ARG, "null plan or output");
    if (!p->star.on) return fail(CHY_ERR_NOT_SETUP, "no external potential set on the plan");
    cudaStream_t s = (cudaStream_t)stream;
    if (ptr_kind == CHY_PTR_DEVICE) {
        CHY_CUDA(launch_star_fill(p->t, p->w, p->star, p->last_slot, starphi, s));
        p->launches += 1;
        return CHY_OK;
    }
    if (ptr_kind != CHY_PTR_HOST) return fail(CHY_ERR_ARG, "ptr_kind");
    int st = ensure_host_staging(p);
    if (st != CHY_OK) return st;
    // the first staging slot is free: every host-pointer solve call has
    // finished with it before returning
    CHY_CUDA(launch_star_fill(p->t, p->w, p->star, p->last_slot, p->stage, s));
    p->launches += 1;
    CHY_CUDA(cudaMemcpyAsync(starphi, p->stage, p->nvol * sizeof(double), cudaMemcpyDeviceToHost, s));
    CHY_CUDA(cudaStreamSynchronize(s));
    return CHY_OK;
}

// chy_source and chy_source_binary: SOURCE's loop nest with the BINARY
// build's terms when q.binary is set (the caller fills q's BINARY fields).
static int run_source(chy_plan *p, const chy_source_args *a, SourceDev &q, void *stream)
{
    if (!p || !a) return fail(CHY_ERR_ARG, "null plan or arguments");
    if (!a->rho || !a->phi || !a->omega || !a->p || !a->s || !a->t || !a->a)
        return fail(CHY_ERR_ARG, "null array");
    const int dst = check_device(p);
    if (dst != CHY_OK) return dst;
    const HostPlan &hp = p->hp;
    if (a->jmax < 1 || a->kmax < 1 || a->jmax > hp.J || a->kmax > hp.K)
        return fail(CHY_ERR_DIMS, "hydro JMAX/KMAX must be in 1..the plan's JMAX/KMAX");
    if (a->jmin < 1) return fail(CHY_ERR_ARG, "JMIN must be >= 1");
    q.J2h = a->jmax + 2;
    q.K2h = a->kmax + 2;
    q.J2p = hp.J + 2;
    q.K2p = hp.K + 2;
    q.L = hp.L;
    q.Jh = a->jmax;
    q.Kh = a->kmax;
    q.j0 = (a->jmin > 2 ? a->jmin : 2) - 1;   // JSTART (radhydro/source.f:33-37)
    q.delt = a->delt;
    q.dr = hp.g.rof3n;
    q.dz = hp.g.zof3n;
    q.dtheta = hp.dtheta;
    // reciprocals of power-of-two spacings are exact: multiplying by them
    // rounds like dividing
    auto pow2_inv = [](double d) {
        int e = 0;
        return std::isfinite(d) && d > 0.0 && std::frexp(d, &e) == 0.5 ? 1.0 / d : 0.0;
    };
    q.inv_dr = pow2_inv(q.dr);
    q.inv_2dr = pow2_inv(2.0 * q.dr);
    q.inv_dz = pow2_inv(q.dz);
    q.R = p->t.r;
    q.rho = a->rho; q.phi = a->phi; q.omega = a->omega; q.p = a->p;
    q.S = a->s; q.T = a->t; q.A = a->a;
    q.rhf = p->t.rhf;
    CHY_CUDA(launch_source(q, (cudaStream_t)stream));
    p->launches += 1;
    return CHY_OK;
}

int chy_source(chy_plan *p, const chy_source_args *a, void *stream)
{
    SourceDev q{};
    return run_source(p, a, q, stream);
}

int chy_source_binary(chy_plan *p, const chy_source_args *a, const chy_binary *b, double mass_star, const double *u,
                      void *stream)
{
    if (!b || !u) return fail(CHY_ERR_ARG, "null binary parameters or U");
    if (!(b->a_bin > 0.0)) return fail(CHY_ERR_ARG, "binary separation must be positive");
    SourceDev q{};
    q.binary = 1;
    // getBinaryPosition (radhydro/ExternalRoutines.f:101-102), as set_binary_orbit
    const double mu = b->mass_bin + mass_star;
    q.omega_bin = std::sqrt((mu) / (b->a_bin * b->a_bin * b->a_bin));
    q.u = u;
    return run_source(p, a, q, stream);
}

long long chy_plan_device_bytes(const chy_plan *p)
{
    if (!p) return 0;
    return (long long)(p->table_bytes + p->work_bytes + p->stage_bytes + p->coef_bytes + chy_mixed_iterate_bytes(p));
}

long long chy_plan_bytes_per_solve(const chy_plan *p)
{
    if (!p) return 0;
    const Work &w = p->w;
    size_t per = w.sX + w.sW + w.sC + w.smom + w.ssub + w.sscan + w.sphac + w.sdiag;
    if (p->precision == CHY_PREC_FP64_BLKTRI) per += (size_t)p->t.blk.nvec * p->t.M * p->t.L;
    return (long long)(per * sizeof(double));
}

// Folds the recorded event sets into stage_ms (waits for the last one).
static int drain_stage_events(chy_plan *p)
{
    for (size_t c = 0; c < p->ev_used; c++) {
        auto &set = p->ev[c];
        CHY_CUDA(cudaEventSynchronize(set[ST_NSTAGE]));
        for (int i = 0; i < ST_NSTAGE; i++) {
            float ms = 0.f;
            CHY_CUDA(cudaEventElapsedTime(&ms, set[i], set[i + 1]));
            p->stage_ms[i] += ms;
        }
        p->stage_calls++;
    }
    p->ev_used = 0;
    return CHY_OK;
}

int chy_plan_set_profiling(chy_plan *p, int on)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    const int st = drain_stage_events(p);
    p->profile = on != 0;
    for (double &v : p->stage_ms) v = 0.0;
    p->stage_calls = 0;
    return st;
}

int chy_plan_stage_times(chy_plan *p, double *ms, int n, long long *calls)
{
    if (!p || !ms) return fail(CHY_ERR_ARG, "null argument");
    const int st = drain_stage_events(p);
    if (st != CHY_OK) return -st;
    for (int i = 0; i < n && i < ST_NSTAGE; i++) ms[i] = p->stage_ms[i];
    if (calls) *calls = p->stage_calls;
    return ST_NSTAGE;
}

long long chy_plan_launch_count(const chy_plan *p) { return p ? p->launches : 0; }

}  // extern "C"

// Event sets kept before older ones are folded in (with a host wait).
static constexpr size_t kMaxEventSets = 4096;

// One launch sequence over nb solves whose caller buffers are in bp.
static int run_batch(chy_plan *p, const BatchPtrs &bp, int nb, cudaStream_t s)
{
    const DevTables &t = p->t;
    const bool prof = p->profile;
    cudaEvent_t *evs = nullptr;
    if (prof) {
        if (p->ev_used == kMaxEventSets) {
            const int st = drain_stage_events(p);
            if (st != CHY_OK) return st;
        }
        if (p->ev_used == p->ev.size()) {
            p->ev.emplace_back();
            for (auto &e : p->ev.back()) e = nullptr;
            for (auto &e : p->ev.back()) CHY_CUDA(cudaEventCreate(&e));
        }
        evs = p->ev[p->ev_used++].data();
    }
    auto mark = [&](int i) -> cudaError_t { return prof ? cudaEventRecord(evs[i], s) : cudaSuccess; };
    CHY_CUDA(mark(0));
    CHY_CUDA(launch_forward(t, bp, p->w, nb, s));
    CHY_CUDA(mark(1));
    CHY_CUDA(launch_bdy_sums(t, p->w, nb, s));
    CHY_CUDA(mark(2));
    CHY_CUDA(launch_bdy_synth(t, p->w, nb, s));
    CHY_CUDA(mark(3));
    int nl = 0;
    if (p->precision == CHY_PREC_FP64) {
        CHY_CUDA(launch_solve_fp64(t, p->w, nb, p->num_sms, s));
        nl = 3;
    } else if (p->precision == CHY_PREC_FP64_BLKTRI) {
        CHY_CUDA(launch_solve_blk(t, p->w, nb, p->num_sms, p->blk_warps, p->blk_ctas_per_sm, s, &nl));
    } else {
        int st = chy_mixed_solve(p, nb, s, &nl);
        if (st != CHY_OK) return st;
    }
    CHY_CUDA(mark(4));
    int ni = 0;
    if (p->star.on && p->star.indirect) {
        CHY_CUDA(launch_star_shift(t, bp, p->w, p->star, nb, s));
        ni = 2;
    }
    int nv = 0;
    CHY_CUDA(launch_inverse(t, bp, p->w, p->star, nb, s, &nv));
    CHY_CUDA(mark(5));
    p->launches += 1 + 2 + 1 + nl + ni + nv;
    p->last_slot = nb - 1;
    return CHY_OK;
}

static int fetch_diag(chy_plan *p, chy_diag *diag, int nb, int first, cudaStream_t s)
{
    if (!diag) return CHY_OK;
    CHY_CUDA(cudaMemcpy2DAsync(p->h_diag, sizeof(double) * kDiagPart, p->w.diag, sizeof(double) * p->w.sdiag,
                               sizeof(double) * kDiagPart, nb, cudaMemcpyDeviceToHost, s));
    CHY_CUDA(cudaStreamSynchronize(s));
    const int st = chy_mixed_collect(p, nb);
    if (st != CHY_OK) return fail(st, st == CHY_ERR_TIMEOUT ? "mode solve: bounded wait expired" : "mode solve readback");
    for (int i = 0; i < nb; i++) {
        chy_diag &d = diag[first + i];
        const double *h = p->h_diag + (size_t)kDiagPart * i;
        d.tmass = h[0];
        d.phichk = h[1];
        d.klocat = (int)h[2];
        d.indirectx = !p->star.on ? 0.0 : p->star.indirect ? h[kDiagStar] : p->star.ix;
        d.indirecty = !p->star.on ? 0.0 : p->star.indirect ? h[kDiagStar + 1] : p->star.iy;
        chy_mixed_fill_diag(p, i, &d);
    }
    return CHY_OK;
}

// Device staging slots and copy streams for host-pointer solves (first use).
static int ensure_host_staging(chy_plan *p)
{
    if (p->stage) return CHY_OK;
    // one solve per chunk: the copies (two grid volumes over PCIe) take several
    // times longer than the solve, so small chunks keep the pipeline's fill
    // and drain short and the solve stays hidden behind the copies
    const int c = 1;
    const size_t bytes = (size_t)chy_plan::kStageSlots * c * 2 * p->nvol * sizeof(double);
    if (cudaMalloc(&p->stage, bytes) != cudaSuccess) {
        cudaGetLastError();
        p->stage = nullptr;
        return fail(CHY_ERR_NOMEM, "host staging slots");
    }
    p->stage_bytes = bytes;
    p->stage_chunk = c;
    CHY_CUDA(cudaStreamCreateWithFlags(&p->s_h2d, cudaStreamNonBlocking));
    CHY_CUDA(cudaStreamCreateWithFlags(&p->s_d2h, cudaStreamNonBlocking));
    CHY_CUDA(cudaEventCreateWithFlags(&p->ev_start, cudaEventDisableTiming));
    for (int i = 0; i < chy_plan::kStageSlots; i++) {
        CHY_CUDA(cudaEventCreateWithFlags(&p->ev_in[i], cudaEventDisableTiming));
        CHY_CUDA(cudaEventCreateWithFlags(&p->ev_done[i], cudaEventDisableTiming));
        CHY_CUDA(cudaEventCreateWithFlags(&p->ev_out[i], cudaEventDisableTiming));
    }
    return CHY_OK;
}

extern "C" int chy_solve_batch(chy_plan *p, int n, const double *const *rho, double *const *phi,
                               chy_diag *diag, int ptr_kind, void *stream)
{
    if (!p || n < 0 || (n > 0 && (!rho || !phi))) return fail(CHY_ERR_ARG, "null plan or buffers");
    cudaStream_t s = (cudaStream_t)stream;
    const HostPlan &hp = p->hp;
    for (int i = 0; i < n; i++)
        if (!rho[i] || !phi[i]) return fail(CHY_ERR_ARG, "null rho/phi pointer");
    if (n > 0) {
        const int dst = check_device(p);
        if (dst != CHY_OK) return dst;
    }
    if (ptr_kind == CHY_PTR_DEVICE) {
        for (int first = 0; first < n;) {
            const int nb = std::min(std::min(n - first, p->max_batch), kMaxBatchPtrs);
            BatchPtrs bp{};
            for (int i = 0; i < nb; i++) { bp.rho[i] = rho[first + i]; bp.phi[i] = phi[first + i]; }
            int st = run_batch(p, bp, nb, s);
            if (st != CHY_OK) return st;
            st = fetch_diag(p, diag, nb, first, s);
            if (st != CHY_OK) return st;
            first += nb;
        }
        return CHY_OK;
    }
    if (ptr_kind != CHY_PTR_HOST) return fail(CHY_ERR_ARG, "ptr_kind");
    if (n == 0) return CHY_OK;
    int st = ensure_host_staging(p);
    if (st != CHY_OK) return st;
    // Three-stage pipeline over chunks of stage_chunk solves: copy in on
    // s_h2d, solve on the caller's stream, copy out on s_d2h.  A slot is
    // reused only after its previous copy out has finished.
    // with a host COEF destination, one solve per chunk (COEF is per solve)
    const int c = p->coef_host ? 1 : p->stage_chunk, R = chy_plan::kStageSlots;
    bool used[chy_plan::kStageSlots] = {};
    CHY_CUDA(cudaEventRecord(p->ev_start, s));
    CHY_CUDA(cudaStreamWaitEvent(p->s_h2d, p->ev_start, 0));
    for (int first = 0, chunk = 0; first < n; first += c, chunk++) {
        const int nb = std::min(c, n - first), slot = chunk % R;
        double *base = p->stage + (size_t)slot * c * 2 * p->nvol;
        if (used[slot]) CHY_CUDA(cudaStreamWaitEvent(p->s_h2d, p->ev_out[slot], 0));
        BatchPtrs bp{};
        const double *mapped[kMaxBatchPtrs] = {};
        for (int i = 0; i < nb; i++) {
            double *dr = base + (size_t)i * 2 * p->nvol, *df = dr + p->nvol;
            const double *hr = rho[first + i];
            CHY_CUDA(copy_rho_in(dr, hr, hp.J, hp.K, hp.L, p->s_h2d));
            // the cells the solve leaves alone start from the caller's values:
            // the external potential updates them, and the copy out returns
            // them with the rest of PHI.  From pinned (mapped) host memory a
            // kernel reads them below; otherwise the copy engine moves them
            mapped[i] = chy_internal_mapped_view(phi[first + i]);
            if (!mapped[i])
                CHY_CUDA(copy_phi_rim(df, phi[first + i], hp.J, hp.K, hp.L, cudaMemcpyHostToDevice, p->s_h2d));
            bp.rho[i] = dr;
            bp.phi[i] = df;
        }
        CHY_CUDA(cudaEventRecord(p->ev_in[slot], p->s_h2d));
        CHY_CUDA(cudaStreamWaitEvent(s, p->ev_in[slot], 0));
        for (int i = 0; i < nb; i++)
            if (mapped[i]) {
                CHY_CUDA(chy_internal_rim_in(bp.phi[i], mapped[i], hp.J, hp.K, hp.L, s));
                p->launches += 1;
            }
        // COEF cells the solve leaves alone (X1 = 0, pot/pot3.f:106) keep the
        // caller's values: the device buffer starts from the host array
        if (p->coef_host)
            CHY_CUDA(cudaMemcpyAsync(p->coef_dev, p->coef_host, p->coef_bytes, cudaMemcpyHostToDevice, s));
        st = run_batch(p, bp, nb, s);
        if (st != CHY_OK) return st;
        if (p->coef_host)
            CHY_CUDA(cudaMemcpyAsync(p->coef_host, p->coef_dev, p->coef_bytes, cudaMemcpyDeviceToHost, s));
        if (diag) {
            // diagnostics are read per chunk: this synchronises the pipeline
            st = fetch_diag(p, diag, nb, first, s);
            if (st != CHY_OK) return st;
        }
        CHY_CUDA(cudaEventRecord(p->ev_done[slot], s));
        CHY_CUDA(cudaStreamWaitEvent(p->s_d2h, p->ev_done[slot], 0));
        for (int i = 0; i < nb; i++) {
            CHY_CUDA(copy_phi_out(phi[first + i], bp.phi[i], hp.J, hp.K, hp.L, p->s_d2h));
            // the cells the external potential updated
            if (p->star.on)
                CHY_CUDA(copy_phi_rim(phi[first + i], bp.phi[i], hp.J, hp.K, hp.L, cudaMemcpyDeviceToHost, p->s_d2h));
        }
        CHY_CUDA(cudaEventRecord(p->ev_out[slot], p->s_d2h));
        used[slot] = true;
    }
    for (int i = 0; i < R; i++)
        if (used[i]) CHY_CUDA(cudaStreamWaitEvent(s, p->ev_out[i], 0));
    // a bounded wait that expired in any of these mode solves (with diag the
    // chunks have reported it already)
    int *err = diag ? nullptr : chy_mixed_host_error_word(p);
    if (err) {
        *err = 0;
        st = chy_mixed_read_error(p, err, s);
        if (st != CHY_OK) return fail(st, "error word readback");
    }
    CHY_CUDA(cudaStreamSynchronize(s));
    if (err && *err != 0) {
        *err = 0;
        return fail(CHY_ERR_TIMEOUT, "mode solve: a bounded wait expired; the affected modes of PHI are NaN");
    }
    return CHY_OK;
}

// ---------------------------------------------------------------------------
// chy_solve_multi: densities of several grids in one stream-ordered call
// ---------------------------------------------------------------------------
namespace {
constexpr int kMultiStreams = 8;
struct StreamPool {
    cudaStream_t streams[kMultiStreams] = {};
    cudaEvent_t join[kMultiStreams] = {};
    cudaEvent_t fork = nullptr;
    bool ready = false;
};
std::mutex g_pool_mu;
StreamPool g_pools[64];

// Per-device side streams and fork/join events, created on first use.
int stream_pool(StreamPool **out)
{
    int dev = 0;
    CHY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CHY_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_pool_mu);
    StreamPool &sp = g_pools[dev];
    if (!sp.ready) {
        CHY_CUDA(cudaEventCreateWithFlags(&sp.fork, cudaEventDisableTiming));
        for (int i = 0; i < kMultiStreams; i++) {
            CHY_CUDA(cudaStreamCreateWithFlags(&sp.streams[i], cudaStreamNonBlocking));
            CHY_CUDA(cudaEventCreateWithFlags(&sp.join[i], cudaEventDisableTiming));
        }
        sp.ready = true;
    }
    *out = &sp;
    return CHY_OK;
}
}  // namespace

extern "C" int chy_solve_multi(int n, chy_plan *const *plans, const double *const *rho, double *const *phi,
                               void *stream)
{
    if (n < 0 || (n > 0 && (!plans || !rho || !phi))) return fail(CHY_ERR_ARG, "null arrays");
    if (n == 0) return CHY_OK;
    // group the requests by plan, largest total volume first
    std::vector<chy_plan *> order;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < n; i++) {
        if (!plans[i] || !rho[i] || !phi[i]) return fail(CHY_ERR_ARG, "null plan or buffer in request list");
        const int dst = check_device(plans[i]);
        if (dst != CHY_OK) return dst;
        size_t g = 0;
        while (g < order.size() && order[g] != plans[i]) g++;
        if (g == order.size()) {
            order.push_back(plans[i]);
            members.emplace_back();
        }
        members[g].push_back(i);
    }
    std::vector<size_t> rank(order.size());
    for (size_t g = 0; g < rank.size(); g++) rank[g] = g;
    std::sort(rank.begin(), rank.end(), [&](size_t a, size_t b) {
        return order[a]->nvol * members[a].size() > order[b]->nvol * members[b].size();
    });
    cudaStream_t s = (cudaStream_t)stream;
    StreamPool *sp = nullptr;
    int st = stream_pool(&sp);
    if (st != CHY_OK) return st;
    int nstreams = kMultiStreams;   // grids in flight at once: the smallest any plan asks for
    for (chy_plan *p : order)
        if (p->streams > 0) nstreams = std::min(nstreams, p->streams);
    const int S = (int)std::min(order.size(), (size_t)nstreams);
    CHY_CUDA(cudaEventRecord(sp->fork, s));
    for (int i = 0; i < S; i++) CHY_CUDA(cudaStreamWaitEvent(sp->streams[i], sp->fork, 0));
    for (size_t r = 0; r < rank.size(); r++) {
        const size_t g = rank[r];
        chy_plan *p = order[g];
        const std::vector<int> &idx = members[g];
        cudaStream_t gs = sp->streams[r % S];
        const int per = std::min(p->chunk > 0 ? std::min(p->chunk, p->max_batch) : p->max_batch, kMaxBatchPtrs);
        for (size_t first = 0; first < idx.size();) {
            const int nb = (int)std::min(idx.size() - first, (size_t)per);
            BatchPtrs bp{};
            for (int i = 0; i < nb; i++) {
                bp.rho[i] = rho[idx[first + i]];
                bp.phi[i] = phi[idx[first + i]];
            }
            st = run_batch(p, bp, nb, gs);
            if (st != CHY_OK) return st;
            first += nb;
        }
    }
    for (int i = 0; i < S; i++) {
        CHY_CUDA(cudaEventRecord(sp->join[i], sp->streams[i]));
        CHY_CUDA(cudaStreamWaitEvent(s, sp->join[i], 0));
    }
    return CHY_OK;
}

// ---------------------------------------------------------------------------
// chy_autotune_multi: the launch schedule of a request set, picked by timing
// ---------------------------------------------------------------------------
namespace {
struct Schedule {
    int streams, chunk, mode_div, blk_warps, blk_cps;
};

void apply_schedule(const std::vector<chy_plan *> &plans, const Schedule &c)
{
    for (chy_plan *p : plans) {
        p->streams = c.streams;
        p->chunk = c.chunk;
        p->mode_ctas = std::max(1, p->num_sms / c.mode_div);
        p->blk_warps = c.blk_warps;
        p->blk_ctas_per_sm = c.blk_cps;
    }
}
}  // namespace

extern "C" int chy_plan_set_schedule(chy_plan *p, const chy_tune *c)
{
    if (!p || !c) return fail(CHY_ERR_ARG, "null plan or schedule");
    if (c->streams < 0 || c->streams > kMultiStreams || c->chunk < 0 || c->mode_ctas < 0 ||
        !blk_schedule_valid(c->blk_warps, c->blk_ctas_per_sm) || c->mode_kernel < 0 || c->mode_kernel > 2)
        return fail(CHY_ERR_ARG, "schedule out of range (streams 0..8, blk_warps 4/8/16, blk_warps * "
                                 "blk_ctas_per_sm <= 16, mode_kernel 0..2)");
    p->streams = c->streams;
    p->chunk = c->chunk;
    p->mode_ctas = c->mode_ctas;
    p->blk_warps = c->blk_warps;
    p->blk_ctas_per_sm = c->blk_ctas_per_sm;
    p->mode_kernel = c->mode_kernel;
    return CHY_OK;
}

extern "C" int chy_plan_get_schedule(const chy_plan *p, chy_tune *c)
{
    if (!p || !c) return fail(CHY_ERR_ARG, "null plan or schedule");
    std::memset(c, 0, sizeof *c);
    c->streams = p->streams;
    c->chunk = p->chunk;
    c->mode_ctas = p->mode_ctas;
    c->blk_warps = p->blk_warps;
    c->blk_ctas_per_sm = p->blk_ctas_per_sm;
    c->mode_kernel = p->mode_kernel;
    return CHY_OK;
}

extern "C" int chy_autotune_multi(int n, chy_plan *const *plans, const double *const *rho, double *const *phi,
                                  void *stream, int repeats, chy_tune *out)
{
    if (n <= 0 || !plans || !rho || !phi) return fail(CHY_ERR_ARG, "empty or null request set");
    if (repeats < 1) repeats = 3;
    std::vector<chy_plan *> uniq;
    bool any_mixed = false, any_blk = false;
    int max_batch = 1;
    for (int i = 0; i < n; i++) {
        if (!plans[i]) return fail(CHY_ERR_ARG, "null plan in request set");
        if (std::find(uniq.begin(), uniq.end(), plans[i]) == uniq.end()) uniq.push_back(plans[i]);
        any_mixed |= plans[i]->precision == CHY_PREC_MIXED;
        any_blk |= plans[i]->precision == CHY_PREC_FP64_BLKTRI;
        max_batch = std::max(max_batch, plans[i]->max_batch);
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CHY_CUDA(cudaEventCreate(&e0));
    CHY_CUDA(cudaEventCreate(&e1));
    auto measure = [&](const Schedule &c, double *ms) -> int {
        apply_schedule(uniq, c);
        int st = chy_solve_multi(n, plans, rho, phi, stream);   // warm-up
        for (int r = 0; r < repeats && st == CHY_OK; r++) {
            if (r == 0 && cudaEventRecord(e0, s) != cudaSuccess) return cuda_fail(cudaGetLastError(), "event");
            st = chy_solve_multi(n, plans, rho, phi, stream);
        }
        if (st != CHY_OK) return st;
        CHY_CUDA(cudaEventRecord(e1, s));
        CHY_CUDA(cudaEventSynchronize(e1));
        float f = 0.f;
        CHY_CUDA(cudaEventElapsedTime(&f, e0, e1));
        *ms = (double)f / repeats;
        return CHY_OK;
    };
    // coordinate descent from the default schedule over each knob's values
    Schedule best{kMultiStreams, 0, 1, 8, 2};
    double best_ms = 0.0, default_ms = 0.0;
    int st = measure(best, &best_ms), tried = 1;
    default_ms = best_ms;
    auto try_values = [&](auto set, const std::vector<int> &values) {
        for (int v : values) {
            if (st != CHY_OK) return;
            Schedule c = best;
            set(c, v);
            if (std::memcmp(&c, &best, sizeof c) == 0) continue;
            double ms = 0.0;
            st = measure(c, &ms);
            tried++;
            if (st == CHY_OK && ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    };
    if (uniq.size() > 1) try_values([](Schedule &c, int v) { c.streams = v; }, {4, 2, 1});
    if (max_batch > 1) try_values([](Schedule &c, int v) { c.chunk = v; }, {(max_batch + 1) / 2, (max_batch + 3) / 4});
    if (any_mixed) try_values([](Schedule &c, int v) { c.mode_div = v; }, {2, 4});
    if (any_blk) {
        for (const auto &wc : std::vector<std::pair<int, int>>{{16, 1}, {4, 4}, {8, 1}, {4, 2}}) {
            if (st != CHY_OK) break;
            Schedule c = best;
            c.blk_warps = wc.first;
            c.blk_cps = wc.second;
            double ms = 0.0;
            st = measure(c, &ms);
            tried++;
            if (st == CHY_OK && ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply_schedule(uniq, best);
    if (st != CHY_OK) return st;
    if (out) {
        out->streams = best.streams;
        out->chunk = best.chunk;
        out->mode_ctas = std::max(1, uniq[0]->num_sms / best.mode_div);
        out->blk_warps = best.blk_warps;
        out->blk_ctas_per_sm = best.blk_cps;
        out->mode_kernel = uniq[0]->mode_kernel;   // kept as set
        out->ms = best_ms;
        out->ms_default = default_ms;
        out->candidates = tried;
    }
    return CHY_OK;
}

int chy_internal_run_batch(chy_plan *p, const BatchPtrs &bp, int nb, cudaStream_t s) { return run_batch(p, bp, nb, s); }

const double *chy_internal_mapped_view(const double *host)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost && a.devicePointer ? static_cast<const double *>(a.devicePointer) : nullptr;
}

// PHI(:, KMAX+2, L) and PHI(JMAX+2, 1, L) of plane L = blockIdx.x, from the
// caller's mapped host array (reads cross PCIe) into the device copy.
__global__ void __launch_bounds__(256) k_phi_rim_in(double *dst, const double *src, int J, int K)
{
    const size_t J2 = (size_t)J + 2, plane = J2 * ((size_t)K + 2), base = (size_t)blockIdx.x * plane;
    const size_t top = base + J2 * ((size_t)K + 1);
    for (size_t j = threadIdx.x; j < J2; j += blockDim.x) dst[top + j] = src[top + j];
    if (threadIdx.x == 0) dst[base + J + 1] = src[base + J + 1];
}

cudaError_t chy_internal_rim_in(double *dev, const double *src, int J, int K, int L, cudaStream_t s)
{
    k_phi_rim_in<<<L, 256, 0, s>>>(dev, src, J, K);
    return cudaGetLastError();
}

extern "C" int chy_solve(chy_plan *p, const double *rho, double *phi, chy_diag *diag, int ptr_kind,
                         void *stream)
{
    const double *r[1] = {rho};
    double *f[1] = {phi};
    return chy_solve_batch(p, 1, r, f, diag, ptr_kind, stream);
}

// Test hook: copies a work array of batch slot 0 to the host (synchronous).
extern "C" long long chy_dbg_work(chy_plan *p, const char *name, double *out, long long cap)
{
    if (!p || !name || !out) return -CHY_ERR_ARG;
    const std::string n(name);
    const double *src = nullptr;
    size_t cnt = 0;
    if (n == "X") { src = p->w.X; cnt = p->w.sX; }
    else if (n == "mom") { src = p->w.mom; cnt = p->w.smom; }
    else if (n == "sub") { src = p->w.sub; cnt = p->w.ssub; }
    else if (n == "scan") { src = p->w.scan; cnt = p->w.sscan; }
    else if (n == "phac") { src = p->w.phac; cnt = p->w.sphac; }
    else if (n == "diag") { src = p->w.diag; cnt = p->w.sdiag; }
    else return -CHY_ERR_ARG;
    if ((long long)cnt > cap) cnt = (size_t)cap;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out, src, cnt * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return -cuda_fail(e, "chy_dbg_work");
    return (long long)cnt;
}

#include <unordered_map>

cudaError_t chy::ensure_smem(const void *kernel, size_t bytes)
{
    static std::mutex mu;
    static std::unordered_map<const void *, int> done[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    auto &m = done[dev & 63];
    auto it = m.find(kernel);
    if (it != m.end() && it->second >= (int)bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) m[kernel] = (int)bytes;
    return e;
}

// ---------------------------------------------------------------------------
// chy_solve_static: the FP64 device-pointer solve with its per-solve work
// space taken from one fixed, statically sized device array instead of the
// plan's allocation.  The call itself allocates nothing (no cudaMalloc, no
// cudaFree, no allocating library routine).  One array per device, shared by
// every plan: overlapping calls on the same device (from several streams or
// threads) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------
static constexpr size_t kStaticScratchBytes = (size_t)8 << 20;   // 8 MiB
static __device__ __align__(256) double g_static_scratch[kStaticScratchBytes / sizeof(double)];

namespace {
std::mutex g_static_mu;
double *g_static_ptr[64] = {};   // per device: address of g_static_scratch
}  // namespace

extern "C" int chy_solve_static(chy_plan *p, const double *rho, double *phi, void *stream)
{
    if (!p || !rho || !phi) return fail(CHY_ERR_ARG, "null plan or buffers");
    if (p->precision != CHY_PREC_FP64) return fail(CHY_ERR_UNSUPPORTED, "chy_solve_static runs FP64 plans only");
    // the plan's per-solve arrays, 256-byte aligned pieces, carved from the static array
    const Work &pw = p->w;
    auto al = [](size_t n) { return (n + 31) & ~(size_t)31; };
    const size_t need = al(pw.sX) + al(pw.sW) + al(pw.sC) + al(pw.smom) + al(pw.ssub) + al(pw.sscan) +
                        al(pw.sphac) + al(pw.sdiag);
    if (need * sizeof(double) > kStaticScratchBytes)
        return fail(CHY_ERR_CAPACITY, "chy_solve_static: this grid needs " + std::to_string(need * sizeof(double)) +
                                          " bytes of work space; the static scratch holds " +
                                          std::to_string(kStaticScratchBytes) + " bytes");
    int dev = 0;
    CHY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CHY_ERR_ARG, "device ordinal out of range");
    if (dev != p->device)
        return fail(CHY_ERR_ARG, "chy_solve_static: plan was created on device " + std::to_string(p->device) +
                                     ", device " + std::to_string(dev) + " is current");
    double *base = nullptr;
    {
        // first call on each device (with that device current): look the
        // array up once; later calls reuse the address, which stays valid
        // for the life of the process's context on that device (a
        // cudaDeviceReset would invalidate it)
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_ptr[dev]) {
            void *ptr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
            g_static_ptr[dev] = static_cast<double *>(ptr);
        }
        base = g_static_ptr[dev];
    }
    Work w = pw;   // strides
    double *q = base;
    w.X = q; q += al(pw.sX);
    w.W = q; q += al(pw.sW);
    w.C = q; q += al(pw.sC);
    w.mom = q; q += al(pw.smom);
    w.sub = q; q += al(pw.ssub);
    w.scan = q; q += al(pw.sscan);
    w.phac = q; q += al(pw.sphac);
    w.diag = q;
    w.coef = nullptr;   // /COEFS/ output only through chy_solve
    cudaStream_t s = (cudaStream_t)stream;
    // every call starts from zeroed work space, as the plan's own allocation does
    CHY_CUDA(cudaMemsetAsync(base, 0, need * sizeof(double), s));
    BatchPtrs bp{};
    bp.rho[0] = rho;
    bp.phi[0] = phi;
    const DevTables &t = p->t;
    CHY_CUDA(launch_forward(t, bp, w, 1, s));
    CHY_CUDA(launch_bdy_sums(t, w, 1, s));
    CHY_CUDA(launch_bdy_synth(t, w, 1, s));
    CHY_CUDA(launch_solve_fp64(t, w, 1, p->num_sms, s));
    int nv = 0;
    CHY_CUDA(launch_inverse(t, bp, w, StarDev{}, 1, s, &nv));   // POT3 alone
    p->launches += 1 + 2 + 1 + 3 + nv;
    return CHY_OK;
}

extern "C" int chy_dbg_mixed_kernel(const chy_plan *p) { return p ? chy_mixed_last_kernel(p) : -CHY_ERR_ARG; }

extern "C" int chy_dbg_mixed_probe(chy_plan *p, int polls)
{
    if (!p) return fail(CHY_ERR_ARG, "null plan");
    const int st = chy_dbg_mixed_probe_set(p, polls);
    return st == CHY_OK ? st : fail(st, "probe needs a mixed plan and polls >= 0");
}

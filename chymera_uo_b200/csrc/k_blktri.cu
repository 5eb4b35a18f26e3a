// k_blktri.cu -- POT3's mode solves in the reference's own algorithm and
// order: FISHPACK BLKTRI generalized cyclic reduction (pot/blktri.f:60-260),
// FP64, replayed from the schedule recorded on the host (blk.h).
//
// Work items are (solve, mode) pairs, 32 to a group: one lane of a warp per
// item.  Every item of a group runs the same stage/task/program sequence
// (the schedule does not depend on the mode), so a warp's lanes never
// diverge; only BM, the radial diagonal, differs between lanes.  Each item's
// vectors (Y(:,1..N) and the intermediate products, M doubles each) are
// stored lane-interleaved, [group][vector][j][lane], so every access of a
// warp is one contiguous 256-byte run.
//
// One CTA owns a group at a time and walks the stages; the tasks of a stage
// are independent PRDCT calls (or element-wise combinations) spread over the
// CTA's warps, with a barrier between stages.  A PRDCT call keeps its
// elimination multipliers D and partial solution W in per-warp scratch.
//
// This file is compiled with --fmad=false and uses IEEE division: every
// product, sum and quotient rounds as the reference's, so the modes equal
// the reference's BLKTRI output bit for bit.
#include "devplan.h"

namespace chy {

constexpr int kBlkLanes = 32;
constexpr int kBlkUnroll = 8;   // rows whose loads are issued ahead of the recurrence

// Y(j,k) = 4 pi G Xhat(j,k) - boundary folds (pot/pot3.f:212-224), in that
// order of operations.
__device__ __forceinline__ double blk_rhs(const DevTables &t, const double *Xl, int j, int k)
{
    double y = t.pig4 * Xl[(size_t)k * t.J + j];
    if (k == t.NZ - 1) y = y - t.cnmax * Xl[(size_t)t.NZ * t.J + j];
    if (j == t.M - 1) y = y - t.cmmax * Xl[(size_t)k * t.J + t.M];
    return y;
}

// X (mode-major) -> lane-interleaved right-hand sides Y(:,k+1) of every item
// of group g.  Grid (groups, NZ); a 32 x 32 tile per pass.
__global__ void __launch_bounds__(256) k_blk_gather(DevTables t, Work w, int nb)
{
    __shared__ double tile[kBlkLanes][kBlkLanes + 1];
    const int g = blockIdx.x, k = blockIdx.y, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int M = t.M, L = t.L;
    const BlkDev &d = t.blk;
    double *out = w.bvec + ((size_t)g * d.nvec + k) * (size_t)M * kBlkLanes;
    for (int j0 = 0; j0 < M; j0 += kBlkLanes) {
        for (int r = ty; r < kBlkLanes; r += 8) {
            const int item = g * kBlkLanes + r, b = item / L, l = item % L, j = j0 + tx;
            double v = 0.0;
            if (b < nb && j < M) v = blk_rhs(t, w.X + (size_t)b * w.sX + (size_t)l * t.K * t.J, j, k);
            tile[r][tx] = v;
        }
        __syncthreads();
        for (int jj = ty; jj < kBlkLanes; jj += 8) {
            const int j = j0 + jj;
            if (j < M) out[(size_t)j * kBlkLanes + tx] = tile[tx][jj];
        }
        __syncthreads();
    }
}

// Solved Y(:,k+1) of every item of group g -> interior of X.
__global__ void __launch_bounds__(256) k_blk_scatter(DevTables t, Work w, int nb)
{
    __shared__ double tile[kBlkLanes][kBlkLanes + 1];
    const int g = blockIdx.x, k = blockIdx.y, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int M = t.M, L = t.L;
    const BlkDev &d = t.blk;
    const double *in = w.bvec + ((size_t)g * d.nvec + k) * (size_t)M * kBlkLanes;
    for (int j0 = 0; j0 < M; j0 += kBlkLanes) {
        for (int jj = ty; jj < kBlkLanes; jj += 8) {
            const int j = j0 + jj;
            tile[tx][jj] = (j < M) ? in[(size_t)j * kBlkLanes + tx] : 0.0;
        }
        __syncthreads();
        for (int r = ty; r < kBlkLanes; r += 8) {
            const int item = g * kBlkLanes + r, b = item / L, l = item % L, j = j0 + tx;
            if (b < nb && j < M) w.X[(size_t)b * w.sX + (size_t)l * t.K * t.J + (size_t)k * t.J + j] = tile[r][tx];
        }
        __syncthreads();
    }
}

// One PRDCT call (pot/blktri.f:177-260) for the 32 items of a warp.  Vector
// pointers are already offset to the lane; consecutive rows are 32 apart.
__device__ __forceinline__ void blk_prdct(const BlkProg &pg, const BlkStep *__restrict__ steps,
                                          const double *__restrict__ X, double *__restrict__ Y,
                                          double *__restrict__ Wv, double *__restrict__ Dv,
                                          const double *__restrict__ bm, const double *am, const double *cm, int m)
{
    constexpr int S = kBlkLanes, U = kBlkUnroll;
    // entry: W = X or -X, Y = W, and Y = AA(NA) W when NA > 0 (:183-208)
#pragma unroll 8
    for (int j = 0; j < m; j++) {
        double v = X[(size_t)j * S];
        if (pg.neg) v = -v;
        Y[(size_t)j * S] = pg.pre ? pg.pre_coef * v : v;
    }
    for (int q = 0; q < pg.nsteps; q++) {
        const BlkStep sp = steps[pg.first + q];
        const double rt = sp.rt;
        // elimination from row M (:214-221)
        const double bl = bm[(size_t)(m - 1) * S] - rt;
        double dn = am[m - 1] / bl;
        double wn = Y[(size_t)(m - 1) * S] / bl;
        Dv[(size_t)(m - 1) * S] = dn;
        Wv[(size_t)(m - 1) * S] = wn;
        // rows m-2 .. 1 in chunks of U; the next chunk's loads are issued
        // before this chunk's recurrence runs
        double yv[U], bv[U], yn[U], bn[U];
        auto load_e = [&](int i0, double *ya, double *ba) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 - u;
                ya[u] = (i >= 1) ? Y[(size_t)i * S] : 0.0;
                ba[u] = (i >= 1) ? bm[(size_t)i * S] : 0.0;
            }
        };
        load_e(m - 2, yv, bv);
        for (int i0 = m - 2; i0 >= 1; i0 -= U) {
            load_e(i0 - U, yn, bn);
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 - u;
                if (i >= 1) {
                    const double den = bv[u] - rt - cm[i] * dn;
                    dn = am[i] / den;
                    wn = (yv[u] - cm[i] * wn) / den;
                    Dv[(size_t)i * S] = dn;
                    Wv[(size_t)i * S] = wn;
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                yv[u] = yn[u];
                bv[u] = bn[u];
            }
        }
        // row 1 (:222-228)
        const double den = bm[0] - rt - cm[0] * dn;
        double w = (den == 0) ? 1. : (Y[0] - cm[0] * wn) / den;
        // substitution (:229-231) fused with the right-hand-side update that
        // follows the pass: Y = W (:234-238), Y = Y + c W (:254-257),
        // Y = c W (:201-208)
        const int post = sp.post;
        const double c = sp.coef;
        const bool rd = post == BLK_AXPY;   // the update reads the pass's right-hand side
        auto put = [&](int j, double v, double y) {
            if (post == BLK_COPY) Y[(size_t)j * S] = v;
            else if (post == BLK_AXPY) Y[(size_t)j * S] = y + c * v;
            else if (post == BLK_SCALE) Y[(size_t)j * S] = c * v;
        };
        put(0, w, rd ? Y[0] : 0.0);
        double wv[U], dv[U], yw[U], wx[U], dx[U], yx[U];
        auto load_f = [&](int j0, double *wa, double *da, double *ya) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u;
                wa[u] = (j < m) ? Wv[(size_t)j * S] : 0.0;
                da[u] = (j < m) ? Dv[(size_t)j * S] : 0.0;
                ya[u] = (rd && j < m) ? Y[(size_t)j * S] : 0.0;
            }
        };
        load_f(1, wv, dv, yw);
        for (int j0 = 1; j0 < m; j0 += U) {
            load_f(j0 + U, wx, dx, yx);
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u;
                if (j < m) {
                    w = wv[u] - dv[u] * w;
                    put(j, w, yw[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                wv[u] = wx[u];
                dv[u] = dx[u];
                yw[u] = yx[u];
            }
        }
    }
}

// Persistent CTAs over groups; NW warps per CTA.  Dynamic shared memory
// holds AM and CM (2 M doubles).
template <int NW>
__global__ void __launch_bounds__(NW * 32) k_blk_solve(DevTables t, Work w, int ngroups)
{
    extern __shared__ double sm[];
    const BlkDev &d = t.blk;
    const int m = t.M, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *am = sm, *cm = sm + m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        am[i] = t.am[i];
        cm[i] = t.cm[i];
    }
    __syncthreads();
    const size_t vlen = (size_t)m * kBlkLanes;
    double *Wv = w.bscr + ((size_t)blockIdx.x * NW + warp) * 2 * vlen + lane;
    double *Dv = Wv + vlen;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        double *base = w.bvec + (size_t)g * d.nvec * vlen;
        const double *bm = d.bmt + (size_t)(g % d.nblk) * vlen + lane;
        for (int s = 0; s < d.nstage; s++) {
            const BlkStage st = d.stages[s];
            if (st.kind == BLK_TASK_PRDCT) {
                for (int i = warp; i < st.ntasks; i += NW) {
                    const BlkTask tk = d.tasks[st.first + i];
                    const BlkProg pg = d.progs[tk.prog];
                    blk_prdct(pg, d.steps, base + (size_t)tk.a * vlen + lane, base + (size_t)tk.out * vlen + lane,
                              Wv, Dv, bm, am, cm, m);
                }
            } else {
                const long long total = (long long)st.ntasks * (long long)vlen;
                for (long long e = threadIdx.x; e < total; e += blockDim.x) {
                    const BlkTask tk = d.tasks[st.first + (int)(e / (long long)vlen)];
                    const size_t r = (size_t)(e % (long long)vlen);
                    const double a = base[(size_t)tk.a * vlen + r];
                    const double b = tk.b < 0 ? 0.0 : base[(size_t)tk.b * vlen + r];
                    const double c = tk.c < 0 ? 0.0 : base[(size_t)tk.c * vlen + r];
                    // Y = W1 + W2 - Y (:106-108); W1 = Y - W1 - W2 (:157-159)
                    base[(size_t)tk.out * vlen + r] = (st.kind == BLK_TASK_SUMSUB) ? (a + b) - c : (a - b) - c;
                }
            }
            __syncthreads();
        }
    }
}

static int blk_groups(const DevTables &t, int nb) { return (nb * t.L + kBlkLanes - 1) / kBlkLanes; }

// Scratch holds two vectors per warp for any stage schedule the launch accepts:
// NW warps per CTA and up to ctas_per_sm CTAs per SM with NW * ctas_per_sm <= 16
// (at most 16 warps per SM, at most one CTA per group).
size_t blk_scratch_doubles(const DevTables &t, int max_batch, int num_sms)
{
    const int g = blk_groups(t, max_batch);
    return (size_t)16 * (g < num_sms ? g : num_sms) * 2 * (size_t)t.M * kBlkLanes;
}

size_t blk_vector_doubles(const DevTables &t, int nb)
{
    return (size_t)blk_groups(t, nb) * t.blk.nvec * (size_t)t.M * kBlkLanes;
}

bool blk_schedule_valid(int nw, int ctas_per_sm)
{
    return (nw == 4 || nw == 8 || nw == 16) && ctas_per_sm >= 1 && nw * ctas_per_sm <= 16;
}

template <int NW>
static cudaError_t blk_launch(const DevTables &t, const Work &w, int ngroups, int ctas, cudaStream_t s)
{
    const size_t smem = (size_t)2 * t.M * sizeof(double);
    cudaError_t e = ensure_smem((const void *)k_blk_solve<NW>, smem);
    if (e != cudaSuccess) return e;
    k_blk_solve<NW><<<ctas, NW * 32, smem, s>>>(t, w, ngroups);
    return cudaGetLastError();
}

cudaError_t launch_solve_blk(const DevTables &t, const Work &w, int nb, int num_sms, int nw, int ctas_per_sm,
                             cudaStream_t s, int *launches)
{
    if (!blk_schedule_valid(nw, ctas_per_sm)) return cudaErrorInvalidValue;
    const int ngroups = blk_groups(t, nb);
    // one CTA per group at most; nw * ctas_per_sm <= 16 keeps the warps within
    // the scratch (16 per SM, no more than 16 per group)
    const int cap = ctas_per_sm * num_sms, ctas = ngroups < cap ? ngroups : cap;
    k_blk_gather<<<dim3(ngroups, t.NZ), 256, 0, s>>>(t, w, nb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (nw == 4) e = blk_launch<4>(t, w, ngroups, ctas, s);
    else if (nw == 8) e = blk_launch<8>(t, w, ngroups, ctas, s);
    else e = blk_launch<16>(t, w, ngroups, ctas, s);
    if (e != cudaSuccess) return e;
    k_blk_scatter<<<dim3(ngroups, t.NZ), 256, 0, s>>>(t, w, nb);
    if (launches) *launches = 3;
    return cudaGetLastError();
}

}  // namespace chy

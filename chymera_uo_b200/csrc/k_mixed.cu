// k_mixed.cu -- mixed-precision mode solve on the 5th-generation tensor cores.
//
// Every azimuthal mode's block-tridiagonal system (pot/pot3.f:201-248) is
// solved by FP64 iterative refinement around an approximate FP32/FP16 solver:
//     x_0 = 0;  r_i = Y - A_m x_i (FP64);  x_{i+1} = x_i + S(r_i)
// S applies the vertical eigenbasis and radial sweeps of the FP64 path
// (see k_solve.cu) with
//   * both vertical transforms on tcgen05 tensor cores: operands as FP16
//     hi/lo pairs scaled by powers of two, three MMA passes (hi*hi + hi*lo +
//     lo*hi) accumulated in FP32 in tensor memory -- about 22 bits;
//   * the radial tridiagonal sweeps in FP32 on the accumulator rows, read and
//     written in tensor memory, two threads per system (top-down and
//     bottom-up elimination meeting in the middle).
// The residual, the update of x and the final result stay FP64, so the
// refined solution converges to the FP64 solution of the same operator.
//
// One CTA owns one mode at a time (persistent over (solve, mode) items) and
// keeps the mode's operand tiles in shared memory and its accumulators in
// tensor memory; only Y, x and the eigenbasis tiles move through L2.
// No TMA multicast is used anywhere.  Every wait is bounded: on a timeout the
// kernel records an error word, stops issuing work, releases its tensor
// memory and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "planimpl.h"

using namespace chy;

namespace {

constexpr int kTiles = 128;         // MMA M and K extent (vertical index, padded)
constexpr int kMaxN = 256;          // MMA N extent (radial index, padded)
constexpr int kAImg = 2 * kTiles * kTiles * 2;   // hi + lo FP16 tile bytes (64 KB)
constexpr float kAScale = 4096.0f;  // eigenbasis tiles are stored times 2^12
constexpr long long kSpinLimit = 1ll << 26;

// Byte offset of element (row r, k) in a K-major, 128-byte-swizzled FP16
// operand tile with R rows and K = 128 (two 64-element row chunks).  Chunk c
// occupies R*128 bytes; within it row r is at r*128 and its 16-byte granule
// g is stored at g ^ (r % 8).
__host__ __device__ inline uint32_t kmaj_off(int r, int k, int R)
{
    const int chunk = k >> 6, kk = k & 63;
    return (uint32_t)(chunk * (R * 128) + r * 128 + (((kk >> 3) ^ (r & 7)) << 4) + ((kk & 7) << 1));
}

}  // namespace

struct MixedDev {
    const uint8_t *aimg;        // [U hi, U lo, V hi, V lo] swizzled tiles (2^12 scaled)
    const float *lam;           // [128]
    double *xbuf;               // [nb][L][K][J] FP64 iterate
    size_t sxb;
    double *corr;               // [nb][L][8][2] per mode: sum delta^2, sum x^2
    size_t scorr;
    int *err;                   // error word
    int nit;                    // approximate solves (1 + corrections)
    int ntile;                  // MMA N = J rounded up to 64 (<= 256)
};

struct MixedState {
    size_t o_aimg = 0, o_lam = 0;   // offsets into the packed table image
    MixedDev dev{};
    double *h_corr = nullptr;       // pinned [max_batch][L][8][2]
    int *h_err = nullptr;           // pinned
};

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    // start >> 4, LBO = 1 (unused for swizzled K-major), SBO = 1024 B >> 4,
    // version 1 (bit 46), layout SWIZZLE_128B (2 at bits 61-63)
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes));
}

// bounded wait on phase `parity`; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tm_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tm_st32(uint32_t taddr, const float *v)
{
    uint32_t r[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) r[i] = __float_as_uint(v[i]);
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tm_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tm_st16(uint32_t taddr, const float *v)
{
    uint32_t r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = __float_as_uint(v[i]);
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// power-of-two scale that maps max|v| below 2^14
__device__ __forceinline__ float pow2_scale(float vmax)
{
    if (!(vmax > 0.0f) || !isfinite(vmax)) return 1.0f;
    int e;
    frexpf(vmax, &e);
    return ldexpf(1.0f, 14 - e);
}

// Writes the FP16 hi/lo split of v (already scaled) for element (row, k).
__device__ __forceinline__ void put_split(uint8_t *hi, uint8_t *lo, int row, int k, int R, float v)
{
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    const uint32_t o = kmaj_off(row, k, R);
    *reinterpret_cast<__half *>(hi + o) = h;
    *reinterpret_cast<__half *>(lo + o) = l;
}

// Three-pass FP16 hi/lo product of the A tile (hi at sA, lo at sA + 32 KB)
// and the B tile (hi at sBh, lo at sBh + NT*256) into TMEM columns [0, NT):
// D = Ahi Bhi + Ahi Blo + Alo Bhi, K = 128 in eight 16-wide steps.  Issued by
// one thread; completion is signalled on bar.
__device__ __forceinline__ void gemm_issue(uint32_t tmem, const uint8_t *sA, const uint8_t *sBh, int NT,
                                           uint32_t idesc, uint64_t *bar)
{
    tc_fence_after();
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sBh);
    const uint32_t a_lo = kTiles * kTiles * 2, b_lo = (uint32_t)NT * 256;
    const uint32_t pa[3] = {0u, 0u, a_lo}, pb[3] = {0u, b_lo, 0u};
#pragma unroll
    for (int pass = 0; pass < 3; ++pass)
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const uint32_t ao = a0 + pa[pass] + (uint32_t)(kk >> 2) * (kTiles * 128) + (uint32_t)(kk & 3) * 32;
            const uint32_t bo = b0 + pb[pass] + (uint32_t)(kk >> 2) * ((uint32_t)NT * 128) + (uint32_t)(kk & 3) * 32;
            umma_f16(tmem, umma_desc(ao), umma_desc(bo), idesc, (pass | kk) ? 1u : 0u);
        }
    umma_commit(bar);
}

}  // namespace

// ---------------------------------------------------------------------------
// The fused per-mode solver
// ---------------------------------------------------------------------------
// Shared memory: A tile (64 KB: hi, lo), B tile (ntile*512 B: hi, lo),
// FP64 stencil rows, FP32 sweep coefficients, reduction scratch, barriers.
struct MixedSmem {
    static constexpr size_t a = 0;
    static constexpr size_t b = kAImg;
    // the B region doubles as the residual/update staging area (>= 72 KB)
    __host__ __device__ static size_t breg(int nt) { return (size_t)nt * 512 > 73728 ? (size_t)nt * 512 : 73728; }
    __host__ __device__ static size_t tables(int nt) { return b + breg(nt); }
    __host__ __device__ static size_t bytes(int nt) { return tables(nt) + 22 * 1024; }
};

__global__ void __launch_bounds__(256, 1) k_mode_mixed(DevTables t, Work w, MixedDev x, int nb)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NT = x.ntile, M = t.M, NZ = t.NZ, J = t.J, K = t.K;
    uint8_t *sA = sm + MixedSmem::a;
    uint8_t *sBh = sm + MixedSmem::b, *sBl = sBh + (size_t)NT * 256;
    double *d_am = reinterpret_cast<double *>(sm + MixedSmem::tables(NT));   // [256]
    double *d_cm = d_am + 256, *d_bm = d_cm + 256;                             // [256] each
    double *d_an = d_bm + 256, *d_bn = d_an + 128, *d_cn = d_bn + 128;         // [128] each
    float *f_am = reinterpret_cast<float *>(d_cn + 128), *f_cm = f_am + 256, *f_bm = f_cm + 256;
    float *f_lam = f_bm + 256;                                                 // [128]
    float *f_red = f_lam + 128;                                                // [8]
    double *d_red = reinterpret_cast<double *>(f_red + 8);                     // [16]
    float *f_xch = reinterpret_cast<float *>(d_red + 16);                      // [128][4]
    uint64_t *bar_mma = reinterpret_cast<uint64_t *>(f_xch + 512);
    uint64_t *bar_a = bar_mma + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_a + 1);
    int *s_flag = reinterpret_cast<int *>(tmem_slot + 1);

    // ---- setup: tensor memory (all 512 columns), barriers, m-independent tables
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar_mma, 1);
        mbar_init(bar_a, 1);
        *s_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int j = tid; j < 256; j += blockDim.x) {
        d_am[j] = j < M ? t.am[j] : 0.0;
        d_cm[j] = j < M ? t.cm[j] : 0.0;
        f_am[j] = (float)d_am[j];
        f_cm[j] = (float)d_cm[j];
    }
    for (int k = tid; k < 128; k += blockDim.x) {
        d_an[k] = k < NZ ? t.an[k] : 0.0;
        d_bn[k] = k < NZ ? t.bn[k] : 0.0;
        d_cn[k] = k < NZ ? t.cn[k] : 0.0;
        f_lam[k] = x.lam[k];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int kq = 32 * (warp & 3) + lane;     // TMEM lane this thread owns
    const int jh = warp >> 2;                  // which half of the columns
    const int NH = NT / 2;                     // columns per half (multiple of 8)
    // MMA: kind::f16, A/B FP16 K-major, D FP32, M = 128, N = NT
    const uint32_t idesc = (1u << 4) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    uint32_t ph_mma = 0, ph_a = 0;
    bool failed = false;

    const long long items = (long long)nb * t.L;
    if (tid == 0 && blockIdx.x < items) {
        mbar_expect_tx(bar_a, kAImg);
        bulk_g2s(sA, x.aimg, kAImg, bar_a);   // U for the first transform
    }
    bool a_inflight = blockIdx.x < items;

    auto wait_all = [&](uint64_t *bar, uint32_t &ph) {
        bool ok = mbar_wait(bar, ph);
        ph ^= 1u;
        if (!ok) *s_flag = 1;
        __syncthreads();
        return *s_flag == 0;
    };
    auto issue_gemm = [&]() {
        if (tid == 0) gemm_issue(tmem, sA, sBh, NT, idesc, bar_mma);
    };

    for (long long item = blockIdx.x; item < items && !failed; item += gridDim.x) {
        const int b = (int)(item / t.L), l = (int)(item % t.L);
        const int m = l <= t.N ? l : l - t.N;
        const double xl2 = 2.0 * (t.xlamm[m] - 1.0);
        // BM_m (pot/pot3.f:226-230) for the FP64 residual, and for the FP32
        // sweeps the diagonal excess g = BM + AM + CM formed directly (no
        // cancellation): 2(cos m dtheta - 1) C(j), plus the axis term at j = 0
        // and -CMMAX at j = M-1
        for (int j = tid; j < 256; j += blockDim.x) {
            double bm = 0.0, gm = 0.0;
            if (j < M) {
                const double axis = (((m & 1) ? -1.0 : 1.0) - 1.0) * t.ammin;
                bm = t.bm0[j] + xl2 * t.cc[j];
                gm = xl2 * t.cc[j];
                if (j == 0) { bm = t.bm0[0] + axis + xl2 * t.cc[0]; gm = axis + gm; }
                if (j == M - 1) gm = gm - t.cmmax;
            }
            d_bm[j] = bm;
            f_bm[j] = (float)gm;
        }
        double *Xl = w.X + (size_t)b * w.sX + (size_t)l * K * J;
        double *xl = x.xbuf + (size_t)b * x.sxb + (size_t)l * K * J;
        double *cr = x.corr + (size_t)b * x.scorr + (size_t)l * 16;
        __syncthreads();

        for (int it = 0; it < x.nit && !failed; ++it) {
            const bool last = it == x.nit - 1;
            // ---- residual r = Y - A_m x (FP64) -> TMEM cols [256, 256+NT) as FP32.
            // Staged in 32-column chunks through the B-tile region (unused until
            // the split below) so global rows are read coalesced: sY[k][jj]
            // (stride 33) and the iterate with a one-cell halo (stride 35).
            // Out-of-range neighbours are staged as 0; their stencil
            // coefficients (AN(1), CN(KMAX-1), AM(1), CM(JMAX-1)) are 0 too.
            float rmax = 0.0f;
            {
                double *sY = reinterpret_cast<double *>(sBh);
                double *sXs = sY + 128 * 33;
                for (int c0 = 0; c0 < NT; c0 += 32) {
                    __syncthreads();
                    for (int i = tid; i < 128 * 32; i += 256) {
                        const int k = i >> 5, jj = i & 31, j = c0 + jj;
                        double y = 0.0;
                        if (j < M && k < NZ) {
                            y = t.pig4 * Xl[(size_t)k * J + j];
                            if (k == NZ - 1) y = y - t.cnmax * Xl[(size_t)NZ * J + j];
                            if (j == M - 1) y = y - t.cmmax * Xl[(size_t)k * J + M];
                        }
                        sY[k * 33 + jj] = y;
                    }
                    if (it > 0) {
                        for (int i = tid; i < 130 * 34; i += 256) {
                            const int kk = i / 34 - 1, jj = i % 34 - 1, j = c0 + jj;
                            sXs[(kk + 1) * 35 + (jj + 1)] =
                                (kk >= 0 && kk < NZ && j >= 0 && j < M) ? xl[(size_t)kk * J + j] : 0.0;
                        }
                    }
                    __syncthreads();
                    float v[16];
                    const int k = kq, jb = jh * 16;
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int jj = jb + u, j = c0 + jj;
                        double r = sY[k * 33 + jj];
                        if (it > 0 && j < M && k < NZ) {
                            const double *xr = sXs + (k + 1) * 35 + (jj + 1);
                            const double ax = (d_bn[k] + d_bm[j]) * xr[0] + d_an[k] * xr[-35] + d_cn[k] * xr[35] +
                                              d_am[j] * xr[-1] + d_cm[j] * xr[1];
                            r = r - ax;
                        }
                        v[u] = (float)r;
                        rmax = fmaxf(rmax, fabsf(v[u]));
                    }
                    tm_st16(tmem + lane_base + 256 + c0 + jb, v);
                }
            }
            rmax = warp_max(rmax);
            if (lane == 0) f_red[warp] = rmax;
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            rmax = f_red[0];
            for (int i = 1; i < 8; ++i) rmax = fmaxf(rmax, f_red[i]);
            const float s1 = pow2_scale(rmax);
            // ---- TMEM r -> B tile (row j, K index k), FP16 hi/lo
            for (int c0 = jh * NH; c0 < (jh + 1) * NH; c0 += 32) {
                float v[32];
                tm_ld32(tmem + lane_base + 256 + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) put_split(sBh, sBl, c0 + u, kq, NT, v[u] * s1);
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            // ---- W = U r (vertical transform) into TMEM cols [0, NT)
            if (a_inflight && !wait_all(bar_a, ph_a)) { failed = true; break; }
            a_inflight = false;
            issue_gemm();
            if (!wait_all(bar_mma, ph_mma)) { failed = true; break; }
            tc_fence_after();
            if (tid == 0) {   // A tile free: bring in V
                mbar_expect_tx(bar_a, kAImg);
                bulk_g2s(sA, x.aimg + kAImg, kAImg, bar_a);
            }
            a_inflight = true;
            // ---- radial sweeps (T_r(m) + lam_p) w = W_p, top-down and bottom-up halves
            float xmax = 0.0f;
            {
                const int p = kq;
                const bool live = p < NZ;
                const float lam = f_lam[p];
                const int h = min(32 * ((M + 63) / 64), M);   // rows [0,h) top, [h,M) bottom
                float yv[32], cv[32];
                float ymid = 0.f, cmid = 0.f;
                // Elimination in excess form: with g = d + a + c (the small
                // diagonal excess) the top-down multipliers c' = c/D are kept as
                // e = 1 + c' = (g - a e_prev)/D, D = (g - a e_prev) - c, so no
                // near-cancelling sum is formed in FP32; bottom-up likewise with
                // f = 1 + a''.
                if (jh == 0) {
                    float e = 0.f, yp = 0.f;
                    for (int c0 = 0; c0 < h; c0 += 32) {
                        tm_ld32(tmem + lane_base + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            const int j = c0 + u;
                            if (j < h && live) {
                                const float tt = (f_bm[j] + lam) - f_am[j] * e;
                                const float rr = __fdividef(1.0f, tt - f_cm[j]);
                                e = tt * rr;
                                yp = (yv[u] - f_am[j] * yp) * rr;
                                yv[u] = yp;
                                cv[u] = e;
                            } else {
                                cv[u] = 0.f;
                            }
                        }
                        tm_st32(tmem + lane_base + c0, yv);
                        tm_st32(tmem + lane_base + 256 + c0, cv);
                    }
                    ymid = yp;
                    cmid = e;
                    f_xch[p * 4 + 0] = ymid;
                    f_xch[p * 4 + 1] = cmid;
                } else if (h < M) {
                    float f = 0.f, yp = 0.f;
                    const int cl = ((M - 1) / 32) * 32;
                    for (int c0 = cl; c0 >= h; c0 -= 32) {
                        tm_ld32(tmem + lane_base + c0, yv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            const int j = c0 + u;
                            if (j < M && live) {
                                const float tt = (f_bm[j] + lam) - f_cm[j] * f;
                                const float rr = __fdividef(1.0f, tt - f_am[j]);
                                f = tt * rr;
                                yp = (yv[u] - f_cm[j] * yp) * rr;
                                yv[u] = yp;
                                cv[u] = f;
                            } else {
                                cv[u] = 0.f;
                            }
                        }
                        tm_st32(tmem + lane_base + c0, yv);
                        tm_st32(tmem + lane_base + 256 + c0, cv);
                    }
                    f_xch[p * 4 + 2] = yp;
                    f_xch[p * 4 + 3] = f;
                }
                __syncthreads();
                // meeting rows h-1 (top) and h (bottom):
                // x_t = y'_t + (1-e_t) x_u, x_u = y''_u + (1-f_u) x_t
                float xt, xu;
                {
                    const float yt = f_xch[p * 4 + 0], et = f_xch[p * 4 + 1];
                    if (h < M) {
                        const float yu = f_xch[p * 4 + 2], fu = f_xch[p * 4 + 3];
                        xt = (yt + (1.0f - et) * yu) / ((et + fu) - et * fu);
                        xu = yu + (1.0f - fu) * xt;
                    } else {
                        xt = yt;
                        xu = 0.f;
                    }
                }
                if (!live) { xt = 0.f; xu = 0.f; }
                if (jh == 0) {
                    float xn = xt;   // x_{j+1} while sweeping up
                    for (int c0 = ((h - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
                        tm_ld32(tmem + lane_base + c0, yv);
                        tm_ld32(tmem + lane_base + 256 + c0, cv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            const int j = c0 + u;
                            float xv = 0.f;
                            if (j < h && live) {
                                xv = (j == h - 1) ? xt : yv[u] + (1.0f - cv[u]) * xn;
                                xn = xv;
                            }
                            yv[u] = xv;
                            xmax = fmaxf(xmax, fabsf(xv));
                        }
                        tm_st32(tmem + lane_base + c0, yv);
                    }
                } else {
                    float xp = xu;   // x_{j-1} while sweeping down
                    for (int c0 = (h / 32) * 32; c0 < NT; c0 += 32) {
                        tm_ld32(tmem + lane_base + c0, yv);
                        tm_ld32(tmem + lane_base + 256 + c0, cv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            const int j = c0 + u;   // h is a multiple of 32: j >= h
                            float xv = 0.f;
                            if (j < M && live) {
                                xv = (j == h) ? xu : yv[u] + (1.0f - cv[u]) * xp;
                                xp = xv;
                            }
                            yv[u] = xv;
                            xmax = fmaxf(xmax, fabsf(xv));
                        }
                        tm_st32(tmem + lane_base + c0, yv);
                    }
                }
            }
            xmax = warp_max(xmax);
            if (lane == 0) f_red[warp] = xmax;
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            xmax = f_red[0];
            for (int i = 1; i < 8; ++i) xmax = fmaxf(xmax, f_red[i]);
            const float s2 = pow2_scale(xmax);
            // ---- TMEM w -> B tile (row j, K index p), FP16 hi/lo
            for (int c0 = jh * NH; c0 < (jh + 1) * NH; c0 += 32) {
                float v[32];
                tm_ld32(tmem + lane_base + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) put_split(sBh, sBl, c0 + u, kq, NT, v[u] * s2);
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            // ---- delta = V w into TMEM cols [0, NT)
            if (!wait_all(bar_a, ph_a)) { failed = true; break; }
            a_inflight = false;
            issue_gemm();
            if (!wait_all(bar_mma, ph_mma)) { failed = true; break; }
            tc_fence_after();
            const bool more = !last || item + gridDim.x < items;
            if (tid == 0 && more) {   // A tile free: U for the next transform
                mbar_expect_tx(bar_a, kAImg);
                bulk_g2s(sA, x.aimg, kAImg, bar_a);
            }
            a_inflight = more;
            // ---- x += delta (FP64); the last pass writes the interior of X
            const double unscale = 1.0 / ((double)kAScale * (double)kAScale * (double)s1 * (double)s2);
            // staged like the residual: TMEM rows -> sD[k][jj] -> coalesced rows
            double sd = 0.0, sx = 0.0;
            {
                double *sD = reinterpret_cast<double *>(sBh);
                for (int c0 = 0; c0 < NT; c0 += 32) {
                    float v[16];
                    const int jb = jh * 16;
                    tm_ld16(tmem + lane_base + c0 + jb, v);
                    __syncthreads();
#pragma unroll
                    for (int u = 0; u < 16; ++u) sD[kq * 33 + jb + u] = (double)v[u] * unscale;
                    __syncthreads();
                    for (int i = tid; i < 128 * 32; i += 256) {
                        const int k = i >> 5, jj = i & 31, j = c0 + jj;
                        if (k < NZ && j < M) {
                            const double dlt = sD[k * 33 + jj];
                            const size_t o = (size_t)k * J + j;
                            const double xn = (it > 0 ? xl[o] : 0.0) + dlt;
                            if (last) Xl[o] = xn;
                            else xl[o] = xn;
                            sd += dlt * dlt;
                            sx += xn * xn;
                        }
                    }
                }
            }
            sd = warp_sum(sd);
            sx = warp_sum(sx);
            if (lane == 0) { d_red[warp] = sd; d_red[8 + warp] = sx; }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                double a = 0.0, c = 0.0;
                for (int i = 0; i < 8; ++i) { a += d_red[i]; c += d_red[8 + i]; }
                cr[2 * it] = a;
                cr[2 * it + 1] = c;
            }
        }
    }
    // drain a transfer still in flight, then release tensor memory
    if (a_inflight && !failed) mbar_wait(bar_a, ph_a);
    if (failed && tid == 0) atomicExch(x.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int round64(int v) { return (v + 63) / 64 * 64; }

bool chy_mixed_supported(const chy::HostPlan *hp) { return hp->NZ <= 127 && hp->J >= 64 && round64(hp->J) <= kMaxN; }

size_t chy_mixed_pack_tables(const chy::HostPlan *hp, std::vector<char> *image)
{
    // [U hi | U lo | V hi | V lo]: K-major swizzled FP16 tiles of 2^12 * U(p,k)
    // (rows p, K index k) and 2^12 * V(k,p) (rows k, K index p)
    std::vector<uint8_t> img((size_t)2 * kAImg, 0);
    const int NZ = hp->NZ;
    auto put = [&](size_t base, int row, int k, double v) {
        v *= (double)kAScale;
        const __half h = __double2half(v);
        const __half l = __double2half(v - (double)__half2float(h));
        const uint32_t o = kmaj_off(row, k, kTiles);
        std::memcpy(&img[base + o], &h, 2);
        std::memcpy(&img[base + kTiles * kTiles * 2 + o], &l, 2);
    };
    for (int p = 0; p < NZ; ++p)
        for (int k = 0; k < NZ; ++k) {
            put(0, p, k, hp->U[(size_t)p * NZ + k]);
            put(kAImg, k, p, hp->V[(size_t)k * NZ + p]);
        }
    size_t off = (image->size() + 1023) & ~(size_t)1023;
    image->resize(off + img.size());
    std::memcpy(image->data() + off, img.data(), img.size());
    // eigenvalues as FP32, padded with -1 (any nonzero diagonal works for the
    // zero padding rows)
    std::vector<float> lam(128, -1.0f);
    for (int p = 0; p < NZ; ++p) lam[p] = (float)hp->lam[p];
    size_t off2 = (image->size() + 255) & ~(size_t)255;
    image->resize(off2 + lam.size() * sizeof(float));
    std::memcpy(image->data() + off2, lam.data(), lam.size() * sizeof(float));
    return off;   // lam follows at the next 256-byte boundary after the tiles
}

void chy_mixed_bind_tables(chy_plan *p, char *dev_base)
{
    if (!p->mx) p->mx = new MixedState();
    p->mx->dev.aimg = reinterpret_cast<const uint8_t *>(dev_base);
    size_t lam_off = (((size_t)(dev_base - p->d_tables) + 2 * kAImg) + 255) & ~(size_t)255;
    p->mx->dev.lam = reinterpret_cast<const float *>(p->d_tables + lam_off);
}

size_t chy_mixed_work_doubles(const chy_plan *p)
{
    if (p->precision != CHY_PREC_MIXED) return 0;
    const chy::HostPlan &hp = p->hp;
    const size_t per = (size_t)hp.L * hp.K * hp.J + (size_t)hp.L * 16;
    return per * p->max_batch + 8;
}

void chy_mixed_bind_work(chy_plan *p, double *base)
{
    if (!p->mx) p->mx = new MixedState();
    MixedDev &d = p->mx->dev;
    const chy::HostPlan &hp = p->hp;
    d.sxb = (size_t)hp.L * hp.K * hp.J;
    d.scorr = (size_t)hp.L * 16;
    d.xbuf = base;
    d.corr = base + d.sxb * p->max_batch;
    d.err = reinterpret_cast<int *>(d.corr + d.scorr * p->max_batch);
    d.ntile = round64(hp.J);
    if (p->precision == CHY_PREC_MIXED) {
        cudaMallocHost(&p->mx->h_corr, sizeof(double) * d.scorr * p->max_batch);
        cudaMallocHost(&p->mx->h_err, sizeof(int));
    }
}

int chy_mixed_solve(chy_plan *p, int nb, cudaStream_t s, int *launches)
{
    *launches = 0;
    MixedDev d = p->mx->dev;
    d.nit = 1 + p->refine;
    if (d.nit > 8) d.nit = 8;
    const size_t sm = MixedSmem::bytes(d.ntile);
    cudaError_t e = ensure_smem((const void *)k_mode_mixed, sm);
    if (e != cudaSuccess) return CHY_ERR_CUDA;
    const long long items = (long long)nb * p->hp.L;
    const int grid = (int)(items < p->num_sms ? items : p->num_sms);
    k_mode_mixed<<<grid, 256, sm, s>>>(p->t, p->w, d, nb);
    if (cudaGetLastError() != cudaSuccess) return CHY_ERR_CUDA;
    *launches = 1;
    return CHY_OK;
}

// Per-step correction norms ||delta_i|| / ||x_i|| summed over modes, and the
// device error word.  Called after the stream has been synchronised.
int chy_mixed_collect(chy_plan *p, int nb)
{
    if (p->precision != CHY_PREC_MIXED || !p->mx) return CHY_OK;
    MixedState &m = *p->mx;
    if (cudaMemcpy(m.h_err, m.dev.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return CHY_ERR_CUDA;
    if (*m.h_err != 0) {
        cudaMemset(m.dev.err, 0, sizeof(int));
        return CHY_ERR_TIMEOUT;
    }
    if (cudaMemcpy(m.h_corr, m.dev.corr, sizeof(double) * m.dev.scorr * nb, cudaMemcpyDeviceToHost) != cudaSuccess)
        return CHY_ERR_CUDA;
    return CHY_OK;
}

void chy_mixed_fill_diag(const chy_plan *p, int slot, chy_diag *d)
{
    d->iterations = 0;
    if (p->precision != CHY_PREC_MIXED || !p->mx || !p->mx->h_corr) return;
    const int nit = std::min(1 + p->refine, 8);
    const double *c = p->mx->h_corr + (size_t)slot * p->mx->dev.scorr;
    d->iterations = nit;
    for (int it = 0; it < nit && it < 8; ++it) {
        double sd = 0.0, sx = 0.0;
        for (int l = 0; l < p->hp.L; ++l) {
            sd += c[(size_t)l * 16 + 2 * it];
            sx += c[(size_t)l * 16 + 2 * it + 1];
        }
        d->corr_rel[it] = sx > 0.0 ? std::sqrt(sd / sx) : 0.0;
    }
}

void chy_mixed_release(chy_plan *p)
{
    if (!p->mx) return;
    cudaFreeHost(p->mx->h_corr);
    cudaFreeHost(p->mx->h_err);
    delete p->mx;
    p->mx = nullptr;
}

// ---------------------------------------------------------------------------
// Self-test of the tensor-core path: D = (2^12 U) * Bm^T for one tile, where
// Bm (NT x 128, row-major FP32) is split to FP16 hi/lo by the same code the
// solver uses.  Writes D (128 x NT, row-major FP32).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_umma_selftest(const uint8_t *aimg, const float *Bm, float *D, int NT, int *err)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t *sA = sm, *sBh = sm + kAImg, *sBl = sBh + (size_t)NT * 256;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sBl + (size_t)NT * 256);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 2);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < NT * 128; i += blockDim.x) {
        const int row = i / 128, k = i % 128;
        put_split(sBh, sBl, row, k, NT, Bm[i]);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    bool ok = true;
    if (tid == 0) {
        mbar_expect_tx(&bars[1], kAImg);
        bulk_g2s(sA, aimg, kAImg, &bars[1]);
    }
    ok = mbar_wait(&bars[1], 0);
    __syncthreads();
    const uint32_t idesc = (1u << 4) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    if (ok && tid == 0) gemm_issue(tmem, sA, sBh, NT, idesc, &bars[0]);
    if (ok) ok = mbar_wait(&bars[0], 0);
    tc_fence_after();
    if (ok) {
        for (int c0 = 0; c0 < NT; c0 += 32) {
            float v[32];
            tm_ld32(tmem + ((uint32_t)(32 * warp) << 16) + c0, v);
#pragma unroll
            for (int u = 0; u < 32; ++u) D[(size_t)(32 * warp + lane) * NT + c0 + u] = v[u];
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// Test hook: which = 0 uses the U tile, 1 the V tile of the plan.
extern "C" int chy_dbg_umma(chy_plan *p, int which, const float *Bm_dev, float *D_dev, int NT)
{
    if (!p || !p->mx || !Bm_dev || !D_dev || NT < 64 || NT > 256 || NT % 64) return CHY_ERR_ARG;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return CHY_ERR_NOMEM;
    cudaMemset(err, 0, sizeof(int));
    const size_t sm = (size_t)kAImg + (size_t)NT * 512 + 64;
    ensure_smem((const void *)k_umma_selftest, sm);
    k_umma_selftest<<<1, 128, sm>>>(p->mx->dev.aimg + (which ? kAImg : 0), Bm_dev, D_dev, NT, err);
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(err);
    if (e != cudaSuccess) return CHY_ERR_CUDA;
    return h ? CHY_ERR_TIMEOUT : CHY_OK;
}

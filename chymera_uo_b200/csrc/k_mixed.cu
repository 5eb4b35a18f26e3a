// k_mixed.cu -- mixed-precision mode solve on the 5th-generation tensor cores.
//
// Every azimuthal mode's block-tridiagonal system (pot/pot3.f:201-248) is
// solved by FP64 iterative refinement around an approximate FP32/FP16 solver:
//     x_0 = 0;  r_i = Y - A_m x_i (FP64);  x_{i+1} = x_i + S(r_i)
// S applies the vertical eigenbasis and radial sweeps of the FP64 path
// (see k_solve.cu) with
//   * both vertical transforms on tcgen05 tensor cores: operands as FP16
//     hi/lo pairs scaled by powers of two, three MMA passes (hi*hi + hi*lo +
//     lo*hi) accumulated in FP32 in tensor memory -- about 22 bits.  The
//     eigenbasis is used in its orthogonal form Q (U = Q^T D, V = D^-1 Q, D
//     the diagonal symmetriser of the vertical operator), so one resident
//     tile serves both transforms, read as Q^T and, through the transposed
//     descriptor, as Q; D scales the residual rows and D^-1 the update;
//   * the radial tridiagonal sweeps in FP32 on the accumulator rows, read and
//     written in tensor memory, two threads per system (top-down and
//     bottom-up elimination meeting in the middle).
// The residual, the update of x and the final result stay FP64, so the
// refined solution converges to the FP64 solution of the same operator.
//
// One CTA owns one mode at a time (persistent over (solve, mode) items) and
// keeps the eigenbasis tile and the mode's operand tiles in shared memory and
// its accumulators in tensor memory; only Y, x and the mode's slice of the
// radial sweep table move through L2.
// No TMA multicast is used anywhere.  Every wait is bounded: on a timeout the
// kernel records an error word, stops issuing work, releases its tensor
// memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
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
// residual staging: chunk width, row strides (doubles) and buffer sizes
constexpr int kRC = 16;
constexpr int kResYS = 18, kResXS = 22;
constexpr int kResY = 128 * kResYS, kResBuf = kResY + 130 * kResXS;
// epilogue staging: sD [128][33] then two [128][32] prefetch buffers
constexpr int kEpiD = 128 * 33;
// resident-iterate residual: three-deep ring of 32-column chunks, row stride 34
constexpr int kRingC = 32, kRingS = 34, kRingBuf = 128 * kRingS;
// tensor-map ring: kRingSlots slots, each two 16-column halves of 128 rows x
// 128 bytes
constexpr int kRingHalf = 128 * 128, kRingSlot = 2 * kRingHalf, kRingSlots = 4;
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kStageBytes = cmax(cmax(cmax((size_t)(kEpiD + 2 * 128 * 32) * 8, (size_t)2 * kResBuf * 8),
                                         (size_t)3 * kRingBuf * 8),
                                    (size_t)kRingSlots * kRingSlot);   // tensor-map ring
static_assert((kRingBuf * 8) % 16 == 0, "16-byte staging");
static_assert((kEpiD * 8) % 16 == 0 && (kResY * 8) % 16 == 0 && (kResBuf * 8) % 16 == 0, "16-byte staging");

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
    const uint8_t *aimg;        // [Q^T hi, Q^T lo] swizzled tile (2^12 scaled), Q the
                                // orthogonal vertical eigenbasis
    const float *lam;           // [128]
    const double *zsc;          // [4][128] per vertical row k: d_k, 1/d_k, d_k AN_k / d_(k-1),
                                // d_k CN_k / d_(k+1) (D = diag(d) symmetrises T_z)
    const float *sw_mul;        // [N+1][ntile][128] multipliers e or f of the radial sweeps
    const float *sw_piv;        // [N+1][ntile][128] pivot reciprocals 1/D
    double *xbuf;               // [nb][L][K][J] FP64 iterate
    size_t sxb;
    double *corr;               // [nb][L][8][2] per mode: sum delta^2, sum x^2
    size_t scorr;
    int *err;                   // error word
    int nit;                    // approximate solves (1 + corrections)
    int ntile;                  // MMA N = J rounded up to 64 (<= 256)
    int probe_polls;            // test hook: > 0 makes every CTA first wait this many
                                // polls on a barrier nothing arrives on (0: off)
};

// Arrays of the multi-kernel mixed pipeline (grids with JMAX > 256 or JMAX
// not a multiple of 16).  item = solve * L + mode; Jt = JMAX rounded up to a
// multiple of 256 (the GEMM N tile).
struct WideDev {
    double *xit;                // [item][K][J] FP64 iterate
    size_t sxit;
    float *R;                   // [item][Jt][128] FP32: residual rows, then the sweep results
    float *O;                   // [item][Jt][128] FP32: products U r (W) and V w (delta)
    size_t sro;
    unsigned *rmax, *wmax;      // [item][Jt/256] bits of max |r| and max |w| per tile
    int Jt, nt;                 // nt = Jt / 256
};

struct MixedState {
    size_t o_aimg = 0, o_lam = 0;   // offsets into the packed table image
    MixedDev dev{};
    double *h_corr = nullptr;       // pinned [max_batch][L][8][2]
    size_t xbuf_bytes = 0;          // FP64 iterate (two or more corrections)
    int *h_err = nullptr;           // pinned
    int probe_polls = 0;            // test hook (chy_dbg_mixed_probe)
    WideDev wide{};                 // the multi-kernel pipeline of grids k_mode_mixed does not cover
    bool is_wide = false;
    int pair_clusters = -1;         // co-resident CTA pairs of k_mode_pair (-1: not asked yet)
    bool paired = false;            // the last mode solve ran k_mode_pair (per-half sums)
    CUtensorMap tm_x{};             // X as rows of JMAX doubles: 16 x KMAX tiles, 128-byte swizzle
    CUtensorMap tm_xs{};            // the same with 16 x (KMAX-1) tiles: stores skip the boundary row
    CUtensorMap tm_pl{};            // k_mode_pair, one warp's rows: 16 x min(KMAX, 32) tiles
    CUtensorMap tm_ps{};            // its stores: 16 x 32 tiles
    CUtensorMap tm_psl{};           // the last warp's stores: 16 x (KMAX-1 - 32 (ceil((KMAX-1)/32) - 1))
    bool tm_ok = false;
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

// The same 128 x 128 tile read as an MN-major operand (its transpose): the
// 64-element row chunks of the K-major layout are the 128-byte MN atoms.
// LBO = 16 KB between the two 64-wide halves of M, SBO = 1 KB between groups
// of eight K rows, SWIZZLE_128B.
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kTiles * 128) >> 4) << 16) | (64ull << 32) |
           (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes));
}

// bounded wait on phase `parity`; returns false after `limit` polls
__device__ __forceinline__ bool mbar_wait_n(uint64_t *bar, uint32_t parity, long long limit)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < limit; ++i) {
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

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) { return mbar_wait_n(bar, parity, kSpinLimit); }

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// One 2-D tile of the tensor map at (x, y) into shared memory, counted on bar.
// No multicast.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// One 2-D tile from shared memory to the tensor map at (x, y), in the
// thread's bulk async-group.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int x, int y, const void *src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most N of this thread's bulk groups still reading shared memory
template <int N>
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory"); }
// all of this thread's bulk groups complete (writes performed)
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

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

__device__ __forceinline__ void tm_st8(uint32_t taddr, const float *v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Stores without the wait: the source registers are consumed at issue;
// tm_wait_st() before another thread or the tensor core reads the columns.
__device__ __forceinline__ void tm_st16_nw(uint32_t taddr, const float *v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
        : "memory");
}

__device__ __forceinline__ void tm_st32_nw(uint32_t taddr, const float *v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]),
        "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]),
        "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}

// Loads without the wait; the values are valid after tm_wait_ld18 names them
// (as read-write operands, so no use can be scheduled before the wait).
__device__ __forceinline__ void tm_ld16_nw(uint32_t taddr, float *v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
          "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tm_ld1_nw(uint32_t taddr, float &v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=f"(v) : "r"(taddr) : "memory");
}

__device__ __forceinline__ void tm_wait_ld32(float *v, float *w)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                   "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                   "+f"(v[15]), "+f"(w[0]), "+f"(w[1]), "+f"(w[2]), "+f"(w[3]), "+f"(w[4]), "+f"(w[5]), "+f"(w[6]),
                   "+f"(w[7]), "+f"(w[8]), "+f"(w[9]), "+f"(w[10]), "+f"(w[11]), "+f"(w[12]), "+f"(w[13]),
                   "+f"(w[14]), "+f"(w[15])
                 :
                 : "memory");
}

__device__ __forceinline__ void tm_wait_ld18(float *v, float &a, float &b)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                   "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                   "+f"(v[15]), "+f"(a), "+f"(b)
                 :
                 : "memory");
}

// 16-byte global -> shared copy; bytes = 0 fills the destination with zeros
// (src must still be a valid address)
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

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
// its exponent k: pow2_scale(vmax) = 2^k
__device__ __forceinline__ int pow2_exp(float vmax)
{
    if (!(vmax > 0.0f) || !isfinite(vmax)) return 0;
    int e;
    frexpf(vmax, &e);
    return 14 - e;
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

// FP16 hi/lo split of 32 consecutive B-tile rows c0..c0+31 (K index kq, the
// caller's TMEM lane), values already scaled.  Lane pairs (2i, 2i+1) swap
// halves so that each thread writes the (k even, k odd) pair of one row as a
// half2: rows c0+u for even lanes, c0+u+4 for odd lanes.  Same roundings as
// put_split, element by element.
__device__ __forceinline__ void split_rows32(uint8_t *hi, uint8_t *lo, const float *v, int c0, int kq, int lane,
                                             int R)
{
    const int odd = lane & 1, ke = kq & ~1, kk = ke & 63, g = kk >> 3;
    const uint32_t base = (uint32_t)((ke >> 6) * (R * 128) + ((kk & 7) << 1));
    // even lanes take rows u with u % 8 < 4, odd lanes rows u + 4: in the
    // 128-byte swizzle the two rows' granules are disjoint, so the 32 lanes'
    // stores fall on 32 distinct banks
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int u = (i & 3) + ((i >> 2) << 3);
        const float send = odd ? v[u] : v[u + 4];
        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
        const float a = odd ? recv : v[u];        // K index ke
        const float b = odd ? v[u + 4] : recv;    // K index ke + 1
        const int row = c0 + u + 4 * odd;
        const uint32_t off = base + (uint32_t)row * 128 + ((uint32_t)(g ^ (row & 7)) << 4);
        const __half2 h = __floats2half2_rn(a, b);
        const float2 hb = __half22float2(h);
        const __half2 l = __floats2half2_rn(a - hb.x, b - hb.y);
        *reinterpret_cast<__half2 *>(hi + off) = h;
        *reinterpret_cast<__half2 *>(lo + off) = l;
    }
}

// Three-pass FP16 hi/lo product of the A tile (hi at sA, lo at sA + 32 KB)
// and the B tile (hi at sBh, lo at sBh + NT*256) into TMEM columns [0, NT):
// D = Ahi Bhi + Ahi Blo + Alo Bhi, K = 128 in eight 16-wide steps.  With
// trans the A tile is used transposed (MN-major descriptor, the instruction's
// transpose-A bit), so one resident tile serves both Q^T r and Q w.  Issued
// by one thread; completion is signalled on bar.
__device__ __forceinline__ void gemm_issue(uint32_t tmem, const uint8_t *sA, const uint8_t *sBh, int NT,
                                           uint32_t idesc, uint64_t *bar, bool trans)
{
    tc_fence_after();
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sBh);
    const uint32_t a_lo = kTiles * kTiles * 2, b_lo = (uint32_t)NT * 256;
    const uint32_t pa[3] = {0u, 0u, a_lo}, pb[3] = {0u, b_lo, 0u};
    const uint32_t id = idesc | (trans ? 1u << 15 : 0u);
#pragma unroll
    for (int pass = 0; pass < 3; ++pass)
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            // K-major: 16 K columns are 32 bytes of a 128-byte row, the second
            // 64 in the next chunk; MN-major: 16 K rows are two 1 KB groups
            const uint32_t ao = trans ? a0 + pa[pass] + (uint32_t)kk * 2048u
                                      : a0 + pa[pass] + (uint32_t)(kk >> 2) * (kTiles * 128) + (uint32_t)(kk & 3) * 32;
            const uint32_t bo = b0 + pb[pass] + (uint32_t)(kk >> 2) * ((uint32_t)NT * 128) + (uint32_t)(kk & 3) * 32;
            umma_f16(tmem, trans ? umma_desc_mn(ao) : umma_desc(ao), umma_desc(bo), id, (pass | kk) ? 1u : 0u);
        }
    umma_commit(bar);
}

}  // namespace

// ---------------------------------------------------------------------------
// The fused per-mode solver
// ---------------------------------------------------------------------------
// Shared memory: A tile (64 KB: hi, lo), the B region (B tile; between the
// products it stages residual and update rows or holds the sweep
// multipliers), then FP64 stencil rows, FP32 sweep coefficients, reduction
// and exchange scratch, barriers.
struct MixedSmem {
    static constexpr size_t a = 0;
    static constexpr size_t b = kAImg;
    __host__ __device__ static size_t breg(int nt) { return (size_t)nt * 512 > kStageBytes ? (size_t)nt * 512 : kStageBytes; }
    __host__ __device__ static size_t tables(int nt) { return b + breg(nt); }
    __host__ __device__ static size_t bytes(int nt) { return tables(nt) + 22 * 1024; }
};

// kRes: at most two approximate solves.  The first solution x0 is an FP32
// accumulator times a power of two, so it stays exactly in tensor memory
// columns [0, NT) and the correction works in columns [256, 256 + NT); the
// FP64 iterate never goes through global memory.  Otherwise (more
// corrections) the iterate is kept in FP64 in x.xbuf.
template <bool kRes>
__global__ void __launch_bounds__(256, 1) k_mode_mixed(DevTables t, Work w, MixedDev x, int nb,
                                                     const __grid_constant__ CUtensorMap tm_x,
                                                     const __grid_constant__ CUtensorMap tm_xs)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NT = x.ntile, M = t.M, NZ = t.NZ, J = t.J, K = t.K;
    uint8_t *sA = sm + MixedSmem::a;
    uint8_t *sBh = sm + MixedSmem::b, *sBl = sBh + (size_t)NT * 256;
    double *d_am = reinterpret_cast<double *>(sm + MixedSmem::tables(NT));   // [256]
    double *d_cm = d_am + 256, *d_bm = d_cm + 256;                             // [256] each
    double *d_an = d_bm + 256, *d_bn = d_an + 128, *d_cn = d_bn + 128;         // [128] each
    float4 *f_t = reinterpret_cast<float4 *>(d_cn + 128);                     // [256] {g, a, c, 0}
    float *f_lam = reinterpret_cast<float *>(f_t + 256);                       // [128]
    float *f_red = f_lam + 128;                                                // [2][8]
    double *d_red = reinterpret_cast<double *>(f_red + 16);                    // [24]
    float *f_xch = reinterpret_cast<float *>(d_red + 24);                      // [128][4]
    float *f_edge = f_xch + 512;                                               // [2][8][2][16]
    uint64_t *bar_mma = reinterpret_cast<uint64_t *>(f_edge + 512);
    uint64_t *bar_a = bar_mma + 1;
    uint64_t *bar_ring = bar_a + 1;   // [kRingSlots] residual ring slots
    uint64_t *bar_cv = bar_ring + kRingSlots;   // sweep multipliers copied in
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_cv + 1);
    int *s_flag = reinterpret_cast<int *>(tmem_slot + 1);

    // ---- setup: tensor memory (all 512 columns), barriers, m-independent tables
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar_mma, 1);
        mbar_init(bar_a, 1);
        for (int i = 0; i < kRingSlots; ++i) mbar_init(bar_ring + i, 1);
        mbar_init(bar_cv, 1);
        *s_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int j = tid; j < 256; j += blockDim.x) {
        d_am[j] = j < M ? t.am[j] : 0.0;
        d_cm[j] = j < M ? t.cm[j] : 0.0;
        f_t[j] = make_float4(0.f, (float)d_am[j], (float)d_cm[j], 0.f);
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
    // Both transforms use the orthogonal Q (one resident tile, read as Q^T
    // and as Q): W = U r = Q^T (D r) and delta = V w = D^-1 (Q w).  The
    // residual is formed times d_k (this thread's row), the product Q w is
    // scaled by 1/d_k; the stencil's vertical terms act on x0 without its 1/d
    // factors, so their coefficients carry d_k/d_(k+-1).
    const double dk = x.zsc[kq], ek = x.zsc[128 + kq];
    const double an_s = x.zsc[256 + kq], cn_s = x.zsc[384 + kq];
    const double pig4k = t.pig4 * dk, cnmaxk = t.cnmax * dk, cmmaxk = t.cmmax * dk;
    // MMA: kind::f16, A/B FP16 K-major, D FP32, M = 128, N = NT
    const uint32_t idesc = (1u << 4) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const int nit = kRes ? min(x.nit, 2) : x.nit;
    uint32_t ph_mma = 0, ph_a = 0;
    uint32_t ring_ph = 0, ring_pend = 0;   // residual ring slots: phase parity, copies in flight
    uint32_t ph_cv = 0;
    bool cv_pend = false;
    bool mma_pend = false;   // a product's completion not yet observed
    bool failed = false;

    const long long items = (long long)nb * t.L;
    // test hook: a bounded wait on a barrier nothing arrives on (the sweep
    // multipliers' barrier, before anything is issued on it), so the failure
    // path runs with no copy or product in flight
    if (x.probe_polls > 0) {
        if (tid == 0 && !mbar_wait_n(bar_cv, 0, x.probe_polls)) *s_flag = 1;
        __syncthreads();
        failed = *s_flag != 0;
    }
    if (tid == 0 && blockIdx.x < items && !failed) {
        mbar_expect_tx(bar_a, kAImg);
        bulk_g2s(sA, x.aimg, kAImg, bar_a);   // Q, resident for every transform
    }
    bool a_inflight = blockIdx.x < items && !failed;
    long long fail_item = blockIdx.x;   // first item of this CTA left unsolved

    // all threads wait; the phase advances only when every thread saw it
    // complete, so after a failure the drain below waits on the same phase
    auto wait_all = [&](uint64_t *bar, uint32_t &ph) {
        const bool ok = mbar_wait(bar, ph);
        if (!ok) *s_flag = 1;
        __syncthreads();
        const bool good = *s_flag == 0;
        if (good) ph ^= 1u;
        return good;
    };
    // block sums of three per-thread values into d_red[0..2] (uniform call)
    auto block_sum3 = [&](double a, double b, double c) {
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
        __syncthreads();
        if (lane == 0) { d_red[warp] = a; d_red[8 + warp] = b; d_red[16 + warp] = c; }
        __syncthreads();
        if (tid == 0) {
            double sa = 0.0, sb = 0.0, sc = 0.0;
            for (int i = 0; i < 8; ++i) { sa += d_red[i]; sb += d_red[8 + i]; sc += d_red[16 + i]; }
            d_red[0] = sa; d_red[8] = sb; d_red[16] = sc;
        }
    };

    for (long long item = blockIdx.x; item < items && !failed; item += gridDim.x) {
        fail_item = item;
        // mode-major order, modes l and l + N (same m) side by side and the
        // batch's solves innermost: the items in flight at once share a few
        // sweep-table slices, which then stay in L2
        const int o = (int)(item / nb), b = (int)(item % nb);
        const int l = (o & 1) ? (o >> 1) + t.N : (o >> 1);
        const int m = l <= t.N ? l : l - t.N;
        const double xl2 = 2.0 * (t.xlamm[m] - 1.0);
        // BM_m (pot/pot3.f:226-230) for the FP64 residual (the sweeps use the
        // tabulated multipliers)
        for (int j = tid; j < 256; j += blockDim.x) {
            double bm = 0.0;
            if (j < M) {
                const double axis = (((m & 1) ? -1.0 : 1.0) - 1.0) * t.ammin;
                bm = t.bm0[j] + xl2 * t.cc[j];
                if (j == 0) bm = t.bm0[0] + axis + xl2 * t.cc[0];
            }
            d_bm[j] = bm;
        }
        double *Xl = w.X + (size_t)b * w.sX + (size_t)l * K * J;
        double *xl = kRes ? nullptr : x.xbuf + (size_t)b * x.sxb + (size_t)l * K * J;
        double *cr = x.corr + (size_t)b * x.scorr + (size_t)l * 16;
        // kRes: scales 2^eu0 of x0 held in tensor memory, per radial half
        // [0, NT/2) and [NT/2, NT): every power-of-two scale is taken per half,
        // exactly as k_mode_pair's two CTAs take them, so both kernels give the
        // same bits
        double u0h0 = 0.0, u0h1 = 0.0;
        int eu0h0 = 0, eu0h1 = 0;
        double ym_keep = 0.0;   // kRes: X(k, M) of this thread's row, for the write-back tiles
        __syncthreads();

        for (int it = 0; it < nit && !failed; ++it) {
            const bool last = it == nit - 1;
            const bool res_x = kRes && it > 0;          // x0 read from tensor memory
            const uint32_t acc = res_x ? 256u : 0u;     // product / sweep columns
            float sxf0 = 0.f, sxf1 = 0.f;               // kRes: sums of x0^2 per half (unscaled)
            // ---- residual r = Y - A_m x (FP64) -> TMEM cols [256, 256+NT) as FP32.
            // Out-of-range neighbours read as 0; their stencil coefficients
            // (AN(1), CN(KMAX-1), AM(1), CM(JMAX-1)) are 0 too.  JMAX is a
            // multiple of 16, so column M is in the chunk of column M-1 and
            // every 16-byte granule of a row is aligned.
            float rmax0 = 0.0f, rmax1 = 0.0f;           // max |r| per half
            if constexpr (kRes) {
                // Raw X rows k = 0..KMAX-1 (boundary row NZ and column M
                // included) stream through a four-deep ring of 32-column
                // chunks loaded by the tensor-memory-access engine: per chunk
                // two 16-column x KMAX-row tiles of the tensor map over X, in
                // the 128-byte swizzle (16-byte granule g of row k at
                // g ^ (k % 8)), so the 16-byte reads of eight consecutive rows
                // fall on distinct banks.  x0 comes from tensor memory, its
                // vertical neighbours by warp shuffles and, across warps,
                // through shared memory.
                uint8_t *ring = sBh;                       // [kRingSlots][2][128 rows][128 B]
                const int nchr = NT / kRingC;
                const int row0 = (b * t.L + l) * K;        // first tensor-map row of this item
                // thread 0 issues chunk c into slot c % kRingSlots (after the
                // barrier that retired the slot's previous chunk); halves past
                // JMAX are zero-filled instead
                auto issue = [&](int c) {
                    if (c >= nchr) return;
                    ring_pend |= 1u << (c % kRingSlots);
                    if (warp != 0) return;
                    const int sl = c % kRingSlots, c0 = c * kRingC;
                    uint8_t *slot = ring + sl * kRingSlot;
                    const int halves = c0 >= J ? 0 : (c0 + 16 >= J ? 1 : 2);
                    if (lane == 0) {
                        if (halves > 0) {
                            mbar_expect_tx(bar_ring + sl, (uint32_t)(halves * K * 128));
                            for (int h = 0; h < halves; ++h)
                                tma_load_2d(slot + h * kRingHalf, &tm_x, c0 + 16 * h, row0, bar_ring + sl);
                        } else {
                            mbar_arrive(bar_ring + sl);
                        }
                    }
                    for (int h = halves; h < 2; ++h)
                        for (int i = lane; i < K * 16; i += 32)
                            reinterpret_cast<double *>(slot + h * kRingHalf)[i] = 0.0;
                };
                // all threads: chunk c has landed (bounded wait; on a timeout
                // the slot stays pending for the drain at the end)
                auto landed = [&](int c) {
                    const int sl = c % kRingSlots;
                    if (mbar_wait(bar_ring + sl, (ring_ph >> sl) & 1u)) {
                        ring_ph ^= 1u << sl;
                        ring_pend &= ~(1u << sl);
                    } else {
                        *s_flag = 1;
                    }
                };
                // element (row k, column cc < 32) of a slot
                auto at = [&](const uint8_t *slot, int k, int cc) -> const double * {
                    const int h = cc >> 4, q = cc & 15;
                    return reinterpret_cast<const double *>(slot + h * kRingHalf + k * 128 +
                                                            ((((q >> 1) ^ (k & 7))) << 4) + ((q & 1) << 3));
                };
                // generic writes to this region (splits, epilogue staging)
                // are ordered before the copy engine's writes
                fence_proxy_async();
                __syncthreads();
                for (int c = 0; c < kRingSlots - 1; ++c) issue(c);
                const int k = kq, jb = jh * 16, quad = warp & 3;
                const bool krow = k < NZ;
                const double an = an_s, cn = cn_s, bnk = d_bn[k];
                for (int c = 0; c < nchr; ++c) {
                    const int c0 = c * kRingC;
                    float xc[16], xlf = 0.f, xrt = 0.f;
                    if (res_x) {
                        // the tensor-memory loads fly while the row copies land
                        const int jl = c0 + jb - 1, jr = c0 + jb + 16;
                        tm_ld16_nw(tmem + lane_base + c0 + jb, xc);
                        tm_ld1_nw(tmem + lane_base + (uint32_t)(jl < 0 ? 0 : jl), xlf);
                        tm_ld1_nw(tmem + lane_base + (uint32_t)(jr < NT ? jr : NT - 1), xrt);
                        landed(c);
                        tm_wait_ld18(xc, xlf, xrt);
                        if (jl < 0) xlf = 0.f;
                        if (jr >= NT) xrt = 0.f;
                        float *ed = f_edge + ((c & 1) * 8 + warp) * 32;
                        if (lane == 0) {
#pragma unroll
                            for (int u = 0; u < 16; ++u) ed[u] = xc[u];
                        }
                        if (lane == 31) {
#pragma unroll
                            for (int u = 0; u < 16; ++u) ed[16 + u] = xc[u];
                        }
                    } else {
                        landed(c);
                    }
                    __syncthreads();
                    if (*s_flag) break;   // a tile did not land: stop (uniform)
                    issue(c + kRingSlots - 1);
                    // right-hand side 4 pi G rho with the boundary folds
                    // (pot/pot3.f:219-224), times d_k: the row below the top
                    // boundary folds row NZ (one thread), the column M fold
                    // lies in one chunk
                    const uint8_t *slot = ring + (c % kRingSlots) * kRingSlot;
                    double yv[16];
#pragma unroll
                    for (int u = 0; u < 16; u += 2) {
                        const double2 t2 = *reinterpret_cast<const double2 *>(at(slot, k, jb + u));
                        yv[u] = pig4k * t2.x;
                        yv[u + 1] = pig4k * t2.y;
                    }
                    if (k == NZ - 1) {
#pragma unroll
                        for (int u = 0; u < 16; u += 2) {
                            const double2 t3 = *reinterpret_cast<const double2 *>(at(slot, NZ, jb + u));
                            yv[u] = fma(-cnmaxk, t3.x, yv[u]);
                            yv[u + 1] = fma(-cnmaxk, t3.y, yv[u + 1]);
                        }
                    }
                    const int uM = M - 1 - (c0 + jb);   // uniform in the warp
                    if (uM >= 0 && uM < 16) {
                        const double yM = *at(slot, k, M - c0);
                        ym_keep = yM;
#pragma unroll
                        for (int u = 0; u < 16; ++u)
                            if (u == uM) yv[u] = fma(-cmmaxk, yM, yv[u]);
                    }
                    float v[16];
                    if (res_x) {
                        // rows above lane 0 and below lane 31 come from the
                        // neighbouring warps' edges (all lanes load, two select)
                        const float *eu = f_edge + ((c & 1) * 8 + (quad > 0 ? warp - 1 : warp)) * 32 + 16;
                        const float *ed = f_edge + ((c & 1) * 8 + (quad < 3 ? warp + 1 : warp)) * 32;
                        const bool top0 = lane == 0, bot31 = lane == 31;
                        const float zu = quad > 0 ? 1.f : 0.f, zd = quad < 3 ? 1.f : 0.f;
                        // x0 at columns j-1 .. j+16 in this half's units; a neighbour
                        // across the halves' boundary is converted exactly
                        const bool hh = c0 >= NH;
                        const double u0 = hh ? u0h1 : u0h0;
                        double xd_[18];
                        xd_[0] = c0 + jb == NH ? ldexp((double)xlf, eu0h0 - eu0h1) : (double)xlf;
                        xd_[17] = c0 + jb + 16 == NH ? ldexp((double)xrt, eu0h1 - eu0h0) : (double)xrt;
#pragma unroll
                        for (int u = 0; u < 16; ++u) xd_[u + 1] = (double)xc[u];
                        float sxf = 0.f, rm = 0.f;
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const int j = c0 + jb + u;
                            float xu = __shfl_up_sync(0xffffffffu, xc[u], 1);
                            float xd = __shfl_down_sync(0xffffffffu, xc[u], 1);
                            const float eu_u = eu[u] * zu, ed_u = ed[u] * zd;
                            xu = top0 ? eu_u : xu;
                            xd = bot31 ? ed_u : xd;
                            // d_k A x0 / u0 (x0 = u0 t / d): u0 is a power of two, so
                            // scaling the sum is exact
                            double ax = (bnk + d_bm[j]) * xd_[u + 1];
                            ax = fma(an, (double)xu, ax);
                            ax = fma(cn, (double)xd, ax);
                            ax = fma(d_am[j], xd_[u], ax);
                            ax = fma(d_cm[j], xd_[u + 2], ax);
                            const double r = fma(-u0, ax, yv[u]);
                            const bool in = krow && j < M;
                            sxf = fmaf(in ? xc[u] : 0.f, xc[u], sxf);
                            v[u] = in ? (float)r : 0.f;
                            rm = fmaxf(rm, fabsf(v[u]));
                        }
                        if (hh) { rmax1 = fmaxf(rmax1, rm); sxf1 += sxf; }
                        else { rmax0 = fmaxf(rmax0, rm); sxf0 += sxf; }
                    } else {
                        float rm = 0.f;
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const int j = c0 + jb + u;
                            v[u] = (krow && j < M) ? (float)yv[u] : 0.f;
                            rm = fmaxf(rm, fabsf(v[u]));
                        }
                        if (c0 >= NH) rmax1 = fmaxf(rmax1, rm);
                        else rmax0 = fmaxf(rmax0, rm);
                    }
                    tm_st16_nw(tmem + lane_base + 256 + c0 + jb, v);
                }
                tm_wait_st();
                if (*s_flag) { failed = true; break; }
            } else {
                // Chunks of kRC columns, double-buffered with cp.async: raw X
                // rows k = 0..KMAX-1 and the iterate rows k = -1..NZ with
                // columns c0-2 .. c0+kRC+1 (out-of-range granules are zero).
                // Row strides of 9 and 11 granules keep the 16-byte reads of
                // eight consecutive rows on distinct banks.
                double *stage = reinterpret_cast<double *>(sBh);
                const bool need_x = it > 0;
                auto issue = [&](int c0, int buf) {
                    double *sy = stage + buf * kResBuf, *sx = sy + kResY;
                    for (int g = tid; g < K * (kRC / 2); g += 256) {
                        const int k = g / (kRC / 2), j = c0 + 2 * (g % (kRC / 2));
                        const bool ok = j < J;
                        cp_async16(sy + k * kResYS + (j - c0), ok ? Xl + (size_t)k * J + j : Xl, ok ? 16 : 0);
                    }
                    if (need_x) {
                        for (int g = tid; g < (NZ + 2) * (kRC / 2 + 2); g += 256) {
                            const int kk = g / (kRC / 2 + 2) - 1, j = c0 - 2 + 2 * (g % (kRC / 2 + 2));
                            const bool ok = kk >= 0 && kk < NZ && j >= 0 && j < J;
                            cp_async16(sx + (kk + 1) * kResXS + (j - c0 + 2), ok ? xl + (size_t)kk * J + j : xl,
                                       ok ? 16 : 0);
                        }
                    }
                    cp_async_commit();
                };
                const int nch = NT / kRC;
                issue(0, 0);
                const int k = kq, jb = jh * (kRC / 2);
                const bool krow = k < NZ;
                const double an = d_an[k], cn = d_cn[k], bnk = d_bn[k];
                for (int c = 0; c < nch; ++c) {
                    const int c0 = c * kRC;
                    if (c + 1 < nch) {
                        issue(c0 + kRC, (c + 1) & 1);
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                    __syncthreads();
                    const double *sy = stage + (c & 1) * kResBuf, *sx = sy + kResY;
                    float v[kRC / 2];
                    double yv[kRC / 2], xc[kRC / 2 + 4], xu[kRC / 2], xd[kRC / 2];
#pragma unroll
                    for (int u = 0; u < kRC / 2; u += 2) {
                        const double2 t2 = *reinterpret_cast<const double2 *>(sy + k * kResYS + jb + u);
                        yv[u] = t2.x;
                        yv[u + 1] = t2.y;
                    }
                    if (need_x) {
#pragma unroll
                        for (int u = 0; u < kRC / 2 + 4; u += 2) {
                            const double2 t2 = *reinterpret_cast<const double2 *>(sx + (k + 1) * kResXS + jb + u);
                            xc[u] = t2.x;
                            xc[u + 1] = t2.y;
                        }
#pragma unroll
                        for (int u = 0; u < kRC / 2; u += 2) {
                            const double2 a2 = *reinterpret_cast<const double2 *>(sx + k * kResXS + jb + 2 + u);
                            const double2 b2 = *reinterpret_cast<const double2 *>(sx + (k + 2) * kResXS + jb + 2 + u);
                            xu[u] = a2.x;
                            xu[u + 1] = a2.y;
                            xd[u] = b2.x;
                            xd[u + 1] = b2.y;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kRC / 2; ++u) {
                        const int jj = jb + u, j = c0 + jj;
                        double r = 0.0;
                        if (krow && j < M) {
                            r = t.pig4 * yv[u];
                            if (k == NZ - 1) r = r - t.cnmax * sy[NZ * kResYS + jj];
                            if (j == M - 1) r = r - t.cmmax * sy[k * kResYS + (M - c0)];
                            if (need_x) {
                                const double ax = (bnk + d_bm[j]) * xc[u + 2] + an * xu[u] + cn * xd[u] +
                                                  d_am[j] * xc[u + 1] + d_cm[j] * xc[u + 3];
                                r = r - ax;
                            }
                        }
                        v[u] = (float)(dk * r);
                        if (c0 >= NH) rmax1 = fmaxf(rmax1, fabsf(v[u]));
                        else rmax0 = fmaxf(rmax0, fabsf(v[u]));
                    }
                    tm_st8(tmem + lane_base + 256 + c0 + jb, v);
                    __syncthreads();
                }
                tm_wait_st();
            }
            rmax0 = warp_max(rmax0);
            rmax1 = warp_max(rmax1);
            if (lane == 0) { f_red[warp] = rmax0; f_red[8 + warp] = rmax1; }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            rmax0 = f_red[0];
            rmax1 = f_red[8];
            for (int i = 1; i < 8; ++i) { rmax0 = fmaxf(rmax0, f_red[i]); rmax1 = fmaxf(rmax1, f_red[8 + i]); }
            const int k1h0 = pow2_exp(rmax0), k1h1 = pow2_exp(rmax1);
            const float s1 = ldexpf(1.0f, jh ? k1h1 : k1h0);   // this thread splits half jh
            // ---- TMEM r -> B tile (row j, K index k), FP16 hi/lo
            for (int c0 = jh * NH; c0 < (jh + 1) * NH; c0 += 32) {
                float v[32];
                tm_ld32(tmem + lane_base + 256 + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) v[u] *= s1;
                split_rows32(sBh, sBl, v, c0, kq, lane, NT);
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            // ---- W = U r (vertical transform) into TMEM cols [acc, acc + NT)
            if (a_inflight && !wait_all(bar_a, ph_a)) { failed = true; break; }
            a_inflight = false;
            if (tid == 0) gemm_issue(tmem + acc, sA, sBh, NT, idesc, bar_mma, false);
            mma_pend = true;
            // the first chunk of pivot reciprocals is loaded while the product runs
            const float *swp = x.sw_piv + (size_t)m * NT * 128 + kq;   // row j at swp[j * 128]
            const int h = 32 * ((M + 63) / 64);   // M >= 63, h < M, h % 32 == 0
            const int cl = ((M - 1) / 32) * 32;   // the bottom-up sweep's first chunk
            float R[32];
#pragma unroll
            for (int u = 0; u < 32; ++u) R[u] = swp[(size_t)((jh == 0 ? 0 : cl) + u) * 128];
            if (!wait_all(bar_mma, ph_mma)) { failed = true; break; }
            mma_pend = false;
            tc_fence_after();
            float *cvs = reinterpret_cast<float *>(sBh);   // [j][p] multipliers for the back sweeps
            if (lane == 0 && (warp & 1) == 0) {
                // B tile free: this m's multipliers for the back sweeps, a
                // quarter per even warp (an issuing thread waits while the
                // copy engine takes in its bytes, so no warp takes all four)
                const int q = warp >> 1;
                const float *src = x.sw_mul + (size_t)m * NT * 128;
                if (q == 0) mbar_expect_tx(bar_cv, (uint32_t)NT * 512);
                bulk_g2s(cvs + q * NT * 32, src + q * NT * 32, (uint32_t)NT * 128, bar_cv);
            }
            cv_pend = true;
            // ---- radial sweeps (T_r(m) + lam_p) w = W_p, top-down over rows
            // [0, h) and bottom-up over [h, M), meeting in the middle.  The
            // multipliers and pivot reciprocals come from the sweep table, so
            // each row costs one dependent FMA.  The elimination reads the
            // pivot reciprocals from global memory one 32-row chunk ahead of
            // the recurrence; the multipliers, which only the back sweeps
            // need, arrive in shared memory as one bulk copy meanwhile.  The
            // multipliers are in excess form (e_j, f_j small for small
            // shifts), so 1 - e_j keeps nearly all of its bits.
            float xmax = 0.0f;
            {
                const int p = kq;
                const bool live = p < NZ;
                const uint32_t tb = tmem + lane_base + acc;
                float yv[32];
                float Rn[32];
                if (jh == 0) {
                    float yp = 0.f;
                    for (int c0 = 0; c0 < h; c0 += 32) {
                        if (c0 + 32 < h) {
#pragma unroll
                            for (int u = 0; u < 32; ++u) Rn[u] = swp[(size_t)(c0 + 32 + u) * 128];
                        }
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            const float rr = R[u], ar = f_t[c0 + u].y * rr;
                            yp = fmaf(-ar, yp, yv[u] * rr);
                            yv[u] = yp;
                        }
                        tm_st32_nw(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) R[u] = Rn[u];
                    }
                    f_xch[p * 4 + 0] = yp;
                } else {
                    float yp = 0.f;
                    for (int c0 = cl; c0 >= h; c0 -= 32) {
                        if (c0 - 32 >= h) {
#pragma unroll
                            for (int u = 0; u < 32; ++u) Rn[u] = swp[(size_t)(c0 - 32 + u) * 128];
                        }
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            const float rr = R[u], cr = f_t[c0 + u].z * rr;
                            const float yn = fmaf(-cr, yp, yv[u] * rr);
                            yp = (c0 + u < M) ? yn : yp;   // uniform
                            yv[u] = yn;
                        }
                        tm_st32_nw(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) R[u] = Rn[u];
                    }
                    f_xch[p * 4 + 2] = yp;
                }
                tm_wait_st();
                // the multipliers have landed (the barrier inside)
                const bool cv_ok = wait_all(bar_cv, ph_cv);
                if (!cv_ok) { failed = true; break; }
                cv_pend = false;
                // meeting rows h-1 (top) and h (bottom), in FP64 from the two
                // halves' values at their own scales 2^(12 + k1):
                // x_t = y'_t + (1-e_t) x_u, x_u = y''_u + (1-f_u) x_t
                float xt, xu;
                {
                    const int ks0 = 12 + k1h0, ks1 = 12 + k1h1;
                    const double yt = ldexp((double)f_xch[p * 4 + 0], -ks0);
                    const double yu = ldexp((double)f_xch[p * 4 + 2], -ks1);
                    const double et = cvs[(h - 1) * 128 + p], fu = cvs[h * 128 + p];
                    const double xtd = (yt + (1.0 - et) * yu) / ((et + fu) - et * fu);
                    const double xud = yu + (1.0 - fu) * xtd;
                    xt = (float)ldexp(xtd, ks0);
                    xu = (float)ldexp(xud, ks1);
                }
                if (jh == 0) {
                    float xn = xt;   // x_{j+1} while sweeping up
                    for (int c0 = h - 32; c0 >= 0; c0 -= 32) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) Rn[u] = cvs[(c0 + u) * 128 + p];
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            float xv = yv[u] + (1.0f - Rn[u]) * xn;
                            xv = (c0 + u == h - 1) ? xt : xv;
                            xn = xv;
                            yv[u] = live ? xv : 0.f;
                            xmax = fmaxf(xmax, fabsf(yv[u]));
                        }
                        tm_st32_nw(tb + c0, yv);
                    }
                } else {
                    float xp = xu;   // x_{j-1} while sweeping down
                    for (int c0 = h; c0 < NT; c0 += 32) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) Rn[u] = cvs[(c0 + u) * 128 + p];
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            float xv = yv[u] + (1.0f - Rn[u]) * xp;
                            xv = (c0 + u == h) ? xu : xv;
                            xp = xv;
                            yv[u] = (live && c0 + u < M) ? xv : 0.f;
                            xmax = fmaxf(xmax, fabsf(yv[u]));
                        }
                        tm_st32_nw(tb + c0, yv);
                    }
                }
                tm_wait_st();
            }
            // per half: warps 0-3 swept half 0, warps 4-7 half 1
            xmax = warp_max(xmax);
            if (lane == 0) f_red[warp] = xmax;
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            float xm0 = f_red[0], xm1 = f_red[4];
            for (int i = 1; i < 4; ++i) { xm0 = fmaxf(xm0, f_red[i]); xm1 = fmaxf(xm1, f_red[4 + i]); }
            const int k2h0 = pow2_exp(xm0), k2h1 = pow2_exp(xm1);
            const float s2 = ldexpf(1.0f, jh ? k2h1 : k2h0);
            // ---- TMEM w -> B tile (row j, K index p), FP16 hi/lo
            for (int c0 = jh * NH; c0 < (jh + 1) * NH; c0 += 32) {
                float v[32];
                tm_ld32(tmem + lane_base + acc + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) v[u] *= s2;
                split_rows32(sBh, sBl, v, c0, kq, lane, NT);
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            // ---- Q w (delta times d) into TMEM cols [acc, acc + NT): the resident
            // tile, transposed
            if (tid == 0) gemm_issue(tmem + acc, sA, sBh, NT, idesc, bar_mma, true);
            mma_pend = true;
            if (!wait_all(bar_mma, ph_mma)) { failed = true; break; }
            mma_pend = false;
            tc_fence_after();
            // this solve's columns are 2^eun times its result, per half
            const int eun0 = -(24 + k1h0 + k2h0), eun1 = -(24 + k1h1 + k2h1);
            const double unscale0 = ldexp(1.0, eun0), unscale1 = ldexp(1.0, eun1);
            if constexpr (kRes) {
                if (!last) {
                    // x0 stays in tensor memory columns [0, NT)
                    u0h0 = unscale0;
                    u0h1 = unscale1;
                    eu0h0 = eun0;
                    eu0h1 = eun1;
                    continue;
                }
                // X = x0 + delta (FP64).  Each 32-column chunk is staged in
                // one of three slots (two 16-column halves, 128-byte swizzle)
                // and written by the copy engine as tiles of rows 0..KMAX-2
                // (the boundary row is not written); column M, which shares
                // the last tile, carries X's own value back.  The next chunk's
                // tensor-memory rows load while this chunk's tiles are stored.
                double sd = 0.0, sx = 0.0;
                const int jb = jh * 16, row0 = (b * t.L + l) * K;
                float dv[16], xv[16];
                tm_ld16_nw(tmem + lane_base + acc + jb, dv);
                if (res_x) tm_ld16_nw(tmem + lane_base + jb, xv);
                for (int c0 = 0, c = 0; c0 < NT; c0 += 32, ++c) {
                    uint8_t *slot = sBh + (c % 3) * kRingSlot;
                    tm_wait_ld32(dv, xv);
                    const bool hh = c0 >= NH;
                    const double uk = (hh ? unscale1 : unscale0) * ek, u0k = (hh ? u0h1 : u0h0) * ek;   // row's 1/d_k
                    double xn[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int j = c0 + jb + u;
                        const double dl = (double)dv[u] * uk;
                        xn[u] = (res_x ? (double)xv[u] * u0k : 0.0) + dl;
                        if (kq < NZ && j < M) {
                            sd += dl * dl;
                            sx += xn[u] * xn[u];
                        }
                        if (j == M) xn[u] = ym_keep;   // column M (uniform in the warp)
                    }
#pragma unroll
                    for (int u = 0; u < 16; u += 2) {
                        const int q = jb + u, h = q >> 4, g = (q & 15) >> 1;
                        *reinterpret_cast<double2 *>(slot + h * kRingHalf + kq * 128 + ((g ^ (kq & 7)) << 4)) =
                            make_double2(xn[u], xn[u + 1]);
                    }
                    fence_proxy_async();
                    if (tid == 0) bulk_wait_read<1>();   // the store from this slot's last chunk has read it
                    __syncthreads();
                    if (c0 + 32 < NT) {
                        tm_ld16_nw(tmem + lane_base + acc + c0 + 32 + jb, dv);
                        if (res_x) tm_ld16_nw(tmem + lane_base + c0 + 32 + jb, xv);
                    }
                    if (tid == 0) {
                        for (int h = 0; h < 2 && c0 + 16 * h < J; ++h)
                            tma_store_2d(&tm_xs, c0 + 16 * h, row0, slot + h * kRingHalf);
                        bulk_commit();
                    }
                }
                if (tid == 0) bulk_wait_all();   // tiles written, staging free for the next item
                __syncthreads();
                block_sum3(sd, sx, ((double)sxf0 * u0h0 * u0h0 + (double)sxf1 * u0h1 * u0h1) * ek * ek);
                if (tid == 0) {
                    if (res_x) {   // the first solve's delta is x0 itself
                        cr[0] = d_red[16];
                        cr[1] = d_red[16];
                    }
                    cr[2 * it] = d_red[0];
                    cr[2 * it + 1] = d_red[8];
                }
                __syncthreads();
            } else {
                // ---- x += delta (FP64); the last pass writes the interior of X.
                // TMEM rows -> sD[k][jj] -> coalesced rows of x; the previous
                // iterate's rows are prefetched one chunk ahead
                double sd = 0.0, sx = 0.0;
                double *sD = reinterpret_cast<double *>(sBh);
                double *sO = sD + kEpiD;
                const bool need_x = it > 0;
                auto issue = [&](int c0, int buf) {
                    double *so = sO + buf * (128 * 32);
                    for (int g = tid; g < 128 * 16; g += 256) {
                        const int k = g >> 4, j = c0 + 2 * (g & 15);
                        const bool ok = k < NZ && j < J;
                        cp_async16(so + k * 32 + (j - c0), ok ? xl + (size_t)k * J + j : xl, ok ? 16 : 0);
                    }
                    cp_async_commit();
                };
                const int nch = NT / 32, jb = jh * 16;
                if (need_x) issue(0, 0);
                for (int c = 0; c < nch; ++c) {
                    const int c0 = c * 32;
                    if (need_x) {
                        if (c + 1 < nch) {
                            issue(c0 + 32, (c + 1) & 1);
                            cp_async_wait<1>();
                        } else {
                            cp_async_wait<0>();
                        }
                    }
                    float v[16];
                    tm_ld16(tmem + lane_base + c0 + jb, v);
#pragma unroll
                    for (int u = 0; u < 16; ++u) sD[kq * 33 + jb + u] = (double)v[u] * ((c0 >= NH ? unscale1 : unscale0) * ek);
                    __syncthreads();
                    const double *so = sO + (c & 1) * (128 * 32);
                    for (int i = tid; i < 128 * 32; i += 256) {
                        const int k = i >> 5, jj = i & 31, j = c0 + jj;
                        if (k < NZ && j < M) {
                            const double dlt = sD[k * 33 + jj];
                            const size_t o = (size_t)k * J + j;
                            const double xn = (need_x ? so[k * 32 + jj] : 0.0) + dlt;
                            if (last) Xl[o] = xn;
                            else xl[o] = xn;
                            sd += dlt * dlt;
                            sx += xn * xn;
                        }
                    }
                    __syncthreads();
                }
                block_sum3(sd, sx, 0.0);
                if (tid == 0) {
                    cr[2 * it] = d_red[0];
                    cr[2 * it + 1] = d_red[8];
                }
                __syncthreads();
            }
        }
    }
    // drain copies and products still in flight (bounded), then release
    // tensor memory
    if (a_inflight) mbar_wait(bar_a, ph_a);
    for (int sl = 0; sl < kRingSlots; ++sl)
        if (ring_pend & (1u << sl)) mbar_wait(bar_ring + sl, (ring_ph >> sl) & 1u);
    if (cv_pend) mbar_wait(bar_cv, ph_cv);
    if (mma_pend) mbar_wait(bar_mma, ph_mma);
    if (failed) {
        // the modes this CTA left unsolved become NaN (interior of X), so the
        // failure reaches PHI instead of passing silently; the error word
        // tells the host
        if (tid == 0) {
            bulk_wait_all();
            atomicExch(x.err, 1);
        }
        __syncthreads();
        const double qnan = __longlong_as_double(0x7ff8000000000000ll);
        for (long long item = fail_item; item < items; item += gridDim.x) {
            const int o = (int)(item / nb), b = (int)(item % nb);
            const int l = (o & 1) ? (o >> 1) + t.N : (o >> 1);
            double *Xl = w.X + (size_t)b * w.sX + (size_t)l * K * J;
            for (int i = tid; i < NZ * M; i += blockDim.x) Xl[(size_t)(i / M) * J + i % M] = qnan;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// ---------------------------------------------------------------------------
// The paired per-mode solver (two approximate solves, one correction)
// ---------------------------------------------------------------------------
// A cluster of two CTAs (two SMs) holds each (solve, mode) item: CTA r owns
// the radial columns [r NH, (r + 1) NH), NH = ntile / 2 -- exactly the rows
// that the two-sided radial elimination runs top-down (r = 0) and bottom-up
// (r = 1), since h = 32 ceil(M / 64) = NH.  Half an item needs half of the
// tensor memory (x0 and one accumulator of NH columns) and half of the
// shared-memory operand region, so each CTA holds two items at once: its two
// groups of four warps take different items and run independently, one
// group's memory phases (right-hand-side intake, write-back) overlapping the
// other's products and sweeps.  Per item, the two CTAs of a pair exchange
// through distributed shared memory (st.async with complete-tx on the peer's
// mbarrier, double-buffered) the rows where the radial sweeps meet, after
// each elimination, and the iterate's edge column for the correction
// residual.  Each CTA scales its half by its own powers of two; exchanged
// values carry their exponents and are converted exactly.  The eigenbasis
// tile is loaded once and shared by both groups.  Every wait is bounded.
constexpr int kPairB = 64 * 1024;        // per-group region: ring, B tile, multipliers, staging
constexpr int kPairTileB = 128 * 128;    // one 16-column x 128-row FP64 tile (bytes)
constexpr int kPairRing = 4;             // residual ring slots (one tile each)
constexpr int kPairStage = 4;            // write-back staging slots
struct PairSmem {
    static constexpr size_t a = 0;
    static constexpr size_t b = kAImg;                              // [2][kPairB]
    static constexpr size_t am = b + 2 * (size_t)kPairB;            // double [128] AM of this CTA's columns
    static constexpr size_t cm = am + 128 * 8;                      // double [128] CM
    static constexpr size_t bm = cm + 128 * 8;                      // double [2][128] BM_m per group
    static constexpr size_t bn = bm + 2 * 128 * 8;                  // double [128] BN
    static constexpr size_t ft = bn + 128 * 8;                      // float4 [128] {0, AM, CM, 0}
    static constexpr size_t dred = ft + 128 * 16;                   // double [2][24]
    static constexpr size_t fred = dred + 2 * 24 * 8;               // float [2][8]
    static constexpr size_t edge = fred + 2 * 8 * 4;                // float [2][4][2][128] x0 edge rows
    static constexpr size_t xch = edge + 2 * 4 * 2 * 128 * 4;       // float4 [2][2][128] incoming exchanges
    static constexpr size_t bars = xch + 2 * 2 * 128 * 16;          // uint64 [3 + 2 * 20]
    static constexpr size_t misc = bars + 43 * 8;                   // tmem slot, flags [2]
    static constexpr size_t bytes = misc + 16;
};
static_assert(PairSmem::bytes <= 227 * 1024, "pair shared memory");
static_assert(PairSmem::xch % 16 == 0 && PairSmem::bars % 8 == 0, "pair alignment");

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id_x()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count_x()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// the peer CTA's shared::cluster address of a variable of this CTA
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t peer)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(peer));
    return r;
}
// 16 bytes into the peer's shared memory, counted on the peer's mbarrier
__device__ __forceinline__ void st_async16(uint32_t raddr, float4 v, uint32_t rbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     raddr),
                 "r"(__float_as_uint(v.x)), "r"(__float_as_uint(v.y)), "r"(__float_as_uint(v.z)),
                 "r"(__float_as_uint(v.w)), "r"(rbar)
                 : "memory");
}
// bounded wait with cluster-scope acquire (data written by the peer CTA)
__device__ __forceinline__ bool mbar_wait_cl(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(256, 1) k_mode_pair(DevTables t, Work w, MixedDev x, int nb,
                                                      const __grid_constant__ CUtensorMap tm_l,
                                                      const __grid_constant__ CUtensorMap tm_s,
                                                      const __grid_constant__ CUtensorMap tm_sl)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = warp >> 2, gt = tid & 127;            // group, thread in group
    const uint32_t rank = cluster_rank(), peer = rank ^ 1u;
    const int NT = x.ntile, NH = NT / 2, col0 = (int)rank * NH;
    const int M = t.M, NZ = t.NZ, J = t.J, K = t.K;
    uint8_t *sA = sm + PairSmem::a;
    uint8_t *sB = sm + PairSmem::b + (size_t)g * kPairB;
    uint8_t *sBh = sB, *sBl = sB + (size_t)NH * 256;
    double *d_am = reinterpret_cast<double *>(sm + PairSmem::am);
    double *d_cm = reinterpret_cast<double *>(sm + PairSmem::cm);
    double *d_bm = reinterpret_cast<double *>(sm + PairSmem::bm) + g * 128;
    double *d_bn = reinterpret_cast<double *>(sm + PairSmem::bn);
    float4 *f_t = reinterpret_cast<float4 *>(sm + PairSmem::ft);
    double *d_red = reinterpret_cast<double *>(sm + PairSmem::dred) + g * 24;
    float *f_red = reinterpret_cast<float *>(sm + PairSmem::fred) + g * 8;
    // x0's edge rows of this group: [warp][top (lane 0), bottom (lane 31)][column]
    float *f_edge = reinterpret_cast<float *>(sm + PairSmem::edge) + g * 1024;
    float4 *xch = reinterpret_cast<float4 *>(sm + PairSmem::xch) + g * 256;   // [2 slots][128]
    uint64_t *bar_a = reinterpret_cast<uint64_t *>(sm + PairSmem::bars);
    uint64_t *bar_stagger = bar_a + 1;                  // group 1 may start
    uint64_t *bar_probe = bar_a + 2;                    // nothing arrives on it (test hook)
    uint64_t *gb = bar_a + 3 + g * 20;                  // this group's barriers
    uint64_t *bar_mma = gb, *bar_cv = gb + 1, *bar_x = gb + 2;   // bar_x[2]
    uint64_t *bar_ring = gb + 4 + 4 * (warp & 3);       // this warp's four ring slots
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + PairSmem::misc);
    int *s_flag = reinterpret_cast<int *>(sm + PairSmem::misc + 8) ;   // [2]

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < 43; ++i) mbar_init(bar_a + i, 1);
        s_flag[0] = s_flag[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int jl = tid; jl < 128; jl += blockDim.x) {
        const int j = col0 + jl;
        const double a = (jl < NH && j < M) ? t.am[j] : 0.0, c = (jl < NH && j < M) ? t.cm[j] : 0.0;
        d_am[jl] = a;
        d_cm[jl] = c;
        f_t[jl] = make_float4(0.f, (float)a, (float)c, 0.f);
        d_bn[jl] = jl < NZ ? t.bn[jl] : 0.0;
    }
    tc_fence_before();
    __syncthreads();
    // the peer's barriers are initialised before anything is sent to them
    cluster_sync_all();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t G = (uint32_t)g * 256u;              // this group's tensor-memory columns
    const int kq = 32 * (warp & 3) + lane;              // the row (TMEM lane) this thread owns
    const double dk = x.zsc[kq], ek = x.zsc[128 + kq];
    const double an_s = x.zsc[256 + kq], cn_s = x.zsc[384 + kq];
    const double pig4k = t.pig4 * dk, cnmaxk = t.cnmax * dk, cmmaxk = t.cmmax * dk;
    const uint32_t idesc = (1u << 4) | ((uint32_t)(NH >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const long long items = (long long)nb * t.L;
    const long long pairs = cluster_count_x(), cl = cluster_id_x();
    const long long first = 2 * cl + g, stride = 2 * pairs;
    const int nch = NH / 16;
    const int nit = x.nit < 2 ? 1 : 2;                 // approximate solves
    const int h = NH;                                   // first bottom-up row (global)
    const int clast = ((M - 1) / 32) * 32;              // the bottom-up sweep's first chunk (global)
    // the peer's incoming-exchange slots and barriers for this group
    const uint32_t r_xch = peer_addr(xch, peer), r_barx = peer_addr(bar_x, peer);

    uint32_t ph_mma = 0, ph_cv = 0, ring_ph = 0, ring_pend = 0;
    uint32_t xq = 0;                                    // exchanges so far (slot xq & 1)
    bool mma_pend = false, cv_pend = false, failed = false;
    bool a_wait = first < items;                        // this group still has to see Q land
    long long fail_item = first;

    if (x.probe_polls > 0) {
        // test hook: a bounded wait on a barrier nothing arrives on, before
        // anything is issued
        if (tid == 0 && !mbar_wait_n(bar_probe, 0, x.probe_polls)) s_flag[0] = s_flag[1] = 1;
        __syncthreads();
        failed = s_flag[g] != 0;
        a_wait = a_wait && !failed;
    }
    if (tid == 0 && 2 * cl < items && !failed) {
        mbar_expect_tx(bar_a, kAImg);
        bulk_g2s(sA, x.aimg, kAImg, bar_a);             // Q, shared by both groups for every transform
    }
    bool a_inflight = 2 * cl < items && !failed;        // drained by thread 0 at the end
    // Group 1 starts when group 0 has finished its first item's last residual
    // (about half an item): the two groups then stay out of step, one in its
    // memory phases while the other runs its products and sweeps.  Group 0
    // releases group 1 at the latest when it leaves its item loop.
    bool stag_wait = g == 1 && first < items && !failed, stag_sent = g == 1;

    auto gbar = [&]() { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); };
    auto gwait = [&](uint64_t *bar, uint32_t &ph, bool cluster_scope) {
        const bool ok = cluster_scope ? mbar_wait_cl(bar, ph) : mbar_wait(bar, ph);
        if (!ok) s_flag[g] = 1;
        gbar();
        const bool good = s_flag[g] == 0;
        if (good) ph ^= 1u;
        return good;
    };
    // one DSMEM exchange with the peer: this thread's 16 bytes out, the
    // peer's 16 bytes for the same row back (false on a timeout)
    auto exchange = [&](float4 v, float4 &in) {
        const uint32_t s = xq & 1u, par = (xq >> 1) & 1u;
        st_async16(r_xch + (s * 128 + gt) * 16, v, r_barx + s * 8);
        if (gt == 0) mbar_expect_tx(bar_x + s, 128 * 16);
        uint32_t p = par;
        const bool ok = gwait(bar_x + s, p, true);
        ++xq;
        if (ok) in = xch[s * 128 + gt];
        return ok;
    };
    auto group_max = [&](float v) {
        v = warp_max(v);
        if (lane == 0) f_red[warp & 3] = v;
        tc_fence_before();
        gbar();
        tc_fence_after();
        return fmaxf(fmaxf(f_red[0], f_red[1]), fmaxf(f_red[2], f_red[3]));
    };

    for (long long item = first; item < items && !failed; item += stride) {
        fail_item = item;
        if (stag_wait) {
            uint32_t ps = 0;
            if (!gwait(bar_stagger, ps, false)) { failed = true; break; }
            stag_wait = false;
        }
        const int o = (int)(item / nb), b = (int)(item % nb);
        const int l = (o & 1) ? (o >> 1) + t.N : (o >> 1);
        const int m = l <= t.N ? l : l - t.N;
        const double xl2 = 2.0 * (t.xlamm[m] - 1.0);
        {   // BM_m (pot/pot3.f:226-230) of this CTA's columns
            const int jl = gt, j = col0 + jl;
            double bm = 0.0;
            if (jl < NH && j < M) {
                bm = t.bm0[j] + xl2 * t.cc[j];
                if (j == 0) bm = t.bm0[0] + (((m & 1) ? -1.0 : 1.0) - 1.0) * t.ammin + xl2 * t.cc[0];
            }
            d_bm[jl] = bm;
        }
        double *cr = x.corr + (size_t)b * x.scorr + (size_t)l * 16 + 8 * rank;
        const int row0 = (b * t.L + l) * K;             // first tensor-map row of this item
        double u0 = 0.0;                                // scale of x0 in tensor memory (2^eu0)
        int eu0 = 0;
        double ym_keep = 0.0, edge_in = 0.0;            // X(k, M); the peer's x0 edge in u0 units
        float sxf = 0.f;
        gbar();

        for (int it = 0; it < nit && !failed; ++it) {
            const bool res_x = it > 0;
            const uint32_t acc = G + (res_x ? 128u : 0u);   // product / sweep columns
            const uint32_t rcol = G + 128u;                 // residual columns
            // ---- residual r = d_k (Y - A_m x) (FP64) -> TMEM as FP32, this
            // CTA's columns in 16-column tiles through a four-slot ring.  Each
            // warp loads, reads and recycles only its own 32 rows of a slot
            // (one tensor-map box per warp and tile, one mbarrier per warp and
            // slot), so the warps of the group never wait for one another in
            // this loop: an issuing thread waits while the copy engine takes
            // in its bytes, and every warp now pays that for its own 4 KB
            const int quad = warp & 3;
            const bool wrows = 32 * quad < K;               // this warp's rows hold data
            auto issue = [&](int c) {
                if (c >= nch || !wrows) return;
                const int sl = c % kPairRing;
                ring_pend |= 1u << sl;
                uint8_t *slot = sB + sl * kPairTileB + quad * 4096;
                const int x0c = col0 + 16 * c;
                if (x0c < J) {
                    if (lane == 0) {
                        fence_proxy_async();
                        mbar_expect_tx(bar_ring + sl, (uint32_t)(min(K, 32) * 128));
                        tma_load_2d(slot, &tm_l, x0c, row0 + 32 * quad, bar_ring + sl);
                    }
                } else {
                    for (int i = lane; i < 32 * 16; i += 32) reinterpret_cast<double *>(slot)[i] = 0.0;
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar_ring + sl);
                }
            };
            bool wbad = false;                              // a wait of this warp ran out
            auto landed = [&](int c) {
                if (!wrows) return;
                const int sl = c % kPairRing;
                if (mbar_wait(bar_ring + sl, (ring_ph >> sl) & 1u)) {
                    ring_ph ^= 1u << sl;
                    ring_pend &= ~(1u << sl);
                } else {
                    s_flag[g] = 1;
                    wbad = true;
                }
            };
            auto at = [&](const uint8_t *slot, int k, int q) -> const double * {
                return reinterpret_cast<const double *>(slot + k * 128 + ((((q >> 1) ^ (k & 7))) << 4) + ((q & 1) << 3));
            };
            const int k = kq;
            const bool krow = k < NZ;
            const double bnk = d_bn[k];
            float rmax = 0.0f;
            if (res_x) {
                // x0's top and bottom rows of every warp for the vertical
                // neighbours across warps, staged once for all chunks
                float *my = f_edge + quad * 256;
                for (int c0 = 0; c0 < NH; c0 += 32) {
                    float v[32];
                    tm_ld32(tmem + lane_base + G + c0, v);
                    if (lane == 0) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) my[c0 + u] = v[u];
                    }
                    if (lane == 31) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) my[128 + c0 + u] = v[u];
                    }
                }
            }
            fence_proxy_async();
            gbar();
            for (int c = 0; c < kPairRing - 1; ++c) issue(c);
            const float *eu = f_edge + (quad > 0 ? quad - 1 : quad) * 256 + 128;   // row 32 quad - 1
            const float *ed = f_edge + (quad < 3 ? quad + 1 : quad) * 256;         // row 32 quad + 32
            const float zu = quad > 0 ? 1.f : 0.f, zd = quad < 3 ? 1.f : 0.f;
            for (int c = 0; c < nch; ++c) {
                const int c0 = 16 * c;
                float xc[16], xlf = 0.f, xrt = 0.f;
                if (res_x) {
                    const int jl = c0 - 1, jr = c0 + 16;
                    tm_ld16_nw(tmem + lane_base + G + c0, xc);
                    tm_ld1_nw(tmem + lane_base + G + (uint32_t)(jl < 0 ? 0 : jl), xlf);
                    tm_ld1_nw(tmem + lane_base + G + (uint32_t)(jr < NH ? jr : NH - 1), xrt);
                    landed(c);
                    tm_wait_ld18(xc, xlf, xrt);
                } else {
                    landed(c);
                }
                if (wbad) break;
                // this warp's rows of the slot of chunk c - 1 are read: reuse it
                __syncwarp();
                issue(c + kPairRing - 1);
                const uint8_t *slot = sB + (c % kPairRing) * kPairTileB;
                double yv[16];
#pragma unroll
                for (int u = 0; u < 16; u += 2) {
                    const double2 t2 = *reinterpret_cast<const double2 *>(at(slot, k, u));
                    yv[u] = pig4k * t2.x;
                    yv[u + 1] = pig4k * t2.y;
                }
                if (k == NZ - 1) {
#pragma unroll
                    for (int u = 0; u < 16; u += 2) {
                        const double2 t3 = *reinterpret_cast<const double2 *>(at(slot, NZ, u));
                        yv[u] = fma(-cnmaxk, t3.x, yv[u]);
                        yv[u + 1] = fma(-cnmaxk, t3.y, yv[u + 1]);
                    }
                }
                const int uM = M - 1 - (col0 + c0);     // column M lies in the tile of column M-1
                if (uM >= 0 && uM < 16) {
                    const double yM = *at(slot, k, uM + 1);
                    ym_keep = yM;
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        if (u == uM) yv[u] = fma(-cmmaxk, yM, yv[u]);
                }
                float v[16];
                if (res_x) {
                    const bool top0 = lane == 0, bot31 = lane == 31;
                    double xd_[18];
                    // the neighbours across the pair's column boundary come from the peer
                    xd_[0] = c0 == 0 ? (rank == 1 ? edge_in : 0.0) : (double)xlf;
                    xd_[17] = c0 + 16 == NH ? (rank == 0 ? edge_in : 0.0) : (double)xrt;
#pragma unroll
                    for (int u = 0; u < 16; ++u) xd_[u + 1] = (double)xc[u];
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int jl = c0 + u, j = col0 + jl;
                        float xu = __shfl_up_sync(0xffffffffu, xc[u], 1);
                        float xd = __shfl_down_sync(0xffffffffu, xc[u], 1);
                        const float eu_u = eu[jl] * zu, ed_u = ed[jl] * zd;
                        xu = top0 ? eu_u : xu;
                        xd = bot31 ? ed_u : xd;
                        double ax = (bnk + d_bm[jl]) * xd_[u + 1];
                        ax = fma(an_s, (double)xu, ax);
                        ax = fma(cn_s, (double)xd, ax);
                        ax = fma(d_am[jl], xd_[u], ax);
                        ax = fma(d_cm[jl], xd_[u + 2], ax);
                        const double r = fma(-u0, ax, yv[u]);
                        const bool in = krow && j < M;
                        sxf = fmaf(in ? xc[u] : 0.f, xc[u], sxf);
                        v[u] = in ? (float)r : 0.f;
                        rmax = fmaxf(rmax, fabsf(v[u]));
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int j = col0 + c0 + u;
                        v[u] = (krow && j < M) ? (float)yv[u] : 0.f;
                        rmax = fmaxf(rmax, fabsf(v[u]));
                    }
                }
                tm_st16_nw(tmem + lane_base + rcol + c0, v);
            }
            tm_wait_st();
            if (!stag_sent && it == nit - 1) {
                if (gt == 0) mbar_arrive(bar_stagger);
                stag_sent = true;
            }
            const int k1 = pow2_exp(group_max(rmax));
            if (s_flag[g]) { failed = true; break; }
            const float s1 = ldexpf(1.0f, k1);
            // ---- TMEM r -> B tile (row j, K index k), FP16 hi/lo
            for (int c0 = 0; c0 < NH; c0 += 32) {
                float v[32];
                tm_ld32(tmem + lane_base + rcol + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) v[u] *= s1;
                split_rows32(sBh, sBl, v, c0, kq, lane, NH);
            }
            fence_proxy_async();
            tc_fence_before();
            gbar();
            // ---- W = Q^T r into TMEM cols [acc, acc + NH)
            if (a_wait) {
                uint32_t pa = 0;
                if (!gwait(bar_a, pa, false)) { failed = true; break; }
                a_wait = false;
            }
            if (gt == 0) gemm_issue(tmem + acc, sA, sBh, NH, idesc, bar_mma, false);
            mma_pend = true;
            // the first chunk of pivot reciprocals is loaded while the product runs
            const float *swp = x.sw_piv + (size_t)m * NT * 128 + kq;    // global row j at swp[j * 128]
            float R[32];
#pragma unroll
            for (int u = 0; u < 32; ++u) R[u] = swp[(size_t)((rank == 0 ? 0 : clast) + u) * 128];
            if (!gwait(bar_mma, ph_mma, false)) { failed = true; break; }
            mma_pend = false;
            tc_fence_after();
            float *cvs = reinterpret_cast<float *>(sB);   // [local row][p] multipliers
            if (lane == 0) {
                // a quarter of the multipliers per warp of the group (an
                // issuing thread waits while the copy engine takes in its
                // bytes, so no warp takes all four)
                const int q = warp & 3;
                const float *src = x.sw_mul + ((size_t)m * NT + col0) * 128;
                if (q == 0) mbar_expect_tx(bar_cv, (uint32_t)NH * 512);
                bulk_g2s(cvs + q * NH * 32, src + q * NH * 32, (uint32_t)NH * 128, bar_cv);
            }
            cv_pend = true;
            // ---- radial sweeps (T_r(m) + lam_p) w = W_p on this CTA's rows:
            // top-down over [0, h) (rank 0) or bottom-up over [h, M) (rank 1),
            // then the meeting rows h-1 and h from both, then the back sweep
            float xmax = 0.0f;
            const int p = kq;
            const bool live = p < NZ;
            const uint32_t tb = tmem + lane_base + acc;
            const int ks = 12 + k1;                     // the sweep values are 2^ks times W
            {
                float yv[32], Rn[32];
                float yp = 0.f;
                if (rank == 0) {
                    for (int c0 = 0; c0 < NH; c0 += 32) {
                        if (c0 + 32 < NH) {
#pragma unroll
                            for (int u = 0; u < 32; ++u) Rn[u] = swp[(size_t)(c0 + 32 + u) * 128];
                        }
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            const float rr = R[u], ar = f_t[c0 + u].y * rr;
                            yp = fmaf(-ar, yp, yv[u] * rr);
                            yv[u] = yp;
                        }
                        tm_st32_nw(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) R[u] = Rn[u];
                    }
                } else {
                    for (int c0 = clast; c0 >= h; c0 -= 32) {
                        if (c0 - 32 >= h) {
#pragma unroll
                            for (int u = 0; u < 32; ++u) Rn[u] = swp[(size_t)(c0 - 32 + u) * 128];
                        }
                        const int cl0 = c0 - col0;
                        tm_ld32(tb + cl0, yv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            const float rr = R[u], cr_ = f_t[cl0 + u].z * rr;
                            const float yn = fmaf(-cr_, yp, yv[u] * rr);
                            yp = (c0 + u < M) ? yn : yp;   // uniform
                            yv[u] = yn;
                        }
                        tm_st32_nw(tb + cl0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) R[u] = Rn[u];
                    }
                }
                tm_wait_st();
                if (!gwait(bar_cv, ph_cv, false)) { failed = true; break; }
                cv_pend = false;
                // meeting rows h-1 (rank 0's last) and h (rank 1's first), in
                // FP64 from both halves' values at their own scales:
                // x_t = y'_t + (1-e_t) x_u, x_u = y''_u + (1-f_u) x_t
                const float mine_c = cvs[(rank == 0 ? NH - 1 : 0) * 128 + p];
                float4 in;
                if (!exchange(make_float4(yp, mine_c, __int_as_float(ks), 0.f), in)) { failed = true; break; }
                const int ks_peer = __float_as_int(in.z);
                const double yt = rank == 0 ? ldexp((double)yp, -ks) : ldexp((double)in.x, -ks_peer);
                const double yu = rank == 0 ? ldexp((double)in.x, -ks_peer) : ldexp((double)yp, -ks);
                const double et = rank == 0 ? (double)mine_c : (double)in.y;
                const double fu = rank == 0 ? (double)in.y : (double)mine_c;
                const double xtd = (yt + (1.0 - et) * yu) / ((et + fu) - et * fu);
                const double xud = yu + (1.0 - fu) * xtd;
                if (rank == 0) {
                    float xn = (float)ldexp(xtd, ks);   // x_{j+1} while sweeping up
                    for (int c0 = NH - 32; c0 >= 0; c0 -= 32) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) Rn[u] = cvs[(c0 + u) * 128 + p];
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 31; u >= 0; --u) {
                            float xv = yv[u] + (1.0f - Rn[u]) * xn;
                            xv = (c0 + u == NH - 1) ? xn : xv;
                            xn = xv;
                            yv[u] = live ? xv : 0.f;
                            xmax = fmaxf(xmax, fabsf(yv[u]));
                        }
                        tm_st32_nw(tb + c0, yv);
                    }
                } else {
                    float xpv = (float)ldexp(xud, ks);  // x_{j-1} while sweeping down
                    for (int c0 = 0; c0 < NH; c0 += 32) {
#pragma unroll
                        for (int u = 0; u < 32; ++u) Rn[u] = cvs[(c0 + u) * 128 + p];
                        tm_ld32(tb + c0, yv);
#pragma unroll
                        for (int u = 0; u < 32; ++u) {
                            float xv = yv[u] + (1.0f - Rn[u]) * xpv;
                            xv = (c0 + u == 0) ? xpv : xv;
                            xpv = xv;
                            yv[u] = (live && col0 + c0 + u < M) ? xv : 0.f;
                            xmax = fmaxf(xmax, fabsf(yv[u]));
                        }
                        tm_st32_nw(tb + c0, yv);
                    }
                }
                tm_wait_st();
            }
            const int k2 = pow2_exp(group_max(xmax));
            const float s2 = ldexpf(1.0f, k2);
            // ---- TMEM w -> B tile (row j, K index p), FP16 hi/lo
            for (int c0 = 0; c0 < NH; c0 += 32) {
                float v[32];
                tm_ld32(tb + c0, v);
#pragma unroll
                for (int u = 0; u < 32; ++u) v[u] *= s2;
                split_rows32(sBh, sBl, v, c0, kq, lane, NH);
            }
            fence_proxy_async();
            tc_fence_before();
            gbar();
            // ---- Q w (delta times d) into TMEM cols [acc, acc + NH): the resident tile, transposed
            if (gt == 0) gemm_issue(tmem + acc, sA, sBh, NH, idesc, bar_mma, true);
            mma_pend = true;
            if (!gwait(bar_mma, ph_mma, false)) { failed = true; break; }
            mma_pend = false;
            tc_fence_after();
            const int eun = -(24 + k1 + k2);            // this solve's result is 2^eun times the columns
            const double unscale = ldexp(1.0, eun);
            if (it + 1 < nit) {
                // x0 stays in tensor memory columns [G, G + NH); its edge column
                // goes to the peer for the correction residual
                u0 = unscale;
                eu0 = eun;
                float te;
                tm_ld1_nw(tmem + lane_base + G + (uint32_t)(rank == 0 ? NH - 1 : 0), te);
                asm volatile("tcgen05.wait::ld.sync.aligned;" : "+f"(te)::"memory");
                float4 in;
                if (!exchange(make_float4(te, 0.f, __int_as_float(eu0), 0.f), in)) { failed = true; break; }
                edge_in = ldexp((double)in.x, __float_as_int(in.z) - eu0);
                continue;
            }
            // ---- X = x0 + delta (FP64), staged as 16-column tiles (128-byte
            // swizzle) and written by the copy engine as rows 0..KMAX-2 (the
            // boundary row is not written); column M carries X's own value
            // back.  Each warp stages and stores its own 32 rows (the last
            // warp with data one row fewer), so no group barrier is needed
            double sd = 0.0, sx = 0.0;
            const double uk = unscale * ek, u0k = u0 * ek;     // this row's 1/d_k
            const int srows = min(32, K - 1 - 32 * quad);
            const CUtensorMap *smap = srows == 32 ? &tm_s : &tm_sl;
            float dv[16], xv[16];
            tm_ld16_nw(tmem + lane_base + acc, dv);
            tm_ld16_nw(tmem + lane_base + G, xv);   // x0 (unused after a single solve)
            for (int c = 0; c < nch; ++c) {
                const int c0 = 16 * c;
                uint8_t *slot = sB + (c % kPairStage) * kPairTileB;
                // this warp's store of the slot's previous chunk has read it
                if (lane == 0) bulk_wait_read<kPairStage - 1>();
                __syncwarp();
                tm_wait_ld32(dv, xv);
                double xn[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int j = col0 + c0 + u;
                    const double dl = (double)dv[u] * uk;
                    xn[u] = (res_x ? (double)xv[u] * u0k : 0.0) + dl;
                    if (kq < NZ && j < M) {
                        sd += dl * dl;
                        sx += xn[u] * xn[u];
                    }
                    if (j == M) xn[u] = ym_keep;        // column M (uniform in the warp)
                }
                if (c + 1 < nch) {
                    tm_ld16_nw(tmem + lane_base + acc + c0 + 16, dv);
                    tm_ld16_nw(tmem + lane_base + G + c0 + 16, xv);
                }
#pragma unroll
                for (int u = 0; u < 16; u += 2)
                    *reinterpret_cast<double2 *>(slot + kq * 128 + (((u >> 1) ^ (kq & 7)) << 4)) =
                        make_double2(xn[u], xn[u + 1]);
                fence_proxy_async();
                __syncwarp();
                if (lane == 0 && srows > 0 && col0 + c0 < J) {
                    tma_store_2d(smap, col0 + c0, row0 + 32 * quad, slot + quad * 4096);
                    bulk_commit();
                }
            }
            if (lane == 0) bulk_wait_all();             // tiles written, staging free for the next item
            // per-half sums (the host adds the two halves)
            sd = warp_sum(sd);
            sx = warp_sum(sx);
            double sq = warp_sum((double)sxf * ek * ek);
            gbar();
            if (lane == 0) { d_red[warp & 3] = sd; d_red[8 + (warp & 3)] = sx; d_red[16 + (warp & 3)] = sq; }
            gbar();
            if (gt == 0) {
                double a = 0.0, bb = 0.0, q = 0.0;
                for (int i = 0; i < 4; ++i) { a += d_red[i]; bb += d_red[8 + i]; q += d_red[16 + i]; }
                if (res_x) {                            // the first solve's delta is x0 itself
                    cr[0] = q * u0 * u0;
                    cr[1] = q * u0 * u0;
                }
                cr[2 * it] = a;
                cr[2 * it + 1] = bb;
            }
            gbar();
        }
    }
    if (!stag_sent && gt == 0) mbar_arrive(bar_stagger);
    // drain this group's copies and products still in flight (bounded)
    for (int sl = 0; sl < kPairRing; ++sl)
        if (ring_pend & (1u << sl)) mbar_wait(bar_ring + sl, (ring_ph >> sl) & 1u);
    if (cv_pend) mbar_wait(bar_cv, ph_cv);
    if (mma_pend) mbar_wait(bar_mma, ph_mma);
    if (failed) {
        // this half of every mode the group left unsolved becomes NaN
        if (gt == 0) {
            bulk_wait_all();
            atomicExch(x.err, 1);
        }
        gbar();
        const double qnan = __longlong_as_double(0x7ff8000000000000ll);
        for (long long item = fail_item; item < items; item += stride) {
            const int o = (int)(item / nb), b = (int)(item % nb);
            const int l = (o & 1) ? (o >> 1) + t.N : (o >> 1);
            double *Xl = w.X + (size_t)b * w.sX + (size_t)l * K * J;
            for (int i = gt; i < NZ * NH; i += 128) {
                const int kk = i / NH, j = col0 + i % NH;
                if (j < M) Xl[(size_t)kk * J + j] = qnan;
            }
        }
    }
    if (tid == 0 && a_inflight) mbar_wait(bar_a, 0);
    tc_fence_before();
    __syncthreads();
    // no peer writes into this CTA's shared memory after this point
    cluster_sync_all();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// ---------------------------------------------------------------------------
// Wide pipeline: grids whose radial extent does not fit one CTA's tiles
// (JMAX > 256, e.g. the 512 x 128 x 512 serving class) or whose rows are not
// 16-byte tiles (JMAX not a multiple of 16).  The same refinement as
// k_mode_mixed -- FP64 residual, FP16 hi/lo tensor-core transforms with FP32
// accumulation, FP32 radial sweeps from the same sweep table, FP64 update --
// as five kernels per approximate solve, with the intermediate FP32 arrays in
// device memory:
//   k_wide_resid   r = Y - A x (FP64) -> R[item][j][k] (FP32), per-tile max |r|
//   k_wide_gemm    W = U r: one CTA per (item, 256-column tile), tcgen05
//   k_wide_sweep   (T_r(m) + lam_p) w = W_p, one thread per (item, p) -> R
//   k_wide_gemm    delta = V w
//   k_wide_update  x += delta (FP64); the last solve writes X's interior
// ---------------------------------------------------------------------------
constexpr int kWideN = 256;      // GEMM N tile (radial columns)
constexpr int kWideMaxJ = 1024;  // largest JMAX of the wide pipeline
constexpr int kWideTiles = kWideMaxJ / kWideN;

template <bool kFirst>
__global__ void __launch_bounds__(256) k_wide_resid(DevTables t, Work w, MixedDev x, WideDev d, int nb)
{
    __shared__ float tile[32][129];
    __shared__ float red[8];
    const int item = blockIdx.y, b = item / t.L, l = item % t.L, j0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, j = j0 + tx;
    const int M = t.M, NZ = t.NZ, J = t.J;
    const int m = l <= t.N ? l : l - t.N;
    const double xl2 = 2.0 * (t.xlamm[m] - 1.0);
    const double *Xl = w.X + (size_t)b * w.sX + (size_t)l * t.K * J;
    const double *xl = d.xit + (size_t)item * d.sxit;
    double bmj = 0.0, amj = 0.0, cmj = 0.0;
    if (j < M) {
        bmj = t.bm0[j] + xl2 * t.cc[j];
        if (j == 0) bmj = t.bm0[0] + (((m & 1) ? -1.0 : 1.0) - 1.0) * t.ammin + xl2 * t.cc[0];
        amj = t.am[j];
        cmj = t.cm[j];
    }
    float vmax = 0.0f;
    for (int k = ty; k < 128; k += 8) {
        float v = 0.0f;
        if (k < NZ && j < M) {
            // 4 pi G rho with the boundary folds (pot/pot3.f:212-224)
            double r = t.pig4 * Xl[(size_t)k * J + j];
            if (k == NZ - 1) r = r - t.cnmax * Xl[(size_t)NZ * J + j];
            if (j == M - 1) r = r - t.cmmax * Xl[(size_t)k * J + M];
            if (!kFirst) {
                const double *xr = xl + (size_t)k * J;
                double ax = (t.bn[k] + bmj) * xr[j];
                if (k > 0) ax += t.an[k] * xl[(size_t)(k - 1) * J + j];
                if (k < NZ - 1) ax += t.cn[k] * xl[(size_t)(k + 1) * J + j];
                if (j > 0) ax += amj * xr[j - 1];
                if (j < M - 1) ax += cmj * xr[j + 1];
                r = r - ax;
            }
            v = (float)(x.zsc[k] * r);   // times d_k for the orthogonal transform
        }
        tile[tx][k] = v;
        vmax = fmaxf(vmax, fabsf(v));
    }
    __syncthreads();
    float *Ri = d.R + (size_t)item * d.sro;
    for (int e = threadIdx.x; e < 32 * 128; e += 256) {
        const int jj = e >> 7, k = e & 127;
        Ri[(size_t)(j0 + jj) * 128 + k] = tile[jj][k];
    }
    vmax = warp_max(vmax);
    if ((threadIdx.x & 31) == 0) red[ty] = vmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mx = red[0];
        for (int i = 1; i < 8; ++i) mx = fmaxf(mx, red[i]);
        if (mx > 0.0f) atomicMax(d.rmax + (size_t)item * d.nt + j0 / kWideN, __float_as_uint(mx));
    }
}

// out[item][j][row] = sum_k A(row, k) in[item][j][k] for one 256-column tile:
// A is the plan's 2^12-scaled FP16 hi/lo image of Q^T, or with trans its
// transpose Q; the input tile is scaled by a power of two from its maximum
// and split to FP16 hi/lo in shared memory, three MMA passes accumulate in
// FP32 in tensor memory.
__global__ void __launch_bounds__(256, 1) k_wide_gemm(const uint8_t *aimg, const float *in, float *out,
                                                      const unsigned *tmax, WideDev d, int trans, int *err)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x, item = blockIdx.y;
    uint8_t *sA = sm, *sBh = sm + kAImg, *sBl = sBh + (size_t)kWideN * 256;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sBl + (size_t)kWideN * 256);   // [0] product, [1] A tile
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 2);
    int *flag = reinterpret_cast<int *>(slot + 1);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        mbar_expect_tx(&bars[1], kAImg);
        bulk_g2s(sA, aimg, kAImg, &bars[1]);
    }
    const float s = pow2_scale(__uint_as_float(tmax[(size_t)item * d.nt + tile]));
    // the tile's rows as 16-byte loads, eight in flight per thread
    const float4 *src = reinterpret_cast<const float4 *>(in + (size_t)item * d.sro + (size_t)tile * kWideN * 128);
#pragma unroll 8
    for (int i = tid; i < kWideN * 32; i += 256) {
        const float4 v = src[i];
        const int row = i >> 5, k = (i & 31) * 4;
        put_split(sBh, sBl, row, k, kWideN, v.x * s);
        put_split(sBh, sBl, row, k + 1, kWideN, v.y * s);
        put_split(sBh, sBl, row, k + 2, kWideN, v.z * s);
        put_split(sBh, sBl, row, k + 3, kWideN, v.w * s);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    // the A tile: every thread waits (bounded); a phase counts only if all saw it
    bool a_ok = mbar_wait(&bars[1], 0);
    if (!a_ok) *flag = 1;
    __syncthreads();
    a_ok = *flag == 0;
    const uint32_t idesc = (1u << 4) | ((uint32_t)(kWideN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    if (a_ok && tid == 0) gemm_issue(tmem, sA, sBh, kWideN, idesc, &bars[0], trans != 0);
    bool d_ok = a_ok && mbar_wait(&bars[0], 0);
    if (a_ok && !d_ok) *flag = 1;
    __syncthreads();
    d_ok = *flag == 0;
    tc_fence_after();
    float *dst = out + (size_t)item * d.sro + (size_t)tile * kWideN * 128;
    const int q = warp & 3, row = 32 * q + lane;
    if (d_ok) {
        const float unscale = 1.0f / (kAScale * s);
        for (int c0 = (warp >> 2) * 128; c0 < (warp >> 2) * 128 + 128; c0 += 32) {
            float v[32];
            tm_ld32(tmem + ((uint32_t)(32 * q) << 16) + c0, v);
#pragma unroll
            for (int u = 0; u < 32; ++u) dst[(size_t)(c0 + u) * 128 + row] = v[u] * unscale;
        }
    } else {
        // drain (bounded) what is still in flight, then make the tile NaN so the
        // failure reaches PHI, and raise the error word
        if (!a_ok) mbar_wait(&bars[1], 0);
        else mbar_wait(&bars[0], 0);
        for (int c0 = (warp >> 2) * 128; c0 < (warp >> 2) * 128 + 128; ++c0) dst[(size_t)c0 * 128 + row] = __int_as_float(0x7fc00000);
        if (tid == 0) atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem));
}

// (T_r(m) + lam_p) w = W_p for each p (thread) of one item (block), with the
// sweep table's pivot reciprocals and multipliers: rows [0, h) top-down,
// [h, M) bottom-up, meeting at rows h-1 and h -- k_mode_mixed's sweeps on
// CUDA cores.  W comes from O, w goes to R (zero past M and for p >= NZ).
__global__ void __launch_bounds__(128) k_wide_sweep(DevTables t, MixedDev x, WideDev d)
{
    extern __shared__ float s_tab[];   // AM, CM as FP32 (M each)
    float *s_am = s_tab, *s_cm = s_tab + t.M;
    __shared__ float red[4][kWideTiles];
    const int item = blockIdx.x, l = item % t.L, p = threadIdx.x, M = t.M;
    const int m = l <= t.N ? l : l - t.N;
    const int NTs = x.ntile, h = 32 * ((M + 63) / 64);
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        s_am[j] = (float)t.am[j];
        s_cm[j] = (float)t.cm[j];
    }
    __syncthreads();
    const float *W = d.O + (size_t)item * d.sro + p;
    float *wo = d.R + (size_t)item * d.sro + p;
    const float *piv = x.sw_piv + (size_t)m * NTs * 128 + p, *mul = x.sw_mul + (size_t)m * NTs * 128 + p;
    float tmx[kWideTiles];
#pragma unroll
    for (int i = 0; i < kWideTiles; ++i) tmx[i] = 0.0f;
    if (p < t.NZ) {
        float yp = 0.0f;
#pragma unroll 8
        for (int j = 0; j < h; ++j) {
            const float rr = piv[(size_t)j * 128], ar = s_am[j] * rr;
            yp = fmaf(-ar, yp, W[(size_t)j * 128] * rr);
            wo[(size_t)j * 128] = yp;
        }
        const float yt = yp;
        yp = 0.0f;
#pragma unroll 8
        for (int j = M - 1; j >= h; --j) {
            const float rr = piv[(size_t)j * 128], cr = s_cm[j] * rr;
            yp = fmaf(-cr, yp, W[(size_t)j * 128] * rr);
            wo[(size_t)j * 128] = yp;
        }
        const float yu = yp, et = mul[(size_t)(h - 1) * 128], fu = mul[(size_t)h * 128];
        const float xt = (yt + (1.0f - et) * yu) / ((et + fu) - et * fu);
        const float xu = yu + (1.0f - fu) * xt;
        float xn = xt;
        wo[(size_t)(h - 1) * 128] = xt;
        tmx[(h - 1) / kWideN] = fmaxf(tmx[(h - 1) / kWideN], fabsf(xt));
#pragma unroll 8
        for (int j = h - 2; j >= 0; --j) {
            xn = wo[(size_t)j * 128] + (1.0f - mul[(size_t)j * 128]) * xn;
            wo[(size_t)j * 128] = xn;
            tmx[j / kWideN] = fmaxf(tmx[j / kWideN], fabsf(xn));
        }
        float xp = xu;
        wo[(size_t)h * 128] = xu;
        tmx[h / kWideN] = fmaxf(tmx[h / kWideN], fabsf(xu));
#pragma unroll 8
        for (int j = h + 1; j < M; ++j) {
            xp = wo[(size_t)j * 128] + (1.0f - mul[(size_t)j * 128]) * xp;
            wo[(size_t)j * 128] = xp;
            tmx[j / kWideN] = fmaxf(tmx[j / kWideN], fabsf(xp));
        }
        for (int j = M; j < d.Jt; ++j) wo[(size_t)j * 128] = 0.0f;
    } else {
        for (int j = 0; j < d.Jt; ++j) wo[(size_t)j * 128] = 0.0f;
    }
    for (int i = 0; i < d.nt; ++i) {
        const float v = warp_max(tmx[i]);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < d.nt) {
        const float v = fmaxf(fmaxf(red[0][threadIdx.x], red[1][threadIdx.x]), fmaxf(red[2][threadIdx.x], red[3][threadIdx.x]));
        if (v > 0.0f) atomicMax(d.wmax + (size_t)item * d.nt + threadIdx.x, __float_as_uint(v));
    }
}

// x += delta (FP64) for one item per block; the last solve writes X's
// interior.  Per-item sums of delta^2 and x^2 go to the correction report.
__global__ void __launch_bounds__(256) k_wide_update(DevTables t, Work w, MixedDev x, WideDev d, int it, int last)
{
    __shared__ float tile[128][33];
    __shared__ double red[2][8];
    const int item = blockIdx.x, b = item / t.L, l = item % t.L, M = t.M, NZ = t.NZ, J = t.J;
    double *Xl = w.X + (size_t)b * w.sX + (size_t)l * t.K * J;
    double *xl = d.xit + (size_t)item * d.sxit;
    const float *O = d.O + (size_t)item * d.sro;
    double sd = 0.0, sx = 0.0;
    for (int j0 = 0; j0 < M; j0 += 32) {
        for (int e = threadIdx.x; e < 32 * 128; e += 256) {
            const int jj = e >> 7, k = e & 127;
            tile[k][jj] = O[(size_t)(j0 + jj) * 128 + k];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 32 * NZ; e += 256) {
            const int k = e >> 5, jj = e & 31, j = j0 + jj;
            if (j < M) {
                const double dl = (double)tile[k][jj] * x.zsc[128 + k];   // Q w / d_k
                const size_t o = (size_t)k * J + j;
                const double xn = (it > 0 ? xl[o] : 0.0) + dl;
                if (last) Xl[o] = xn;
                else xl[o] = xn;
                sd += dl * dl;
                sx += xn * xn;
            }
        }
        __syncthreads();
    }
    sd = warp_sum(sd);
    sx = warp_sum(sx);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sd;
        red[1][threadIdx.x >> 5] = sx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int i = 0; i < 8; ++i) {
            a += red[0][i];
            c += red[1][i];
        }
        double *cr = x.corr + (size_t)item * 16;
        cr[2 * it] = a;
        cr[2 * it + 1] = c;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int round64(int v) { return (v + 63) / 64 * 64; }

// Grids the single-kernel mode solve covers; the others take the wide
// pipeline.
static bool mixed_fused(const chy::HostPlan *hp) { return hp->J % 16 == 0 && round64(hp->J) <= kMaxN; }

bool chy_mixed_supported(const chy::HostPlan *hp)
{
    return hp->NZ <= 127 && hp->J >= 64 && (mixed_fused(hp) || hp->J <= kWideMaxJ);
}

// Radial sweep table: for every azimuthal index m = 0..N and vertical
// eigenvalue p (padding rows use -1), the multipliers of the two-sided
// elimination of (T_r(m) + lam_p) in excess form and the pivot reciprocals,
// as two FP32 planes, the multipliers e_j or f_j, then the pivot reciprocals
// 1/D_j, each of layout [m][j][p] (j < ntile, p < 128).
// Rows [0, h) are eliminated top-down, rows [h, M) bottom-up,
// h = 32 ceil(M / 64).  They do not depend on the data, so they are formed
// once, in FP64, here.
std::vector<float> chy::mixed_sweep_table(const chy::HostPlan &hp)
{
    const int M = hp.M, NT = round64(hp.J), n = hp.N, h = 32 * ((M + 63) / 64);
    const size_t plane = (size_t)(n + 1) * NT * 128;
    std::vector<float> t(plane * 2, 0.0f);
    std::vector<double> g(M);
    for (int m = 0; m <= n; ++m) {
        const double xl2 = 2.0 * (hp.xlamm[m] - 1.0);
        const double axis = (((m & 1) ? -1.0 : 1.0) - 1.0) * hp.ammin;
        for (int j = 0; j < M; ++j) {
            g[j] = xl2 * hp.cc[j];
            if (j == 0) g[j] = axis + g[j];
            if (j == M - 1) g[j] = g[j] - hp.cmmax;
        }
        for (int p = 0; p < 128; ++p) {
            const double lam = p < hp.NZ ? hp.lam[p] : -1.0;
            auto put = [&](int j, double c, double r) {
                const size_t o = ((size_t)m * NT + j) * 128 + p;
                t[o] = (float)c;
                t[plane + o] = (float)r;
            };
            double e = 0.0;
            for (int j = 0; j < h; ++j) {
                const double tt = (g[j] + lam) - hp.am[j] * e, rr = 1.0 / (tt - hp.cm[j]);
                e = tt * rr;
                put(j, e, rr);
            }
            double f = 0.0;
            for (int j = M - 1; j >= h; --j) {
                const double tt = (g[j] + lam) - hp.cm[j] * f, rr = 1.0 / (tt - hp.am[j]);
                f = tt * rr;
                put(j, f, rr);
            }
        }
    }
    return t;
}

// Per vertical row k (128, padding rows 1, 1, 0, 0): d_k, 1/d_k,
// d_k AN_k / d_(k-1) and d_k CN_k / d_(k+1), with D = diag(d) the symmetriser
// of T_z (U = Q^T D, V = D^-1 Q).
std::vector<double> chy::mixed_row_scales(const chy::HostPlan &hp)
{
    const int NZ = hp.NZ;
    std::vector<double> z(4 * 128, 0.0);
    for (int k = 0; k < 128; ++k) z[k] = z[128 + k] = 1.0;
    for (int k = 0; k < NZ; ++k) {
        z[k] = hp.dsc[k];
        z[128 + k] = 1.0 / hp.dsc[k];
    }
    for (int k = 0; k < NZ; ++k) {
        z[256 + k] = k > 0 ? hp.dsc[k] * hp.an[k] / hp.dsc[k - 1] : 0.0;
        z[384 + k] = k + 1 < NZ ? hp.dsc[k] * hp.cn[k] / hp.dsc[k + 1] : 0.0;
    }
    return z;
}

size_t chy_mixed_pack_tables(const chy::HostPlan *hp, std::vector<char> *image, bool mixed)
{
    if (!mixed) return image->size();
    // [Q^T hi | Q^T lo]: a K-major swizzled FP16 tile of 2^12 * Q(k,p) (rows p,
    // K index k); read through the MN-major descriptor it is 2^12 * Q
    std::vector<uint8_t> img((size_t)kAImg, 0);
    const int NZ = hp->NZ;
    for (int p = 0; p < NZ; ++p)
        for (int k = 0; k < NZ; ++k) {
            const double v = (double)kAScale * hp->Qt[(size_t)p * NZ + k];
            const __half h = __double2half(v);
            const __half l = __double2half(v - (double)__half2float(h));
            const uint32_t o = kmaj_off(p, k, kTiles);
            std::memcpy(&img[o], &h, 2);
            std::memcpy(&img[kTiles * kTiles * 2 + o], &l, 2);
        }
    size_t off = (image->size() + 1023) & ~(size_t)1023;
    image->resize(off + img.size());
    std::memcpy(image->data() + off, img.data(), img.size());
    // eigenvalues as FP32, padded with -1 (any nonzero diagonal works for the
    // zero padding rows), then the row scales, then the sweep table, each at
    // the next 256-byte boundary
    std::vector<float> lam(128, -1.0f);
    for (int p = 0; p < NZ; ++p) lam[p] = (float)hp->lam[p];
    auto append = [&](const void *src, size_t bytes) {
        const size_t o = (image->size() + 255) & ~(size_t)255;
        image->resize(o + bytes);
        std::memcpy(image->data() + o, src, bytes);
    };
    append(lam.data(), lam.size() * sizeof(float));
    const std::vector<double> zsc = chy::mixed_row_scales(*hp);
    append(zsc.data(), zsc.size() * sizeof(double));
    const std::vector<float> sw = chy::mixed_sweep_table(*hp);
    append(sw.data(), sw.size() * sizeof(float));
    return off;
}

std::vector<double> chy::mixed_operand_tiles(const chy::HostPlan &hp)
{
    std::vector<char> image;
    const size_t off = chy_mixed_pack_tables(&hp, &image, true);
    std::vector<double> out((size_t)2 * kTiles * kTiles);
    for (int t = 0; t < 2; ++t) {
        const size_t base = off + (size_t)t * kTiles * kTiles * 2;
        for (int r = 0; r < kTiles; ++r)
            for (int k = 0; k < kTiles; ++k) {
                __half h;
                std::memcpy(&h, image.data() + base + kmaj_off(r, k, kTiles), 2);
                out[((size_t)t * kTiles + r) * kTiles + k] = (double)__half2float(h);
            }
    }
    return out;
}

void chy_mixed_bind_tables(chy_plan *p, char *dev_base)
{
    if (!p->mx) p->mx = new MixedState();
    if (p->precision != CHY_PREC_MIXED) return;   // no mixed tables packed
    p->mx->dev.aimg = reinterpret_cast<const uint8_t *>(dev_base);
    const size_t lam_off = (((size_t)(dev_base - p->d_tables) + kAImg) + 255) & ~(size_t)255;
    p->mx->dev.lam = reinterpret_cast<const float *>(p->d_tables + lam_off);
    const size_t zsc_off = (lam_off + 128 * sizeof(float) + 255) & ~(size_t)255;
    p->mx->dev.zsc = reinterpret_cast<const double *>(p->d_tables + zsc_off);
    const size_t sw_off = (zsc_off + 4 * 128 * sizeof(double) + 255) & ~(size_t)255;
    p->mx->dev.sw_mul = reinterpret_cast<const float *>(p->d_tables + sw_off);
    p->mx->dev.sw_piv = p->mx->dev.sw_mul + (size_t)(p->hp.N + 1) * round64(p->hp.J) * 128;
}

// Per-mode correction sums and the error word; the FP64 iterate of the
// general path (two or more corrections) is allocated by
// chy_mixed_ensure_iterate when such a count is set.
static size_t al32(size_t n) { return (n + 31) & ~(size_t)31; }   // doubles, 256-byte pieces

size_t chy_mixed_work_doubles(const chy_plan *p)
{
    if (p->precision != CHY_PREC_MIXED) return 0;
    const chy::HostPlan &hp = p->hp;
    size_t n = al32((size_t)hp.L * 16 * p->max_batch + 8);
    if (!mixed_fused(&hp)) {
        const size_t items = (size_t)hp.L * p->max_batch, Jt = (size_t)(hp.J + 255) / 256 * 256;
        n += al32(items * hp.K * hp.J);                  // iterate
        n += 2 * al32(items * Jt * 128 / 2);             // R, O (FP32)
        n += 2 * al32(items * (Jt / 256) / 2 + 1);       // rmax, wmax
    }
    return n;
}

void chy_mixed_bind_work(chy_plan *p, double *base)
{
    if (!p->mx) p->mx = new MixedState();
    MixedDev &d = p->mx->dev;
    const chy::HostPlan &hp = p->hp;
    d.sxb = (size_t)hp.L * hp.K * hp.J;
    d.scorr = (size_t)hp.L * 16;
    d.xbuf = nullptr;
    d.corr = base;
    d.err = reinterpret_cast<int *>(d.corr + d.scorr * p->max_batch);
    d.ntile = round64(hp.J);
    if (p->precision == CHY_PREC_MIXED && !mixed_fused(&hp)) {
        WideDev &wd = p->mx->wide;
        p->mx->is_wide = true;
        const size_t items = (size_t)hp.L * p->max_batch;
        wd.Jt = (hp.J + 255) / 256 * 256;
        wd.nt = wd.Jt / 256;
        double *q = base + al32((size_t)hp.L * 16 * p->max_batch + 8);
        wd.xit = q;
        wd.sxit = (size_t)hp.K * hp.J;
        q += al32(items * hp.K * hp.J);
        wd.sro = (size_t)wd.Jt * 128;
        wd.R = reinterpret_cast<float *>(q);
        q += al32(items * wd.sro / 2);
        wd.O = reinterpret_cast<float *>(q);
        q += al32(items * wd.sro / 2);
        wd.rmax = reinterpret_cast<unsigned *>(q);
        q += al32(items * wd.nt / 2 + 1);
        wd.wmax = reinterpret_cast<unsigned *>(q);
    }
    if (p->precision == CHY_PREC_MIXED) {
        cudaMallocHost(&p->mx->h_corr, sizeof(double) * d.scorr * p->max_batch);
        cudaMallocHost(&p->mx->h_err, sizeof(int));
        // the residual's right-hand-side tiles: X viewed as max_batch*L*K rows
        // of J doubles; one item is K consecutive rows
        PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
        if (enc && hp.K <= 256 && hp.J % 16 == 0) {
            const cuuint64_t dims[2] = {(cuuint64_t)hp.J, (cuuint64_t)p->max_batch * hp.L * hp.K};
            const cuuint64_t strides[1] = {(cuuint64_t)hp.J * sizeof(double)};
            const cuuint32_t box[2] = {16, (cuuint32_t)hp.K}, box_s[2] = {16, (cuuint32_t)(hp.K - 1)};
            const cuuint32_t es[2] = {1, 1};
            p->mx->tm_ok = enc(&p->mx->tm_x, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, p->w.X, dims, strides, box, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                           enc(&p->mx->tm_xs, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, p->w.X, dims, strides, box_s, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
            // k_mode_pair's per-warp boxes (rows 32 q .. 32 q + 31 of an item)
            const int nsw = (hp.K - 1 + 31) / 32, last = hp.K - 1 - 32 * (nsw - 1);
            const cuuint32_t box_pl[2] = {16, (cuuint32_t)std::min(hp.K, 32)}, box_ps[2] = {16, 32},
                             box_psl[2] = {16, (cuuint32_t)last};
            p->mx->tm_ok = p->mx->tm_ok &&
                           enc(&p->mx->tm_pl, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, p->w.X, dims, strides, box_pl, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                           enc(&p->mx->tm_ps, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, p->w.X, dims, strides, box_ps, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                           enc(&p->mx->tm_psl, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, p->w.X, dims, strides, box_psl, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }
    }
}

static int wide_solve(chy_plan *p, int nb, cudaStream_t s, int *launches)
{
    const MixedDev &x = p->mx->dev;
    const WideDev &d = p->mx->wide;
    const chy::DevTables &t = p->t;
    const int nit = std::min(1 + p->refine, 8), items = nb * t.L;
    const size_t gsm = (size_t)kAImg + (size_t)kWideN * 512 + 64;
    if (ensure_smem((const void *)k_wide_gemm, gsm) != cudaSuccess) return CHY_ERR_CUDA;
    for (int it = 0; it < nit; ++it) {
        const size_t mb = (size_t)items * d.nt * sizeof(unsigned);
        if (cudaMemsetAsync(d.rmax, 0, mb, s) != cudaSuccess || cudaMemsetAsync(d.wmax, 0, mb, s) != cudaSuccess)
            return CHY_ERR_CUDA;
        const dim3 rg(d.Jt / 32, items), gg(d.nt, items);
        if (it == 0) k_wide_resid<true><<<rg, 256, 0, s>>>(t, p->w, x, d, nb);
        else k_wide_resid<false><<<rg, 256, 0, s>>>(t, p->w, x, d, nb);
        k_wide_gemm<<<gg, 256, gsm, s>>>(x.aimg, d.R, d.O, d.rmax, d, 0, x.err);
        k_wide_sweep<<<items, 128, 2 * t.M * sizeof(float), s>>>(t, x, d);
        k_wide_gemm<<<gg, 256, gsm, s>>>(x.aimg, d.R, d.O, d.wmax, d, 1, x.err);
        k_wide_update<<<items, 256, 0, s>>>(t, p->w, x, d, it, it == nit - 1 ? 1 : 0);
        if (cudaGetLastError() != cudaSuccess) return CHY_ERR_CUDA;
    }
    *launches = 5 * nit;
    return CHY_OK;
}

int chy_mixed_solve(chy_plan *p, int nb, cudaStream_t s, int *launches)
{
    *launches = 0;
    if (p->mx->is_wide) return wide_solve(p, nb, s, launches);
    MixedDev d = p->mx->dev;
    d.probe_polls = p->mx->probe_polls;
    d.nit = 1 + p->refine;
    if (d.nit > 8) d.nit = 8;
    if (d.nit > 2 && !d.xbuf) return CHY_ERR_NOT_SETUP;
    // the kernel streams X and the iterate with 16-byte async copies
    if ((reinterpret_cast<uintptr_t>(p->w.X) | reinterpret_cast<uintptr_t>(d.xbuf)) % 16 != 0 || p->hp.J % 16 != 0)
        return CHY_ERR_ARG;
    const size_t sm = MixedSmem::bytes(d.ntile);
    // two approximate solves (one correction) keep the iterate in tensor memory
    if (d.nit <= 2 && !p->mx->tm_ok) return CHY_ERR_CUDA;   // tensor map over X not encoded
    const long long items = (long long)nb * p->hp.L;
    const int cap = p->mode_ctas > 0 && p->mode_ctas < p->num_sms ? p->mode_ctas : p->num_sms;
    if (d.nit <= 2 && p->mode_kernel != 1) {
        // CTA pairs, two items per CTA: chosen (mode_kernel 0) when each group
        // gets at least 16 items, so that the second group's half-item start
        // delay is paid back; both kernels give the same bits
        MixedState &ms = *p->mx;
        if (ms.pair_clusters < 0) {
            ms.pair_clusters = 0;
            if (ensure_smem((const void *)k_mode_pair, PairSmem::bytes) == cudaSuccess) {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = 2;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3(2 * (unsigned)p->num_sms, 1, 1);
                cfg.blockDim = dim3(256, 1, 1);
                cfg.dynamicSmemBytes = PairSmem::bytes;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                int n = 0;
                if (cudaOccupancyMaxActiveClusters(&n, (const void *)k_mode_pair, &cfg) == cudaSuccess) ms.pair_clusters = n;
                cudaGetLastError();
            }
        }
        if (ms.pair_clusters > 0 && (p->mode_kernel == 2 || items >= 32ll * ms.pair_clusters)) {
            long long pairs = (items + 1) / 2;
            pairs = std::min<long long>(pairs, ms.pair_clusters);
            pairs = std::min<long long>(pairs, std::max(1, cap / 2));
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = 2;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(2 * (unsigned)pairs, 1, 1);
            cfg.blockDim = dim3(256, 1, 1);
            cfg.dynamicSmemBytes = PairSmem::bytes;
            cfg.stream = s;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            if (cudaLaunchKernelEx(&cfg, k_mode_pair, p->t, p->w, d, nb, p->mx->tm_pl, p->mx->tm_ps, p->mx->tm_psl) != cudaSuccess)
                return CHY_ERR_CUDA;
            ms.paired = true;
            *launches = 1;
            return CHY_OK;
        }
    }
    p->mx->paired = false;
    const void *kern = d.nit <= 2 ? (const void *)k_mode_mixed<true> : (const void *)k_mode_mixed<false>;
    cudaError_t e = ensure_smem(kern, sm);
    if (e != cudaSuccess) return CHY_ERR_CUDA;
    const int grid = (int)(items < cap ? items : cap);
    if (d.nit <= 2) k_mode_mixed<true><<<grid, 256, sm, s>>>(p->t, p->w, d, nb, p->mx->tm_x, p->mx->tm_xs);
    else k_mode_mixed<false><<<grid, 256, sm, s>>>(p->t, p->w, d, nb, p->mx->tm_x, p->mx->tm_xs);
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

int chy_mixed_read_error(chy_plan *p, int *host_word, cudaStream_t s)
{
    if (p->precision != CHY_PREC_MIXED || !p->mx || !host_word) return CHY_OK;
    if (cudaMemcpyAsync(host_word, p->mx->dev.err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemsetAsync(p->mx->dev.err, 0, sizeof(int), s) != cudaSuccess)
        return CHY_ERR_CUDA;
    return CHY_OK;
}

int *chy_mixed_host_error_word(chy_plan *p)
{
    return (p->precision == CHY_PREC_MIXED && p->mx) ? p->mx->h_err : nullptr;
}

int chy_mixed_last_kernel(const chy_plan *p)
{
    if (p->precision != CHY_PREC_MIXED || !p->mx) return 0;
    if (p->mx->is_wide) return 3;
    return p->mx->paired ? 2 : 1;
}

int chy_dbg_mixed_probe_set(chy_plan *p, int polls)
{
    if (p->precision != CHY_PREC_MIXED || !p->mx || polls < 0) return CHY_ERR_ARG;
    p->mx->probe_polls = polls;
    return CHY_OK;
}

void chy_mixed_fill_diag(const chy_plan *p, int slot, chy_diag *d)
{
    d->iterations = 0;
    if (p->precision != CHY_PREC_MIXED || !p->mx || !p->mx->h_corr) return;
    const int nit = std::min(1 + p->refine, 8);
    const double *c = p->mx->h_corr + (size_t)slot * p->mx->dev.scorr;
    d->iterations = nit;
    // k_mode_pair leaves one sum per radial half: [0, 4) and [8, 12)
    const bool halves = p->mx->paired;
    for (int it = 0; it < nit && it < 8; ++it) {
        double sd = 0.0, sx = 0.0;
        for (int l = 0; l < p->hp.L; ++l) {
            sd += c[(size_t)l * 16 + 2 * it];
            sx += c[(size_t)l * 16 + 2 * it + 1];
            if (halves) {
                sd += c[(size_t)l * 16 + 8 + 2 * it];
                sx += c[(size_t)l * 16 + 8 + 2 * it + 1];
            }
        }
        d->corr_rel[it] = sx > 0.0 ? std::sqrt(sd / sx) : 0.0;
    }
}

size_t chy_mixed_iterate_bytes(const chy_plan *p) { return p->mx ? p->mx->xbuf_bytes : 0; }

int chy_mixed_ensure_iterate(chy_plan *p)
{
    // the wide pipeline keeps its own FP64 iterate for any number of corrections
    if (p->precision != CHY_PREC_MIXED || !p->mx || p->mx->dev.xbuf || p->mx->is_wide) return CHY_OK;
    MixedDev &d = p->mx->dev;
    const size_t bytes = d.sxb * p->max_batch * sizeof(double);
    if (cudaMalloc(&d.xbuf, bytes) != cudaSuccess) {
        cudaGetLastError();
        d.xbuf = nullptr;
        return CHY_ERR_NOMEM;
    }
    p->mx->xbuf_bytes = bytes;
    // columns >= M and rows >= NZ are read as zeros and never written
    return cudaMemset(d.xbuf, 0, bytes) == cudaSuccess ? CHY_OK : CHY_ERR_CUDA;
}

void chy_mixed_release(chy_plan *p)
{
    if (!p->mx) return;
    cudaFree(p->mx->dev.xbuf);
    cudaFreeHost(p->mx->h_corr);
    cudaFreeHost(p->mx->h_err);
    delete p->mx;
    p->mx = nullptr;
}

// ---------------------------------------------------------------------------
// Self-test of the tensor-core path: D = (2^12 Q^T) * Bm^T for one tile (with
// trans: 2^12 Q, the same tile through the transposed descriptor), where Bm
// (NT x 128, row-major FP32) is split to FP16 hi/lo by the same code the
// solver uses.  Writes D (128 x NT, row-major FP32).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_umma_selftest(const uint8_t *aimg, const float *Bm, float *D, int NT,
                                                          int trans, int *err)
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
    if (ok && tid == 0) gemm_issue(tmem, sA, sBh, NT, idesc, &bars[0], trans != 0);
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

// Test hook: which = 0 multiplies by the plan's tile (2^12 Q^T), 1 by its
// transpose (2^12 Q).
extern "C" int chy_dbg_umma(chy_plan *p, int which, const float *Bm_dev, float *D_dev, int NT)
{
    if (!p || !p->mx || !Bm_dev || !D_dev || NT < 64 || NT > 256 || NT % 64) return CHY_ERR_ARG;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return CHY_ERR_NOMEM;
    cudaMemset(err, 0, sizeof(int));
    const size_t sm = (size_t)kAImg + (size_t)NT * 512 + 64;
    ensure_smem((const void *)k_umma_selftest, sm);
    k_umma_selftest<<<1, 128, sm>>>(p->mx->dev.aimg, Bm_dev, D_dev, NT, which ? 1 : 0, err);
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(err);
    if (e != cudaSuccess) return CHY_ERR_CUDA;
    return h ? CHY_ERR_TIMEOUT : CHY_OK;
}

// k_fft.cu -- azimuthal transforms and everything fused with them.
//
// Compiled with --fmad=false: every product and sum of the transforms is a
// separately rounded IEEE operation, in the order pot/fft.f performs it, so
// the device transform reproduces the reference's (single-precision-angle)
// transform bit for bit.  Fused multiply-adds are requested explicitly
// (__fma_rn) only where the reference order is not reproduced anyway (ring
// moments, boundary synthesis).
//
// One CTA owns TC adjacent (J,K) columns and holds their LMAX samples in
// shared memory.  The forward tile has rows of stride RS = TC+2 doubles: row
// 2q is Re(z_q) and row 2q+1 is Im(z_q) of the LMAX/2-point complex sequence
// z_q = rho(2q) + i rho(2q+1) that POT3 builds (pot/pot3.f:95-98).  The
// inverse tile has rows of stride TC in split layout: Re(z_q) in row q, Im(z_q)
// in row IM0+q.  Tiles arrive as TMA boxes of tensor maps over RHO and X
// (16-byte aligned rows), else as asynchronous copies; global stores run along
// J, the fastest dimension of the reference's arrays, so they are coalesced.
// The stage structure is fixed at compile time per LMAX; the rotations, output
// permutation and REALTR recurrence values are the recorded tables, staged in
// shared memory.
#include "devplan.h"

#include <cstring>
#include <type_traits>

namespace chy {

// ---------------------------------------------------------------------------
// Compile-time stage structure of pot/fft.f's factorisation for N = 2^e
// (fft.f:147-187): [4]^a, middle, [4]^a with e = 4a + r and middle = {},
// {2}, {4}, {2,2,2} for r = 0..3.
// ---------------------------------------------------------------------------
template <int N>
struct Shape {
    static constexpr int log2n()
    {
        int e = 0;
        while ((1 << e) < N) ++e;
        return e;
    }
    static constexpr int nst()
    {
        const int e = log2n(), a = e / 4, r = e % 4;
        return 2 * a + (r == 0 ? 0 : (r == 3 ? 3 : 1));
    }
    static constexpr int radix(int s)
    {
        const int e = log2n(), a = e / 4, r = e % 4;
        if (s < a || s >= nst() - a) return 4;
        return r == 2 ? 4 : 2;
    }
    static constexpr int span(int s)
    {
        int sp = N;
        for (int i = 0; i <= s; ++i) sp /= radix(i);
        return sp;
    }
};

template <int L>
struct Tile {
    static constexpr int N = L / 2;
    static constexpr int TC = L <= 128 ? 32 : (L <= 256 ? 16 : 8);  // columns per CTA
    static constexpr int RS = TC + 2;                               // row stride (doubles, even)
    static constexpr int ROWS = L + 2;
    static constexpr int TPC = 256 / TC;                            // threads per column
    // inverse tile (split layout, row stride TC): Re rows 0..N, Im rows from
    // IM0 (a 128-byte boundary, for the tensor-map copies)
    static constexpr int IM0 = (TC * 8) % 128 == 0 ? N + 1 : N + 2;
    static constexpr int ROWSI = IM0 + N + 1;
};

// Shared-memory copy of one direction's tables.
struct FftSmem {
    double *tw;        // [ncompact][6]
    uint8_t *on;       // [ncompact]
    int *perm;         // [n]
    double *rt;        // [nh][2]
};

// 3-D tensor maps over each solve's RHO(J+2, K+2, L), one per batch slot:
// boxes of TC+2 columns x one K x up to 256 L, no swizzle, no multicast.  A
// box lands as L rows of TC+2 doubles, the tile's own row stride.
struct RhoMaps {
    CUtensorMap m[kMaxBatchPtrs];
};

__device__ __forceinline__ uint32_t sm32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            sm32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(sm32(bar))
        : "memory");
}
// bounded wait on an mbarrier phase; false on timeout
__device__ __forceinline__ bool fwd_bar_wait(uint64_t *bar, uint32_t parity)
{
    for (long long i = 0; i < (1ll << 26); ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(sm32(bar)), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// Asynchronous global -> shared copies (bytes = 0: the destination is zeroed;
// src must still be a valid address).  cp_async_wait_all() then a barrier
// make them visible to the block.
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Starts the copies of one direction's tables (completed by the caller's
// cp_async_wait_all + barrier).
__device__ __forceinline__ void load_fft_tables(const FftDev &f, const FftSmem &s)
{
    for (int i = threadIdx.x; i < f.ncompact * 6; i += blockDim.x) cp_async8(s.tw + i, f.twc + i, 8);
    for (int i = threadIdx.x; i < f.n; i += blockDim.x) cp_async4(s.perm + i, f.perm + i);
    for (int i = threadIdx.x; i < 2 * f.nh; i += blockDim.x) cp_async8(s.rt + i, f.rt + i, 8);
    for (int i = threadIdx.x; i < f.ncompact; i += blockDim.x) s.on[i] = f.onc[i];
}

// Bytes of one direction's tables as bulk_fft_tables moves them.
__device__ __forceinline__ uint32_t fft_bulk_bytes(const FftDev &f)
{
    return (uint32_t)(f.ncompact * 48 + f.nh * 16 + f.n * 4 + ((f.ncompact + 15) & ~15));
}

// One direction's tables as four bulk copies (one per table, issued by
// lane 0 of warps w0 .. w0+3) counted on bar: every source and destination
// starts on a 16-byte boundary and the flag bytes are padded to 16 (the
// packed table image leaves 256-byte gaps).  A bulk copy holds its issuing
// thread while the copy engine takes it in, so no warp issues more than one.
__device__ __forceinline__ void bulk_fft_tables(const FftDev &f, const FftSmem &s, uint64_t *bar, int w0)
{
    const int w = (int)(threadIdx.x >> 5) - w0;
    if ((threadIdx.x & 31) != 0 || w < 0 || w > 3) return;
    const void *src = w == 0 ? (const void *)f.twc : w == 1 ? (const void *)f.rt : w == 2 ? (const void *)f.perm : (const void *)f.onc;
    void *dst = w == 0 ? (void *)s.tw : w == 1 ? (void *)s.rt : w == 2 ? (void *)s.perm : (void *)s.on;
    const uint32_t bytes = w == 0 ? f.ncompact * 48 : w == 1 ? f.nh * 16 : w == 2 ? f.n * 4 : (f.ncompact + 15) & ~15;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sm32(dst)),
                 "l"(src), "r"(bytes), "r"(sm32(bar))
                 : "memory");
}

template <int L>
__host__ __device__ constexpr size_t fft_table_bytes()
{
    // twiddles <= N entries x 6 doubles, flags, perm, REALTR (N/2+1) x 2
    return (size_t)(L / 2) * 6 * 8 + (size_t)(L / 2) + (size_t)(L / 2) * 4 + (size_t)(L / 4 + 1) * 16 + 64;
}

template <int L>
__device__ __forceinline__ FftSmem carve_fft(char *p)
{
    constexpr int N = L / 2;
    FftSmem s;
    s.tw = (double *)p;
    p += (size_t)N * 6 * 8;
    s.rt = (double *)p;
    p += (size_t)(N / 2 + 1) * 16;
    s.perm = (int *)p;
    p += (size_t)N * 4;
    s.on = (uint8_t *)p;
    return s;
}

// One butterfly of pot/fft.f's radix-2 or radix-4 step on values held in
// registers, in the reference's operation order (compiled without FMA
// contraction, so every product and sum rounds as there).  tw: the recorded
// rotations of this position, on: whether they apply.
template <int R, bool FWD>
__device__ __forceinline__ void butterfly(double &a0, double &b0, double &a1, double &b1, double &a2, double &b2,
                                          double &a3, double &b3, bool on, const double *tw)
{
    if constexpr (R == 2) {
        if (!on) {
            const double ak = a1, bk = b1;
            a1 = a0 - ak;
            b1 = b0 - bk;
            a0 = a0 + ak;
            b0 = b0 + bk;
        } else {
            const double c1 = tw[0], s1 = tw[1];
            const double ak = a0 - a1, bk = b0 - b1;
            a0 = a0 + a1;
            b0 = b0 + b1;
            a1 = c1 * ak - s1 * bk;
            b1 = s1 * ak + c1 * bk;
        }
    } else {
        double akp = a0 + a2, akm = a0 - a2, ajp = a1 + a3, ajm = a1 - a3;
        const double A0 = akp + ajp;
        ajp = akp - ajp;
        double bkp = b0 + b2, bkm = b0 - b2, bjp = b1 + b3, bjm = b1 - b3;
        const double B0 = bkp + bjp;
        bjp = bkp - bjp;
        if constexpr (FWD) {
            akp = akm - bjm; akm = akm + bjm; bkp = bkm + ajm; bkm = bkm - ajm;
        } else {
            akp = akm + bjm; akm = akm - bjm; bkp = bkm - ajm; bkm = bkm + ajm;
        }
        a0 = A0;
        b0 = B0;
        if (on) {
            a1 = akp * tw[0] - bkp * tw[1]; b1 = akp * tw[1] + bkp * tw[0];
            a2 = ajp * tw[2] - bjp * tw[3]; b2 = ajp * tw[3] + bjp * tw[2];
            a3 = akm * tw[4] - bkm * tw[5]; b3 = akm * tw[5] + bkm * tw[4];
        } else {
            a1 = akp; b1 = bkp; a2 = ajp; b2 = bjp; a3 = akm; b3 = bkm;
        }
    }
}

// Stages S and S+1 of the transform in one pass over shared memory (S alone
// when it is the last).  Stage S+1 works inside the blocks of stage S, so the
// R_S * R_{S+1} elements base + i H_{S+1} of a group are closed under both
// stages: a thread loads them, applies stage S's R_{S+1} butterflies and then
// stage S+1's R_S butterflies in registers, and stores them back.  Each
// butterfly is the one the element-by-element stage loop would apply.
//
// Layout of the complex element e in the tile (row stride RS): interleaved
// (Re in row 2e, Im in row 2e+1) or split (Re in row e, Im in row IM0+e).
template <int L, int S, bool FWD, int RS = Tile<L>::RS, bool SPLIT = false>
__device__ __forceinline__ void stage_pairs(double *A, const FftSmem &s, const FftDev &f)
{
    using T = Tile<L>;
    using Sh = Shape<T::N>;
    auto rre = [](int e) { return SPLIT ? e : 2 * e; };
    auto rim = [](int e) { return SPLIT ? T::IM0 + e : 2 * e + 1; };
    if constexpr (S < Sh::nst()) {
        constexpr bool two = S + 1 < Sh::nst();
        constexpr int R1 = Sh::radix(S), H1 = Sh::span(S);
        constexpr int R2 = two ? Sh::radix(S + 1) : 1, H2 = two ? Sh::span(S + 1) : H1;
        constexpr int G = R1 * R2, NG = T::N / G;
        const int off1 = f.off[S], off2 = two ? f.off[S + 1] : 0;
        for (int w = threadIdx.x; w < NG * T::TC; w += blockDim.x) {
            const int c = w % T::TC, gi = w / T::TC;
            const int j = gi % H2, base = (gi / H2) * (R1 * H1) + j;
            double re[G], im[G];
#pragma unroll
            for (int i = 0; i < G; ++i) {
                re[i] = A[rre(base + i * H2) * RS + c];
                im[i] = A[rim(base + i * H2) * RS + c];
            }
            // stage S: butterflies m = 0..R2-1 on elements m + t R2 (t < R1)
#pragma unroll
            for (int m = 0; m < R2; ++m) {
                const int js = j + m * H2;
                const bool on = s.on[off1 + js] != 0;
                const double *tw = s.tw + (size_t)(off1 + js) * 6;
                if constexpr (R1 == 2)
                    butterfly<2, FWD>(re[m], im[m], re[m + R2], im[m + R2], re[m], im[m], re[m], im[m], on, tw);
                else
                    butterfly<4, FWD>(re[m], im[m], re[m + R2], im[m + R2], re[m + 2 * R2], im[m + 2 * R2],
                                      re[m + 3 * R2], im[m + 3 * R2], on, tw);
            }
            if constexpr (two) {
                // stage S+1: butterflies t = 0..R1-1 on elements t R2 + m' (m' < R2)
                const bool on = s.on[off2 + j] != 0;
                const double *tw = s.tw + (size_t)(off2 + j) * 6;
#pragma unroll
                for (int t = 0; t < R1; ++t) {
                    const int e = t * R2;
                    if constexpr (R2 == 2)
                        butterfly<2, FWD>(re[e], im[e], re[e + 1], im[e + 1], re[e], im[e], re[e], im[e], on, tw);
                    else
                        butterfly<4, FWD>(re[e], im[e], re[e + 1], im[e + 1], re[e + 2], im[e + 2], re[e + 3],
                                          im[e + 3], on, tw);
                }
            }
#pragma unroll
            for (int i = 0; i < G; ++i) {
                A[rre(base + i * H2) * RS + c] = re[i];
                A[rim(base + i * H2) * RS + c] = im[i];
            }
        }
        __syncthreads();
        stage_pairs<L, two ? S + 2 : S + 1, FWD, RS, SPLIT>(A, s, f);
    }
}

// REALTR (pot/fft.f:2-70): the N/2+1 (j, N-j) pairs are independent once the
// recurrence values are tabulated.  On the inverse tile: split layout, row
// stride TC (Re of element e in row e, Im in row IM0+e).
template <int L>
__device__ __forceinline__ void realtr_pairs(double *A, const FftSmem &s)
{
    using T = Tile<L>;
    constexpr int n = T::N, nh = n / 2 + 1, RS = T::TC, I0 = T::IM0;
#pragma unroll
    for (int it = 0; it < (nh * T::TC + 255) / 256; ++it) {
        const int w = threadIdx.x + 256 * it;
        if (w >= nh * T::TC) break;
        const int c = w % T::TC, j = w / T::TC, k = n - j;
        const double cn = s.rt[2 * j], sn = s.rt[2 * j + 1];
        const double aj = A[j * RS + c], bj = A[(I0 + j) * RS + c];
        const double ak = A[k * RS + c], bk = A[(I0 + k) * RS + c];
        const double aa = aj + ak, ab = aj - ak, ba = bj + bk, bb = bj - bk;
        const double re = cn * ba + sn * ab, im = sn * ba - cn * ab;
        if (j != k) {
            A[(I0 + k) * RS + c] = im - bb;
            A[k * RS + c] = aa - re;
        }
        A[(I0 + j) * RS + c] = im + bb;
        A[j * RS + c] = aa + re;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Forward transform of the interior columns + ring moments
// ---------------------------------------------------------------------------
// Grid: (ceil(M/TC), NZ, batch).  Reads RHO(2:JMAX, 2:KMAX, :) -- the cells
// POT3 copies into PHI (pot/pot3.f:70-82) and BDYGEN integrates
// (pot/boundary.f:366-370) -- and writes X interior plus MOM.
template <int L>
__global__ void __launch_bounds__(256) k_forward(DevTables t, BatchPtrs bp, Work w, int vec16,
                                                 const __grid_constant__ RhoMaps maps)
{
    using T = Tile<L>;
    extern __shared__ __align__(128) char smem_raw[];
    // Row l of the tile holds RHO(J0+1 .. J0+TC+2, K, L) at columns -1 .. TC:
    // the view A is shifted by one element, so A[l*RS + c] is column
    // j = j0 + c (RHO(j + 2, ...)), and the 16-byte granules of a row start
    // on 16-byte boundaries (RS even).
    double *A0 = (double *)smem_raw;
    double *A = A0 + 1;
    double *mtab = A0 + (size_t)T::ROWS * T::RS;           // [20][L/4] cos, sin of m psi
    FftSmem fs = carve_fft<L>((char *)(mtab + 20 * (L / 4)));
    const int J2 = t.J + 2, K2 = t.K + 2;
    const int j0 = blockIdx.x * T::TC, k = blockIdx.y, b = blockIdx.z;
    const double *rho = bp.rho[b];
    // vec16 == 2: the tile arrives as TMA boxes of the tensor map of this
    // solve's RHO, counted on tbar (after the tables)
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smem_raw + (size_t)T::ROWS * T::RS * 8 + (size_t)20 * (L / 4) * 8 +
                                                  fft_table_bytes<L>());
    if (vec16 == 2) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm32(tbar)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm32(tbar)),
                         "r"((uint32_t)(L * T::RS * 8) + fft_bulk_bytes(t.fwd) + 20u * (L / 4) * 8u));
            for (int l0 = 0; l0 < L; l0 += 256) tma_load_3d(A0 + (size_t)l0 * T::RS, &maps.m[b], j0, k + 1, l0, tbar);
        }
        // the tables on the same barrier: the transform's by lane 0 of warps
        // 1-4, the 20 moment rows (L/4 cos or sin values each) by lanes 0-3
        // of warps 5-7, 0 and 1, one row per thread
        bulk_fft_tables(t.fwd, fs, tbar, 1);
        {
            const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
            const int m = ln < 4 ? (w >= 5 ? (w - 5) * 4 + ln : 12 + w * 4 + ln) : 99;
            if (m < 20) {
                const double *src = m < 10 ? t.cosm + (size_t)m * L : t.sinm + (size_t)(m - 10) * L;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        sm32(mtab + (size_t)m * (L / 4))),
                    "l"(src), "r"((uint32_t)(L / 4) * 8u), "r"(sm32(tbar))
                    : "memory");
            }
        }
    } else {
        // tables and the tile's samples: every copy in flight at once
        load_fft_tables(t.fwd, fs);
        for (int i = threadIdx.x; i < 20 * (L / 4); i += blockDim.x) {
            const int m = i / (L / 4), l = i % (L / 4);
            cp_async8(mtab + i, m < 10 ? t.cosm + (size_t)m * L + l : t.sinm + (size_t)(m - 10) * L + l, 8);
        }
    }
    if (vec16 == 2) {
        // copies issued above
    } else if (vec16) {
        // 16-byte copies of the granules e = j0 .. j0+TC+1 of each row (RHO
        // 16-byte aligned, JMAX+2 even); granules past the row read as zero
        constexpr int NG = T::TC / 2 + 1;
        for (int i = threadIdx.x; i < L * NG; i += blockDim.x) {
            const int g = i % NG, l = i / NG, e = j0 + 2 * g;
            const bool ok = e + 1 < J2;
            cp_async16(A0 + l * T::RS + 2 * g, ok ? rho + (size_t)e + (size_t)J2 * ((k + 1) + (size_t)K2 * l) : rho,
                       ok ? 16 : 0);
        }
    } else {
        for (int i = threadIdx.x; i < L * T::TC; i += blockDim.x) {
            const int c = i % T::TC, l = i / T::TC, j = j0 + c;
            const bool ok = j < t.M;
            cp_async8(A + l * T::RS + c, ok ? rho + (size_t)(j + 1) + (size_t)J2 * ((k + 1) + (size_t)K2 * l) : rho,
                      ok ? 8 : 0);
        }
    }
    cp_async_wait_all();
    // a tile that did not arrive in time makes this tile's modes NaN, so the
    // failure reaches PHI instead of passing silently
    const bool landed = vec16 != 2 || fwd_bar_wait(tbar, 0);
    __syncthreads();

    // azimuthal moments of each ring (pot/boundary.f:527-538), before DV, using
    // psi -> pi - psi, pi + psi, 2 pi - psi to fold the sum to a quarter period
    {
        // The first half of the block forms the cosine sums (q = 0..10), the
        // second half the sine sums (q = 11..20), of every column of the tile
        // at once, TPM = 128/TC threads per column.  With 8 threads per
        // column, lanes alternate between a half-warp's two columns (so that
        // a half-warp reads 8 rows of 2 columns: no bank conflict at the even
        // row stride); otherwise a column's threads are consecutive lanes.
        // SH is the lane distance between a column's threads g and g+1.
        // A warp's table reads serve 4 (TC = 16) columns at a time.
        constexpr int TPM = 128 / T::TC;
        constexpr int SH = TPM == 8 ? 2 : 1;
        const int th = threadIdx.x & 127;
        const int c = SH == 2 ? 2 * (th >> 4) + (th & 1) : th / TPM;
        const int g = SH == 2 ? (th & 15) >> 1 : th % TPM;
        constexpr int Q = L / 4;
        // Butterfly reduce-scatter over the column's TPM lanes (the half's
        // sums padded to NS): at each level a lane keeps half of its live
        // sums and adds the partner's copy of them, so lane g ends with the
        // column totals of sums base(g) .. base(g) + NS/TPM - 1.  Every total
        // is the same pairwise tree over the TPM lanes whichever lane ends
        // with it.
        constexpr int NS = TPM > 16 ? TPM : 16;
        const int j = j0 + c;
        double *mom = w.mom + (size_t)b * w.smom + (size_t)k * t.M + j;
        auto pass = [&](auto sine) {
            constexpr bool S = decltype(sine)::value;
            constexpr int NQ = S ? 10 : 11, Q0 = S ? 11 : 0;
            double a[NS];
#pragma unroll
            for (int q = 0; q < NS; ++q) a[q] = 0.0;
#pragma unroll
            for (int il = 0; il < Q / TPM; ++il) {
                const int l = g + il * TPM;
                const double r1 = A[l * T::RS + c], r2 = A[(L / 2 - 1 - l) * T::RS + c];
                const double r3 = A[(L / 2 + l) * T::RS + c], r4 = A[(L - 1 - l) * T::RS + c];
                if constexpr (!S) {
                    const double e = r1 + r4, f = r2 + r3;
                    const double ce = e + f, co = e - f;
                    a[0] += ce;
#pragma unroll
                    for (int m = 1; m <= 10; ++m) a[m] = __fma_rn(mtab[(m - 1) * Q + l], (m & 1) ? co : ce, a[m]);
                } else {
                    const double gg = r1 - r4, h = r3 - r2;
                    const double se = gg + h, so = gg - h;
#pragma unroll
                    for (int m = 1; m <= 10; ++m)
                        a[m - 1] = __fma_rn(mtab[(9 + m) * Q + l], (m & 1) ? so : se, a[m - 1]);
                }
            }
            int base = 0;
#pragma unroll
            for (int lev = 0; (TPM >> (lev + 1)) >= 1; ++lev) {
                const int o = TPM >> (lev + 1), W = NS >> lev;
                const bool up = (g & o) != 0;
#pragma unroll
                for (int i = 0; i < W / 2; ++i) {
                    const double send = up ? a[i] : a[W / 2 + i];
                    const double keep = up ? a[W / 2 + i] : a[i];
                    a[i] = keep + __shfl_xor_sync(0xffffffffu, send, o * SH);
                }
                base += up ? W / 2 : 0;
            }
            if (j < t.M) {
#pragma unroll
                for (int i = 0; i < NS / TPM; ++i)
                    if (base + i < NQ) mom[(size_t)(Q0 + base + i) * t.nring] = a[i];
            }
        };
        if (threadIdx.x < 128) pass(std::integral_constant<bool, false>{});
        else pass(std::integral_constant<bool, true>{});
    }
    __syncthreads();

    stage_pairs<L, 0, true>(A, fs, t.fwd);

    // REALTR (pot/fft.f:2-70) on the transform in natural order -- its sample
    // q is row perm[q], and A(N+1) = A(1) (pot/fft.f:44-45) -- with the modes
    // of pot/pot3.f:135-140 written straight to X: A1(q+1) is mode q
    // (q = 0..N), B1(q+1) mode N+q (q = 1..N-1).  The (j, N-j) pairs are
    // independent, and each row is read by exactly one pair.
    double *X = w.X + (size_t)b * w.sX;
    constexpr int n = T::N, nh = n / 2 + 1;
    const size_t pl = (size_t)t.K * t.J;
#pragma unroll
    for (int it = 0; it < (nh * T::TC + 255) / 256; ++it) {
        const int i = threadIdx.x + 256 * it;
        if (i >= nh * T::TC) break;
        const int c = i % T::TC, jp = i / T::TC, kp = n - jp, j = j0 + c;
        const int sj = fs.perm[jp], sk = fs.perm[kp < n ? kp : 0];
        const double cn = fs.rt[2 * jp], sn = fs.rt[2 * jp + 1];
        const double aj = A[(2 * sj) * T::RS + c], bj = A[(2 * sj + 1) * T::RS + c];
        const double ak = A[(2 * sk) * T::RS + c], bk = A[(2 * sk + 1) * T::RS + c];
        const double aa = aj + ak, ab = aj - ak, ba = bj + bk, bb = bj - bk;
        const double re = cn * ba + sn * ab, im = sn * ba - cn * ab;
        if (j < t.M) {
            double *xc = X + (size_t)k * t.J + j;
            xc[(size_t)jp * pl] = (aa + re) * t.sf1;
            if (jp != kp) xc[(size_t)kp * pl] = (aa - re) * t.sf1;
            if (jp >= 1) xc[(size_t)(n + jp) * pl] = (im + bb) * t.sf1;
            if (jp >= 1 && jp != kp) xc[(size_t)(n + kp) * pl] = (im - bb) * t.sf1;
            if (!landed) xc[0] = __longlong_as_double(0x7ff8000000000000ll);
        }
    }
}

// ---------------------------------------------------------------------------
// Boundary potentials (pot/boundary.f:659-833) and their transform
// ---------------------------------------------------------------------------
// Grid: (ceil(njk/8), 1, batch).  For each boundary point: MASSIN/MASSOUT
// from the prefix/suffix sums and TRMTOT (pot/boundary.f:782-806).  The
// boundary potential (pot/boundary.f:814-830) is
//   PHI(psi_l) = -G [c_0 + sum_m (c_m cos m psi_l + s_m sin m psi_l)]
// with c_0 = sum_L TRMTOT(1,(L,0)), c_m = 2 sum_L TRMTOT(1,(L,m)),
// s_m = 2 sum_L TRMTOT(2,(L,m)).  POT3 then transforms the boundary columns
// (pot/pot3.f:93-140); the transform being linear, the modes are the same
// combination of the recorded transforms of {1, cos m psi, sin m psi}.
__global__ void __launch_bounds__(256) k_bdy_synth(DevTables t, Work w)
{
    constexpr int kPts = 8;
    __shared__ double trm[kPts][132];
    __shared__ double cq[kPts][21];
    __shared__ int colidx[132];
    const int q0 = blockIdx.x * kPts, b = blockIdx.z, L = t.L;
    const double *scan = w.scan + (size_t)b * w.sscan;

    for (int i = threadIdx.x; i < 132; i += blockDim.x) colidx[i] = -1;
    __syncthreads();
    for (int i = threadIdx.x; i < t.ncol; i += blockDim.x) colidx[t.col_part[i] * 66 + t.col_term[i]] = i;
    __syncthreads();
    for (int i = threadIdx.x; i < kPts * 132; i += blockDim.x) {
        const int c = i / 132, r = i % 132, part = r / 66, term = r % 66, q = q0 + c;
        double v = 0.0;
        if (q < t.njk && term < t.ntrm) {
            const int col = colidx[part * 66 + term];
            const size_t srow = (size_t)t.jk_sub[q] * 2 * t.ncol;
            const double min_ = col >= 0 ? scan[srow + col] : 0.0;
            const double mout = col >= 0 ? scan[srow + t.ncol + col] : 0.0;
            v = t.jk_bin[(size_t)q * 66 + term] * min_ + t.jk_hout[(size_t)q * 66 + term] * mout;
        }
        trm[c][r] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPts * 21; i += blockDim.x) {
        const int c = i / 21, q = i % 21;
        const int m = q <= 10 ? q : q - 10, part = q <= 10 ? 0 : 1;
        double s = 0.0;
        for (int ll = m; ll <= t.maxtrm; ++ll) s = s + trm[c][part * 66 + ll * (ll + 1) / 2 + m];
        cq[c][q] = -t.grav * (q == 0 ? s : 2.0 * s);
    }
    __syncthreads();
    // one azimuth l per thread: its 21 basis values are read once and serve
    // the block's kPts boundary points
    double *X = w.X + (size_t)b * w.sX;
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        double f[21];
#pragma unroll
        for (int p = 0; p < 21; ++p) f[p] = __ldg(t.fbasis + (size_t)p * L + l);
#pragma unroll 2
        for (int c = 0; c < kPts; ++c) {
            const int q = q0 + c;
            if (q < t.njk) {
                double v = 0.0;
#pragma unroll
                for (int p = 0; p < 21; ++p) v = __fma_rn(cq[c][p], f[p], v);
                X[((size_t)l * t.K + t.jk_k[q]) * t.J + t.jk_j[q]] = v;
            }
        }
    }
}

// /COEFS/ amplitude and phase diagnostics (pot/pot3.f:105-132) of every
// transformed column of solve 0, read back from X before the mode solve
// overwrites it.  SF1 = 0.5/N is a power of two, so A1 = X/SF1 exactly.
// Grid: (ceil(J/32), K), block (32, 8).
__global__ void k_coef(DevTables t, Work w)
{
    const int j = blockIdx.x * 32 + threadIdx.x, k = blockIdx.y, n = t.N;
    if (j >= t.J) return;
    const double pi = 3.1415926535897932, inv = 1.0 / t.sf1;
    const size_t pl = (size_t)t.K * t.J, col = (size_t)k * t.J + j;
    const int J2 = t.J + 2, K2 = t.K + 2;
    const size_t ldl = (size_t)J2 * K2, ldi = ldl * (t.L / 2), off = (size_t)(j + 1) + (size_t)J2 * (k + 1);
    const double a1 = w.X[col] * inv, x1 = fabs(a1);
    for (int l = 2 + threadIdx.y; l <= n + 1; l += blockDim.y) {
        if (l <= n) {
            const double a = w.X[(size_t)(l - 1) * pl + col] * inv, bb = w.X[(size_t)(n + l - 1) * pl + col] * inv;
            if (x1 != 0.0) w.coef[off + ldl * (l - 2)] = 2.0 * sqrt(a * a + bb * bb) / x1;
            double philag;
            if (a > 0.0) philag = atan(bb / a);
            else if (a < 0.0) philag = atan(bb / a) + pi;
            else if (bb > 0.0) philag = 0.5 * pi;
            else if (bb < 0.0) philag = -0.5 * pi;
            else philag = 4.0 * pi;
            w.coef[off + ldl * (l - 2) + ldi] = philag * 180. / pi;
        } else {
            if (x1 != 0.0) w.coef[off + ldl * (n - 1)] = fabs(w.X[(size_t)n * pl + col] * inv) / x1;
            w.coef[off + ldl * (n - 1) + ldi] = a1;
        }
    }
}

// ---------------------------------------------------------------------------
// Inverse transform, ghost cells and z-axis extrapolation
// ---------------------------------------------------------------------------
// Grid: (ceil(J/TC), K, batch) over every column POT3 inverts (J = 2..JMAX+1,
// K = 2..KMAX+1, pot/pot3.f:258-281).  CTAs holding J = 2 also write the axis
// ghosts (pot/pot3.f:289-292) and the ZAXPHI row PHI(JMAX+2, K, :)
// (pot/pot3.f:350-387); CTAs at K = 2 write the midplane ghosts
// (pot/pot3.f:293-296).
// ZAXPHI's Neville extrapolation to r = 0 (pot/pot3.f:354-378) for azimuth
// l from NP samples PHI(2.., K, L) and PHI(2.., K, L+N) at the abscissae ZX,
// every operation as the reference orders it.  The table P2 is held as its
// live tail Q(S) = P2(II+S), which shifts down one place per step II, so
// that every index is static and the table stays in registers.
template <int NP, class F>
__device__ __forceinline__ double neville_axis(const double (&zx)[11], F sample, int l, int lm)
{
    constexpr int ichk = NP % 2, num = (NP - ichk) / 2, jsp = num + 1;
    double q[NP];   // q[i] = P2(i + 1) before the first step
#pragma unroll
    for (int jj = 2; jj <= jsp; ++jj) {
        q[num + (jj - 1) - 1] = sample(l, jj - 2);
        q[num - (jj - 2) - 1] = sample(l + lm, jj - 2);
    }
    if constexpr (ichk == 1) q[num + num] = sample(l, num);
    const double xpoint = 0.0;
#pragma unroll 1
    for (int ii = 1; ii <= NP - 1; ++ii) {
        const double p1 = q[0], xinv = 1.0 / zx[ii], xr = xpoint * xinv;
#pragma unroll
        for (int s = 0; s < NP - 1; ++s) {
            if (s < NP - ii) {   // JJ = II + 1 + S
                const double xratio = zx[ii + 1 + s] * xinv, pp = q[s + 1];
                q[s] = (p1 * (xratio - xr) + pp * (xr - 1.0)) / (xratio - 1.0);
            }
        }
    }
    return q[0];
}

// STARPHI of the cell (j, k, l) of PHI(J+2, K+2, L), 0-based, with the star at
// (ix, iy): the reference's expression in its order of operations, every
// product and sum rounded on its own (pot/ExternalPot.f:44-49).  COS/SIN of
// (L-1/2)*DTHETA are the m = 1 rows of COSM/SINM, the same numbers.
__device__ __forceinline__ double star_phi(const DevTables &t, const StarDev &x, double ix, double iy, int j, int k,
                                           int l)
{
    const double r = t.rhf[j], z = t.zhf[k], c = t.cosm[l], s = t.sinm[l];
    double q = __dadd_rn(__dmul_rn(r, r), __dmul_rn(z, z));
    q = __dadd_rn(q, __dmul_rn(ix, ix));
    q = __dadd_rn(q, __dmul_rn(iy, iy));
    q = __dsub_rn(q, __dmul_rn(__dmul_rn(2.0, r), __dadd_rn(__dmul_rn(c, ix), __dmul_rn(s, iy))));
    return __ddiv_rn(-x.mass, __dsqrt_rn(q));
}

// The BINARY build's companion term (pot/ExternalPot.f:57-69) added to v, the
// cell's PHI after STARPHI: v - MASSBIN/RDIST - HALF*OMEGABIN**2*((X+RCOM)**2
// + Y**2) with RDIST = SQRT(RBIN**2 + RHF**2 - 2 RBIN RHF COS(THETA-PI) +
// ZHF**2), X = RHF COS(THETA), Y = RHF SIN(THETA), THETA = (L-1/2) DTHETA,
// in the reference's order of operations.
__device__ __forceinline__ double binary_add(const DevTables &t, const StarDev &x, double v, int j, int k, int l)
{
    const double r = t.rhf[j], z = t.zhf[k];
    double q = __dadd_rn(__dmul_rn(x.rbin, x.rbin), __dmul_rn(r, r));
    q = __dsub_rn(q, __dmul_rn(__dmul_rn(__dmul_rn(2.0, x.rbin), r), t.bcos[l]));
    q = __dadd_rn(q, __dmul_rn(z, z));
    const double rdist = __dsqrt_rn(q);
    const double xp = __dadd_rn(__dmul_rn(r, t.cosm[l]), x.rcom), yp = __dmul_rn(r, t.sinm[l]);
    const double e = __dadd_rn(__dmul_rn(xp, xp), __dmul_rn(yp, yp));
    v = __dsub_rn(v, __ddiv_rn(x.mass_bin, rdist));
    return __dsub_rn(v, __dmul_rn(__dmul_rn(0.5, x.omega2), e));
}

// Star position of solve b: fixed, or the solve's INDIRECT shift.
__device__ __forceinline__ void star_pos(const StarDev &x, const Work &w, int b, double *ix, double *iy)
{
    if (x.indirect) {
        const double *d = w.diag + (size_t)b * w.sdiag;
        *ix = d[kDiagStar];
        *iy = d[kDiagStar + 1];
    } else {
        *ix = x.ix;
        *iy = x.iy;
    }
}

template <int L>
__global__ void __launch_bounds__(256) k_inverse(DevTables t, BatchPtrs bp, Work w, StarDev x, int xmode,
                                                 const __grid_constant__ CUtensorMap xmap)
{
    using T = Tile<L>;
    constexpr int n = T::N, RS = T::TC, I0 = T::IM0;
    extern __shared__ __align__(128) char smem_raw[];
    // Split layout, row stride TC: row q holds A1(q+1) = mode q (q = 0..N),
    // row IM0+q holds B1(q+1) = mode N+q (q = 1..N-1); B1(1) = B1(N+1) = 0.
    double *A = (double *)smem_raw;
    double *red = A + (size_t)T::ROWSI * RS;   // [L/2] ZAXPHI values
    FftSmem fs = carve_fft<L>((char *)(red + L / 2));
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smem_raw + (size_t)T::ROWSI * RS * 8 + (size_t)(L / 2) * 8 +
                                                  fft_table_bytes<L>());
    const int J2 = t.J + 2, K2 = t.K + 2;
    const int j0 = blockIdx.x * T::TC, k = blockIdx.y, b = blockIdx.z;
    const double *X = w.X + (size_t)b * w.sX;
    double *phi = bp.phi[b];

    // xmode 2: two sets of TMA boxes of the tensor map over X (J, K, L x batch),
    // TC columns x one K x up to 256 modes: modes 0..N-1 into rows 0..N-1 and
    // modes N..2N-1 into rows IM0..IM0+N-1; mode N then moves to row N and rows
    // IM0 and IM0+N become B1(1) = B1(N+1) = 0
    if (xmode == 2) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm32(tbar)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            constexpr int B = n < 256 ? n : 256;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm32(tbar)),
                         "r"((uint32_t)(2 * n * RS * 8) + fft_bulk_bytes(t.inv)));
            for (int z0 = 0; z0 < n; z0 += B) {
                tma_load_3d(A + (size_t)z0 * RS, &xmap, j0, k, b * L + z0, tbar);
                tma_load_3d(A + (size_t)(I0 + z0) * RS, &xmap, j0, k, b * L + n + z0, tbar);
            }
        }
        // the tables on the same barrier (lane 0 of warps 1-4)
        bulk_fft_tables(t.inv, fs, tbar, 1);
    } else {
        load_fft_tables(t.inv, fs);
    }
    if (xmode == 2) {
        // copies issued above
    } else if (xmode == 1) {
        // JMAX even: 16-byte granules (columns j, j+1 both in range or both
        // out), aligned since X, JMAX and j0 are
        constexpr int NG = T::TC / 2;
        for (int i = threadIdx.x; i < (n + 1) * NG; i += blockDim.x) {
            const int g = i % NG, q = i / NG, j = j0 + 2 * g;
            const bool ok = j < t.J, okim = ok && q >= 1 && q < n;
            const size_t col = (size_t)k * t.J + j, pl = (size_t)t.K * t.J;
            cp_async16(A + q * RS + 2 * g, ok ? X + (size_t)q * pl + col : X, ok ? 16 : 0);
            cp_async16(A + (I0 + q) * RS + 2 * g, okim ? X + (size_t)(n + q) * pl + col : X, okim ? 16 : 0);
        }
    } else {
        for (int i = threadIdx.x; i < (n + 1) * T::TC; i += blockDim.x) {
            const int c = i % T::TC, q = i / T::TC, j = j0 + c;
            const bool ok = j < t.J, okim = ok && q >= 1 && q < n;
            const size_t col = (size_t)k * t.J + j, pl = (size_t)t.K * t.J;
            cp_async8(A + q * RS + c, ok ? X + (size_t)q * pl + col : X, ok ? 8 : 0);
            cp_async8(A + (I0 + q) * RS + c, okim ? X + (size_t)(n + q) * pl + col : X, okim ? 8 : 0);
        }
    }
    cp_async_wait_all();
    // a tile that did not arrive in time makes this tile's PHI NaN, so the
    // failure shows instead of passing silently
    const bool landed = xmode != 2 || fwd_bar_wait(tbar, 0);
    __syncthreads();
    if (xmode == 2) {
        if (threadIdx.x < T::TC) {
            const int c = threadIdx.x;
            A[n * RS + c] = landed ? A[I0 * RS + c] : __longlong_as_double(0x7ff8000000000000ll);
            A[I0 * RS + c] = 0.0;
            A[(I0 + n) * RS + c] = 0.0;
        }
        __syncthreads();
    }
    realtr_pairs<L>(A, fs);
    stage_pairs<L, 0, false, T::TC, true>(A, fs, t.inv);

    // sample l of column c in natural order, times SF2 = 0.5 (pot/pot3.f:276-279)
    auto sample = [&](int l, int c) -> double {
        const int src = fs.perm[l >> 1];
        return 0.5 * A[((l & 1) ? I0 + src : src) * RS + c];
    };
    // PHI = PHI + STARPHI after POT3 (pot/ExternalPot.f:50), fused into the
    // stores: v is POT3's value of the cell (jj, kk, l)
    double ix = 0.0, iy = 0.0;
    if (x.on) star_pos(x, w, b, &ix, &iy);
    auto out = [&](int jj, int kk, int l, double v) -> double {
        if (!x.on) return v;
        v = __dadd_rn(v, star_phi(t, x, ix, iy, jj, kk, l));
        return x.binary ? binary_add(t, x, v, jj, kk, l) : v;
    };
    auto store = [&](int i) {
        const int c = i % T::TC, l = i / T::TC, j = j0 + c;
        if (j < t.J) {
            const double v = sample(l, c);
            phi[(size_t)(j + 1) + (size_t)J2 * ((k + 1) + (size_t)K2 * l)] = out(j + 1, k + 1, l, v);
            if (k == 0) phi[(size_t)(j + 1) + (size_t)J2 * ((size_t)K2 * l)] = out(j + 1, 0, l, v);   // PHI(J,1,L)
        }
    };
    if (x.on) {
        for (int i = threadIdx.x; i < L * T::TC; i += blockDim.x) store(i);
    } else {
        // 256 threads: a compile-time trip count, so that the shared-memory
        // reads of several cells issue together
#pragma unroll 4
        for (int it = 0; it < L * T::TC / 256; ++it) store(threadIdx.x + 256 * it);
    }
    if (j0 == 0) {
        for (int l = threadIdx.x; l < L; l += blockDim.x) {
            const double v = sample((l + n) % L, 0);                             // PHI(2,K,L+-N)
            phi[(size_t)J2 * ((k + 1) + (size_t)K2 * l)] = out(0, k + 1, l, v);   // PHI(1,K,L)
            if (k == 0) phi[(size_t)J2 * ((size_t)K2 * l)] = out(0, 0, l, v);     // PHI(1,1,L)
        }
        // ZAXPHI: Neville extrapolation to r = 0 across +-RHF (pot/pot3.f:354-378)
        const int lm = L / 2;
        for (int l = threadIdx.x; l < lm; l += blockDim.x) {
            double ph;
            switch (t.npoint) {   // 2..10, checked at plan creation
            case 2: ph = neville_axis<2>(t.zx, sample, l, lm); break;
            case 3: ph = neville_axis<3>(t.zx, sample, l, lm); break;
            case 4: ph = neville_axis<4>(t.zx, sample, l, lm); break;
            case 5: ph = neville_axis<5>(t.zx, sample, l, lm); break;
            case 6: ph = neville_axis<6>(t.zx, sample, l, lm); break;
            case 7: ph = neville_axis<7>(t.zx, sample, l, lm); break;
            case 8: ph = neville_axis<8>(t.zx, sample, l, lm); break;
            case 9: ph = neville_axis<9>(t.zx, sample, l, lm); break;
            default: ph = neville_axis<10>(t.zx, sample, l, lm); break;
            }
            red[l] = ph;
            phi[(size_t)(t.J + 1) + (size_t)J2 * ((k + 1) + (size_t)K2 * l)] = out(t.J + 1, k + 1, l, ph);
            phi[(size_t)(t.J + 1) + (size_t)J2 * ((k + 1) + (size_t)K2 * (l + lm))] = out(t.J + 1, k + 1, l + lm, ph);
        }
        __syncthreads();
        // PHAC(K): the first largest-|ER| deviation, ER = 1 - PH(L)/PHMAX,
        // PHMAX the first largest-|PH| value (pot/pot3.f:351,376,381-386)
        if (threadIdx.x < 32) {
            double pm = 0.0;
            int pl = 0x7fffffff;
            for (int l = threadIdx.x; l < lm; l += 32)
                if (fabs(red[l]) > fabs(pm)) { pm = red[l]; pl = l; }
            for (int o = 16; o > 0; o >>= 1) {
                const double v = __shfl_xor_sync(0xffffffffu, pm, o);
                const int vl = __shfl_xor_sync(0xffffffffu, pl, o);
                if (fabs(v) > fabs(pm) || (fabs(v) == fabs(pm) && vl < pl)) { pm = v; pl = vl; }
            }
            double em = 0.0;
            int el = 0x7fffffff;
            for (int l = threadIdx.x; l < lm; l += 32) {
                const double er = 1.0 - red[l] / pm;
                if (fabs(er) > fabs(em)) { em = er; el = l; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double v = __shfl_xor_sync(0xffffffffu, em, o);
                const int vl = __shfl_xor_sync(0xffffffffu, el, o);
                if (fabs(v) > fabs(em) || (fabs(v) == fabs(em) && vl < el)) { em = v; el = vl; }
            }
            if (threadIdx.x == 0) w.phac[(size_t)b * w.sphac + (k + 2)] = em;
        }
    }
}

// ---------------------------------------------------------------------------
// ExternalPot's other cells, its INDIRECT star position and STARPHI itself
// ---------------------------------------------------------------------------
// PHI = PHI + STARPHI on the cells POT3 does not write: PHI(:, KMAX+2, L) and
// PHI(JMAX+2, 1, L) (pot/ExternalPot.f:42-50 covers the whole grid).
// Grid (L, batch).
__global__ void __launch_bounds__(128) k_star_rim(DevTables t, BatchPtrs bp, Work w, StarDev x)
{
    const int l = blockIdx.x, b = blockIdx.y, J2 = t.J + 2, K2 = t.K + 2;
    double *phi = bp.phi[b];
    double ix, iy;
    star_pos(x, w, b, &ix, &iy);
    for (int j = threadIdx.x; j <= J2; j += blockDim.x) {
        // j < J2: row K = KMAX+2; j == J2: the cell (JMAX+2, 1)
        const int jj = j < J2 ? j : t.J + 1, kk = j < J2 ? t.K + 1 : 0;
        const size_t at = (size_t)jj + (size_t)J2 * ((size_t)kk + (size_t)K2 * l);
        const double v = __dadd_rn(phi[at], star_phi(t, x, ix, iy, jj, kk, l));
        phi[at] = x.binary ? binary_add(t, x, v, jj, kk, l) : v;
    }
}

// INDIRECT (pot/ExternalPot.f:21-34): the disk's mass moment of plane L,
//   sum over K = 2..KMAX1, J = JMIN..JMAX1 of THISMASS*COS(PSI_L)*RHF(J)
//   (and SIN), THISMASS = RHO*RHF(J)*ROF3N*ZOF3N*2*DTHETA,
// into DIAG[kDiagPart + 2L..].  Grid (L, batch); fixed summation order.
__global__ void __launch_bounds__(256) k_star_moment(DevTables t, BatchPtrs bp, Work w, StarDev x)
{
    const int l = blockIdx.x, b = blockIdx.y, J2 = t.J + 2, K2 = t.K + 2;
    const double *rho = bp.rho[b] + (size_t)J2 * K2 * l;
    const int j0 = x.jmin - 1, nj = t.J + 1 - j0;   // 0-based J = JMIN-1 .. JMAX
    const double c = t.cosm[l], s = t.sinm[l];
    double sx = 0.0, sy = 0.0;
    if (nj > 0) {
        for (int i = threadIdx.x; i < nj * t.K; i += blockDim.x) {
            const int j = j0 + i % nj, k = 1 + i / nj;
            const double r = t.rhf[j];
            double m = __dmul_rn(rho[(size_t)j + (size_t)J2 * k], r);
            m = __dmul_rn(m, x.rof3n);
            m = __dmul_rn(m, x.zof3n);
            m = __dmul_rn(m, 2.0);
            m = __dmul_rn(m, x.dtheta);
            sx = __dadd_rn(sx, __dmul_rn(__dmul_rn(m, c), r));
            sy = __dadd_rn(sy, __dmul_rn(__dmul_rn(m, s), r));
        }
    }
    __shared__ double part[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    const int wp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { part[0][wp] = sx; part[1][wp] = sy; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ax = 0.0, ay = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) { ax += part[0][i]; ay += part[1][i]; }
        double *d = w.diag + (size_t)b * w.sdiag + kDiagPart + 2 * l;
        d[0] = ax;
        d[1] = ay;
    }
}

// INDIRECTX/Y = -(RPSTAR*COS/SIN(PHI_STAR) + moment)/MASS_STAR
// (pot/ExternalPot.f:18-19,35-36).  One warp per solve.
__global__ void k_star_shift(DevTables t, Work w, StarDev x)
{
    const int b = blockIdx.x;
    double *d = w.diag + (size_t)b * w.sdiag;
    double sx = 0.0, sy = 0.0;
    for (int l = threadIdx.x; l < t.L; l += 32) {
        sx += d[kDiagPart + 2 * l];
        sy += d[kDiagPart + 2 * l + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (threadIdx.x == 0) {
        d[kDiagStar] = -(x.ix + sx) / x.mass_star;
        d[kDiagStar + 1] = -(x.iy + sy) / x.mass_star;
    }
}

// STARPHI(J+2, K+2, L) (/GAP/) for the star position of batch slot `slot`.
// Grid (K+2, L).
__global__ void __launch_bounds__(128) k_star_fill(DevTables t, Work w, StarDev x, int slot, double *out)
{
    const int k = blockIdx.x, l = blockIdx.y, J2 = t.J + 2, K2 = t.K + 2;
    double ix, iy;
    star_pos(x, w, slot, &ix, &iy);
    for (int j = threadIdx.x; j < J2; j += blockDim.x)
        out[(size_t)j + (size_t)J2 * ((size_t)k + (size_t)K2 * l)] = star_phi(t, x, ix, iy, j, k, l);
}

// PHICHK / KLOCAT (pot/pot3.f:391-399) and TMASS (pot/boundary.f:554).
__global__ void k_diag(DevTables t, Work w)
{
    const int b = blockIdx.x;
    if (threadIdx.x != 0) return;
    const double *phac = w.phac + (size_t)b * w.sphac;
    double err = 0.0;
    int klocat = 0;
    for (int k = 2; k <= t.K + 1; ++k) {
        const double xx = fabs(phac[k]);
        if (xx > fabs(err)) { err = phac[k]; klocat = k; }
    }
    double *d = w.diag + (size_t)b * w.sdiag;
    const double *scan = w.scan + (size_t)b * w.sscan;
    d[0] = scan[(size_t)t.nsub * 2 * t.ncol + 0];   // column 0 = TERM(1)*SUMASS, inside sum over all rings
    d[1] = err;
    d[2] = (double)klocat;
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <int L>
static size_t tile_bytes() { return (size_t)Tile<L>::ROWS * Tile<L>::RS * sizeof(double); }

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        cudaGetLastError();
        return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }();
    return fn;
}

template <int L>
static cudaError_t forward_l(const DevTables &t, const BatchPtrs &bp, const Work &w, int nb, cudaStream_t s)
{
    using T = Tile<L>;
    const size_t sm = tile_bytes<L>() + (size_t)20 * (L / 4) * 8 + fft_table_bytes<L>() + 16;
    cudaError_t e = ensure_smem((const void *)k_forward<L>, sm);
    if (e != cudaSuccess) return e;
    // 16-byte row copies need every RHO 16-byte aligned and JMAX+2 even
    int vec16 = (t.J + 2) % 2 == 0;
    for (int i = 0; i < nb; ++i) vec16 = vec16 && reinterpret_cast<uintptr_t>(bp.rho[i]) % 16 == 0;
    // with 16-byte aligned rows, the tiles come through one tensor map per
    // solve (encoded here: host arithmetic only, passed by value)
    RhoMaps maps{};
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (vec16 && enc) {
        bool ok = true;
        for (int i = 0; i < nb && ok; ++i) {
            const cuuint64_t dims[3] = {(cuuint64_t)(t.J + 2), (cuuint64_t)(t.K + 2), (cuuint64_t)L};
            const cuuint64_t strides[2] = {(cuuint64_t)(t.J + 2) * 8, (cuuint64_t)(t.J + 2) * (t.K + 2) * 8};
            const cuuint32_t box[3] = {(cuuint32_t)T::RS, 1u, (cuuint32_t)(L < 256 ? L : 256)}, es[3] = {1, 1, 1};
            ok = enc(&maps.m[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(bp.rho[i]), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }
        if (ok) vec16 = 2;
    }
    // 256 threads: the table copies, the moment halves and the compile-time
    // trip counts of k_forward assume eight warps
    k_forward<L><<<dim3((t.M + T::TC - 1) / T::TC, t.NZ, nb), 256, sm, s>>>(t, bp, w, vec16, maps);
    return cudaGetLastError();
}

template <int L>
static cudaError_t inverse_l(const DevTables &t, const BatchPtrs &bp, const Work &w, const StarDev &x, int nb,
                             cudaStream_t s, int *launches)
{
    using T = Tile<L>;
    const size_t sm = (size_t)T::ROWSI * T::TC * sizeof(double) + (size_t)(L / 2) * 8 + fft_table_bytes<L>() + 16;
    cudaError_t e = ensure_smem((const void *)k_inverse<L>, sm);
    if (e != cudaSuccess) return e;
    // X rows through a tensor map when JMAX is even (16-byte strides), else
    // 8-byte copies
    int xmode = (t.J & 1) == 0 ? 1 : 0;
    CUtensorMap xmap;
    std::memset(&xmap, 0, sizeof xmap);
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (xmode == 1 && enc && reinterpret_cast<uintptr_t>(w.X) % 16 == 0) {
        const cuuint64_t dims[3] = {(cuuint64_t)t.J, (cuuint64_t)t.K, (cuuint64_t)L * nb};
        const cuuint64_t strides[2] = {(cuuint64_t)t.J * 8, (cuuint64_t)t.J * t.K * 8};
        const cuuint32_t box[3] = {(cuuint32_t)T::TC, 1u, (cuuint32_t)(T::N < 256 ? T::N : 256)}, es[3] = {1, 1, 1};
        if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, w.X, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
            xmode = 2;
    }
    // 256 threads: the table copies and the compile-time trip counts of
    // k_inverse assume eight warps
    k_inverse<L><<<dim3((t.J + T::TC - 1) / T::TC, t.K, nb), 256, sm, s>>>(t, bp, w, x, xmode, xmap);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *launches = 2;
    if (x.on) {
        k_star_rim<<<dim3(L, nb), 128, 0, s>>>(t, bp, w, x);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *launches = 3;
    }
    k_diag<<<nb, 32, 0, s>>>(t, w);
    return cudaGetLastError();
}

#define CHY_DISPATCH_L(FN, ...)                     \
    switch (t.L) {                                  \
    case 32: return FN<32>(__VA_ARGS__);            \
    case 64: return FN<64>(__VA_ARGS__);            \
    case 128: return FN<128>(__VA_ARGS__);          \
    case 256: return FN<256>(__VA_ARGS__);          \
    case 512: return FN<512>(__VA_ARGS__);          \
    case 1024: return FN<1024>(__VA_ARGS__);        \
    default: return cudaErrorInvalidValue;          \
    }

cudaError_t launch_forward(const DevTables &t, const BatchPtrs &bp, const Work &w, int nb, cudaStream_t s)
{
    CHY_DISPATCH_L(forward_l, t, bp, w, nb, s)
}

cudaError_t launch_bdy_synth(const DevTables &t, const Work &w, int nb, cudaStream_t s)
{
    k_bdy_synth<<<dim3((t.njk + 7) / 8, 1, nb), 256, 0, s>>>(t, w);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || w.coef == nullptr) return e;
    k_coef<<<dim3((t.J + 31) / 32, t.K, 1), dim3(32, 8), 0, s>>>(t, w);
    return cudaGetLastError();
}

cudaError_t launch_inverse(const DevTables &t, const BatchPtrs &bp, const Work &w, const StarDev &x, int nb,
                           cudaStream_t s, int *launches)
{
    CHY_DISPATCH_L(inverse_l, t, bp, w, x, nb, s, launches)
}

cudaError_t launch_star_shift(const DevTables &t, const BatchPtrs &bp, const Work &w, const StarDev &x, int nb,
                              cudaStream_t s)
{
    k_star_moment<<<dim3(t.L, nb), 256, 0, s>>>(t, bp, w, x);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_star_shift<<<nb, 32, 0, s>>>(t, w, x);
    return cudaGetLastError();
}

cudaError_t launch_star_fill(const DevTables &t, const Work &w, const StarDev &x, int slot, double *out,
                             cudaStream_t s)
{
    k_star_fill<<<dim3(t.K + 2, t.L), 128, 0, s>>>(t, w, x, slot, out);
    return cudaGetLastError();
}

// Compile-time stage structure used by the kernels, for the plan to compare
// with the recorded schedule.
template <int L>
static bool shape_ok(const FftDev &f)
{
    using Sh = Shape<L / 2>;
    if (f.nst != Sh::nst() || f.n != L / 2) return false;
    for (int s = 0; s < Sh::nst(); ++s)
        if (f.radix[s] != Sh::radix(s) || f.span[s] != Sh::span(s)) return false;
    return true;
}

bool fft_shape_supported(const FftDev &f, int L)
{
    switch (L) {
    case 32: return shape_ok<32>(f);
    case 64: return shape_ok<64>(f);
    case 128: return shape_ok<128>(f);
    case 256: return shape_ok<256>(f);
    case 512: return shape_ok<512>(f);
    case 1024: return shape_ok<1024>(f);
    default: return false;
    }
}

}  // namespace chy

// k_bdy.cu -- BDYGEN's mass integrals without the O(rings x boundary points)
// masked accumulation.
//
// The reference adds every ring's multipole contribution MRING into
// MASSIN(JK) for each boundary point JK with RSPHER <= RBDY(JK), and its
// r^-(2l+1)-scaled contribution into MASSOUT(JK) for RSPHER > RBDY(JK)
// (pot/boundary.f:558-604): ~1.6 G adds at 256x128.  With the rings sorted by
// spherical radius, MASSIN(JK) is a prefix sum and MASSOUT(JK) a suffix sum
// of the same sequence, cut at the number of rings inside RBDY(JK).  The
// sorted sequence is split into sub-chunks that never straddle a cut; one CTA
// sums each sub-chunk, and each column's sub-chunk sums are scanned in
// in-order runs.  Every sum has a fixed order, so results are bit-reproducible
// alone or in a batch.
// The outside sums are accumulated from the outermost ring inward, so the
// huge r^-(2l+1) factors of inner rings never enter a difference.
//
// Compiled with --fmad=false: each product and sum rounds separately, in a
// fixed order.
#include "devplan.h"

namespace chy {

// Grid: (nsub, 1, ceil(batch / kSubBatch)), four threads per column.  The
// ring-table slice of a sub-chunk is loaded once and serves up to kSubBatch
// solves, two solves per pass.  Every column sum keeps its order, whatever
// the pairing.
constexpr int kSubBatch = 8;
constexpr int kSubThreads = 512;
__global__ void __launch_bounds__(kSubThreads) k_bdy_sub(DevTables t, Work w, int nb, int spp)
{
    extern __shared__ double smem[];
    const int RL = t.srow, NT_ = t.ntrm;
    double *s_row = smem;                                      // [ns][RL]: TERM, r^-(2l+1), DV
    double *s_mom = smem + kSubChunk * RL;                     // [spp][ns][21]
    int *s_ring = reinterpret_cast<int *>(s_mom + (size_t)spp * kSubChunk * 21);   // [ns] ring index
    const int sc = blockIdx.x;
    const int s0 = t.sub_start[sc], s1 = t.sub_start[sc + 1], ns = s1 - s0;

    // per ring, geometry from the plan (TERM(I) of pot/boundary.f:385-502,
    // r^-(2l+1) of :587, DV of :516)
    for (int i = threadIdx.x; i < ns * RL; i += blockDim.x) s_row[i] = t.sterm[(size_t)s0 * RL + i];
    for (int i = threadIdx.x; i < ns; i += blockDim.x) s_ring[i] = t.ring_sorted[s0 + i];
    const int b0 = blockIdx.z * kSubBatch, b1 = min(nb, b0 + kSubBatch);
    for (int b = b0; b < b1; b += spp) {
        const int nsl = min(spp, b1 - b);
        __syncthreads();   // s_row loaded / s_mom of the previous solves consumed
        // DV * moments of these solves
        for (int it = threadIdx.x; it < nsl * ns * 21; it += blockDim.x) {
            const int sl = it / (ns * 21), rq = it % (ns * 21), r = rq / 21, q = rq % 21;
            const double *mom = w.mom + (size_t)(b + sl) * w.smom;
            s_mom[((size_t)sl * kSubChunk + r) * 21 + q] = s_row[r * RL + NT_ + 11] * mom[(size_t)q * t.nring + s_ring[r]];
        }
        __syncthreads();
        // Column col's inside and outside sums of these solves, each as four
        // partial sums (rings 4i .. 4i+3 into a0 .. a3, a remainder into a0)
        // added as (a0 + a1) + (a2 + a3): a fixed order with a quarter of the
        // dependent chain.  Lane 4 c + i of a warp holds partial sum a_i of
        // its column for both sums and both solves, so a ring's TERM and
        // r^-(2l+1) are read once for four accumulations and the product
        // TERM * DV * MRING once for the inside and the outside sum.
        {
            const int col = threadIdx.x >> 2, ph = threadIdx.x & 3;
            const bool live = col < t.ncol;
            int term = 0, l = 0, mq = 0;
            if (live) {
                term = t.col_term[col];
                l = t.col_l[col];
                mq = t.col_part[col] == 0 ? t.col_m[col] : 10 + t.col_m[col];
            }
            const double *sm0 = s_mom, *sm1 = s_mom + (size_t)kSubChunk * 21;
            double ai0 = 0.0, ao0 = 0.0, ai1 = 0.0, ao1 = 0.0;
            auto ring = [&](int r) {
                const double tt = s_row[r * RL + term], qh = s_row[r * RL + NT_ + l];
                const double p0 = tt * sm0[r * 21 + mq];
                ai0 = ai0 + p0;
                ao0 = ao0 + p0 * qh;
                if (nsl > 1) {
                    const double p1 = tt * sm1[r * 21 + mq];
                    ai1 = ai1 + p1;
                    ao1 = ao1 + p1 * qh;
                }
            };
            const int q4 = ns & ~3;
            if (live) {
                for (int r = ph; r < q4; r += 4) ring(r);
                if (ph == 0)
                    for (int r = q4; r < ns; ++r) ring(r);
            }
            // (a0 + a1) + (a2 + a3); IEEE addition commutes, so every lane of
            // the four ends with the same bits
            auto tree = [&](double v) {
                v = v + __shfl_xor_sync(0xffffffffu, v, 1);
                return v + __shfl_xor_sync(0xffffffffu, v, 2);
            };
            ai0 = tree(ai0);
            ao0 = tree(ao0);
            ai1 = tree(ai1);
            ao1 = tree(ao1);
            if (live && ph == 0) {
                double *sub = w.sub + (size_t)b * w.ssub + (size_t)sc * 2 * t.ncol + col;
                sub[0] = ai0;
                sub[t.ncol] = ao0;
                if (nsl > 1) {
                    sub[w.ssub] = ai1;
                    sub[w.ssub + t.ncol] = ao1;
                }
            }
        }
    }
}

// Grid: (ceil(2*ncol / 32), 1, batch), 512 threads: lane i of every warp
// takes column 32 blockIdx.x + i of the [2][ncol] row (inside sums, then
// outside sums), so each row is read and written in one coalesced piece;
// warp s takes the s-th of kScanRuns consecutive runs of sub-chunks in scan
// order.
// scan[i][0][col] = sum of inside sums of sub-chunks < i (prefix from the
// innermost ring); scan[i][1][col] = sum of outside sums of sub-chunks >= i
// (suffix from the outermost ring).  Each run is summed in order, the run
// totals are added in order, and every prefix is that base plus the run's
// running sum: a fixed order, so the result is bit-reproducible.
constexpr int kScanRuns = 16;
__global__ void __launch_bounds__(32 * kScanRuns) k_bdy_scan(DevTables t, Work w)
{
    __shared__ double run_tot[kScanRuns][32];
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5, b = blockIdx.z;
    const int cc = blockIdx.x * 32 + lane, ld = 2 * t.ncol;
    const bool live = cc < ld, out = cc >= t.ncol;
    const double *__restrict__ sub = w.sub + (size_t)b * w.ssub;
    double *__restrict__ scan = w.scan + (size_t)b * w.sscan;
    const int ns = t.nsub, per = (ns + kScanRuns - 1) / kScanRuns;
    const int lo = min(seg * per, ns), hi = min(lo + per, ns);
    // position p in scan order -> sub-chunk index
    auto idx = [&](int p) { return out ? ns - 1 - p : p; };
    // loads go eight at a time, so that their latencies overlap; the sums
    // stay in order
    constexpr int kU = 8;
    double local = 0.0;
    if (live)
        for (int p0 = lo; p0 < hi; p0 += kU) {
            double v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) v[u] = p0 + u < hi ? sub[(size_t)idx(p0 + u) * ld + cc] : 0.0;
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (p0 + u < hi) local = local + v[u];
        }
    run_tot[seg][lane] = local;
    __syncthreads();
    double base = 0.0;
    for (int i = 0; i < seg; ++i) base = base + run_tot[i][lane];
    if (!live) return;
    double run = base;
    for (int p0 = lo; p0 < hi; p0 += kU) {
        double v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) v[u] = p0 + u < hi ? sub[(size_t)idx(p0 + u) * ld + cc] : 0.0;
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (p0 + u >= hi) break;
            const size_t at = (size_t)idx(p0 + u) * ld + cc;
            if (!out) {
                scan[at] = run;
                run = run + v[u];
            } else {
                run = run + v[u];
                scan[at] = run;
            }
        }
    }
    if (seg == kScanRuns - 1) scan[(size_t)ns * ld + cc] = out ? 0.0 : run;   // the inside total
}

cudaError_t launch_bdy_sums(const DevTables &t, const Work &w, int nb, cudaStream_t s)
{
    // four lanes per column (one per partial sum), two solves per pass
    // when there are two
    if (4 * t.ncol > kSubThreads) return cudaErrorInvalidConfiguration;
    const int spp = nb >= 2 ? 2 : 1;
    const int threads = ((4 * t.ncol + 31) / 32) * 32;
    const size_t sm = (size_t)kSubChunk * (t.srow + 21 * spp) * sizeof(double) + (size_t)kSubChunk * sizeof(int);
    cudaError_t e = ensure_smem((const void *)k_bdy_sub, sm);
    if (e != cudaSuccess) return e;
    k_bdy_sub<<<dim3(t.nsub, 1, (nb + kSubBatch - 1) / kSubBatch), threads, sm, s>>>(t, w, nb, spp);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_bdy_scan<<<dim3((2 * t.ncol + 31) / 32, 1, nb), 32 * kScanRuns, 0, s>>>(t, w);
    return cudaGetLastError();
}

}  // namespace chy

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
// sums each sub-chunk, one thread per column scans the sub-chunk sums.  Every
// sum has a fixed order, so results are bit-reproducible alone or in a batch.
// The outside sums are accumulated from the outermost ring inward, so the
// huge r^-(2l+1) factors of inner rings never enter a difference.
//
// Compiled with --fmad=false: each product and sum rounds separately, in a
// fixed order.
#include "devplan.h"

namespace chy {

// Grid: (nsub, 1, ceil(batch / kSubBatch)).  The ring-table slice of a
// sub-chunk is loaded once and serves up to kSubBatch solves; when the 2*ncol
// column sums of one solve fill at most half the block, two solves are summed
// side by side.  Every column sum keeps its order, whatever the pairing.
constexpr int kSubBatch = 8;
constexpr int kSubThreads = 512;
__global__ void __launch_bounds__(kSubThreads) k_bdy_sub(DevTables t, Work w, int nb, int spp)
{
    extern __shared__ double smem[];
    const int RL = t.srow, NT_ = t.ntrm, per = 2 * t.ncol;
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
        for (int task = threadIdx.x; task < nsl * per; task += blockDim.x) {
            const int sl = task / per, cc = task % per;
            const int col = cc % t.ncol, out = cc / t.ncol;
            const int term = t.col_term[col], m = t.col_m[col], l = t.col_l[col];
            const int mq = t.col_part[col] == 0 ? m : 10 + m;
            const double *sm = s_mom + (size_t)sl * kSubChunk * 21;
            // four partial sums (rings 4i .. 4i+3 into a0 .. a3, a remainder
            // into a0), then (a0 + a1) + (a2 + a3): a fixed order with a
            // quarter of the dependent chain
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            int r = 0;
            if (!out) {
                for (; r + 4 <= ns; r += 4) {
                    a0 = a0 + s_row[r * RL + term] * sm[r * 21 + mq];
                    a1 = a1 + s_row[(r + 1) * RL + term] * sm[(r + 1) * 21 + mq];
                    a2 = a2 + s_row[(r + 2) * RL + term] * sm[(r + 2) * 21 + mq];
                    a3 = a3 + s_row[(r + 3) * RL + term] * sm[(r + 3) * 21 + mq];
                }
                for (; r < ns; ++r) a0 = a0 + s_row[r * RL + term] * sm[r * 21 + mq];
            } else {
                for (; r + 4 <= ns; r += 4) {
                    a0 = a0 + (s_row[r * RL + term] * sm[r * 21 + mq]) * s_row[r * RL + NT_ + l];
                    a1 = a1 + (s_row[(r + 1) * RL + term] * sm[(r + 1) * 21 + mq]) * s_row[(r + 1) * RL + NT_ + l];
                    a2 = a2 + (s_row[(r + 2) * RL + term] * sm[(r + 2) * 21 + mq]) * s_row[(r + 2) * RL + NT_ + l];
                    a3 = a3 + (s_row[(r + 3) * RL + term] * sm[(r + 3) * 21 + mq]) * s_row[(r + 3) * RL + NT_ + l];
                }
                for (; r < ns; ++r) a0 = a0 + (s_row[r * RL + term] * sm[r * 21 + mq]) * s_row[r * RL + NT_ + l];
            }
            const double acc = (a0 + a1) + (a2 + a3);
            w.sub[(size_t)(b + sl) * w.ssub + (size_t)sc * 2 * t.ncol + (size_t)out * t.ncol + col] = acc;
        }
    }
}

// Grid: (2*ncol, 1, batch), 256 threads: one CTA scans one column.
// scan[i][0][col] = sum of inside sums of sub-chunks < i (prefix from the
// innermost ring); scan[i][1][col] = sum of outside sums of sub-chunks >= i
// (suffix from the outermost ring).  Each thread owns a contiguous run of
// sub-chunks; runs are combined by a fixed-shape block scan, so the result is
// bit-reproducible.
__global__ void __launch_bounds__(256) k_bdy_scan(DevTables t, Work w)
{
    __shared__ double warp_tot[8];
    const int cc = blockIdx.x, b = blockIdx.z;
    const int col = cc % t.ncol, out = cc / t.ncol;
    const double *__restrict__ sub = w.sub + (size_t)b * w.ssub;
    double *__restrict__ scan = w.scan + (size_t)b * w.sscan;
    const size_t ld = (size_t)2 * t.ncol, off = (size_t)out * t.ncol + col;
    const int ns = t.nsub, per = (ns + 255) / 256;
    const int lo = threadIdx.x * per, hi = min(lo + per, ns);
    // position p in scan order -> sub-chunk index
    auto idx = [&](int p) { return out ? ns - 1 - p : p; };
    double local = 0.0;
    for (int p = lo; p < hi; ++p) local = local + sub[(size_t)idx(p) * ld + off];
    // exclusive block scan of the per-thread totals
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl = incl + v;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    double base = 0.0;
    for (int i = 0; i < wid; ++i) base = base + warp_tot[i];
    double run = base + (incl - local);
    for (int p = lo; p < hi; ++p) {
        const int i = idx(p);
        const double v = sub[(size_t)i * ld + off];
        if (!out) {
            scan[(size_t)i * ld + off] = run;
            run = run + v;
        } else {
            run = run + v;
            scan[(size_t)i * ld + off] = run;
        }
    }
    if (threadIdx.x == 255) {
        double tot = 0.0;
        for (int i = 0; i < 8; ++i) tot = tot + warp_tot[i];
        scan[(size_t)ns * ld + off] = out ? 0.0 : tot;
    }
}

cudaError_t launch_bdy_sums(const DevTables &t, const Work &w, int nb, cudaStream_t s)
{
    // two solves per pass when there are two and a solve's column sums fill
    // at most half the block
    const int per = 2 * t.ncol, spp = (nb >= 2 && 2 * per <= kSubThreads) ? 2 : 1;
    const int threads = spp == 2 ? ((2 * per + 31) / 32) * 32 : 256;
    const size_t sm = (size_t)kSubChunk * (t.srow + 21 * spp) * sizeof(double) + (size_t)kSubChunk * sizeof(int);
    cudaError_t e = ensure_smem((const void *)k_bdy_sub, sm);
    if (e != cudaSuccess) return e;
    k_bdy_sub<<<dim3(t.nsub, 1, (nb + kSubBatch - 1) / kSubBatch), threads, sm, s>>>(t, w, nb, spp);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_bdy_scan<<<dim3(2 * t.ncol, 1, nb), 256, 0, s>>>(t, w);
    return cudaGetLastError();
}

}  // namespace chy

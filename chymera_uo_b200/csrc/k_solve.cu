// k_solve.cu -- the per-mode (R,Z) solves of POT3 (pot/pot3.f:201-248).
//
// For every azimuthal mode l (m = l for the cosine half, l - N for the sine
// half) POT3 solves the block-tridiagonal system
//     AN(k) x(j,k-1) + BN(k) x(j,k) + CN(k) x(j,k+1)
//   + AM(j) x(j-1,k) + BM_m(j) x(j,k) + CM(j) x(j+1,k) = Y(j,k)
// with FISHPACK BLKTRI.  The vertical operator T_z = (AN, BN, CN) does not
// depend on m, so this library diagonalises it once per grid,
// T_z = V diag(lam) U, and solves each mode as
//     W = U Y              (vertical transform, a GEMM over all modes)
//     (T_r(m) + lam_p) w_p = W_p  for each p   (radial tridiagonal sweeps)
//     x = V W              (inverse vertical transform)
// This file holds the plain FP64 version of that pipeline.
//
// W layout: [l][j][p] (p fastest, leading dimension K) so the radial sweeps
// of 32 consecutive p's read and write coalesced rows.
#include "devplan.h"

namespace chy {

constexpr int kPB = 128;   // p / k extent held in shared memory (NZ <= 127)
constexpr int kJT = 32;    // j columns per GEMM tile

__device__ __forceinline__ int mode_m(int l, int n) { return l <= n ? l : l - n; }

// Y(j,k) = 4 pi G Xhat(j,k) with the Dirichlet boundary folded in
// (pot/pot3.f:212-224).
__device__ __forceinline__ double rhs_value(const DevTables &t, const double *Xl, int j, int k)
{
    double y = t.pig4 * Xl[(size_t)k * t.J + j];
    if (k == t.NZ - 1) y = y - t.cnmax * Xl[(size_t)t.NZ * t.J + j];
    if (j == t.M - 1) y = y - t.cmmax * Xl[(size_t)k * t.J + t.M];
    return y;
}

// W[l][j][p] = sum_k U(p,k) Y_l(j,k).  Persistent: each CTA keeps U in shared
// memory and walks (batch, l, j-tile) items.
__global__ void __launch_bounds__(256) k_zfwd_f64(DevTables t, Work w, int nb)
{
    extern __shared__ double smem[];
    double *Us = smem;                  // [k][p], kPB x kPB
    double *Ys = smem + kPB * kPB;      // [k][j], kPB x kJT
    const int NZ = t.NZ, tid = threadIdx.x;
    for (int i = tid; i < kPB * kPB; i += blockDim.x) {
        const int k = i / kPB, p = i % kPB;
        Us[i] = (k < NZ && p < NZ) ? t.U[(size_t)p * NZ + k] : 0.0;
    }
    const int njt = (t.M + kJT - 1) / kJT;
    const long long items = (long long)nb * t.L * njt;
    const int tp = tid / 8, tj = tid % 8, p0 = tp * 4, jj0 = tj * 4;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int jt = (int)(it % njt), l = (int)((it / njt) % t.L), b = (int)(it / ((long long)njt * t.L));
        const int j0 = jt * kJT;
        const double *Xl = w.X + (size_t)b * w.sX + (size_t)l * t.K * t.J;
        __syncthreads();
        for (int i = tid; i < NZ * kJT; i += blockDim.x) {
            const int k = i / kJT, jj = i % kJT, j = j0 + jj;
            Ys[k * kJT + jj] = (j < t.M) ? rhs_value(t, Xl, j, k) : 0.0;
        }
        __syncthreads();
        double acc[4][4] = {};
        for (int k = 0; k < NZ; ++k) {
            double u[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) { u[a] = Us[k * kPB + p0 + a]; y[a] = Ys[k * kJT + jj0 + a]; }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] = fma(u[a], y[c], acc[a][c]);
        }
        double *Wl = w.W + (size_t)b * w.sW + (size_t)l * t.J * t.K;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = j0 + jj0 + c;
            if (j < t.M)
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    if (p0 + a < NZ) Wl[(size_t)j * t.K + p0 + a] = acc[a][c];
        }
    }
}

// Radial tridiagonal sweeps (T_r(m) + lam_p) w = W_p, one thread per (l, p).
// BM_m(j) as pot/pot3.f:226-230 builds it.  Forward elimination stores the
// multipliers in C (same layout as W), back substitution overwrites W.
__global__ void __launch_bounds__(128) k_thomas_f64(DevTables t, Work w)
{
    const int p = threadIdx.x, l = blockIdx.x, b = blockIdx.z;
    if (p >= t.NZ) return;
    const int m = mode_m(l, t.N), M = t.M, K = t.K;
    const double xl2 = 2.0 * (t.xlamm[m] - 1.0);
    const double axis = ((m % 2 == 0) ? 1.0 : -1.0) - 1.0;
    const double lam = t.lam[p];
    double *__restrict__ Wp = w.W + (size_t)b * w.sW + (size_t)l * t.J * K + p;
    double *__restrict__ Cp = w.C + (size_t)b * w.sC + (size_t)l * t.J * K + p;
    constexpr int kU = 8;   // rows whose loads are issued ahead of the recurrence
    double d = t.bm0[0] + axis * t.ammin + xl2 * t.cc[0] + lam;
    double r = 1.0 / d;
    double cprev = t.cm[0] * r, yprev = Wp[0] * r;
    Cp[0] = cprev;
    Wp[0] = yprev;
    for (int j0 = 1; j0 < M; j0 += kU) {
        double yv[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) yv[u] = (j0 + u < M) ? Wp[(size_t)(j0 + u) * K] : 0.0;
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int j = j0 + u;
            if (j < M) {
                const double a = t.am[j];
                d = (t.bm0[j] + xl2 * t.cc[j]) + lam - a * cprev;
                r = 1.0 / d;
                cprev = t.cm[j] * r;
                yprev = (yv[u] - a * yprev) * r;
                Cp[(size_t)j * K] = cprev;
                Wp[(size_t)j * K] = yprev;
            }
        }
    }
    double x = yprev;
    for (int j0 = M - 2; j0 >= 0; j0 -= kU) {
        double yv[kU], cv[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            yv[u] = (j0 - u >= 0) ? Wp[(size_t)(j0 - u) * K] : 0.0;
            cv[u] = (j0 - u >= 0) ? Cp[(size_t)(j0 - u) * K] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (j0 - u >= 0) {
                x = yv[u] - cv[u] * x;
                Wp[(size_t)(j0 - u) * K] = x;
            }
    }
}

// X_l(j,k) = sum_p V(k,p) W[l][j][p] for the interior (k < NZ, j < M).
__global__ void __launch_bounds__(256) k_zinv_f64(DevTables t, Work w, int nb)
{
    extern __shared__ double smem[];
    double *Vs = smem;                  // [p][k], kPB x kPB
    double *Ws = smem + kPB * kPB;      // [p][j], kPB x (kJT+1)
    constexpr int ldw = kJT + 1;
    const int NZ = t.NZ, tid = threadIdx.x;
    for (int i = tid; i < kPB * kPB; i += blockDim.x) {
        const int p = i / kPB, k = i % kPB;
        Vs[i] = (k < NZ && p < NZ) ? t.V[(size_t)k * NZ + p] : 0.0;
    }
    const int njt = (t.M + kJT - 1) / kJT;
    const long long items = (long long)nb * t.L * njt;
    const int tk = tid / 8, tj = tid % 8, k0 = tk * 4, jj0 = tj * 4;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int jt = (int)(it % njt), l = (int)((it / njt) % t.L), b = (int)(it / ((long long)njt * t.L));
        const int j0 = jt * kJT;
        const double *Wl = w.W + (size_t)b * w.sW + (size_t)l * t.J * t.K;
        __syncthreads();
        for (int i = tid; i < kJT * NZ; i += blockDim.x) {
            const int jj = i / NZ, p = i % NZ, j = j0 + jj;
            Ws[p * ldw + jj] = (j < t.M) ? Wl[(size_t)j * t.K + p] : 0.0;
        }
        __syncthreads();
        double acc[4][4] = {};
        for (int p = 0; p < NZ; ++p) {
            double v[4], x[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) { v[a] = Vs[p * kPB + k0 + a]; x[a] = Ws[p * ldw + jj0 + a]; }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][c] = fma(v[a], x[c], acc[a][c]);
        }
        double *Xl = w.X + (size_t)b * w.sX + (size_t)l * t.K * t.J;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int k = k0 + a;
            if (k < NZ)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int j = j0 + jj0 + c;
                    if (j < t.M) Xl[(size_t)k * t.J + j] = acc[a][c];
                }
        }
    }
}

cudaError_t launch_solve_fp64(const DevTables &t, const Work &w, int nb, int num_sms, cudaStream_t s)
{
    const size_t sm1 = (size_t)(kPB * kPB + kPB * kJT) * sizeof(double);
    const size_t sm3 = (size_t)(kPB * kPB + kPB * (kJT + 1)) * sizeof(double);
    cudaError_t e = ensure_smem((const void *)k_zfwd_f64, sm1);
    if (e == cudaSuccess) e = ensure_smem((const void *)k_zinv_f64, sm3);
    if (e != cudaSuccess) return e;
    if (t.NZ > kPB) return cudaErrorInvalidValue;
    const int njt = (t.M + kJT - 1) / kJT;
    const long long items = (long long)nb * t.L * njt;
    const int grid = (int)(items < num_sms ? items : num_sms);
    k_zfwd_f64<<<grid, 256, sm1, s>>>(t, w, nb);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_thomas_f64<<<dim3(t.L, 1, nb), 128, 0, s>>>(t, w);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_zinv_f64<<<grid, 256, sm3, s>>>(t, w, nb);
    return cudaGetLastError();
}


}  // namespace chy

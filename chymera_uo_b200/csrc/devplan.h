// devplan.h -- device-resident tables of one grid and the launch interface of
// the kernels (internal to libchy_pot3).
//
// HBM layout of one solve's work space:
//   X    [L][K][J]   FP64  azimuthal mode coefficients.  X[l][k][j] is mode l of
//                          PHI(J=j+2, K=k+2): j < J-1, k < K-1 is the interior
//                          (the unknowns of the mode solve), j = J-1 the outer
//                          boundary column, k = K-1 the top boundary row.
//   W    [L][J][K]   FP64  vertical eigen coefficients of the mode solve
//   C    [L][J][K]   FP64  radial elimination multipliers (FP64 solve path)
//   MOM  [21][nring] FP64  per-ring azimuthal moments sum_l {1, cos m psi_l,
//                          sin m psi_l} rho, ring = k*(J-1) + j.
//   SUB  [nsub][2][ncol]   per sub-chunk sums of the boundary integrands.
//   SCAN [nsub+1][2][ncol] exclusive prefix (inside) / suffix (outside) sums.
//   PHAC [K+2]             ZAXPHI deviations
//   DIAG [8 + 2L]          TMASS, PHICHK, KLOCAT, -, INDIRECTX, INDIRECTY, -, -,
//                          then per-L partial mass moments of the INDIRECT shift.
// BLKTRI-order FP64 path only (k_blktri.cu), not per solve but per group of
// 32 (solve, mode) items, item = solve * L + mode:
//   BVEC [group][NVEC][M][32] FP64 each item's BLKTRI vectors, lane-interleaved
//   BSCR [cta][warp][2][M][32] FP64 PRDCT's elimination scratch (W, D)
#pragma once

#include <cstdint>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cuda_runtime.h>

#include "blk.h"

namespace chy {

constexpr int kMaxStage = 16;
constexpr int kMaxBatchPtrs = 64;   // caller pointers passed per launch
constexpr int kSubChunk = 64;       // rings per boundary sub-chunk

struct FftDev {
    int n, isn, nst, nh, ncompact;
    int radix[kMaxStage], span[kMaxStage], off[kMaxStage];
    const double *twc;     // [ncompact][6] rotation of position j of stage s at off[s]+j
    const uint8_t *onc;    // [ncompact]
    const int *perm;       // [n]
    const double *rt;      // [nh][2]
};

// True when the device kernels' compile-time stage structure for this LMAX
// equals the recorded schedule.
bool fft_shape_supported(const FftDev &f, int L);

// The recorded BLKTRI schedule (blk.h) and BM of every mode, laid out
// [mode block][j][32 lanes] with lane -> mode (32 * block + lane) mod L.
struct BlkDev {
    int nvec, nstage, nblk;
    const BlkStep *steps;
    const BlkProg *progs;
    const BlkTask *tasks;
    const BlkStage *stages;
    const double *bmt;
};

struct DevTables {
    int J, K, L, N, M, NZ, nring, nkeep, njk, ncol, nsub, ntrm, maxtrm, isyma, npoint;
    double sf1, pig4, grav, F1, cmmax, ammin, cnmax;
    FftDev fwd, inv;
    const double *cosm, *sinm;      // [10][L]
    const double *bcos;             // [L] COS((L-1/2) DTHETA - PI) (the BINARY companion's angle)
    const double *rhf, *zhf;        // RHF(J+2), ZHF(K+2)
    const double *r;                // R(J+2)
    const double *fbasis;           // [21][L] transforms of {1, cos m psi, sin m psi}
    // kept rings in ascending spherical radius: ring index, and rsph, C1, S1, DV
    const int *ring_sorted;
    const double *sring;            // [nkeep][4]
    const double *sterm;            // [nkeep][srow]: TERM(1..NTRM), r^-(2l+1) l=0..10, DV
    int srow;
    const int *sub_start;           // [nsub+1] sub-chunk boundaries in sorted order
    const int *col_term, *col_part, *col_m, *col_l;   // [ncol]
    const int *jk_j, *jk_k, *jk_sub;                  // [njk]; jk_sub = first sub-chunk outside
    const double *jk_bin, *jk_hout;                   // [njk][66]
    // stencil (radial length M, vertical length NZ)
    const double *am, *cm, *cc, *bm0, *xlamm, *an, *bn, *cn;
    // vertical eigenbasis, row-major [NZ][NZ]: U(p,k) and V(k,p)
    const double *U, *V, *lam;
    double zx[11];
    BlkDev blk;                     // CHY_PREC_FP64_BLKTRI plans only
};

// Per-launch batch addressing.  Caller arrays come as pointer lists; the
// library's work arrays are one allocation with a fixed per-solve stride.
struct BatchPtrs {
    const double *rho[kMaxBatchPtrs];
    double *phi[kMaxBatchPtrs];
};

struct Work {
    double *X, *W, *C, *mom, *sub, *scan, *phac, *diag;
    size_t sX, sW, sC, smom, ssub, sscan, sphac, sdiag;   // per-solve strides (elements)
    double *coef;                                    // optional /COEFS/ output (solve 0 only)
    double *bvec, *bscr;                             // BLKTRI-order path (k_blktri.cu)
};

// ExternalPot (pot/ExternalPot.f:1-80): the star potential added after POT3.
struct StarDev {
    int on = 0;          // add STARPHI to PHI
    int indirect = 0;    // star position shifted by each solve's disk mass moment
    int jmin = 2;        // first J of that moment (1-based)
    double mass = 0.0;   // MASS_STAR + TMASSACC
    double mass_star = 0.0;
    double ix = 0.0, iy = 0.0;   // RPSTAR cos PHI_STAR, RPSTAR sin PHI_STAR
    double rof3n = 0.0, zof3n = 0.0, dtheta = 0.0;
    // the BINARY build's companion (pot/ExternalPot.f:12-16, 57-69)
    int binary = 0;
    double mass_bin = 0.0, rbin = 0.0, omega2 = 0.0, rcom = 0.0;
};
constexpr int kDiagStar = 4;     // DIAG slots of INDIRECTX, INDIRECTY
constexpr int kDiagPart = 8;     // first DIAG slot of the per-L moments

// SOURCE's potential, pressure and rotation terms (radhydro/source.f:45-81).
// Hydro arrays (OMEGA, P, S, T, A) are (J2h, K2h, L); RHO and PHI are the
// potential grid's (J2p, K2p, L).  All pointers are device pointers.
struct SourceDev {
    int J2h, K2h, J2p, K2p, L;
    int Jh, Kh;          // hydro JMAX, KMAX
    int j0;              // JSTART - 1 (0-based first J of T and A)
    double delt, dr, dz, dtheta;
    double inv_dr, inv_2dr, inv_dz;   // 1/DR, 1/(2 DR), 1/DZ when powers of two, else 0
    const double *R;     // R(POT3JMAX+2)
    const double *rho, *phi, *omega, *p;
    double *S, *T, *A;
    // BINARY build's terms (binary != 0): OMEGABIN, RHF(POT3JMAX+2), U
    int binary;
    double omega_bin;
    const double *rhf, *u;
};

// Raises a kernel's dynamic shared-memory limit on the current device the
// first time a launch needs it; the attribute persists, so later launches make
// no runtime call (a per-launch cudaFuncSetAttribute stalls the issue stream).
cudaError_t ensure_smem(const void *kernel, size_t bytes);

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on the driver library); null when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// kernels (k_fft.cu, k_bdy.cu, k_solve.cu)
cudaError_t launch_forward(const DevTables &t, const BatchPtrs &bp, const Work &w, int nb, cudaStream_t s);
cudaError_t launch_bdy_sums(const DevTables &t, const Work &w, int nb, cudaStream_t s);
cudaError_t launch_bdy_synth(const DevTables &t, const Work &w, int nb, cudaStream_t s);
cudaError_t launch_solve_fp64(const DevTables &t, const Work &w, int nb, int num_sms, cudaStream_t s);
// BLKTRI-order FP64 mode solves (k_blktri.cu): gather, cyclic reduction, scatter.
// Stage schedule: nw warps per CTA (4, 8 or 16), up to ctas_per_sm CTAs per SM,
// nw * ctas_per_sm <= 16.
cudaError_t launch_solve_blk(const DevTables &t, const Work &w, int nb, int num_sms, int nw, int ctas_per_sm,
                             cudaStream_t s, int *launches);
bool blk_schedule_valid(int nw, int ctas_per_sm);
// Its work-space sizes in doubles: BVEC for nb solves, BSCR for a plan of max_batch.
size_t blk_vector_doubles(const DevTables &t, int nb);
size_t blk_scratch_doubles(const DevTables &t, int max_batch, int num_sms);
// Inverse transform into PHI (plus STARPHI when x.on) and the diagnostics;
// with x.on also the cells POT3 leaves alone; reports its launch count.
cudaError_t launch_inverse(const DevTables &t, const BatchPtrs &bp, const Work &w, const StarDev &x, int nb,
                           cudaStream_t s, int *launches);
// INDIRECT star position of each solve into DIAG (x.on && x.indirect).
cudaError_t launch_star_shift(const DevTables &t, const BatchPtrs &bp, const Work &w, const StarDev &x, int nb,
                              cudaStream_t s);
// SOURCE's first loop nest on device arrays (k_source.cu).
cudaError_t launch_source(const SourceDev &a, cudaStream_t s);
// STARPHI(J+2, K+2, L) into out (star position of batch slot `slot` if indirect).
cudaError_t launch_star_fill(const DevTables &t, const Work &w, const StarDev &x, int slot, double *out,
                             cudaStream_t s);

}  // namespace chy

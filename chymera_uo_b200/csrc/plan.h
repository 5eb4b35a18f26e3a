// plan.h -- host-side tables of one pot3 grid (internal to libchy_pot3).
//
// Everything here depends only on the grid, never on the density, and is
// built once per plan on the host in FP64 (compiled with -ffp-contract=off so
// every value equals the one the reference's own arithmetic produces):
//   * the azimuthal transform schedule: the stage radices, per-butterfly
//     twiddles and output permutation that Singleton's FFT (pot/fft.f:73-629)
//     and REALTR (pot/fft.f:2-70) use for LMAX/2 points, recorded by walking
//     their loop structure;
//   * BDYGEN geometry (pot/boundary.f:366-617, 659-806): per-ring Legendre x
//     r^l terms, volumes and r^-(2l+1) factors, the rings sorted by spherical
//     radius, and for each boundary point the number of rings inside it;
//   * the POT3 stencil (pot/pot3.f:158-194) and the eigenbasis of its
//     vertical operator, which turns every mode's block-tridiagonal system into
//     KMAX-1 independent radial tridiagonal systems.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "chy_pot3.h"

namespace chy {

// One direction (ISN = +1 forward, -1 inverse) of the LMAX/2-point complex
// transform plus its real-data pass.
struct FftSchedule {
    int n = 0;           // complex length N = LMAX/2
    int isn = 1;
    int nstage = 0;
    int radix[24] = {};  // 2 or 4
    int span[24] = {};   // distance between the elements of one butterfly
    // per stage, per first-element index kk (0..n-1): c1,s1,c2,s2,c3,s3
    std::vector<double> tw;
    std::vector<uint8_t> twon;  // per stage, per kk: 1 if the butterfly rotates
    std::vector<int> perm;      // out[p] = in[perm[p]] (square-factor permutation)
    int nh = 0;                 // REALTR steps (N/2 + 1)
    std::vector<double> rt;     // per step: cn, sn
    // compact form: the rotation of a butterfly depends only on its position
    // j < span within the block; stage s occupies entries [off[s], off[s]+span[s])
    int off[24] = {};
    int ncompact = 0;
    std::vector<double> twc;    // [ncompact][6]
    std::vector<uint8_t> onc;   // [ncompact]
};

// Records the schedule.  Returns CHY_OK or CHY_ERR_DIMS (N not a power of 2).
int build_fft_schedule(int n, int isn, int literal_r8, FftSchedule &s);
// Table-driven execution on the host (used by tests through chy_dbg_*).
void fft_apply_host(const FftSchedule &s, double *a, double *b);
void realtr_apply_host(const FftSchedule &s, double *a, double *b);

struct HostPlan {
    chy_grid g{};
    int J = 0, K = 0, L = 0, N = 0, M = 0, NZ = 0;  // M = J-1, NZ = K-1
    int nring = 0, njk = 0, ntrm = 0;
    double dtheta = 0, sf1 = 0, pig4 = 0;
    std::vector<double> r, z, rhf, zhf;      // (J+2), (K+2)

    FftSchedule fwd, inv;
    std::vector<double> cosm, sinm;          // [m-1][l]  (m = 1..10)
    std::vector<double> bcos;                // [l] COS((L-1/2) DTHETA - PI)
    // POT3's forward transform (times SF1) of the 21 azimuthal basis columns
    // {1, cos m psi_l, sin m psi_l}, m = 1..10: [q][mode]
    std::vector<double> fbasis;

    // rings (j < M, k < NZ), ring index = k*M + j
    std::vector<double> ring_rsph;           // spherical radius
    std::vector<double> ring_dv;             // DV (0 for rings cut by REDGE)
    std::vector<double> ring_term;           // [ring][66]
    std::vector<double> ring_qh;             // [ring][11]: r^-(2l+1)
    std::vector<int> ring_sorted;            // rings (REDGE-kept) by ascending radius
    int nkeep = 0;

    // boundary points JK (top edge, then outer edge; ISYM 1/8 bottom edge is
    // skipped: POT3 overwrites it with the midplane ghost)
    std::vector<int> jk_j, jk_k;             // X coordinates (j in [0,J), k in [0,K))
    std::vector<double> jk_rbdy;
    std::vector<int> jk_split;               // rings (sorted) with r <= RBDY(JK)
    std::vector<int> sub_start;              // sub-chunk cuts in sorted order (never inside a split)
    std::vector<int> jk_sub;                 // sub-chunk index starting at jk_split
    std::vector<double> sring;               // [nkeep][4] rsph, C1, S1, DV in sorted order
    int srow = 0;                            // row length of sterm (NTRM + 12)
    std::vector<double> sterm;               // [nkeep][srow] TERM(1..NTRM), r^-(2l+1), DV
    std::vector<double> jk_bin, jk_hout;     // [jk][66]: TERM*RSPHER^-(l+1), TERM*RSPHER^l

    // active MRING columns: col -> (term index i (0-based), part 0=cos/mass, 1=sin)
    std::vector<int> col_term, col_part, col_m, col_l;
    int ncol = 0;

    // stencil (pot/pot3.f:158-194), radial arrays length M, vertical length NZ
    std::vector<double> am, cm, cc, bm0;     // bm0 = -CM-AM (row 0 and M-1 special)
    std::vector<double> an, bn, cn;
    double cmmax = 0, ammin = 0, cnmax = 0;
    std::vector<double> xlamm;               // cos(m*dtheta), m = 0..N

    // vertical eigenbasis: T_z = V diag(lam) U, U = V^-1; row-major [NZ][NZ].
    // U = Q^T D and V = D^-1 Q with Q orthogonal (Qt = Q^T, row-major
    // [p][k]) and D = diag(dsc) the symmetriser of T_z
    std::vector<double> lam, U, V, Qt, dsc;

    // ZAXPHI abscissae X(1..NPOINT)
    int npoint = 8;
    double zx[11] = {};
};

// Validates the descriptor and fills every table.  Returns a CHY_* status and
// a message in err.
int build_host_plan(const chy_grid &g, HostPlan &hp, std::string &err);

// Symmetric-tridiagonal eigen decomposition by implicit QL with Wilkinson
// shifts: d (n) diagonal, e (n) couplings e[i] between i and i+1, z (n*n)
// column-major eigenvectors.  Returns 0 or the index that failed to converge.
int tridiag_eigen(int n, double *d, double *e, double *z);

// The mixed path's radial sweep table of a grid (k_mixed.cu): two FP32
// planes [N+1][64 ceil(JMAX/64)][128], multipliers then pivot reciprocals.
std::vector<float> mixed_sweep_table(const HostPlan &hp);
// Its eigenbasis operand tile read back through its swizzled layout:
// [Q^T hi, Q^T lo], each [128 rows][128 K] (test hook).
std::vector<double> mixed_operand_tiles(const HostPlan &hp);
// Its per-row scales [4][128]: d_k, 1/d_k, d_k AN_k / d_(k-1),
// d_k CN_k / d_(k+1).
std::vector<double> mixed_row_scales(const HostPlan &hp);

}  // namespace chy

// blk.h -- the reference's own mode solver, FISHPACK BLKTRI (pot/blktri.f),
// recorded on the host as a schedule the GPU replays (internal to
// libchy_pot3).
//
// POT3 solves every azimuthal mode with BLKTRI(IFLG=1, NP=1, N=KMAX-1, ...,
// M=JMAX-1) (pot/pot3.f:233-239): generalized cyclic reduction over the
// vertical index (BLKTR1, pot/blktri.f:60-173) whose unit of work is PRDCT
// (pot/blktri.f:177-260), a product of shifted radial tridiagonal inverses
// applied to one vector of length M.  Which passes PRDCT makes, with which
// shifts, and how it updates its right-hand side between passes depends only
// on the root table COMPB builds (pot/blktri.f:264-344) -- never on the
// density and never on the mode -- so the host walks PRDCT's control flow
// once per grid and records each call as a program:
//
//   entry   W = X or -X, Y = W, optionally Y = c * W  (pot/blktri.f:183-208)
//   step    solve (B - rt I) W = Y by PRDCT's elimination and
//           substitution (:210-231), then Y = W (:234-238),
//           Y = Y + c W (:240-257) or Y = c W (:201-208), or nothing
//
// BLKTR1's loops are recorded as stages of independent tasks: at each
// reduction level the odd-position products (the W3 of :88-89 and :102-103)
// are computed first, then both neighbour products of every even position
// (:100-101, :104-105), then the combination (:106-108); back-substitution
// levels run their two neighbour products, the combination (:157-159) and the
// centre product (:160-161).  Every task of a stage is independent of the
// others, and each does exactly the reference's operations in the reference's
// order, so a replay gives the reference's rounding bit for bit.
#pragma once

#include <string>
#include <vector>

namespace chy {

// Right-hand-side update after a tridiagonal pass of PRDCT.
enum : int { BLK_NONE = 0, BLK_COPY = 1, BLK_AXPY = 2, BLK_SCALE = 3 };

struct BlkStep {
    double rt;     // shift BD(ID) of the pass
    double coef;   // c of Y = Y + c W (RT - BM1/BM2 root) or Y = c W (AA(IA))
    int post;      // BLK_*
    int pad;
};

struct BlkProg {       // one PRDCT call
    int first;         // steps [first, first + nsteps)
    int nsteps;
    int neg;           // W = -X at entry (ND > 0 and IS <= 0)
    int pre;           // Y = pre_coef * W before the first pass (NA > 0)
    double pre_coef;
};

// Task kinds.  Vector ids index an item's vectors; -1 stands for a zero vector.
enum : int { BLK_TASK_PRDCT = 0, BLK_TASK_SUMSUB = 1, BLK_TASK_SUBSUB = 2 };
struct BlkTask {
    int prog;   // PRDCT: program index
    int a;      // PRDCT: input X.  SUMSUB: out = (a + b) - c.  SUBSUB: out = (a - b) - c
    int b, c;
    int out;
    int pad;
};
struct BlkStage {
    int kind;    // BLK_TASK_* of every task in the stage
    int first;   // tasks [first, first + ntasks)
    int ntasks;
    int pad;
};

// Per-item vectors (each M long): Y(:,1..N) at ids [0, N), the odd-position
// products / back-substitution right-hand sides at [N, N+H), the two
// neighbour products at [N+H, N+2H) and [N+2H, N+3H); H = (N+1)/2.
struct BlkSchedule {
    int n = 0, m = 0, kx = 0;
    int nvec = 0;
    std::vector<double> roots;   // COMPB's B(1..IWCN-1), 0-based
    std::vector<double> cns;     // CN as BLKTR1 receives it, W(IWCN..IWCN+N-1)
    std::vector<BlkStep> steps;
    std::vector<BlkProg> progs;
    std::vector<BlkTask> tasks;
    std::vector<BlkStage> stages;
    int max_steps = 0;           // longest program
};

// Records the schedule for N = an.size() vertical and M radial unknowns
// (NP = 1).  an, bn, cn are POT3's AN, BN, CN (pot/pot3.f:177-191).  Returns
// 0, or BLKTRI's IERROR (1: M < 2, 2: N != 2**k - 1, 4: COMPB's eigenvalue
// iteration failed) with a message.
int build_blk_schedule(const std::vector<double> &an, const std::vector<double> &bn,
                       const std::vector<double> &cn, int m, BlkSchedule &s, std::string &err);

// Replays the schedule on the host for one mode: y is Y(M, N) column-major
// (column k = Y(:,k+1)), solved in place; am, bm, cm are BLKTRI's AM, BM, CM.
// The device kernel performs the same operations in the same order.
void blk_solve_host(const BlkSchedule &s, const double *am, const double *bm, const double *cm, double *y);

struct HostPlan;
// BM of mode l (0-based: m = l for l <= LMAX/2, else l - LMAX/2) with POT3's
// expression and order of operations (pot/pot3.f:226-230), M entries.
void blk_mode_bm(const HostPlan &hp, int l, double *bm);
// BM of every mode as the kernel reads it: [max(1, L/32)][M][32], lane ->
// mode (32 * block + lane) mod L.
std::vector<double> blk_bm_table(const HostPlan &hp);

}  // namespace chy

/*
 * chy_pot3_testing.h -- hooks of libchy_pot3 for its test suite.  Only
 * chy_dbg_work and chy_dbg_umma touch the GPU.
 */
#ifndef CHY_POT3_TESTING_H
#define CHY_POT3_TESTING_H

#include "chy_pot3.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The library's recorded transform schedule applied on the host to a[0..n),
 * b[0..n) (complex FFT of pot/fft.f:73 with ISN = isn); no device work. */
int chy_dbg_fft(int n, int isn, int literal_kind, double *a, double *b);
/* REALTR (pot/fft.f:2) from the recorded table; a, b hold n+1 entries. */
int chy_dbg_realtr(int n, int isn, int literal_kind, double *a, double *b);
/* Copies a named host table of the plan for grid g into out (capacity cap
 * entries) and returns its length, or a negative CHY_* status.  Names:
 * "U", "V", "lam", "an", "bn", "cn", "am", "cm", "cc", "bm0", "xlamm",
 * "ring_term" ([ring][66]), "ring_dv", "ring_rsph", "jk_split", "jk_bin",
 * "jk_hout", "sub_start", "jk_sub", "scalars" (sf1, pig4, cmmax, ammin,
 * cnmax, nkeep, ncol, nsub), and for the BLKTRI-order path "blk_roots"
 * (COMPB's root table B), "blk_cns" (CN as BLKTR1 receives it), "blk_bm"
 * ([mode][j] BM) and "blk_bm_table" (BM as the kernel reads it). */
long long chy_dbg_table(const chy_grid *g, const char *name, double *out, long long cap);

/* The recorded BLKTRI schedule replayed on the host for mode l of grid g:
 * y is Y(JMAX-1, KMAX-1) column-major, solved in place with the plan's AM,
 * BM(l) and CM, exactly as the device kernel does it; no device work. */
int chy_dbg_blktri(const chy_grid *g, int l, double *y);

/* Copies work array `name` of batch slot 0 ("X", "mom", "sub", "scan",
 * "phac", "diag") to host memory after a device synchronisation; returns the
 * count copied or a negative CHY_* status.  Layouts are described in
 * chymera_uo_b200/csrc/devplan.h. */
long long chy_dbg_work(chy_plan *p, const char *name, double *out, long long cap);

/* One tensor-core tile product of a CHY_PREC_MIXED plan:
 * D(128 x nt) = 4096 * A_pad(128 x 128) * Bm(nt x 128)^T with A the plan's
 * orthogonal vertical eigenbasis split into FP16 hi/lo parts exactly as the
 * mode solve uses it: which = 0 reads the tile as Q^T (K-major descriptor),
 * 1 as Q (the same tile through the transposed, MN-major descriptor).
 * Bm and D are device pointers (FP32, row-major); nt is 64, 128, 192 or 256.
 * Returns a CHY_* status after synchronising the device. */
int chy_dbg_umma(chy_plan *p, int which, const float *Bm_dev, float *D_dev, int nt);

/* Failure-path hook of a CHY_PREC_MIXED plan: with polls > 0, every CTA of
 * the plan's later mode solves first waits `polls` polls on a barrier that
 * nothing arrives on, before it issues any copy or product; the wait runs
 * out, the CTA poisons its modes with NaN, sets the device error word and
 * exits, and the solve reports CHY_ERR_TIMEOUT.  0 switches it off. */
int chy_dbg_mixed_probe(chy_plan *p, int polls);

/* The kernel that ran the plan's last mixed mode solve: 1 k_mode_mixed (one
 * CTA per mode), 2 k_mode_pair (CTA pairs), 3 the wide pipeline, 0 none yet or
 * not a CHY_PREC_MIXED plan; -CHY_ERR_ARG for a null plan. */
int chy_dbg_mixed_kernel(const chy_plan *p);

#ifdef __cplusplus
}
#endif
#endif

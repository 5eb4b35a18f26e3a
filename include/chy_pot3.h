/*
 * chy_pot3.h -- C ABI of the B200 gravitational-potential solve (CHYMERA pot3).
 *
 * One call replaces the reference's SETBDY + BDYGEN + POT3 sequence
 * (pot/boundary.f:2, pot/boundary.f:88, pot/pot3.f:15) as the ITYPE=71
 * potential run (radhydro/io.f:212-218) and the per-step update
 * (radhydro/3dhyd-main.f:474-477) issue it.  Arrays use the reference's
 * Fortran column-major layout: RHO and PHI are (JMAX+2, KMAX+2, LMAX) doubles
 * (headers/globals.h:55-58, /POIS/), J fastest.  POT3JMAX = JMAX and
 * POT3KMAX = KMAX.
 *
 * Write-set of a solve (identical to the reference's):
 *   PHI(1:JMAX+1, 1:KMAX+1, :)  except PHI(JMAX+2, 1, :)   -- written
 *   PHI(JMAX+2, 2:KMAX+1, :)                                -- written (ZAXPHI)
 *   PHI(:, KMAX+2, :) and PHI(JMAX+2, 1, :)                 -- never touched
 *   RHO is read-only; only RHO(2:JMAX, 2:KMAX, :) is read.
 *
 * No entry point calls exit(); every failure returns a status code.
 */
#ifndef CHY_POT3_H
#define CHY_POT3_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CHY_OK 0
/* 1..5 keep the meaning of FISHPACK BLKTRI's IERROR (pot/blktri.f:14-34;
 * the meanings are spelled out in Poisson/blktri.f90:105-120).  The reference
 * ignores IERROR (pot/pot3.f:238-239); this library reports it. */
#define CHY_ERR_M_LT_2 1          /* JMAX-1 < 2 radial unknowns                    */
#define CHY_ERR_N_NOT_POW2 2      /* KMAX-1 is not 2**k-1 (KMAX not a power of 2)  */
#define CHY_ERR_EIGEN 4           /* vertical-operator eigen solve failed           */
#define CHY_ERR_IDIMY 5           /* leading dimension too small                    */
#define CHY_ERR_ARG 10            /* NULL pointer or invalid argument              */
#define CHY_ERR_DIMS 11           /* LMAX not a power of 2 (pot/fft.f factor rule), */
                                  /* or a size out of the supported range          */
#define CHY_ERR_UNSUPPORTED 12    /* ISYM / MAXTRM / NPOINT outside supported set   */
#define CHY_ERR_NOT_SETUP 13      /* BDYGEN before SETBDY (pot/boundary.f:311)      */
#define CHY_ERR_CUDA 20           /* a CUDA runtime call failed                     */
#define CHY_ERR_NOMEM 21          /* device allocation failed                       */
#define CHY_ERR_NOCONV 30         /* mixed-precision refinement missed tolerance    */
#define CHY_ERR_TIMEOUT 31        /* a device-side bounded wait expired             */
#define CHY_ERR_CAPACITY 32       /* batch larger than the plan's capacity         */

/* ---- descriptors --------------------------------------------------------- */
enum { CHY_LITERAL_GCC = 0, CHY_LITERAL_R8 = 1 };
/* Mode-solve precisions.
 *   CHY_PREC_FP64_BLKTRI  the reference's own mode solver, FISHPACK BLKTRI
 *                         generalized cyclic reduction (pot/blktri.f:3-423,
 *                         called from pot/pot3.f:233-239), in FP64 with the
 *                         reference's operations in the reference's order:
 *                         the plain FP64 pot3, equal to the reference's
 *                         rounding.
 *   CHY_PREC_FP64         FP64 through the eigenbasis of the m-independent
 *                         vertical operator and radial Thomas sweeps; several
 *                         times faster, ~10x closer to the exact solution
 *                         than BLKTRI's rounding (so a few 1e-12 away from the
 *                         reference's result on 256 x 128 grids).
 *   CHY_PREC_MIXED        tensor-core FP16 hi/lo transforms, FP32 sweeps and
 *                         an FP64 refinement (<= 1e-10 of the reference). */
enum { CHY_PREC_FP64 = 0, CHY_PREC_MIXED = 1, CHY_PREC_FP64_BLKTRI = 2 };
enum { CHY_PTR_DEVICE = 0, CHY_PTR_HOST = 1 };

/* Grid and call parameters.  Fields mirror COMMON /GRID/ and /BLOK6/
 * (headers/globals.h:10,104-109) plus the constant call arguments of
 * radhydro/3dhyd-main.f:166-167,477 (MAXTRM=10, ISYM=2, NPOINT=8). */
typedef struct chy_grid {
    int jmax, kmax, lmax;      /* POT3JMAX=JMAX, POT3KMAX=KMAX, LMAX             */
    double rof3n, zof3n;       /* radial / vertical spacing (DELR, DELZ)        */
    const double *r, *z;       /* R(JMAX+2), Z(KMAX+2); NULL: uniform from      */
    const double *rhf, *zhf;   /* RHF, ZHF;  ROF3N/ZOF3N as radhydro/io.f:194-203 */
    double pi, grav;           /* PI, GRAV; DTHETA = 2*PI/LMAX (io.f:136-140)   */
    int isym;                  /* BDYGEN symmetry flag (2 is the production one) */
    int maxtrm;                /* multipole order l <= MAXTRM (<= 10)           */
    double redge;              /* BDYGEN REDGE: 0, or R(JMAX+1) per time step   */
    int npoint;                /* ZAXPHI interpolation points (<= 10)           */
    int literal_kind;          /* CHY_LITERAL_GCC (chymera-omp) or _R8          */
} chy_grid;

/* /INSIDE/ diagnostics (pot/boundary.f:112, pot/pot3.f:317) and the
 * mixed-precision refinement report. */
typedef struct chy_diag {
    double tmass;              /* TMASS: total mass seen by BDYGEN              */
    double phichk;             /* PHICHK: largest z-axis deviation (ZAXPHI)     */
    int klocat;                /* KLOCAT: K of PHICHK                           */
    int iterations;            /* approximate solves performed (mixed: 1 +      */
                               /* corrections; 0 for the FP64 path)             */
    double corr_rel[8];        /* ||delta_i|| / ||x_{i+1}|| of solve i           */
    double indirectx, indirecty; /* star position the external potential used  */
                               /* (/POIS/ INDIRECTX/Y); 0 without one           */
} chy_diag;

typedef struct chy_plan chy_plan;

/* Fills a descriptor with the reference's defaults for a JMAX x KMAX x LMAX
 * grid: ROF3N = 1/JMAX, ZOF3N = 0.5/KMAX, PI = 3.1415926535897932, GRAV = 1,
 * ISYM = 2, MAXTRM = 10, REDGE = 0, NPOINT = 8, gcc literals. */
void chy_grid_defaults(chy_grid *g, int jmax, int kmax, int lmax);

/* Builds every per-grid table (FFT schedule, ring and boundary geometry,
 * stencil, vertical eigenbasis) on the host, uploads them to the current
 * device and allocates work space for up to max_batch concurrent solves.
 * Replaces the once-per-run SETBDY(0,ISYM) (pot/boundary.f:2-82) and
 * BLKTRI(IFLG=0) (pot/blktri.f:13-46). */
int chy_plan_create(const chy_grid *g, int precision, int max_batch, chy_plan **out);
void chy_plan_destroy(chy_plan *p);

/* Every solve entry point needs the device that was current at
 * chy_plan_create to be current when it is called; otherwise it returns
 * CHY_ERR_ARG. */

/* One solve: BDYGEN(MAXTRM,ISYM,REDGE) then POT3(NPOINT,IPRINT=0).
 * rho/phi are device pointers (CHY_PTR_DEVICE) or host pointers
 * (CHY_PTR_HOST; pinned memory gives full copy bandwidth).  A device PHI
 * changes in the reference's write set only.  A host PHI comes back as one
 * contiguous copy: the cells outside the write set (PHI(:,KMAX+2,:),
 * PHI(JMAX+2,1,:)) are read at the start of the call and written back with
 * the same values.  stream may be
 * NULL (legacy default stream).  diag may be NULL.  For device pointers the
 * call is asynchronous unless diag is non-NULL.  Device RHO arrays that start
 * on a 16-byte boundary (cudaMalloc and torch allocations do) with JMAX even
 * are read through tensor-memory-access copies; others through 8-byte copies,
 * with bitwise the same results. */
int chy_solve(chy_plan *p, const double *rho, double *phi, chy_diag *diag, int ptr_kind,
              void *stream);

/* n independent solves of the plan's grid in one launch sequence.  rho[i],
 * phi[i] as above; diag may be NULL or an array of n. */
int chy_solve_batch(chy_plan *p, int n, const double *const *rho, double *const *phi,
                    chy_diag *diag, int ptr_kind, void *stream);

/* n densities of possibly different grids (device pointers): request i is
 * solved with plans[i].  Requests that share a plan are batched (up to its
 * max_batch per launch sequence); different plans run concurrently on side
 * streams forked from `stream` and joined back into it, so the call is
 * ordered on `stream` like chy_solve_batch and makes no host wait.  The first
 * call on a device creates the side streams.  A plan may appear in only one
 * call at a time; calls from several host threads must be serialised.  No
 * reference counterpart (the reference solves one grid per run). */
int chy_solve_multi(int n, chy_plan *const *plans, const double *const *rho, double *const *phi, void *stream);

/* Launch-schedule autotuner for a request set (no reference counterpart).
 * Times chy_solve_multi over the given requests under candidate schedules
 * and keeps the fastest in the plans, where later chy_solve_multi calls (and
 * CUDA graphs captured after this call) use it:
 *   streams      grids in flight at once (8, 4, 2, 1);
 *   chunk        solves per launch sequence (max_batch, /2, /4);
 *   mode_ctas    persistent CTAs of each fused mixed mode solve (all SMs, 1/2,
 *                1/4: grids running side by side then share the SMs);
 *   mode_kernel  not searched; the plan's own setting for the fused mixed
 *                mode solve: 0 = automatic (CTA pairs when the launch holds
 *                at least 16 (solve, mode) items per group of warps, else
 *                one CTA per item), 1 = one CTA per item, 2 = CTA pairs
 *                holding two items per SM.  Both kernels give the same bits;
 *   blk_warps,   the BLKTRI-order path's stage schedule: warps per CTA (the
 *   blk_ctas_per_sm  cyclic-reduction tasks of a stage in flight at once) and
 *                CTAs per SM.
 * Search: from the default schedule, each knob in turn (coordinate descent),
 * `repeats` timed calls per candidate after one warm-up call, CUDA events on
 * `stream`.  The call synchronises `stream`; make it before any capture.  The
 * results of the last call are in phi. */
typedef struct chy_tune {
    int streams, chunk, mode_ctas, blk_warps, blk_ctas_per_sm, mode_kernel;
    double ms;           /* one chy_solve_multi call under the chosen schedule */
    double ms_default;   /* the same under the default schedule              */
    int candidates;      /* schedules timed                                   */
} chy_tune;
int chy_autotune_multi(int n, chy_plan *const *plans, const double *const *rho, double *const *phi, void *stream,
                       int repeats, chy_tune *out);
/* A plan's launch schedule (the first six fields of chy_tune; 0 = default
 * for streams, chunk, mode_ctas and mode_kernel), e.g. to reuse a tuned schedule in a
 * later run.  The timing fields are ignored / returned as 0. */
int chy_plan_set_schedule(chy_plan *p, const chy_tune *c);
int chy_plan_get_schedule(const chy_plan *p, chy_tune *c);

/* ---- serving: continuous batching of solve requests ----------------------
 * No reference counterpart.  A server keeps one size class per distinct grid
 * (resident plans: tables + work space, two lanes so that the copies of one
 * batch overlap the solves of the previous one) and a dispatcher thread.
 * Requests queue from any thread; a request is admitted into its class's next
 * batch as soon as device buffers for it fit in the server's arena, so
 * requests that arrive while others run join the next batch of their grid;
 * classes run concurrently on their own streams.  Results do not depend on
 * batching (every reduction has a fixed per-solve order). */
typedef struct chy_server chy_server;
typedef struct chy_server_opts {
    long long hbm_budget;      /* device bytes for plans + request buffers; 0: 3/4 of free */
    int precision;             /* CHY_PREC_MIXED (grids it does not cover use FP64), _FP64 or */
                               /* _FP64_BLKTRI                                                 */
    int max_batch;             /* solves per launch sequence (default 8, <= 64)            */
    double arena_fraction;     /* share of the budget for request buffers (default 0.5)    */
} chy_server_opts;
typedef struct chy_server_stats {
    long long completed, batches;
    int size_classes;
    long long plan_bytes, arena_bytes;
} chy_server_stats;
/* Starts the dispatcher on the current device; allocates the arena. */
int chy_server_create(const chy_server_opts *o, chy_server **out);
/* Queues one solve of grid g (arrays copied now): rho is read and phi written
 * (the reference's write set; the cells outside it are read and written back
 * unchanged, as for CHY_PTR_HOST solves) asynchronously; both must stay valid
 * until chy_server_wait returns.  Pinned host memory gives full copy
 * bandwidth. */
int chy_server_submit(chy_server *s, const chy_grid *g, const double *rho, double *phi, long long *ticket);
/* Blocks until the request is done; returns its status and the latency from
 * submission to completion (host clock, ms). */
int chy_server_wait(chy_server *s, long long ticket, double *latency_ms);
int chy_server_get_stats(chy_server *s, chy_server_stats *out);
/* Finishes the queued requests, then releases everything. */
void chy_server_destroy(chy_server *s);

/* Optional /COEFS/ output (pot/pot3.f:105-132): when set, the next solves
 * also write COEF(JMAX+2, KMAX+2, LMAX/2, 2) (amplitude, phase in degrees)
 * at coef_dev (device pointer, or NULL to stop). */
int chy_plan_set_coef(chy_plan *p, double *coef_dev);
/* The same for host-pointer solves into a host array (COEF as in /COEFS/):
 * the plan allocates a device copy once, here, and each host-pointer solve
 * copies it in before and out after the solve, so cells the reference leaves
 * alone keep their values.  Host-pointer batches then run one solve per
 * chunk.  NULL stops the output. */
int chy_plan_set_coef_host(chy_plan *p, double *coef_host);

/* The text POT3 writes to unit 3 with IPRINT = 1 (pot/pot3.f:402-418), for
 * the first solve of the plan's latest solve call: "PHAC(1:KMAX1):",
 * PHAC(2:KMAX1) as FORMAT(1P11E11.3), "Fourier amplitudes and phases:" and,
 * for LMAX > 8, per J = 2..JMAX the amplitudes and phases COEF(J,2,M,1:2),
 * M = 1..8, as FORMAT(20X,I5,' COEFS=',1P8E12.3,/,25X,' PHASE=',0P8F12.2).
 * Needs the COEF output of that solve (chy_plan_set_coef or
 * chy_plan_set_coef_host; CHY_ERR_NOT_SETUP otherwise).  Synchronises the
 * device.  Copies at most cap-1 characters and a NUL into buf and returns the
 * full length, or a negative CHY_* status.  The ITYPE=71 run, which calls
 * POT3 with IPRINT = 1 before unit 3 is opened (radhydro/io.f:208-218,
 * :869), writes it to fort.3. */
long long chy_plan_report(chy_plan *p, char *buf, long long cap);

/* Fixed number of refinement corrections for CHY_PREC_MIXED, 0..7 (default
 * 1).  Up to one correction the first solution stays in tensor memory; two or
 * more keep an FP64 iterate in device memory, allocated by this call (one
 * more grid volume per batch slot). */
int chy_plan_set_refine(chy_plan *p, int corrections);

/* ---- ExternalPot (pot/ExternalPot.f:1-80) --------------------------------
 * The central star's potential, added to PHI right after POT3 as the
 * EXTERNAL_POT build does every time step (radhydro/3dhyd-main.f:510-512):
 *   STARPHI(J,K,L) = -(MASS_STAR+TMASSACC) / SQRT(RHF(J)**2 + ZHF(K)**2
 *       + IX**2 + IY**2 - 2 RHF(J) (COS(PSI_L) IX + SIN(PSI_L) IY)),
 *   PSI_L = (L-1/2) DTHETA, PHI = PHI + STARPHI on every cell of the grid.
 * IX, IY = RPSTAR*COS(PHI_STAR), RPSTAR*SIN(PHI_STAR) (ExternalPot.f:18-19);
 * with `indirect` set (INDIRECT builds, ExternalPot.f:21-40) each solve adds
 * its disk's mass moment over J = JMIN..JMAX+1, K = 2..KMAX+1 and divides by
 * -MASS_STAR.  The add is fused into the inverse transform's stores; the
 * cells POT3 does not write (K = KMAX+2, and J = JMAX+2 at K = 1) are updated
 * in place, so for host-pointer solves those cells of the caller's PHI are
 * read in as well as written back. */
typedef struct chy_external {
    double mass_star, tmassacc;  /* MASS_STAR, TMASSACC (/GAP/, globals.h:28)    */
    double rpstar, phi_star;     /* star position (/movingstar/, globals.h:5-6)  */
    int indirect;                /* 1: INDIRECT build's centre-of-mass shift     */
    int jmin;                    /* JMIN of that shift (hydroparam.h:23: 2)      */
} chy_external;
/* Sets (ext non-NULL) or clears (NULL) the external potential of the plan's
 * later solves through chy_solve / chy_solve_batch / chy_solve_multi.
 * chy_solve_static and the server solve POT3 alone. */
int chy_plan_set_external(chy_plan *p, const chy_external *ext);
/* The BINARY build's companion (pot/ExternalPot.f:12-16, 57-69), added after
 * STARPHI on every cell while the external potential is set:
 *   PHI = PHI - MASSBIN/RDIST - OMEGABIN**2/2 ((X+RCOM)**2 + Y**2),
 *   RDIST = SQRT(RBIN**2 + RHF(J)**2 - 2 RBIN RHF(J) COS(THETA-PI) + ZHF(K)**2),
 *   X, Y = RHF(J) COS(THETA), RHF(J) SIN(THETA), THETA = (L-1/2) DTHETA,
 * for getBinaryPosition's circular orbit (radhydro/ExternalRoutines.f:91-105):
 * MUBIN = MASSBIN + MASS_STAR, OMEGABIN = SQRT(MUBIN/ABIN**3), RBIN = ABIN,
 * RCOM = RBIN - RBIN*MASS_STAR/MUBIN.  The reference's parameters are
 * MASSBIN = 1, ABIN = 100 (headers/units.h:25).  STARPHI itself does not
 * include it, as in the reference. */
typedef struct chy_binary {
    double mass_bin;             /* MASSBIN                                      */
    double a_bin;                /* ABIN (> 0)                                   */
} chy_binary;
/* Sets (b non-NULL) or clears (NULL) the companion of the plan's later solves. */
int chy_plan_set_binary(chy_plan *p, const chy_binary *b);
/* Writes STARPHI(JMAX+2, KMAX+2, LMAX) (/GAP/ STARPHI) for the plan's
 * external potential: with `indirect`, for the star position of the plan's
 * latest solve (the last one of its most recent solve call), as the
 * reference's array holds it after the time step's solve.  Call it on the
 * stream of that solve, or after it.  starphi is a device or host pointer per
 * ptr_kind; host-pointer calls synchronise `stream`. */
int chy_plan_star_potential(chy_plan *p, double *starphi, int ptr_kind, void *stream);

/* ---- SOURCE's potential, pressure and rotation terms ----------------------
 * The first loop nest of SOURCE (radhydro/source.f:45-81, BINARY = 0), the
 * consumer of the PHI a solve writes, on device arrays in the reference's
 * layouts, with the plan's R, ROF3N (DR), ZOF3N (DZ) and DTHETA.  For
 * L = 1..LMAX (periodic in L), K = 2..KMAX+1 of the hydro grid:
 *   S += DELT*(R(J)(RHO_J+RHO_J-1)(OMEGA_J+OMEGA_J-1)**2/8
 *              - (RHO_J+RHO_J-1)(PHI_J-PHI_J-1)/(2 DR) - (P_J-P_J-1)/DR),
 *        J = JSTART+1..JMAX+1;
 *   T -= DELT*((RHO_K+RHO_K-1)/2 (PHI_K-PHI_K-1)/DZ + (P_K-P_K-1)/DZ),
 *   A -= DELT*(RHO (PHI_L+1-PHI_L-1) + P_L+1 - P_L-1)/(2 DTHETA),
 *        J = JSTART..JMAX+1;  JSTART = MAX(JMIN, 2).
 * Each operation rounds as the reference's does: bit-identical results.
 * Issued on `stream` after a solve on the same stream, it finds most of PHI
 * still in L2. */
typedef struct chy_source_args {
    int jmax, kmax;            /* hydro JMAX, KMAX (<= the plan's; hydroparam.h:16-17) */
    int jmin;                  /* JMIN (hydroparam.h:23)                             */
    double delt;               /* DELT                                               */
    const double *rho, *phi;   /* RHO, PHI(POT3JMAX+2, POT3KMAX+2, LMAX) (/POIS/)    */
    const double *omega, *p;   /* OMEGA, P(JMAX+2, KMAX+2, LMAX)                     */
    double *s, *t, *a;         /* S, T, A(JMAX+2, KMAX+2, LMAX), updated in place     */
} chy_source_args;
/* Device pointers only; S, T, A must not overlap the input arrays.
 * Asynchronous on `stream`. */
int chy_source(chy_plan *p, const chy_source_args *args, void *stream);
/* The same loop nest as a BINARY build compiles it (radhydro/source.f:38-40,
 * 61-62, 76-77): chy_source's updates, then in the same statements
 *   S += OMEGABIN*OMEGA(J)*RHF(J)*2*RHO(J)*DELT,      J = JSTART+1..JMAX+1,
 *   A -= RHO(J)*OMEGABIN*(U(J+1)+U(J))*DELT*RHF(J),   J = JSTART..JMAX+1,
 * each product formed left to right, with OMEGABIN of getBinaryPosition's
 * circular orbit (radhydro/ExternalRoutines.f:91-105):
 * SQRT((MASSBIN + MASS_STAR)/ABIN**3), the orbit chy_plan_set_binary's
 * companion uses.  u is U(JMAX+2, KMAX+2, LMAX), the radial velocity, a
 * device array that must not overlap S, T, A; mass_star is MASS_STAR (/GAP/).
 * Bit-identical to the reference's statements, like chy_source. */
int chy_source_binary(chy_plan *p, const chy_source_args *args, const chy_binary *b, double mass_star,
                      const double *u, void *stream);

/* Bytes of device work space the plan holds (tables + per-solve scratch). */
long long chy_plan_device_bytes(const chy_plan *p);
/* Device work-space bytes one more concurrent solve of this grid needs. */
long long chy_plan_bytes_per_solve(const chy_plan *p);

const char *chy_status_string(int status);
/* Message of the last failure on the calling thread, and the CUDA error code
 * behind the last CHY_ERR_CUDA. */
const char *chy_last_error(void);
int chy_last_cuda_error(void);

/* Per-stage device timing with CUDA events recorded on the solve stream:
 * stage 0 forward transform + ring moments, 1 boundary mass integrals,
 * 2 boundary potentials + their transform, 3 mode solves, 4 inverse
 * transform + ghosts + ZAXPHI.  Recording adds no host waits; the events are
 * read when chy_plan_stage_times is called (or every 4096 launch
 * sequences).  Switching profiling on or off resets the totals. */
int chy_plan_set_profiling(chy_plan *p, int on);
/* Waits for the recorded events, then returns the accumulated milliseconds
 * per stage (n >= 5) and the number of timed launch sequences; returns the
 * number of stages, or a negative CHY_* status. */
int chy_plan_stage_times(chy_plan *p, double *ms, int n, long long *calls);
/* Kernel launches this plan has issued so far. */
long long chy_plan_launch_count(const chy_plan *p);

/* One FP64 solve (device pointers, as chy_solve with CHY_PTR_DEVICE and no
 * diag) that allocates nothing: no device allocation, no free, no allocating
 * library routine during the call.  It has no reference counterpart.  It is
 * for callers whose device memory is fully committed once the plan exists,
 * for example a simulation that reserves the rest of the GPU for its own
 * arrays, or a time-step loop that must not call the allocator.
 * Its per-solve work space is one static 8 MiB device array per device:
 * enough for the FP64 work space of a 64 x 32 x 64 grid (3.5 MiB, the
 * reference's CPU-run size) or 64 x 32 x 128 (6.5 MiB).  Grids that need more
 * return CHY_ERR_CAPACITY (chy_last_error gives the size); mixed plans return
 * CHY_ERR_UNSUPPORTED.  The array is cleared (cudaMemsetAsync) at the
 * start of every call.  The first call on each device looks the array up
 * (cudaGetSymbolAddress) with that device current; make it before any
 * stream capture starts.  The address is kept for the process's life, so a
 * cudaDeviceReset in between is not supported.  All calls on one device share
 * the array, so calls that overlap in time (several streams or threads) race:
 * serialise them.  The plan's device must be current (CHY_ERR_ARG
 * otherwise).  Asynchronous on `stream` like chy_solve. */
int chy_solve_static(chy_plan *p, const double *rho, double *phi, void *stream);

#ifdef __cplusplus
}
#endif
#endif

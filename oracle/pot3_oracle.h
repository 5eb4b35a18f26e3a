/*
 * pot3_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of CHYMERA's gravitational-potential solve (SETBDY, BDYGEN,
 * POT3, ZAXPHI, FFT, REALTR, BLKTRI) used as the checker for the CUDA library
 * and as the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity status: UNPINNED against the reference binary.  The reference is
 * Fortran and no Fortran compiler exists on this machine or the GPU hosts, and
 * the reference ships no tests, fixtures or golden outputs.  The restatement
 * is pinned instead by independent checks (numpy FFT, scipy sparse per-mode
 * solves, a manufactured solution, multipole known answers); see tests/.
 *
 * All arrays follow the reference's Fortran column-major layout.
 */
#ifndef POT3_ORACLE_H
#define POT3_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_ctx ora_ctx;

/* literal_r8 = 0: default-REAL(4) literals as in the gcc build
 *                 (bin/Makefile.gcc: no -r8), e.g. pot/fft.f:38 and :129 use
 *                 single-precision ATAN(1.0).
 * literal_r8 = 1: all default-real literals promoted to REAL(8) as in the
 *                 -r8 / -fdefault-real-8 builds (bin/Makefile.intel:19,
 *                 Poisson/Makefile:14).
 * nthreads: OpenMP threads for BDYGEN/POT3 (1 = serial, bit-reproducible).
 * want_coef: allocate /COEFS/ COEF(JMAX2,KMAX2,LMAX/2,2) (pot/pot3.f:20). */
ora_ctx *ora_new(int jmax, int kmax, int lmax, int literal_r8, int nthreads, int want_coef);
void ora_free(ora_ctx *c);

/* Pointers into the context's COMMON-block stand-ins (caller fills / reads). */
double *ora_phi(ora_ctx *c);   /* PHI(JMAX2,KMAX2,LMAX)   headers/globals.h:55-58 */
double *ora_rho(ora_ctx *c);   /* RHO(JMAX2,KMAX2,LMAX)   */
double *ora_r(ora_ctx *c);     /* R(JMAX2)                headers/globals.h:104-109 */
double *ora_z(ora_ctx *c);     /* Z(KMAX2)                */
double *ora_rhf(ora_ctx *c);   /* RHF(JMAX2)              */
double *ora_zhf(ora_ctx *c);   /* ZHF(KMAX2)              */
double *ora_coef(ora_ctx *c);  /* COEF or NULL            */
double *ora_massin(ora_ctx *c);  /* MASSIN(2,66,JKM1) of the last BDYGEN  */
double *ora_massout(ora_ctx *c); /* MASSOUT(2,66,JKM1) of the last BDYGEN */
double *ora_rbdy(ora_ctx *c);  /* RBDY(JKM1) from SETBDY  */
int ora_jkmax(ora_ctx *c);

/* /BLOK6/ and /GRID/ scalars */
void ora_set_scalars(ora_ctx *c, double rof3n, double zof3n, double dtheta,
                     double pi, double grav);
/* Fills R, Z, RHF, ZHF exactly as radhydro/io.f:194-203 does. */
void ora_make_grid(ora_ctx *c, double delr, double delz);

/* The three entry points of the hot path. */
void ora_setbdy(ora_ctx *c, int ncall, int isym);                 /* pot/boundary.f:2   */
int  ora_bdygen(ora_ctx *c, int maxtrm, int isym, double redge);  /* pot/boundary.f:88  */
void ora_pot3(ora_ctx *c, int npoint, int iprint);                /* pot/pot3.f:15      */

/* /INSIDE/ diagnostics: out[0]=TMASS, out[1]=PHICHK, out[2]=KLOCAT */
void ora_inside(ora_ctx *c, double *out3);
/* PHAC(K), K=1..KMAX2, from the last ZAXPHI */
double *ora_phac(ora_ctx *c);

/* ExternalPot (pot/ExternalPot.f:1-80) on the context's PHI after POT3:
 * adds STARPHI = -(MASS_STAR+TMASSACC)/|x - x_star| everywhere (starphi, if
 * not NULL, receives it) with the star at INDIRECTX/Y = RPSTAR*COS/SIN(PHI_STAR),
 * or, indirect != 0 (INDIRECT builds), shifted by the disk's mass moment over
 * J = JMIN..JMAX1 (ExternalPot.f:21-40).  ixy (if not NULL) gets INDIRECTX/Y. */
void ora_external_pot(ora_ctx *c, double mass_star, double tmassacc, double rpstar, double phi_star,
                      int indirect, int jmin, double *starphi, double *ixy);
/* The same with the BINARY build's companion term (binary != 0): massBin,
 * aBin as in headers/units.h:25 (1 and 100 there). */
void ora_external_pot_binary(ora_ctx *c, double mass_star, double tmassacc, double rpstar, double phi_star,
                             int indirect, int jmin, int binary, double mass_bin, double a_bin, double *starphi,
                             double *ixy);

/* SOURCE's potential, pressure and rotation terms (radhydro/source.f:45-81,
 * BINARY = 0) for a hydro grid jmax x kmax x lmax: omega, p, s, t, a are
 * (jmax+2, kmax+2, lmax); rho, phi are (j2p, k2p, lmax); r is R(j2p).  s, t, a
 * are updated in place. */
void ora_source(int jmax, int kmax, int lmax, int j2p, int k2p, int jmin, double delt, double dr, double dz,
                double dtheta, const double *r, const double *rho, const double *phi, const double *omega,
                const double *p, double *s, double *t, double *a);
/* The same with the BINARY build's terms when binary != 0 (source.f:38-40,
 * 61-62, 76-77): omegaBin = sqrt((mass_bin + mass_star)/a_bin**3),
 * S += omegaBin*OMEGA*RHF*2*RHO*DELT, A -= RHO*omegaBin*(U(J+1)+U(J))*DELT*RHF;
 * u is U(jmax+2, kmax+2, lmax), rhf is RHF(j2p). */
void ora_source_binary(int jmax, int kmax, int lmax, int j2p, int k2p, int jmin, double delt, double dr, double dz,
                       double dtheta, const double *r, const double *rho, const double *phi, const double *omega,
                       const double *p, double *s, double *t, double *a, int binary, double mass_star,
                       double mass_bin, double a_bin, const double *rhf, const double *u);

/* Low-level routines, exported for unit tests. Arrays are 0-based views of the
 * Fortran 1-based arrays. */
void ora_fft(double *a, double *b, int ntot, int n, int nspan, int isn, int literal_r8);
void ora_realtr(double *a, double *b, int n, int isn, int literal_r8);
/* BLKTRI with its own /CBLKT/ + /BLOKJ1/ state block; state must hold at least
 * ora_blktri_state_size() bytes and persists between the IFLG=0 and IFLG=1 calls. */
int  ora_blktri_state_size(void);
void ora_blktri(void *state, int iflg, int np, int n, const double *an, const double *bn,
                const double *cn, int mp, int m, const double *am, const double *bm,
                const double *cm, int idimy, double *y, int *ierror, double *w);
/* Size of the BLKTRI workspace that POT3 gives it (pot/pot3.f:30) for the grid. */
int  ora_blktri_wsize(int jmax, int kmax);

#ifdef __cplusplus
}
#endif
#endif

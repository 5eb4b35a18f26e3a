// k_source.cu -- the potential, pressure and rotation source terms of the
// momentum equations, SOURCE's first loop nest (radhydro/source.f:45-81), on
// the device, for the PHI a solve has just written; with the BINARY build's
// rotating-frame terms as an option.
//
// Per cell of the hydro grid, L = 1..LMAX (periodic), K = 2..KMAX+1:
//   S(J) += DELT*( R(J)*(RHO_J+RHO_J-1)*(OMEGA_J+OMEGA_J-1)**2 * 1/4 * 1/2
//                 - (RHO_J+RHO_J-1)*(PHI_J-PHI_J-1)/(2 DR) - (P_J-P_J-1)/DR )
//                                                  J = JSTART+1..JMAX+1
//   T(J) -= DELT*( 1/2 (RHO_K+RHO_K-1)*(PHI_K-PHI_K-1)/DZ + (P_K-P_K-1)/DZ )
//   A(J) -= DELT*( RHO*(PHI_L+1-PHI_L-1) + P_L+1 - P_L-1 )/(2 DTHETA)
//                                                  J = JSTART..JMAX+1
// JSTART = MAX(JMIN, 2).  Every product, quotient and sum is rounded on its
// own, in the reference's order, so the result is the reference's to the bit.
//
// BINARY builds add, in the same statements (source.f:61-62, 76-77),
//   S += OMEGABIN*OMEGA(J)*RHF(J)*2*RHO(J)*DELT
//   A -= RHO(J)*OMEGABIN*(U(J+1)+U(J))*DELT*RHF(J)
// HBM-bound: per updated cell 7 reads and 3 writes of 8 bytes (one more read,
// U, in BINARY builds).  One CTA per (K, L) row; the neighbour rows K-1 and
// planes L+-1 that a CTA reads were read by CTAs just before it (blockIdx.x =
// K runs fastest), so they come from L2 and DRAM traffic stays at the
// algorithmic 80 bytes per cell.
#include <cuda_runtime.h>

#include "devplan.h"

namespace chy {

// x / d.  When d is a power of two (inv = 1/d, exact, nonzero) the quotient
// and x * inv are the same exactly rounded number, the exact x * 2^-n, and
// the product costs one instruction instead of a division sequence.
__device__ __forceinline__ double quot(double x, double d, double inv)
{
    return inv != 0.0 ? __dmul_rn(x, inv) : __ddiv_rn(x, d);
}

// BIN: the BINARY build's terms (radhydro/source.f:61-62, 76-77), each added
// after the DELT term of its statement, its product formed left to right.
template <bool BIN>
__global__ void __launch_bounds__(256) k_source(SourceDev a)
{
    const int k = blockIdx.x + 1, l = blockIdx.y;   // 0-based K = 1..KMAX, L
    const int lp = l + 1 == a.L ? 0 : l + 1, lm = l == 0 ? a.L - 1 : l - 1;
    const size_t hp = (size_t)a.J2h * a.K2h, pp = (size_t)a.J2p * a.K2p;
    const size_t h0 = (size_t)a.J2h * k + hp * l;          // hydro row (K, L)
    const size_t p0 = (size_t)a.J2p * k + pp * l;          // potential row (K, L)
    const size_t hk = h0 - a.J2h, pk = p0 - a.J2p;          // rows K-1
    const size_t hlp = (size_t)a.J2h * k + hp * lp, hlm = (size_t)a.J2h * k + hp * lm;
    const size_t plp = (size_t)a.J2p * k + pp * lp, plm = (size_t)a.J2p * k + pp * lm;
    const double two_dr = __dmul_rn(2.0, a.dr), two_dth = __dmul_rn(2.0, a.dtheta);
    const double *__restrict__ rho = a.rho;
    const double *__restrict__ phi = a.phi;
    const double *__restrict__ om = a.omega;
    const double *__restrict__ pr = a.p;
    for (int j = a.j0 + threadIdx.x; j <= a.Jh; j += blockDim.x) {
        // every operand first (J-1 >= 0 at J = JSTART too), so that the loads
        // of the three updates are in flight together
        const double r0 = __ldg(rho + p0 + j), rj = __ldg(rho + p0 + j - 1), rk = __ldg(rho + pk + j);
        const double f0 = __ldg(phi + p0 + j), fj = __ldg(phi + p0 + j - 1), fk = __ldg(phi + pk + j);
        const double fp = __ldg(phi + plp + j), fm = __ldg(phi + plm + j);
        const double q0 = __ldg(pr + h0 + j), qj = __ldg(pr + h0 + j - 1), qk = __ldg(pr + hk + j);
        const double qp = __ldg(pr + hlp + j), qm = __ldg(pr + hlm + j);
        const double o0 = __ldg(om + h0 + j), oj = __ldg(om + h0 + j - 1);
        const double R = __ldg(a.R + j);
        const double s0 = a.S[h0 + j], t0 = a.T[h0 + j], a0 = a.A[h0 + j];
        // S (radhydro/source.f:55-60), J = JSTART+1..JMAX+1
        if (j > a.j0) {
            const double rs = __dadd_rn(r0, rj);
            const double os = __dadd_rn(o0, oj);
            double x1 = __dmul_rn(R, rs);
            x1 = __dmul_rn(x1, __dmul_rn(os, os));
            x1 = __dmul_rn(x1, 0.25);
            x1 = __dmul_rn(x1, 0.5);
            const double x2 = quot(__dmul_rn(rs, __dsub_rn(f0, fj)), two_dr, a.inv_2dr);
            const double x3 = quot(__dsub_rn(q0, qj), a.dr, a.inv_dr);
            double sn = __dadd_rn(s0, __dmul_rn(a.delt, __dsub_rn(__dsub_rn(x1, x2), x3)));
            if constexpr (BIN) {
                // + OMEGABIN*OMEGA(J)*RHF(J)*2*RHO(J)*DELT
                double b = __dmul_rn(a.omega_bin, o0);
                b = __dmul_rn(b, __ldg(a.rhf + j));
                b = __dmul_rn(b, 2.0);
                b = __dmul_rn(b, r0);
                sn = __dadd_rn(sn, __dmul_rn(b, a.delt));
            }
            a.S[h0 + j] = sn;
        }
        // T (radhydro/source.f:67-70)
        const double rz = __dadd_rn(r0, rk);
        const double y1 = quot(__dmul_rn(__dmul_rn(0.5, rz), __dsub_rn(f0, fk)), a.dz, a.inv_dz);
        const double y2 = quot(__dsub_rn(q0, qk), a.dz, a.inv_dz);
        a.T[h0 + j] = __dsub_rn(t0, __dmul_rn(a.delt, __dadd_rn(y1, y2)));
        // A (radhydro/source.f:74-75)
        double z = __dmul_rn(r0, __dsub_rn(fp, fm));
        z = __dsub_rn(__dadd_rn(z, qp), qm);
        double an = __dsub_rn(a0, __ddiv_rn(__dmul_rn(a.delt, z), two_dth));
        if constexpr (BIN) {
            // - RHO(J)*OMEGABIN*(U(J+1)+U(J))*DELT*RHF(J); J+1 <= JMAX+1 is in U
            double b = __dmul_rn(r0, a.omega_bin);
            b = __dmul_rn(b, __dadd_rn(__ldg(a.u + h0 + j + 1), __ldg(a.u + h0 + j)));
            b = __dmul_rn(b, a.delt);
            an = __dsub_rn(an, __dmul_rn(b, __ldg(a.rhf + j)));
        }
        a.A[h0 + j] = an;
    }
}

cudaError_t launch_source(const SourceDev &a, cudaStream_t s)
{
    if (a.Kh < 1 || a.L < 1 || a.j0 > a.Jh) return cudaSuccess;
    if (a.binary)
        k_source<true><<<dim3(a.Kh, a.L), 256, 0, s>>>(a);
    else
        k_source<false><<<dim3(a.Kh, a.L), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace chy

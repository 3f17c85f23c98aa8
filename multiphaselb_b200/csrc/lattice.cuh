// lattice.cuh -- lattice traits, parameter block and node-local physics.
//
// Everything here is __host__ __device__ arithmetic on one node.  The
// expressions keep the reference's evaluation order term by term (C
// left-to-right association, no contraction: the translation units that
// include this header are compiled with -fmad=false) so that the device
// results equal the reference's binary64 results bit for bit.
#pragma once

#include <cmath>

#include <stdint.h>
#include <utility>
#include <type_traits>
#include "../../include/mplb_gpu.h"

#ifndef MPLB_HD
#define MPLB_HD __host__ __device__ __forceinline__
#endif

namespace mplb {

// ----------------------------------------------------------------- lattices
// Velocity sets in the reference's order (D2Q9_Vel.c:20-55, D3Q15_Vel.c) and
// their reverse maps (D2Q9_Reverse.c, D3Q15_Reverse.c).  Components are packed
// two bits each (value+1) and reverse indices four bits each, so both compile
// time (static_for indices) and runtime indices work in device code.
struct D2Q9T {
    static constexpr int lattice = MPLB_D2Q9;
    static constexpr int Q = 9, D = 2, NAX = 4;
    static constexpr uint32_t PX = 133401u, PY = 10341u, PZ = 87381u;
    static constexpr uint64_t PREV = 27253675056ull;
};
struct D3Q15T {
    static constexpr int lattice = MPLB_D3Q15;
    static constexpr int Q = 15, D = 3, NAX = 6;
    static constexpr uint32_t PX = 143168841u, PY = 42112149u, PZ = 2787669u;
    static constexpr uint64_t PREV = 543154130879988000ull;
};

template <class L> MPLB_HD constexpr int cxk(int k) { return (int)((L::PX >> (2 * k)) & 3u) - 1; }
template <class L> MPLB_HD constexpr int cyk(int k) { return (int)((L::PY >> (2 * k)) & 3u) - 1; }
template <class L> MPLB_HD constexpr int czk(int k) { return (int)((L::PZ >> (2 * k)) & 3u) - 1; }
template <class L> MPLB_HD constexpr int ck(int k, int j) { return j == 0 ? cxk<L>(k) : j == 1 ? cyk<L>(k) : czk<L>(k); }
template <class L> MPLB_HD constexpr int revk(int k) { return (int)((L::PREV >> (4 * k)) & 15ull); }
// Axis finite-difference directions (scalarGradient.c:22-23,62-63,108-109,148-149,189-190):
// a = direction whose pull source is x + e_d (c = -e_d), b = the one with c = +e_d.
template <class L> MPLB_HD constexpr int fda(int d) { return L::Q == 9 ? (d == 0 ? 3 : 4) : 2 * d + 2; }
template <class L> MPLB_HD constexpr int fdb(int d) { return L::Q == 9 ? (d == 0 ? 1 : 2) : 2 * d + 1; }

// Moment polynomials of the MRT basis evaluated on a velocity (integers):
// D2Q9 Lallemand-Luo rows (D2Q9_MRT.c:20-108), D3Q15 d'Humieres rows
// (D3Q15_MRT.c).  Used at compile time for M f and on the host for M^-1.
MPLB_HD constexpr int moment(int lat, int r, int cx, int cy, int cz) {
    int c2 = cx * cx + cy * cy + cz * cz;
    if (lat == MPLB_D2Q9) {
        return r == 0 ? 1 : r == 1 ? -4 + 3 * c2 : r == 2 ? (8 - 21 * c2 + 9 * c2 * c2) / 2
             : r == 3 ? cx : r == 4 ? (-5 + 3 * c2) * cx : r == 5 ? cy
             : r == 6 ? (-5 + 3 * c2) * cy : r == 7 ? cx * cx - cy * cy : cx * cy;
    }
    return r == 0 ? 1 : r == 1 ? c2 - 2 : r == 2 ? (15 * c2 * c2 - 55 * c2 + 32) / 2
         : r == 3 ? cx : r == 4 ? (5 * c2 - 13) * cx / 2 : r == 5 ? cy
         : r == 6 ? (5 * c2 - 13) * cy / 2 : r == 7 ? cz : r == 8 ? (5 * c2 - 13) * cz / 2
         : r == 9 ? 3 * cx * cx - c2 : r == 10 ? cy * cy - cz * cz : r == 11 ? cx * cy
         : r == 12 ? cy * cz : r == 13 ? cx * cz : cx * cy * cz;
}

template <class L>
MPLB_HD constexpr int Mint(int r, int k) { return moment(L::lattice, r, cxk<L>(k), cyk<L>(k), czk<L>(k)); }

// ----------------------------------------------------------- parameter block
// Passed by value to every kernel (lives in the kernel-parameter constant
// bank), so several handles on one device never share mutable globals.
struct Params {
    int32_t lat, Q;
    uint32_t n;
    double cs2;
    double w[MPLB_MAX_Q];      // LB weights (D2Q9_omega.c, D3Q15_omega.c)
    double ppw[MPLB_MAX_Q];    // pseudopotential force weights (D2Q9_ppw.c, D3Q15_ppw.c)
    double Mi[MPLB_MAX_Q][MPLB_MAX_Q];  // M^-1, host-computed as M[c][r]/|row c|^2
    // flow field
    int32_t f_model, f_update;
    double Lf[MPLB_MAX_Q];
    double relax_f[MPLB_MAX_Q];  // (1 - 0.5*Lambda[k])            liMRTCollision.c:92
    double s1_den, s2_den;       // ((1/Lambda[1])-0.5), ((1/Lambda[2])-0.5)  liMRTForce.c:35-36
    double sig12, sig6;          // 12*sigma (liMRTForce.c:35), 6.0*sigma (xuMRTForce.c:43)
    double sigma_p;              // sigma of the pressure's gradient term (liMRTPressure.c:246)
    // thermal field
    int32_t g_model, g_update;
    double Lg[MPLB_MAX_Q];
    double corr3, corr5;         // (1 - L3/2)*L4, (1 - L5/2)*L6   liTempMRTCollision.c:75-77
    double lam_fac;              // (1/Lambda[3] - 0.5)           heatSource.c:40,105
    // myMRT thermal model (myMRTCollision.c, myMRTEquilibriumMS.c, heatSource.c:28-90)
    double my_a1, my_a2;         // alpha_1, alpha_2
    double my_qo[3];             // off-diagonal rates Q[3][4], Q[5][6], Q[7][8]   myMRTCollision.c:80-116
    double my_qa0;               // (I - Q/2)[0][0] = 1.0 + (-0.5*Lambda[0])      myMRTCollision.c:125-140
    double my_lgeo, my_ldiv;     // conductivity factor: (4 + 3a1 + 2a2), 6 (D2Q9); (6 + 11a1 + a2), 9 (D3Q15)
    // EOS (EOSInfo.h:80-102)
    int32_t eos;
    double a, b, R, G, M, Cv, rho_0;
    double g[3], fext[3];
    double pr_tc, pr_kappa;      // Peng-Robinson: 0.170151343*a/(b*R), 0.37464+1.5422w-0.26992w^2
    // exact shortcuts, decided on the host: x/G == -x when G == -1,
    // x/Cv == x when Cv == 1, x/(M*M) == x when M*M == 1
    int32_t g_neg1, cv_one, m2_one;
    // surface-tension term of the flow field (liMRT/xuMRT surfaceTension, kappa_st)
    int32_t st_on;
    double kappa_st;
};

// ----------------------------------------------------------- exact division
// Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990; see also
// Muller et al., Handbook of Floating-Point Arithmetic, ch. 5): if yr is the
// correctly rounded reciprocal RN(1/y) and q = RN(x*yr), the remainder
// e = x - q*y is exact in one FMA and RN(q + e*yr) = RN(x/y), for results
// that neither overflow nor underflow.  So several quotients with the same
// divisor cost one reciprocal and three operations each, and are bit-equal to
// IEEE division.  A zero numerator returns q, which keeps the sign of x/y.
MPLB_HD double div_rcp(double x, double y, double yr) {
    const double q = x * yr;
    const double e = fma(-q, y, x);
    return q == 0.0 ? q : fma(e, yr, q);
}
// RN(1/3) for x/3.0.
constexpr double RCP3 = 1.0 / 3.0;
MPLB_HD double div3(double x) { return div_rcp(x, 3.0, RCP3); }

#ifdef __CUDA_ARCH__
__device__ __forceinline__ double rcp_rn(double y) { return __drcp_rn(y); }
#else
inline double rcp_rn(double y) { return 1.0 / y; }
#endif

// ---------------------------------------------------------------------- EOS
// p_eos.c:7-64
MPLB_HD double p_eos(const Params& P, double rho, double T) {
    switch (P.eos) {
    case MPLB_EOS_IDEAL:
        return rho * P.R * T;
    case MPLB_EOS_CS: {
        double al = P.b * rho / 4.0;
        double be = 1 - al;
        return rho * P.R * T * ((1 + al + al * al - al * al * al) / (be * be * be)) - P.a * rho * rho;
    }
    case MPLB_EOS_PR: {
        double be = (1 + P.pr_kappa * (1 - sqrt(T / P.pr_tc)));
        return rho * P.R * T / (1 - P.b * rho) - P.a * be * be * rho * rho / (1 + 2 * P.b * rho - P.b * rho * P.b * rho);
    }
    case MPLB_EOS_VDW:
        return rho * P.R * T / (P.M - rho * P.b) - (P.m2_one ? P.a * rho * rho : P.a * rho * rho / (P.M * P.M));
    default:
        return 0;
    }
}

// potential.c:7-13, given p_EOS(rho, T)
MPLB_HD double potential_p(const Params& P, double rho, double p) {
    const double v = 2 * (p - rho * P.cs2);
    return sqrt(P.g_neg1 ? -v : v / (P.G));
}
MPLB_HD double potential(const Params& P, double rho, double T) { return potential_p(P, rho, p_eos(P, rho, T)); }

// p_eos for several temperatures at one density: the density-only parts are
// evaluated once (each is the same operation on the same operands as in
// p_eos, so the values are identical); quotients whose numerator depends on T
// use one shared reciprocal and div_rcp.
struct EosRho {
    double z;   // CS: (1+al+al^2-al^3)/(be^3)
    double d;   // VdW: M - rho*b; PR: 1 - b*rho
    double dr;  // RN(1/d)
    double d2;  // PR: 1 + 2*b*rho - b*rho*b*rho
    double d2r;
    double att; // VdW: a*rho*rho/(M*M)
};
MPLB_HD EosRho eos_rho(const Params& P, double rho) {
    EosRho e{};
    switch (P.eos) {
    case MPLB_EOS_CS: {
        double al = P.b * rho / 4.0;
        double be = 1 - al;
        e.z = (1 + al + al * al - al * al * al) / (be * be * be);
        break;
    }
    case MPLB_EOS_PR:
        e.d = 1 - P.b * rho;
        e.dr = rcp_rn(e.d);
        e.d2 = 1 + 2 * P.b * rho - P.b * rho * P.b * rho;
        e.d2r = rcp_rn(e.d2);
        break;
    case MPLB_EOS_VDW:
        e.d = P.M - rho * P.b;
        e.dr = rcp_rn(e.d);
        e.att = P.m2_one ? P.a * rho * rho : P.a * rho * rho / (P.M * P.M);
        break;
    default:
        break;
    }
    return e;
}
MPLB_HD double p_eos_at(const Params& P, const EosRho& e, double rho, double T) {
    switch (P.eos) {
    case MPLB_EOS_IDEAL:
        return rho * P.R * T;
    case MPLB_EOS_CS:
        return rho * P.R * T * e.z - P.a * rho * rho;
    case MPLB_EOS_PR: {
        double be = (1 + P.pr_kappa * (1 - sqrt(T / P.pr_tc)));
        return div_rcp(rho * P.R * T, e.d, e.dr) - div_rcp(P.a * be * be * rho * rho, e.d2, e.d2r);
    }
    case MPLB_EOS_VDW:
        return div_rcp(rho * P.R * T, e.d, e.dr) - e.att;
    default:
        return 0;
    }
}

// --------------------------------------------------------------- matvecs
// Compile-time loop: calls f(integral_constant<int, 0..N-1>) in order.
template <class F, int... I>
MPLB_HD void static_for_impl(F& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
MPLB_HD void static_for(F&& f) { static_for_impl(f, std::make_integer_sequence<int, N>{}); }

// matVecMult.c:4-20 evaluates res_i = sum_j M_ij v_j left to right from 0.
// M has integer entries, so each product is exact; terms with a zero
// coefficient are skipped (they add +-0 and leave a finite sum unchanged).
// s + c v for an integer c with |c| a power of two >= 2: c v is exact, so one
// fused multiply-add rounds exactly as the separate multiply and add.
MPLB_HD constexpr bool pow2_ge2(int c) {
    const int a = c < 0 ? -c : c;
    return a >= 2 && (a & (a - 1)) == 0;
}
MPLB_HD double add_exact_product(double s, double c, double v) {
#ifdef __CUDA_ARCH__
    return __fma_rn(c, v, s);
#else
    return std::fma(c, v, s);
#endif
}

template <class L>
MPLB_HD void mul_M(const double* v, double* r) {
    static_for<L::Q>([&](auto i) {
        double s = 0;
        static_for<L::Q>([&](auto j) {
            constexpr int c = Mint<L>(decltype(i)::value, decltype(j)::value);
            if constexpr (c == 1) s = s + v[j];
            else if constexpr (c == -1) s = s - v[j];
            else if constexpr (pow2_ge2(c)) s = add_exact_product(s, (double)c, v[j]);
            else if constexpr (c != 0) s = s + (double)c * v[j];
        });
        r[i] = s;
    });
}

// Squared norm of moment row r (rows of M are orthogonal: M^-1 = M^T D^-1).
template <class L>
MPLB_HD constexpr int row_norm2(int r) {
    int s = 0;
    for (int k = 0; k < L::Q; k++) s += Mint<L>(r, k) * Mint<L>(r, k);
    return s;
}

// M^-1 m.  The reference's M^-1 entries are RN(M[j][i] / |row j|^2)
// (D2Q9_MRTInv.c, D3Q15_MRTInv.c), and every |M[j][i]| is a power of two,
// so each entry is exactly M[j][i] * RN(1/|row j|^2) and each rounded product
// RN(entry * m_j) is exactly M[j][i] * p_j with p_j = RN(RN(1/|row j|^2) * m_j).
// One multiply per column, then the reference's row sums in j order.
template <class L>
MPLB_HD void mul_Mi(const Params& P, const double* v, double* r) {
    (void)P;
    double p[L::Q];
    static_for<L::Q>([&](auto j) {
        constexpr double c = 1.0 / (double)row_norm2<L>(decltype(j)::value);
        p[j] = c * v[j];
    });
    static_for<L::Q>([&](auto i) {
        double s = 0;
        static_for<L::Q>([&](auto j) {
            constexpr int c = Mint<L>(decltype(j)::value, decltype(i)::value);
            if constexpr (c == 1) s = s + p[j];
            else if constexpr (c == -1) s = s - p[j];
            else if constexpr (pow2_ge2(c)) s = add_exact_product(s, (double)c, p[j]);
            else if constexpr (c != 0) s = s + (double)c * p[j];
        });
        r[i] = s;
    });
}

// ------------------------------------------------------------ equilibria
// liMRTEquilibrium.c:3-29 / xuMRTEquilibrium.c:3-29
template <class L>
MPLB_HD double eq_flow_k(const Params& P, int k, double rho, const double* v) {
    double al = 0, be = 0;
    const int c[3] = {cxk<L>(k), cyk<L>(k), czk<L>(k)};
#pragma unroll
    for (int j = 0; j < 3; j++) {
        al += c[j] * v[j];
        be += v[j] * v[j];
    }
    return rho * P.w[k] * (1 + al / P.cs2 + 0.5 * al * al / (P.cs2 * P.cs2) - 0.5 * be / P.cs2);
}

// liTempMRTEquilibrium.c:5-44 (D2Q9): g = M^-1 n_eq(T, U)
MPLB_HD void eq_heat(const Params& P, double T, double u0, double u1, double* g) {
    double n[9];
    n[0] = T;
    n[1] = -2.0 * T;
    n[2] = 2.0 * T;
    n[3] = T * u0;
    n[4] = T * (-u0);
    n[5] = T * u1;
    n[6] = T * (-u1);
    n[7] = 0;
    n[8] = 0;
    mul_Mi<D2Q9T>(P, n, g);
}

// ---------------------------------------------------------- node collisions
// liMRTCollision.c:48-106 with liMRTForce.c:18-42.  f in/out (9 values).
// Surface-tension moments C of an interior node: liMRTSurfaceTension.c:7-150
// (D2Q9, full 2x2 tensor) and xuMRTSurfaceTension.c:7-168 (D3Q15, upper
// triangle).  Q_ij = sum_k ppw_k (psi(x + c_k) - psi(x)) c_ki c_kj -- the
// reference's lattice.weights are the pseudopotential weights
// (setLatticeInfo.c:80) -- then Q *= 0.5 psi G kappa left to right.  With
// c in {-1, 0, 1} the products are exact: zero terms are skipped, the others
// add or subtract alpha.  nbpsi(k) = psi at x + c_k.
template <class L, class PsiAt>
MPLB_HD void surface_tension(const Params& P, double ps, PsiAt nbpsi, double* C) {
    double Q00 = 0, Q01 = 0, Q02 = 0, Q11 = 0, Q12 = 0, Q22 = 0;
    static_for<L::Q - 1>([&](auto km1) {
        constexpr int k = decltype(km1)::value + 1;
        const double al = P.ppw[k] * (nbpsi(k) - ps);
        auto acc = [&](double& q, int c) {
            if (c == 1) q += al;
            else if (c == -1) q -= al;
        };
        acc(Q00, cxk<L>(k) * cxk<L>(k));
        acc(Q01, cxk<L>(k) * cyk<L>(k));
        acc(Q11, cyk<L>(k) * cyk<L>(k));
        if constexpr (L::D == 3) {
            acc(Q02, cxk<L>(k) * czk<L>(k));
            acc(Q12, cyk<L>(k) * czk<L>(k));
            acc(Q22, czk<L>(k) * czk<L>(k));
        }
    });
    const double kap = P.kappa_st;
    Q00 = Q00 * 0.5 * ps * P.G * kap;
    Q01 = Q01 * 0.5 * ps * P.G * kap;
    Q11 = Q11 * 0.5 * ps * P.G * kap;
#pragma unroll
    for (int k = 0; k < L::Q; k++) C[k] = 0;
    if constexpr (L::D == 2) {
        C[1] = 1.5 * P.Lf[1] * (Q00 + Q11);
        C[2] = -1.5 * P.Lf[2] * (Q00 + Q11);
        C[7] = -P.Lf[8] * (Q00 - Q11);
        C[8] = -P.Lf[8] * Q01;
    } else {
        Q02 = Q02 * 0.5 * ps * P.G * kap;
        Q12 = Q12 * 0.5 * ps * P.G * kap;
        Q22 = Q22 * 0.5 * ps * P.G * kap;
        C[1] = 4.0 * P.Lf[1] * (Q00 + Q11 + Q22) / 5.0;
        C[9] = -P.Lf[10] * (2 * Q00 - Q11 - Q22);
        C[10] = -P.Lf[10] * (Q11 - Q22);
        C[11] = -P.Lf[10] * Q01;
        C[12] = -P.Lf[10] * Q12;
        C[13] = -P.Lf[10] * Q02;
    }
}

// C (may be NULL) is the surface-tension term, added to every moment after
// the relaxation (liMRTCollision.c:90-98).
MPLB_HD void collide_limrt_psi(const Params& P, double* f, double rho, const double* U,
                               const double* F, const double* Fi, double ps, const double* C = nullptr) {
    double um = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) um += U[k] * U[k];
    double meq[9], m[9], S[9];
    meq[0] = rho;
    meq[1] = rho * (-2 + 3 * um);
    meq[2] = rho * (1 - 3 * um);
    meq[3] = rho * U[0];
    meq[4] = rho * (-U[0]);
    meq[5] = rho * U[1];
    meq[6] = rho * (-U[1]);
    meq[7] = rho * (U[0] * U[0] - U[1] * U[1]);
    meq[8] = rho * U[0] * U[1];
    mul_M<D2Q9T>(f, m);
    double uf = U[0] * F[0] + U[1] * F[1];
    double fi2 = Fi[0] * Fi[0] + Fi[1] * Fi[1];
    S[0] = 0;
    S[1] = 6 * uf + P.sig12 * fi2 / (ps * ps * P.s1_den);
    S[2] = -6 * uf - P.sig12 * fi2 / (ps * ps * P.s2_den);
    S[3] = F[0];
    S[4] = -F[0];
    S[5] = F[1];
    S[6] = -F[1];
    S[7] = 2 * (U[0] * F[0] - U[1] * F[1]);
    S[8] = U[0] * F[1] + U[1] * F[0];
#pragma unroll
    for (int k = 0; k < 9; k++) m[k] = m[k] - P.Lf[k] * (m[k] - meq[k]) + P.relax_f[k] * S[k];
    if (C) {
#pragma unroll
        for (int k = 0; k < 9; k++) m[k] = m[k] + C[k];
    }
    mul_Mi<D2Q9T>(P, m, f);
}
MPLB_HD void collide_limrt(const Params& P, double* f, double rho, const double* U, const double* F,
                           const double* Fi, double T) {
    collide_limrt_psi(P, f, rho, U, F, Fi, potential(P, rho, T));
}

// xuMRTCollision.c:46-89, xuMRTEquilibriumMS.c:12-51, xuMRTForce.c:14-69.
// F here is Fi + (rho - rho_0) g (no fext), xuMRTForce.c:18-22.
MPLB_HD void collide_xumrt_psi(const Params& P, double* f, double rho, const double* U,
                               const double* Fi, double ps, const double* C = nullptr) {
    double um = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) um += U[k] * U[k];
    double meq[15], m[15], S[15], F[3];
    meq[0] = rho;
    meq[1] = rho * (-1.0 + um);
    meq[2] = rho * (1.0 - 5.0 * um);
    meq[3] = rho * U[0];
    meq[4] = div3(rho * -7.0 * U[0]);
    meq[5] = rho * U[1];
    meq[6] = div3(rho * -7.0 * U[1]);
    meq[7] = rho * U[2];
    meq[8] = div3(rho * -7.0 * U[2]);
    meq[9] = rho * (2.0 * U[0] * U[0] - U[1] * U[1] - U[2] * U[2]);
    meq[10] = rho * (U[1] * U[1] - U[2] * U[2]);
    meq[11] = rho * U[0] * U[1];
    meq[12] = rho * U[1] * U[2];
    meq[13] = rho * U[0] * U[2];
    meq[14] = 0;
    mul_M<D3Q15T>(f, m);
#pragma unroll
    for (int j = 0; j < 3; j++) F[j] = Fi[j] + (rho - P.rho_0) * P.g[j];
    double uf = U[0] * F[0] + U[1] * F[1] + U[2] * F[2];
    double f2 = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) f2 += F[k] * F[k];
    S[0] = 0;
    S[1] = 2.0 * uf + (P.sig6 * f2) / (ps * ps * P.s1_den);
    S[2] = -10.0 * uf;
    S[3] = F[0];
    S[4] = div3(-7.0 * F[0]);
    S[5] = F[1];
    S[6] = div3(-7.0 * F[1]);
    S[7] = F[2];
    S[8] = div3(-7.0 * F[2]);
    S[9] = 4.0 * U[0] * F[0] - 2.0 * U[1] * F[1] - 2.0 * U[2] * F[2];
    S[10] = 2.0 * U[1] * F[1] - 2.0 * U[2] * F[2];
    S[11] = U[0] * F[1] + U[1] * F[0];
    S[12] = U[1] * F[2] + U[2] * F[1];
    S[13] = U[0] * F[2] + U[2] * F[0];
    S[14] = 0;
#pragma unroll
    for (int k = 0; k < 15; k++) m[k] = m[k] - P.Lf[k] * (m[k] - meq[k]) + P.relax_f[k] * S[k];
    if (C) {
#pragma unroll
        for (int k = 0; k < 15; k++) m[k] = m[k] + C[k];
    }
    mul_Mi<D3Q15T>(P, m, f);
}
MPLB_HD void collide_xumrt(const Params& P, double* f, double rho, const double* U, const double* Fi, double T) {
    collide_xumrt_psi(P, f, rho, U, Fi, potential(P, rho, T));
}

// liTempMRTCollision.c:38-84, liTempMRTEquilibriumMS.c:20-38, liTempMRTSource.c:17-24.
MPLB_HD void collide_litemp(const Params& P, double* g, double T, double u0, double u1, double src) {
    double neq[9], n[9];
    neq[0] = T;
    neq[1] = -2.0 * T;
    neq[2] = 2.0 * T;
    neq[3] = T * u0;
    neq[4] = T * (-u0);
    neq[5] = T * u1;
    neq[6] = T * (-u1);
    neq[7] = 0;
    neq[8] = 0;
    mul_M<D2Q9T>(g, n);
    double n4 = n[4], n6 = n[6];
    n[0] = n[0] - P.Lg[0] * (n[0] - neq[0]) + src;
#pragma unroll
    for (int k = 1; k < 9; k++) n[k] = n[k] - P.Lg[k] * (n[k] - neq[k]) + 0.0;
    n[3] = n[3] + P.corr3 * n4;
    n[5] = n[5] + P.corr5 * n6;
    mul_Mi<D2Q9T>(P, n, g);
}

// ------------------------------------------------------------ myMRT (thermal)
// Moments of the equilibrium, myMRTEquilibriumMS.c:17-75 (= myMRTEquilibrium.c:
// 10-88): T, alpha_1 T, alpha_2 T, +-T u_d, zeros.  T*(-u) and -(T*u) (the
// D3Q15 form) are the same double.
template <class L>
MPLB_HD void neq_mymrt(const Params& P, double T, const double* u, double* ne) {
    ne[0] = T;
    ne[1] = P.my_a1 * T;
    ne[2] = P.my_a2 * T;
    ne[3] = T * u[0];
    ne[4] = T * (-u[0]);
    ne[5] = T * u[1];
    ne[6] = T * (-u[1]);
    if constexpr (L::Q == 15) {
        ne[7] = T * u[2];
        ne[8] = T * (-u[2]);
#pragma unroll
        for (int k = 9; k < 15; k++) ne[k] = 0;
    } else {
        ne[7] = 0;
        ne[8] = 0;
    }
}

// myMRTEquilibrium.c: g = M^-1 n_eq.
template <class L>
MPLB_HD void eq_mymrt(const Params& P, double T, const double* u, double* g) {
    double ne[L::Q];
    neq_mymrt<L>(P, T, u, ne);
    mul_Mi<L>(P, ne, g);
}

// myMRTCollision.c:150-210: n = M g; n <- n - Q (n - n_eq) + (I - Q/2) Gamma,
// Q diagonal (Lambda) plus the pairs (3,4), (5,6) [, (7,8)], Gamma =
// (scalarSource, 0, ...) (myMRTSource.c:17-25), both products as the sparse
// row sums of sparseMatVecMult.c:4-28.  Rows k >= 1 of (I - Q/2) Gamma are
// +-0, and n - Q (n - n_eq) is never -0 (M g sums start from +0), so those
// additions leave it unchanged and are not made.
template <class L>
MPLB_HD void collide_mymrt(const Params& P, double* g, double T, const double* u, double src) {
    double ne[L::Q], n[L::Q], a[L::Q];
    neq_mymrt<L>(P, T, u, ne);
    mul_M<L>(g, n);
#pragma unroll
    for (int k = 0; k < L::Q; k++) a[k] = P.Lg[k] * (n[k] - ne[k]);
    a[3] = a[3] + P.my_qo[0] * (n[4] - ne[4]);
    a[5] = a[5] + P.my_qo[1] * (n[6] - ne[6]);
    if constexpr (L::Q == 15) a[7] = a[7] + P.my_qo[2] * (n[8] - ne[8]);
    n[0] = n[0] - a[0] + P.my_qa0 * src;
#pragma unroll
    for (int k = 1; k < L::Q; k++) n[k] = n[k] - a[k];
    mul_Mi<L>(P, n, g);
}

// heatSource.c:28-90 (myMRT): the liTempMRT source without the time
// extrapolation, conductivity rho Cv (1/L3 - 1/2) (geo) / div.
MPLB_HD double heat_source_value_my(const Params& P, double rho, double T, double dot, double divU) {
    double lambda = rho * P.Cv * P.lam_fac * P.my_lgeo / P.my_ldiv;
    double dpdT = p_eos(P, rho, 1.1 * T) - p_eos(P, rho, 0.9 * T);
    dpdT = dpdT / (0.2 * T);
    return -lambda * dot / P.Cv + divU * T * (1.0 - dpdT / (rho * P.Cv));
}

// heatSource.c:144-165: source from gradients (dot), divergence, rho, T_old.
MPLB_HD double heat_source_value(const Params& P, double rho, double T, double dot, double divU,
                                 double oldss) {
    double lambda = rho * P.Cv * P.lam_fac;
    double dpdT = p_eos(P, rho, 1.1 * T) - p_eos(P, rho, 0.9 * T);
    dpdT = dpdT / (0.2 * T);
    double s = -lambda * dot / P.Cv + divU * T * (1.0 - dpdT / (rho * P.Cv));
    return s + 0.5 * (s - oldss);
}
// Same value, with the density's EOS parts er and rr = RN(1/rho) shared.
MPLB_HD double heat_source_value_er(const Params& P, const EosRho& er, double rho, double rr, double T,
                                    double dot, double divU, double oldss) {
    double lambda = rho * P.Cv * P.lam_fac;
    double dpdT = p_eos_at(P, er, rho, 1.1 * T) - p_eos_at(P, er, rho, 0.9 * T);
    dpdT = dpdT / (0.2 * T);
    double a = P.cv_one ? -lambda * dot : -lambda * dot / P.Cv;
    double b = P.cv_one ? div_rcp(dpdT, rho, rr) : dpdT / (rho * P.Cv);
    double s = a + divU * T * (1.0 - b);
    return s + 0.5 * (s - oldss);
}

// ------------------------------------------------------- dependent launch
// Fused step kernels are launched with programmatic stream serialization: a
// step's grid may be scheduled while the previous step drains.  Only kernels
// whose inputs come through plain (non-restrict) pointers and __ldg take part:
// a load through a const __restrict__ parameter may be compiled as an
// invariant load, which the compiler is free to move above the wait.  Every kernel waits
// for the previous grid to complete (and its writes to be visible) before it
// reads anything, then lets the next step's grid be scheduled.  Launched
// without the attribute, the wait returns at once.
__device__ __forceinline__ void step_dependency_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// A fused-step launch with programmatic stream serialization (the kernels
// start with step_dependency_wait).  Launch errors surface through
// cudaGetLastError, which every caller checks.
template <class... KArgs, class... Args>
void launch_step(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                 Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace mplb

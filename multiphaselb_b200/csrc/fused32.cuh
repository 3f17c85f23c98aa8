// fused32.cuh -- FP32-deviation form of the fused box kernels.
//
// Populations are stored in FP32 as deviations from the rest state,
//   f~_k = f_k - w_k * rho_ref,   g~_k = g_k - wg_k * T_ref,
// (w: LB weights; wg = M^-1 (1, -2, 2, 0, ..., 0), the liTempMRT rest state)
// and collided in FP32 in moment space.  The equilibria are written in terms
// of d_rho = rho - rho_ref and d_T = T - T_ref (M w rho_ref = rho_ref (1,-2,1,0..)
// for D2Q9 and rho_ref (1,-1,1,0..) for D3Q15), so no large rest-state moment
// is subtracted in FP32.  The density and temperature sums, the equation of
// state and psi, the interaction force, the heat source, and the carried T,
// U, S stay FP64.  Bounce-back and fixedT act on deviations exactly: the rest
// terms cancel (w_k = w_rev(k); fixedT's difference of two equilibria).
//
// This translation unit is compiled with multiply-add contraction on: it is
// not a bitwise path; its error against the FP64 path is measured.
#pragma once

#include "fused.cuh"

namespace mplb {

struct FusedArgs32 {
    int nx, ny, nz, px, py, pz, tiles_x, tiles_y, zchunk;
    uint32_t n;  // nodes of this lattice (array stride)
    const float* fin;
    float* fout;
    const float* gin;
    float* gout;
    const double* Told;
    double* Tnew;
    const double* Uold;
    double* Unew;
    double* S;
    const double* rho_c;
    double rho_ref, T_ref;
    float wf[MPLB_MAX_Q];  // w_k
    float wg[9];           // M^-1 (1, -2, 2, 0, ...)
    // FP32 copies of the collision constants
    float Lf[MPLB_MAX_Q], relax_f[MPLB_MAX_Q], Lg[9];
    float s1_den, s2_den, sig12, sig6, corr3, corr5;
    const uint8_t* bcmap;
    int bc_margin;  // FusedArgs::bc_margin
    double Twall[MPLB_MAX_PATCHES];
    BCProg prog[FUSED_MAX_PROGS];
};

template <class L>
__device__ __forceinline__ void mul_M32(const float* v, float* r) {
    static_for<L::Q>([&](auto i) {
        float s = 0.f;
        static_for<L::Q>([&](auto j) {
            constexpr int c = Mint<L>(decltype(i)::value, decltype(j)::value);
            if constexpr (c == 1) s += v[j];
            else if constexpr (c == -1) s -= v[j];
            else if constexpr (c != 0) s += (float)c * v[j];
        });
        r[i] = s;
    });
}

template <class L>
__device__ __forceinline__ void mul_Mi32(const float* v, float* r) {
    float p[L::Q];
    static_for<L::Q>([&](auto j) {
        constexpr float c = (float)(1.0 / (double)row_norm2<L>(decltype(j)::value));
        p[j] = c * v[j];
    });
    static_for<L::Q>([&](auto i) {
        float s = 0.f;
        static_for<L::Q>([&](auto j) {
            constexpr int c = Mint<L>(decltype(j)::value, decltype(i)::value);
            if constexpr (c == 1) s += p[j];
            else if constexpr (c == -1) s -= p[j];
            else if constexpr (c != 0) s += (float)c * p[j];
        });
        r[i] = s;
    });
}

// First direction with every component non-zero (the smallest lattice weight).
template <class L>
constexpr int first_diagonal() {
    for (int k = 0; k < L::Q; k++) {
        int c2 = cxk<L>(k) * cxk<L>(k) + cyk<L>(k) * cyk<L>(k) + czk<L>(k) * czk<L>(k);
        if (c2 == L::D) return k;
    }
    return L::Q - 1;
}

// Exact bookkeeping of the conserved moments for the FP32 collision.  In
// exact arithmetic the collision keeps the node's mass and adds the force to
// its momentum.  In FP32 it conserves rounded moments (FP32 sums of the
// inputs), and rounding in M^-1 m and in the stores adds more; at a steady
// state those errors repeat every step at every node, so the lattice mass
// drifts (measured: +2.7e-10 per node and step on a 128^2 CS bubble) and the
// momentum wanders, which moves the interface and holds max |drho/dt| near
// 1e-9 instead of letting it decay.  Here the stored outputs are corrected so
// that their exact sums (FP64 sums of FP32 values: exact) equal the targets:
//   momentum, axis by axis: half the residual onto the population along +e_d,
//     half off the one along -e_d (mass unchanged);
//   mass: the residual onto the rest population (momentum unchanged), what
//     it cannot represent split evenly over an opposite diagonal pair.
// What remains is a fraction of an ulp of the populations involved, of
// either sign.  (Putting the mass residual into two populations that do not
// cancel in momentum drives a spurious flow: tried, unstable.)
template <class L>
constexpr int axis_population(int d) {
    for (int k = 1; k < L::Q; k++)
        if (ck<L>(k, d) == 1 && cxk<L>(k) * cxk<L>(k) + cyk<L>(k) * cyk<L>(k) + czk<L>(k) * czk<L>(k) == 1)
            return k;
    return 0;
}

template <class L>
__device__ __forceinline__ void restore_conserved(float* f, double mass, const double* mom) {
    static_for<L::D>([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        double j = 0.0;
        static_for<L::Q>([&](auto kk) {
            constexpr int c = ck<L>(decltype(kk)::value, d);
            if constexpr (c == 1) j += (double)f[kk];
            else if constexpr (c == -1) j -= (double)f[kk];
        });
        const double half = 0.5 * (mom[d] - j);
        constexpr int a = axis_population<L>(d), b = revk<L>(a);
        f[a] = (float)((double)f[a] + half);
        f[b] = (float)((double)f[b] - half);
    });
    double post = 0.0;
#pragma unroll
    for (int k = 0; k < L::Q; k++) post += (double)f[k];
    const double v = (double)f[0] + (mass - post);
    f[0] = (float)v;
    const double half = 0.5 * (v - (double)f[0]);
    constexpr int a = first_diagonal<L>(), b = revk<L>(a);
    f[a] = (float)((double)f[a] + half);
    f[b] = (float)((double)f[b] + half);
}

// Total momentum of a periodic lattice without net body force is conserved
// exactly by the model; FP32 rounding (below an ulp per node and step, but
// not of zero mean at a steady state) lets it drift, and the drift carries
// the bubble along (|drho/dt| = |grad rho| v at the interface).  Equilibrium
// runs of the FP32 form therefore reset the total momentum to its value at
// the start of the run at every convergence check.  The total is kept in
// fixed point (resolution 2^-40): each node's exact FP64 momentum is rounded
// to a multiple of 2^-40 and the integers are summed, so the result does not
// depend on summation order or tiling.
constexpr double MOM_SCALE = 1099511627776.0;  // 2^40

template <class L>
__device__ __forceinline__ void node_momentum_fx(const float* __restrict__ f, uint32_t n, uint32_t id,
                                                 long long* m) {
    static_for<L::D>([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        double j = 0.0;
        static_for<L::Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            constexpr int c = ck<L>(k, d);
            if constexpr (c == 1) j += (double)f[(size_t)k * n + id];
            else if constexpr (c == -1) j -= (double)f[(size_t)k * n + id];
        });
        m[d] = __double2ll_rn(j * MOM_SCALE);
    });
}

// Warp sum (exact: integers) and one atomic per warp.
__device__ __forceinline__ void warp_add_ll(long long v, long long* out) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(reinterpret_cast<unsigned long long*>(out), (unsigned long long)v);
}

// Remove a lattice's momentum excess J - J0 at the nodes id = 0, s, 2s, ...:
// at each, half of its share off the population along +e_d and half onto
// the one along -e_d (mass unchanged but for the two roundings).  Spread
// over all n nodes, the share of a small excess lies far below the FP32
// resolution of the populations and every correction rounds away (a 256^2
// lattice whose excess grows by 2e-6 per thousand steps would get 1.5e-11
// per population against an ulp near 4e-9, and its bubble drifts).  So the
// stride s is chosen for shares of at least MOM_FIX_MIN, a few ulps of the
// largest axis-population deviations; s = 1 (every node) for large excesses.
// What rounding still leaves is measured and removed at the next check.
constexpr double MOM_FIX_MIN = 2e-8;

template <class L>
__device__ __forceinline__ uint32_t momentum_fix_stride(uint32_t n, const long long* J, const long long* J0) {
    double mx = 0.0;
#pragma unroll
    for (int d = 0; d < L::D; d++) mx = fmax(mx, fabs((double)(J[d] - J0[d])) / MOM_SCALE);
    if (mx == 0.0) return n;
    const double s = ceil(MOM_FIX_MIN * (double)n / (0.5 * mx));
    return s <= 1.0 ? 1u : (s >= (double)n ? n : (uint32_t)s);
}

template <class L>
__device__ __forceinline__ void momentum_fix_node(float* __restrict__ f, uint32_t n, uint32_t id,
                                                  const long long* J, const long long* J0) {
    const uint32_t s = momentum_fix_stride<L>(n, J, J0);
    if (id % s != 0) return;
    const double count = (double)((n + s - 1) / s);
    static_for<L::D>([&](auto dd) {
        constexpr int d = decltype(dd)::value;
        const double half = 0.5 * ((double)(J[d] - J0[d]) / MOM_SCALE / count);
        constexpr int a = axis_population<L>(d), b = revk<L>(a);
        f[(size_t)a * n + id] = (float)((double)f[(size_t)a * n + id] - half);
        f[(size_t)b * n + id] = (float)((double)f[(size_t)b * n + id] + half);
    });
}

// liMRT collision on deviations (liMRTCollision.c / liMRTForce.c in FP32).
__device__ __forceinline__ void collide_limrt32(const FusedArgs32& A, float* f, double rho, float dr, const float* U,
                                                const float* F, const float* Fi, double psi) {
    const float r = (float)rho;
    const float um = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    float meq[9], m[9], S[9];
    meq[0] = dr;
    meq[1] = -2.f * dr + 3.f * r * um;
    meq[2] = dr - 3.f * r * um;
    meq[3] = r * U[0];
    meq[4] = -r * U[0];
    meq[5] = r * U[1];
    meq[6] = -r * U[1];
    meq[7] = r * (U[0] * U[0] - U[1] * U[1]);
    meq[8] = r * U[0] * U[1];
    mul_M32<D2Q9T>(f, m);
    const float ps2 = (float)(psi * psi);
    const float uf = U[0] * F[0] + U[1] * F[1];
    const float fi2 = Fi[0] * Fi[0] + Fi[1] * Fi[1];
    S[0] = 0.f;
    S[1] = 6.f * uf + A.sig12 * fi2 / (ps2 * A.s1_den);
    S[2] = -6.f * uf - A.sig12 * fi2 / (ps2 * A.s2_den);
    S[3] = F[0];
    S[4] = -F[0];
    S[5] = F[1];
    S[6] = -F[1];
    S[7] = 2.f * (U[0] * F[0] - U[1] * F[1]);
    S[8] = U[0] * F[1] + U[1] * F[0];
#pragma unroll
    for (int k = 0; k < 9; k++) m[k] = m[k] - A.Lf[k] * (m[k] - meq[k]) + A.relax_f[k] * S[k];
    mul_Mi32<D2Q9T>(m, f);
}

// xuMRT collision on deviations.
__device__ __forceinline__ void collide_xumrt32(const FusedArgs32& A, float* f, double rho, float dr, const float* U,
                                                const float* F, double psi) {
    const float r = (float)rho;
    const float um = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    constexpr float S73 = 7.f / 3.f;
    float meq[15], m[15], S[15];
    meq[0] = dr;
    meq[1] = -dr + r * um;
    meq[2] = dr - 5.f * r * um;
    meq[3] = r * U[0];
    meq[4] = -S73 * r * U[0];
    meq[5] = r * U[1];
    meq[6] = -S73 * r * U[1];
    meq[7] = r * U[2];
    meq[8] = -S73 * r * U[2];
    meq[9] = r * (2.f * U[0] * U[0] - U[1] * U[1] - U[2] * U[2]);
    meq[10] = r * (U[1] * U[1] - U[2] * U[2]);
    meq[11] = r * U[0] * U[1];
    meq[12] = r * U[1] * U[2];
    meq[13] = r * U[0] * U[2];
    meq[14] = 0.f;
    mul_M32<D3Q15T>(f, m);
    const float uf = U[0] * F[0] + U[1] * F[1] + U[2] * F[2];
    const float f2 = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
    S[0] = 0.f;
    S[1] = 2.f * uf + A.sig6 * f2 / ((float)(psi * psi) * A.s1_den);
    S[2] = -10.f * uf;
    S[3] = F[0];
    S[4] = -S73 * F[0];
    S[5] = F[1];
    S[6] = -S73 * F[1];
    S[7] = F[2];
    S[8] = -S73 * F[2];
    S[9] = 4.f * U[0] * F[0] - 2.f * U[1] * F[1] - 2.f * U[2] * F[2];
    S[10] = 2.f * U[1] * F[1] - 2.f * U[2] * F[2];
    S[11] = U[0] * F[1] + U[1] * F[0];
    S[12] = U[1] * F[2] + U[2] * F[1];
    S[13] = U[0] * F[2] + U[2] * F[0];
    S[14] = 0.f;
#pragma unroll
    for (int k = 0; k < 15; k++) m[k] = m[k] - A.Lf[k] * (m[k] - meq[k]) + A.relax_f[k] * S[k];
    mul_Mi32<D3Q15T>(m, f);
}

// liTempMRT collision on deviations.
__device__ __forceinline__ void collide_litemp32(const FusedArgs32& A, float* g, double T, float dT, float u0, float u1,
                                                 float src) {
    const float t = (float)T;
    float neq[9], n[9];
    neq[0] = dT;
    neq[1] = -2.f * dT;
    neq[2] = 2.f * dT;
    neq[3] = t * u0;
    neq[4] = -t * u0;
    neq[5] = t * u1;
    neq[6] = -t * u1;
    neq[7] = 0.f;
    neq[8] = 0.f;
    mul_M32<D2Q9T>(g, n);
    const float n4 = n[4], n6 = n[6];
#pragma unroll
    for (int k = 0; k < 9; k++) n[k] = n[k] - A.Lg[k] * (n[k] - neq[k]);
    n[0] += src;
    n[3] += A.corr3 * n4;
    n[5] += A.corr5 * n6;
    mul_Mi32<D2Q9T>(n, g);
}

// Pull one node's deviations, apply its boundary program, return FP64 moments.
template <class L, bool F_ON, bool G_ON, bool HAS_BC>
__device__ __forceinline__ void pull_node32(const Params& P, const FusedArgs32& A, int x, int y, int z, uint32_t id,
                                            float* f, float* g, double& rho, double& T, float& dr, float& dT) {
    const uint32_t n = A.n;
    FusedArgs G{};
    G.nx = A.nx; G.ny = A.ny; G.nz = A.nz; G.px = A.px; G.py = A.py; G.pz = A.pz;
    const NodeOffsets no = node_offsets(G, x, y, L::D == 3 ? z : 0, L::D);
    uint32_t miss = 0;
    static_for<L::Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        bool m;
        const uint32_t src = source_of(no, id, cxk<L>(k), cyk<L>(k), czk<L>(k), m);
        if constexpr (F_ON) f[k] = __ldg(A.fin + (size_t)k * n + src);
        if constexpr (G_ON) g[k] = __ldg(A.gin + (size_t)k * n + src);
        miss |= (uint32_t)m << k;
    });
    if constexpr (HAS_BC) {
        const uint8_t pi = A.bcmap[id];
        if (pi) {
            const BCProg& pr = A.prog[pi];
            auto bounce = [&](float* v) {
#pragma unroll
                for (int k = 0; k < L::Q; k++) {
                    const int r = revk<L>(k);
                    if ((miss >> k) & 1u) v[k] = v[r];
                    else if (!((miss >> r) & 1u) && k >= 1 && k <= L::NAX) {
                        v[k] = 0.5f * v[k] + 0.5f * v[r];
                        v[r] = v[k];
                    }
                }
            };
            if constexpr (F_ON)
                for (int o = 0; o < pr.nf; o++) bounce(f);
            if constexpr (G_ON) {
                for (int o = 0; o < pr.ng; o++) {
                    if (pr.gt[o] == MPLB_BC_BOUNCEBACK) {
                        bounce(g);
                    } else {
                        const double Tw = A.Twall[pr.gp[o]];
#pragma unroll
                        for (int k = 0; k < L::Q; k++) {
                            if (!((miss >> k) & 1u)) continue;
                            int mx = wrap1(x + cxk<L>(k), A.nx, A.px);
                            int my = wrap1(y + cyk<L>(k), A.ny, A.py);
                            if (mx < 0 || my < 0) continue;
                            const uint32_t m = (uint32_t)mx + (uint32_t)A.nx * (uint32_t)my;
                            const double u0 = A.Uold[m], u1 = A.Uold[n + m];
                            const double diff = eq_heat_k(P, k, Tw, u0, u1) - eq_heat_k(P, k, A.Told[m], u0, u1);
                            g[k] = (float)diff + A.gin[(size_t)k * n + id];
                        }
                    }
                }
            }
        }
    }
    if constexpr (F_ON) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += f[k];
        dr = s;
        rho = A.rho_ref + (double)s;
    } else {
        rho = A.rho_c[id];
        dr = (float)(rho - A.rho_ref);
    }
    if constexpr (G_ON) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += g[k];
        dT = s;
        T = A.T_ref + (double)s;
    } else {
        T = A.Told[id];
        dT = (float)(T - A.T_ref);
    }
}

// pull_node32 for a node of an inner tile (no wrap, no missing source, no
// boundary program).
template <class L, bool F_ON, bool G_ON>
__device__ __forceinline__ void pull_node32_inner(const Params& P, const FusedArgs32& A, uint32_t id, float* f,
                                                  float* g, double& rho, double& T, float& dr, float& dT) {
    (void)P;
    const uint32_t n = A.n;
    const int nx = A.nx, nxy = A.nx * A.ny;
    static_for<L::Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        const uint32_t src = (uint32_t)((int)id - cxk<L>(k) - cyk<L>(k) * nx - czk<L>(k) * nxy);
        if constexpr (F_ON) f[k] = __ldg(A.fin + (size_t)k * n + src);
        if constexpr (G_ON) g[k] = __ldg(A.gin + (size_t)k * n + src);
    });
    if constexpr (F_ON) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += f[k];
        dr = s;
        rho = A.rho_ref + (double)s;
    } else {
        rho = A.rho_c[id];
        dr = (float)(rho - A.rho_ref);
    }
    if constexpr (G_ON) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += g[k];
        dT = s;
        T = A.T_ref + (double)s;
    } else {
        T = A.Told[id];
        dT = (float)(T - A.T_ref);
    }
}

// L2 prefetch of what pull_node32 and the heat source load for node (x, y).
template <class L, bool F_ON, bool G_ON>
__device__ __forceinline__ void prefetch_node32(const FusedArgs32& A, int x, int y, uint32_t id) {
    const uint32_t n = A.n;
    FusedArgs G{};
    G.nx = A.nx; G.ny = A.ny; G.nz = 1; G.px = A.px; G.py = A.py; G.pz = 1;
    const NodeOffsets no = node_offsets(G, x, y, 0, L::D);
    static_for<L::Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        bool m;
        const uint32_t src = source_of(no, id, cxk<L>(k), cyk<L>(k), czk<L>(k), m);
        if constexpr (F_ON) prefetch_l2(A.fin + (size_t)k * n + src);
        if constexpr (G_ON) prefetch_l2(A.gin + (size_t)k * n + src);
    });
    if constexpr (G_ON) {
        prefetch_l2(A.Told + id);
        prefetch_l2(A.Uold + id);
        prefetch_l2(A.Uold + n + id);
        prefetch_l2(A.S + id);
    }
}

// After the macros: force (FP64), heat source (FP64, computed by the caller),
// velocity, then FP32 collisions; or (EMIT) the FP64 reference state.
template <class L, bool F_ON, bool G_ON, bool EMIT, class PsiAt>
__device__ __forceinline__ void finish_node32(const Params& P, const FusedArgs32& A, uint32_t id, bool onb, float* f,
                                              float* g, double rho, float dr, double T, float dT, double psi,
                                              PsiAt nbpsi, double heat, double* emit_f, double* emit_g,
                                              double* rho_out, double* Fi_out, double* Ft_out) {
    const uint32_t n = A.n;
    double Fi[3] = {0, 0, 0}, Ft[3], Ud[3];
    if constexpr (F_ON) {
        if (!onb) {
            double F[3] = {0.0, 0.0, 0.0};
            static_for<L::Q - 1>([&](auto km1) {
                constexpr int k = decltype(km1)::value + 1;
                const double al = P.ppw[k] * nbpsi(k);
                static_for<3>([&](auto i) {
                    constexpr int c = ck<L>(k, decltype(i)::value);
                    if constexpr (c == 1) F[i] += al;
                    else if constexpr (c == -1) F[i] -= al;
                });
            });
            const double be = -P.G * psi;
#pragma unroll
            for (int i = 0; i < 3; i++) Fi[i] = F[i] * be;
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double t = Fi[j] + (rho - P.rho_0) * P.g[j];
            if (!onb) t += P.fext[j];
            Ft[j] = t;
        }
        // sum_k c_k f_k == sum_k c_k f~_k (sum_k c_k w_k = 0)
        static_for<3>([&](auto jj) {
            constexpr int j = decltype(jj)::value;
            float lv = 0.f;
            static_for<L::Q>([&](auto kk) {
                constexpr int c = ck<L>(decltype(kk)::value, j);
                if constexpr (c == 1) lv += f[kk];
                else if constexpr (c == -1) lv -= f[kk];
            });
            const double Fj = L::Q == 9 ? Ft[j] : Fi[j] + (rho - P.rho_0) * P.g[j];
            Ud[j] = ((double)lv + Fj * 0.5) / rho;
        });
    } else {
#pragma unroll
        for (int j = 0; j < 3; j++) Ud[j] = A.Uold[(size_t)j * n + id];
    }
    if constexpr (EMIT) {
        if constexpr (F_ON) {
#pragma unroll
            for (int k = 0; k < L::Q; k++) emit_f[(size_t)k * n + id] = (double)f[k] + (double)A.wf[k] * A.rho_ref;
            rho_out[id] = rho;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                Fi_out[(size_t)j * n + id] = Fi[j];
                Ft_out[(size_t)j * n + id] = Ft[j];
                A.Unew[(size_t)j * n + id] = Ud[j];
            }
        }
        if constexpr (G_ON) {
#pragma unroll
            for (int k = 0; k < 9; k++) emit_g[(size_t)k * n + id] = (double)g[k] + (double)A.wg[k] * A.T_ref;
            A.Tnew[id] = T;
        }
        return;
    }
    const float U[3] = {(float)Ud[0], (float)Ud[1], (float)Ud[2]};
    if constexpr (F_ON) {
        // conserved moments the collision must produce: the input mass, and
        // the input momentum plus the force the collision applies
        double mass = 0.0, mom[3] = {0.0, 0.0, 0.0};
        static_for<L::Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            mass += (double)f[k];
            static_for<L::D>([&](auto dd) {
                constexpr int c = ck<L>(k, decltype(dd)::value);
                if constexpr (c == 1) mom[dd] += (double)f[k];
                else if constexpr (c == -1) mom[dd] -= (double)f[k];
            });
        });
        if constexpr (L::Q == 9) {
            const float F[3] = {(float)Ft[0], (float)Ft[1], (float)Ft[2]};
            const float Fv[3] = {(float)Fi[0], (float)Fi[1], (float)Fi[2]};
            collide_limrt32(A, f, rho, dr, U, F, Fv, psi);
#pragma unroll
            for (int j = 0; j < 3; j++) mom[j] += Ft[j];
        } else {
            double Fx[3];
#pragma unroll
            for (int j = 0; j < 3; j++) Fx[j] = Fi[j] + (rho - P.rho_0) * P.g[j];
            const float F[3] = {(float)Fx[0], (float)Fx[1], (float)Fx[2]};
            collide_xumrt32(A, f, rho, dr, U, F, psi);
#pragma unroll
            for (int j = 0; j < 3; j++) mom[j] += Fx[j];
        }
        restore_conserved<L>(f, mass, mom);
#pragma unroll
        for (int k = 0; k < L::Q; k++) A.fout[(size_t)k * n + id] = f[k];
        if constexpr (G_ON) {
            A.Unew[id] = Ud[0];
            A.Unew[n + id] = Ud[1];
        }
    }
    if constexpr (G_ON) {
        collide_litemp32(A, g, T, dT, U[0], U[1], (float)heat);
#pragma unroll
        for (int k = 0; k < 9; k++) A.gout[(size_t)k * n + id] = g[k];
        A.Tnew[id] = T;
        A.S[id] = heat;
    }
}

}  // namespace mplb

// fused.cuh -- one kernel per time step on structured boxes.
//
// The reference advances a step with eleven passes over the lattice
// (multiPhasePP.c:163-240).  On a box mesh the whole step is one kernel that
// reads each population once and writes it once:
//
//   step n:  pull-stream f*_n, g*_n  ->  f''_n, g''_n         (lbstream.c)
//            boundary programs at wall nodes                   (bounceBack.c, fixedT.c)
//            rho_n = sum f'', T_n = sum g''                    (macroDensity/Temperature)
//            psi_n, 1/rho_n on the tile + a one-node ring      (potential.c)
//            heat source S_n from rho_n, T_{n-1}, U_{n-1}      (heatSource.c)
//            Fi_n, Ft_n, U_n                                   (interForce.c, liMRTVelocity.c)
//            collide -> f*_{n+1}, g*_{n+1}                     (liMRTCollision.c, ...)
//
// so the state carried between kernels is the post-collision populations
// (double-buffered), T and U (double-buffered: neighbours read the previous
// step's values) and S.  The reference's own state after step n (f''_n,
// rho_n, Fi_n, Ft_n) is rebuilt on demand by the same kernel in EMIT mode from
// the retained input buffer of the last step.
//
// Arithmetic per node is the shared code of lattice.cuh, so results equal
// the operator path (and the reference) bit for bit.
#pragma once

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ops.cuh"

namespace mplb {

constexpr int FUSED_MAX_PROGS = 64;
constexpr int FUSED_MAX_OPS = 3;

// Boundary operations of one node, per field, in patch order.
struct BCProg {
    uint8_t nf, ng;
    uint8_t ft[FUSED_MAX_OPS], gt[FUSED_MAX_OPS];  // MPLB_BC_BOUNCEBACK or MPLB_BC_FIXEDT
    uint8_t gp[FUSED_MAX_OPS];                      // patch index of a fixedT op
};

// Slabs on the fused path (mplb_gpu_add_mirror): the step outputs of owned
// nodes [lo, lo + cnt) are also stored into nodes [dst, dst + cnt) of a
// neighbouring slab's next-step input buffers (its halo); f / g / T / U are
// that slab's arrays (stride n_dst per component), NULL when not mirrored.
struct MirrorRange {
    uint32_t lo, cnt, dst, n_dst;
    double* f;
    double* g;
    double* T;
    double* U;
};
constexpr int MPLB_MAX_MIRRORS = 2;

struct FusedArgs {
    int nx, ny, nz;
    int px, py, pz;     // 1 = periodic axis
    int tiles_x, tiles_y, zchunk;
    const double* fin;
    double* fout;
    const double* gin;
    double* gout;
    const double* Told;  // T of the previous step (the only T when g is frozen)
    double* Tnew;
    const double* Uold;  // U of the previous step (the only U when f is frozen)
    double* Unew;
    double* S;
    const double* rho_c;  // density when f is frozen
    double* rho_out;      // EMIT outputs
    double* Fi_out;
    double* Ft_out;
    const uint8_t* bcmap;  // per node: 0 = no boundary op, else index into prog
    int bc_margin;         // largest distance of a node with a boundary op from its nearest face, -1 = none
    int* kerr;             // kernel-side error flag (a bounded wait that ran out), read by the host
    double* rho_a;         // myMRT thermal field: rho_n and sum g''_n of every node (k_pullsum_d2q9)
    double* gsum_a;
    uint32_t own_lo, own_cnt;  // a step stores the outputs of nodes [own_lo, own_lo + own_cnt) only
    int nmirror;               // slabs: mirrored ranges in mirror[0 .. nmirror)
    MirrorRange mirror[MPLB_MAX_MIRRORS];
    double Twall[MPLB_MAX_PATCHES];
    BCProg prog[FUSED_MAX_PROGS];
};

// ------------------------------------------------------------- geometry
// Wrap a coordinate one step outside [0, ext): periodic -> wrapped,
// walled -> -1 (absent).  Inputs are within [-1, ext].
MPLB_HD int wrap1(int c, int ext, int periodic) {
    if (c < 0) return periodic ? c + ext : -1;
    if (c >= ext) return periodic ? c - ext : -1;
    return c;
}

// Node held by ext-grid slot e (0..T+1) of a tile starting at t0 along an
// axis: -1 when absent.  Only slots within one node of the box are ever read,
// so slots further out are absent too.
MPLB_HD int slot_coord(int t0, int e, int ext, int periodic) {
    const int c = t0 - 1 + e;
    return c <= ext ? wrap1(c, ext, periodic) : -1;
}

// Ring slot r (0..2*(TX+2)+2*TY-1) of a TX x TY tile -> ext coordinates.
MPLB_HD void ring_slot(int r, int TX, int TY, int& ex, int& ey) {
    const int EX = TX + 2;
    if (r < EX) { ex = r; ey = 0; }
    else if (r < 2 * EX) { ex = r - EX; ey = TY + 1; }
    else if (r < 2 * EX + TY) { ex = 0; ey = r - 2 * EX + 1; }
    else { ex = EX - 1; ey = r - 2 * EX - TY + 1; }
}

// Pull source of population (cx, cy, cz) at node (x, y, z); -1 if missing.
MPLB_HD int64_t pull_src(int nx, int ny, int nz, int px, int py, int pz, int x, int y, int z, int cx, int cy,
                         int cz) {
    int sx = wrap1(x - cx, nx, px), sy = wrap1(y - cy, ny, py), sz = wrap1(z - cz, nz, pz);
    if (sx < 0 || sy < 0 || sz < 0) return -1;
    return (int64_t)sx + (int64_t)nx * ((int64_t)sy + (int64_t)ny * (int64_t)sz);
}

// Offsets from a node to its axis neighbours (wrapped on periodic axes) and
// which of them lie beyond a walled face.  Computed once per node; the pull
// source of population k (x - c_k) is then one offset per non-zero component.
struct NodeOffsets {
    int xm, xp, ym, yp, zm, zp;  // index offsets to the sources at x-1, x+1, y-1, ...
    bool mxm, mxp, mym, myp, mzm, mzp;  // that source is missing
};
MPLB_HD NodeOffsets node_offsets(const FusedArgs& A, int x, int y, int z, int D) {
    NodeOffsets o;
    const int nxy = A.nx * A.ny;
    const bool xlo = x == 0, xhi = x == A.nx - 1, ylo = y == 0, yhi = y == A.ny - 1;
    const bool zlo = D == 3 && z == 0, zhi = D == 3 && z == A.nz - 1;
    o.xm = xlo ? A.nx - 1 : -1;
    o.xp = xhi ? 1 - A.nx : 1;
    o.ym = ylo ? (A.ny - 1) * A.nx : -A.nx;
    o.yp = yhi ? (1 - A.ny) * A.nx : A.nx;
    o.zm = zlo ? (A.nz - 1) * nxy : -nxy;
    o.zp = zhi ? (1 - A.nz) * nxy : nxy;
    o.mxm = xlo && !A.px;
    o.mxp = xhi && !A.px;
    o.mym = ylo && !A.py;
    o.myp = yhi && !A.py;
    o.mzm = zlo && !A.pz;
    o.mzp = zhi && !A.pz;
    return o;
}
// Pull source of the population with velocity (cx, cy, cz) at node id: the
// node id itself when the source is missing (lbstream.c:36-42 keeps the value).
MPLB_HD uint32_t source_of(const NodeOffsets& o, uint32_t id, int cx, int cy, int cz, bool& missing) {
    int off = 0;
    bool m = false;
    if (cx == 1) { off += o.xm; m |= o.mxm; }
    if (cx == -1) { off += o.xp; m |= o.mxp; }
    if (cy == 1) { off += o.ym; m |= o.mym; }
    if (cy == -1) { off += o.yp; m |= o.myp; }
    if (cz == 1) { off += o.zm; m |= o.mzm; }
    if (cz == -1) { off += o.zp; m |= o.mzp; }
    missing = m;
    return m ? id : (uint32_t)((int)id + off);
}

// Node on a walled face: it has a missing neighbour (readLatticeMesh.c:171-203).
MPLB_HD bool on_wall(const FusedArgs& A, int x, int y, int z) {
    return (!A.px && (x == 0 || x == A.nx - 1)) || (!A.py && (y == 0 || y == A.ny - 1)) ||
           (!A.pz && (z == 0 || z == A.nz - 1));
}

// bounceBack.c:21-70 on registers, k ascending, in place.
template <class L>
__device__ __forceinline__ void bounce_back(uint32_t miss, double* v) {
#pragma unroll
    for (int k = 0; k < L::Q; k++) {
        const int r = revk<L>(k);
        if ((miss >> k) & 1u) {
            v[k] = v[r];
        } else if (!((miss >> r) & 1u) && k >= 1 && k <= L::NAX) {
            v[k] = 0.5 * v[k] + 0.5 * v[r];
            v[r] = v[k];
        }
    }
}

// The flow field's boundary program of node id (bounce-back ops in patch order).
template <class L>
__device__ __forceinline__ void apply_flow_program(const FusedArgs& A, uint32_t id, uint32_t miss, double* f) {
    const BCProg& pr = A.prog[A.bcmap[id]];
    for (int o = 0; o < pr.nf; o++) bounce_back<L>(miss, f);
}

// Prefetch into L2 what pull_node and the heat source will load for node
// (x, y): the pulled populations, and T, U, S of the node.  Issued at kernel
// start so these misses overlap the ring work instead of following it.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
template <class L, bool F_ON, bool G_ON>
__device__ __forceinline__ void prefetch_node(const Params& P, const FusedArgs& A, int x, int y, uint32_t id) {
    const uint32_t n = P.n;
    const NodeOffsets no = node_offsets(A, x, y, 0, L::D);
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

// ------------------------------------------------------------ phase A
// Pull-stream one node, apply its boundary program, sum moments.
// f, g receive f''_n, g''_n; miss bit k = population k has no source.
template <class L, bool F_ON, bool G_ON, bool HAS_BC>
__device__ __forceinline__ void pull_node(const Params& P, const FusedArgs& A, int x, int y, int z,
                                          uint32_t id, double* f, double* g, double& rho, double& T) {
    const uint32_t n = P.n;
    const NodeOffsets no = node_offsets(A, x, y, L::D == 3 ? z : 0, L::D);
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
        uint8_t pi = A.bcmap[id];
        if (pi) {
            const BCProg& pr = A.prog[pi];
            auto bounce = [&](double* v) { bounce_back<L>(miss, v); };
            if constexpr (F_ON)
                for (int o = 0; o < pr.nf; o++) bounce(f);
            if constexpr (G_ON) {
                for (int o = 0; o < pr.ng; o++) {
                    if (pr.gt[o] == MPLB_BC_BOUNCEBACK) {
                        bounce(g);
                    } else {
                        // fixedT.c:119-200.  The neighbour nbid = x + c_k; its
                        // post-stream population k came from this node: g*_n(x)[k].
                        const double Tw = A.Twall[pr.gp[o]];
#pragma unroll
                        for (int k = 0; k < L::Q; k++) {
                            if (!((miss >> k) & 1u)) continue;
                            int mx = wrap1(x + cxk<L>(k), A.nx, A.px);
                            int my = wrap1(y + cyk<L>(k), A.ny, A.py);
                            if (mx < 0 || my < 0) continue;
                            uint32_t m = (uint32_t)mx + (uint32_t)A.nx * (uint32_t)my;
                            double u0 = A.Uold[m], u1 = A.Uold[n + m];
                            double eq_nb, eq_bnd;
                            if (P.g_model == MPLB_MYMRT) {
                                const double u[3] = {u0, u1, A.Uold[2 * (size_t)n + m]};
                                eq_nb = eq_my_k<L>(P, k, A.Told[m], u);
                                eq_bnd = eq_my_k<L>(P, k, Tw, u);
                            } else {
                                eq_nb = eq_heat_k(P, k, A.Told[m], u0, u1);
                                eq_bnd = eq_heat_k(P, k, Tw, u0, u1);
                            }
                            g[k] = eq_bnd + (A.gin[(size_t)k * n + id] - eq_nb);
                        }
                    }
                }
            }
        }
    }
    if constexpr (F_ON) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += f[k];
        rho = s;
    } else {
        rho = A.rho_c[id];
    }
    if constexpr (G_ON) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += g[k];
        T = s;
    } else {
        T = A.Told[id];
    }
}

// ------------------------------------------------------------ phase B
// Interaction force, total force and velocity of one node from its
// post-stream populations f, density rho (rr = RN(1/rho)) and psi
// (nbpsi(k) = psi_n at x + c_k).
template <class L, class PsiAt>
__device__ __forceinline__ void force_velocity(const Params& P, bool onb, const double* f, double rho, double rr,
                                               double psi, PsiAt nbpsi, double* Fi, double* Ft, double* U) {
    Fi[0] = Fi[1] = Fi[2] = 0;
    // interactionForce.c:47-79 (zero force on boundary nodes)
    if (!onb) {
        double F[3] = {0.0, 0.0, 0.0};
        static_for<L::Q - 1>([&](auto km1) {
            constexpr int k = decltype(km1)::value + 1;
            double al = P.ppw[k] * nbpsi(k);
            static_for<3>([&](auto i) {
                constexpr int c = ck<L>(k, decltype(i)::value);
                if constexpr (c == 1) F[i] = F[i] + al;
                else if constexpr (c == -1) F[i] = F[i] - al;
            });
        });
        double be = -P.G * psi;
#pragma unroll
        for (int i = 0; i < 3; i++) Fi[i] = F[i] * be;
    }
    // interForce.c:27-39
#pragma unroll
    for (int j = 0; j < 3; j++) {
        double t = Fi[j] + (rho - P.rho_0) * P.g[j];
        if (!onb) t += P.fext[j];
        Ft[j] = t;
    }
    // liMRTVelocity.c:27-44 (F = Ft) / xuMRTVelocity.c:19-44 (F = Fi + (rho - rho_0) g).
    // Zero velocity components contribute +-0 and are skipped.
    static_for<3>([&](auto jj) {
        constexpr int j = decltype(jj)::value;
        double lv = 0;
        static_for<L::Q>([&](auto kk) {
            constexpr int c = ck<L>(decltype(kk)::value, j);
            if constexpr (c == 1) lv = lv + f[kk];
            else if constexpr (c == -1) lv = lv - f[kk];
        });
        double Fj = L::Q == 9 ? Ft[j] : Fi[j] + (rho - P.rho_0) * P.g[j];
        U[j] = div_rcp(lv + Fj * 0.5, rho, rr);  // == (lv + Fj*0.5)/rho
    });
}

// Everything after the macros for one node that owns an output.
// nbpsi(k) returns psi_n at x + c_k.
template <class L, bool F_ON, bool G_ON, bool EMIT, class PsiAt, bool MY = false>
__device__ __forceinline__ void finish_node(const Params& P, const FusedArgs& A, uint32_t id, bool onb,
                                            double* f, double* g, double rho, double rr, double T, double psi,
                                            PsiAt nbpsi, double src_heat) {
    const uint32_t n = P.n;
    // slabs: a halo node's step outputs are stored by the neighbour that owns it
    if constexpr (!EMIT)
        if (id - A.own_lo >= A.own_cnt) return;
    double Fi[3] = {0, 0, 0}, Ft[3], U[3];
    if constexpr (F_ON) {
        force_velocity<L>(P, onb, f, rho, rr, psi, nbpsi, Fi, Ft, U);
    } else {
#pragma unroll
        for (int j = 0; j < 3; j++) U[j] = A.Uold[(size_t)j * n + id];
    }
    if constexpr (EMIT) {
        if constexpr (F_ON) {
#pragma unroll
            for (int k = 0; k < L::Q; k++) A.fout[(size_t)k * n + id] = f[k];
            A.rho_out[id] = rho;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                A.Fi_out[(size_t)j * n + id] = Fi[j];
                A.Ft_out[(size_t)j * n + id] = Ft[j];
                A.Unew[(size_t)j * n + id] = U[j];
            }
        }
        if constexpr (G_ON) {
#pragma unroll
            for (int k = 0; k < L::Q; k++) A.gout[(size_t)k * n + id] = g[k];
        }
        return;
    }
    if constexpr (F_ON) {
        // surface-tension term (zero on wall nodes, which miss a neighbour)
        double C[L::Q];
        const double* Cp = nullptr;
        if (P.st_on) {
            if (!onb) {
                surface_tension<L>(P, psi, nbpsi, C);
            } else {
#pragma unroll
                for (int k = 0; k < L::Q; k++) C[k] = 0;
            }
            Cp = C;
        }
        if constexpr (L::Q == 9) collide_limrt_psi(P, f, rho, U, Ft, Fi, psi, Cp);
        else collide_xumrt_psi(P, f, rho, U, Fi, psi, Cp);
#pragma unroll
        for (int k = 0; k < L::Q; k++) A.fout[(size_t)k * n + id] = f[k];
        if constexpr (G_ON) {
            // only the heat source and fixedT read U of the previous step
            A.Unew[id] = U[0];
            A.Unew[n + id] = U[1];
        }
    }
    if constexpr (G_ON) {
        if constexpr (MY) collide_mymrt<L>(P, g, T, U, src_heat);
        else collide_litemp(P, g, T, U[0], U[1], src_heat);
#pragma unroll
        for (int k = 0; k < 9; k++) A.gout[(size_t)k * n + id] = g[k];
        A.Tnew[id] = T;
        A.S[id] = src_heat;
    }
    // slabs: the same outputs into a neighbour's halo (the input of its next step)
    for (int m = 0; m < A.nmirror; m++) {
        const MirrorRange& M = A.mirror[m];
        if (id - M.lo >= M.cnt) continue;
        const size_t d = (size_t)M.dst + (id - M.lo), nd = M.n_dst;
        if constexpr (F_ON) {
#pragma unroll
            for (int k = 0; k < L::Q; k++) M.f[(size_t)k * nd + d] = f[k];
            if constexpr (G_ON) {
                M.U[d] = U[0];
                M.U[nd + d] = U[1];
            }
        }
        if constexpr (G_ON) {
#pragma unroll
            for (int k = 0; k < 9; k++) M.g[(size_t)k * nd + d] = g[k];
            M.T[d] = T;
        }
    }
}

// ------------------------------------------------------------ 2D kernel
// Tile of TX x TY nodes, one thread each, plus the one-node ring around it
// (psi, 1/rho, T_{n-1}, U_{n-1}) computed by the first threads.
constexpr int min_blocks(int threads) { return threads <= 128 ? 4 : (threads <= 256 ? 2 : 1); }

// Pull-stream one node of an inner tile (no wrap, no missing source, no
// boundary program): the arithmetic of pull_node without its bookkeeping.
template <class L, bool F_ON, bool G_ON>
__device__ __forceinline__ void pull_node_inner(const Params& P, const FusedArgs& A, uint32_t id, double* f,
                                                double* g, double& rho, double& T) {
    const uint32_t n = P.n;
    const int nx = A.nx;
    static_for<L::Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        const uint32_t src = (uint32_t)((int)id - cxk<L>(k) - cyk<L>(k) * nx);
        if constexpr (F_ON) f[k] = __ldg(A.fin + (size_t)k * n + src);
        if constexpr (G_ON) g[k] = __ldg(A.gin + (size_t)k * n + src);
    });
    if constexpr (F_ON) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += f[k];
        rho = s;
    } else {
        rho = A.rho_c[id];
    }
    if constexpr (G_ON) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < L::Q; k++) s += g[k];
        T = s;
    } else {
        T = A.Told[id];
    }
}

// Is the tile at (x0, y0), with its ring and the ring's pull sources, inside
// the box (nothing wraps, nothing is missing) and free of boundary programs?
// Such a tile takes the INNER body.  Every node with a program lies within
// bc_margin of a face, so a ring farther in than that holds none; the test
// is arithmetic only (uniform over the block, no load before the work).
template <int TX, int TY>
__device__ __forceinline__ bool inner_tile(const FusedArgs& A, int x0, int y0) {
    const int m = A.bc_margin > 0 ? A.bc_margin : 0;
    return x0 - 1 > m && x0 + TX < A.nx - 1 - m && y0 - 1 > m && y0 + TY < A.ny - 1 - m;
}

// myMRT heat source of node (x, y) from the arrays of k_pullsum_d2q9
// (heatSource.c:28-90): gradients of T_{n-1} and 1/rho_n, divergence of
// U_{n-1}, one-sided at a missing axis neighbour, as the operator kernel.
template <bool INNER>
__device__ __forceinline__ double heat_my(const Params& P, const FusedArgs& A, int x, int y, uint32_t id) {
    const uint32_t n = P.n;
    double gT[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, div = 0;
    const double Ti = A.Told[id], ri = A.rho_a[id];
#pragma unroll
    for (int d = 0; d < 2; d++) {
        int xa = x, ya = y, xb = x, yb = y;
        if (d == 0) {
            xa = INNER ? x + 1 : wrap1(x + 1, A.nx, A.px);
            xb = INNER ? x - 1 : wrap1(x - 1, A.nx, A.px);
        } else {
            ya = INNER ? y + 1 : wrap1(y + 1, A.ny, A.py);
            yb = INNER ? y - 1 : wrap1(y - 1, A.ny, A.py);
        }
        const bool pa = xa >= 0 && ya >= 0, pb = xb >= 0 && yb >= 0;
        const uint32_t ia = pa ? (uint32_t)xa + (uint32_t)A.nx * (uint32_t)ya : id;
        const uint32_t ib = pb ? (uint32_t)xb + (uint32_t)A.nx * (uint32_t)yb : id;
        const FD t = fd_pair(pa ? 0 : -1, pb ? 0 : -1, A.Told[ia], A.Told[ib], Ti);
        const FD r = fd_pair(pa ? 0 : -1, pb ? 0 : -1, 1.0 / A.rho_a[ia], 1.0 / A.rho_a[ib], 1.0 / ri);
        const FD u = fd_pair(pa ? 0 : -1, pb ? 0 : -1, A.Uold[(size_t)d * n + ia], A.Uold[(size_t)d * n + ib],
                             A.Uold[(size_t)d * n + id]);
        gT[d] = t.v;
        gR[d] = r.v;
        if (u.present) div += u.v;
    }
    double dot = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) dot += gT[k] * gR[k];
    return heat_source_value_my(P, ri, Ti, dot, div);
}

// myMRT steps: rho_n and sum g''_n of every node (pull, boundary program,
// sums), so the fused kernel can take the heat source, T_n = sum g'' + S/2
// and psi of its ring from them (the heat source of a ring node needs rho_n
// one node further out).
template <bool F_ON, bool HAS_BC>
__global__ void __launch_bounds__(256) k_pullsum_d2q9(Params P, FusedArgs A) {
    step_dependency_wait();
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= P.n) return;
    const int x = (int)(id % (uint32_t)A.nx), y = (int)(id / (uint32_t)A.nx);
    double f[9], g[9], rho, T;
    pull_node<D2Q9T, F_ON, true, HAS_BC>(P, A, x, y, 0, id, f, g, rho, T);
    A.rho_a[id] = rho;
    A.gsum_a[id] = T;
}

// The tile: TX x TY nodes, one thread each, plus the one-node ring around it
// (psi, 1/rho, T_{n-1}, U_{n-1}) computed by the first threads.  INNER
// tiles skip the wrap / missing-source / boundary bookkeeping; the
// arithmetic is the same code either way.
template <int F2_TX, int F2_TY, bool F_ON, bool G_ON, bool HAS_BC, bool EMIT, bool INNER, int EX, int EY, int GX,
          int GY, bool MY = false, int RINGW = 0>
__device__ __forceinline__ void fused2_tile(const Params& P, const FusedArgs& A, int x0, int y0,
                                            double (*s_psi)[EX], double (*s_inv)[GX], double (*s_To)[GX],
                                            double (*s_U0)[GX], double (*s_U1)[GX]) {
    using L = D2Q9T;
    constexpr int NRING = 2 * EX + 2 * F2_TY;
    const uint32_t n = P.n;
    const int tx = threadIdx.x % F2_TX, ty = threadIdx.x / F2_TX;

    // one ext-grid slot: pull, moments, psi; shared-memory record.  The own
    // slot keeps RN(1/rho) and the density's EOS parts for phase B.
    double s_own = 0;  // myMRT: heat source of the own node
    auto slot = [&](int ex, int ey, double* f, double* g, double& rho, double& T, uint32_t& id, bool mine,
                    double& rr, EosRho& er) -> bool {
        int x, y;
        if constexpr (INNER) {
            x = x0 - 1 + ex;
            y = y0 - 1 + ey;
        } else {
            x = slot_coord(x0, ex, A.nx, A.px);
            y = slot_coord(y0, ey, A.ny, A.py);
            if (x < 0 || y < 0) return false;
        }
        id = (uint32_t)x + (uint32_t)A.nx * (uint32_t)y;
        if constexpr (MY && !EMIT) {
            // myMRT step: a ring node's rho_n, sum g'' come from k_pullsum_d2q9
            if (!mine) {
                rho = A.rho_a[id];
                T = A.gsum_a[id] + 0.5 * heat_my<INNER>(P, A, x, y, id);
                if constexpr (F_ON) s_psi[ey][ex] = potential(P, rho, T);
                return true;
            }
        }
        if constexpr (INNER) pull_node_inner<L, F_ON, G_ON>(P, A, id, f, g, rho, T);
        else pull_node<L, F_ON, G_ON, HAS_BC>(P, A, x, y, 0, id, f, g, rho, T);
        if constexpr (MY) {
            // myMRTTemperature.c:22-31: T_n = sum g'' + S_n / 2
            if constexpr (EMIT) {
                T = T + 0.5 * A.S[id];
            } else {
                s_own = heat_my<INNER>(P, A, x, y, id);
                T = T + 0.5 * s_own;
            }
        }
        if (mine) {
            rr = rcp_rn(rho);
            er = eos_rho(P, rho);
            if constexpr (F_ON) s_psi[ey][ex] = potential_p(P, rho, p_eos_at(P, er, rho, T));
            if constexpr (G_ON) s_inv[ey][ex] = rr;
        } else {
            if constexpr (F_ON) s_psi[ey][ex] = potential(P, rho, T);
            if constexpr (G_ON) s_inv[ey][ex] = 1.0 / rho;
        }
        if constexpr (G_ON) {
            s_To[ey][ex] = A.Told[id];
            s_U0[ey][ex] = A.Uold[id];
            s_U1[ey][ex] = A.Uold[n + id];
        }
        return true;
    };

    // RINGW > 0: the block has RINGW more warps after its TX x TY node
    // threads, one thread per ring slot, so every thread fills one slot
    // before the barrier (a node thread: its own node) through one copy of
    // the slot code; RINGW == 0: the node threads fill the ring first.
    constexpr int NT = F2_TX * F2_TY;
    static_assert(RINGW == 0 || NRING <= 32 * RINGW, "one ring slot per ring thread");
    const bool ringer = RINGW > 0 && (int)threadIdx.x >= NT;
    if (RINGW == 0) {
        // the own node's loads start now; the ring work below overlaps them
        // (with ring warps the node threads load their pulls at once)
        const int px = x0 + tx, py = y0 + ty;
        if (px < A.nx && py < A.ny)
            prefetch_node<L, F_ON, G_ON>(P, A, px, py, (uint32_t)px + (uint32_t)A.nx * (uint32_t)py);
    }
    if constexpr (RINGW == 0) {
        // the ring first, so the own node's populations are live only across the barrier
        for (int r = threadIdx.x; r < NRING; r += blockDim.x) {
            int ex, ey;
            ring_slot(r, F2_TX, F2_TY, ex, ey);
            double rf[9], rg[9], rrho, rt, rrr;
            EosRho rer;
            uint32_t rid;
            slot(ex, ey, rf, rg, rrho, rt, rid, false, rrr, rer);
        }
    }
    double f[9], g[9], rho = 0, T = 0, rr = 0;
    EosRho er{};
    uint32_t id = 0;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool own = !ringer && (INNER || (gx < A.nx && gy < A.ny));
    // interior slot (threads outside the box still fill the slot of the
    // wrapped node, so partial tiles see their periodic neighbours); a ring
    // thread's slot is its ring slot
    int sx = tx + 1, sy = ty + 1;
    bool act = true;
    if (ringer) {
        const int r = (int)threadIdx.x - NT;
        act = r < NRING;
        if (act) ring_slot(r, F2_TX, F2_TY, sx, sy);
    }
    const bool have = act && slot(sx, sy, f, g, rho, T, id, own, rr, er);
    __syncthreads();
    if (!own || !have) return;

    const int ex = tx + 1, ey = ty + 1;
    const bool onb = INNER ? false : on_wall(A, gx, gy, 0);
    double heat = 0;
    if constexpr (MY && !EMIT) heat = s_own;
    if constexpr (G_ON && !EMIT && !MY) {
        // heatSource.c:119-165 with the one-sided differences of finiteDifference/*.c
        double gT[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, div = 0;
        const double To = s_To[ey][ex], iv = s_inv[ey][ex];
        // x: a = x+1, b = x-1
        {
            bool a = INNER || wrap1(gx + 1, A.nx, A.px) >= 0, b = INNER || wrap1(gx - 1, A.nx, A.px) >= 0;
            FD t = fd_pair(a ? 0 : -1, b ? 0 : -1, s_To[ey][ex + 1], s_To[ey][ex - 1], To);
            FD r = fd_pair(a ? 0 : -1, b ? 0 : -1, s_inv[ey][ex + 1], s_inv[ey][ex - 1], iv);
            FD u = fd_pair(a ? 0 : -1, b ? 0 : -1, s_U0[ey][ex + 1], s_U0[ey][ex - 1], s_U0[ey][ex]);
            gT[0] = t.v;
            gR[0] = r.v;
            if (u.present) div += u.v;
        }
        {
            bool a = INNER || wrap1(gy + 1, A.ny, A.py) >= 0, b = INNER || wrap1(gy - 1, A.ny, A.py) >= 0;
            FD t = fd_pair(a ? 0 : -1, b ? 0 : -1, s_To[ey + 1][ex], s_To[ey - 1][ex], To);
            FD r = fd_pair(a ? 0 : -1, b ? 0 : -1, s_inv[ey + 1][ex], s_inv[ey - 1][ex], iv);
            FD u = fd_pair(a ? 0 : -1, b ? 0 : -1, s_U1[ey + 1][ex], s_U1[ey - 1][ex], s_U1[ey][ex]);
            gT[1] = t.v;
            gR[1] = r.v;
            if (u.present) div += u.v;
        }
        double dot = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) dot += gT[k] * gR[k];
        heat = heat_source_value_er(P, er, rho, rr, To, dot, div, A.S[id]);
    }
    double psi = 0;
    if constexpr (F_ON) psi = s_psi[ey][ex];
    auto nbpsi = [&](int k) { return s_psi[ey + cyk<L>(k)][ex + cxk<L>(k)]; };
    finish_node<L, F_ON, G_ON, EMIT, decltype(nbpsi), MY>(P, A, id, onb, f, g, rho, rr, T, psi, nbpsi, heat);
}

// MINB: resident blocks per SM asked of the register allocator (0 = the
// default of min_blocks); a higher value trades registers for warps.
// TRY_INNER: the kernel also carries the INNER body for tiles away from the
// faces; without it the kernel holds the general body alone (a smaller
// instruction footprint, which a lattice of one wave notices).
// MY: the thermal field is myMRT (T = sum g'' + S/2; non-EMIT steps follow
// k_pullsum_d2q9).
// RINGW: warps added to the block that compute the tile's ring (launch with
// TX * TY + 32 * RINGW threads); 0: the node threads compute it first.
template <int F2_TX, int F2_TY, int MINB, bool F_ON, bool G_ON, bool HAS_BC, bool EMIT, bool TRY_INNER = false,
          bool MY = false, int RINGW = 0>
__global__ void __launch_bounds__(F2_TX * F2_TY + 32 * RINGW, MINB ? MINB : min_blocks(F2_TX * F2_TY))
    k_fused_d2q9(Params P, FusedArgs A) {
    step_dependency_wait();
    constexpr int EX = F2_TX + 2, EY = F2_TY + 2;
    constexpr int GY = G_ON ? EY : 1, GX = G_ON ? EX : 1;
    __shared__ double s_psi[EY][EX];
    __shared__ double s_inv[GY][GX];
    __shared__ double s_To[GY][GX];
    __shared__ double s_U0[GY][GX];
    __shared__ double s_U1[GY][GX];
    const int bx = blockIdx.x % A.tiles_x, by = blockIdx.x / A.tiles_x;
    const int x0 = bx * F2_TX, y0 = by * F2_TY;
    if constexpr (TRY_INNER) {
        if (inner_tile<F2_TX, F2_TY>(A, x0, y0)) {
            fused2_tile<F2_TX, F2_TY, F_ON, G_ON, HAS_BC, EMIT, true, EX, EY, GX, GY, MY, RINGW>(
                P, A, x0, y0, s_psi, s_inv, s_To, s_U0, s_U1);
            return;
        }
    }
    fused2_tile<F2_TX, F2_TY, F_ON, G_ON, HAS_BC, EMIT, false, EX, EY, GX, GY, MY, RINGW>(P, A, x0, y0, s_psi, s_inv,
                                                                                          s_To, s_U0, s_U1);
}

// ------------------------------------------------------------ 3D kernels
// xy tile of TX x TY columns marching along z over a chunk of planes.
// Shared memory: a three-plane ring buffer of psi (tile + one-node ring) and
// the pulled populations of the current and next plane (k-major, thread
// fastest: conflict-free), so only a few scalars stay in registers across
// the plane barriers.  Isothermal: liTempMRT is D2Q9 only, so T is read,
// never written.
template <int TX, int TY, bool PIPE>
constexpr size_t f3_smem() {
    return (size_t)(3 * (TY + 2) * (TX + 2) + (PIPE ? 3 : 2) * 15 * TX * TY) * sizeof(double);
}

template <int F3_TX, int F3_TY, bool HAS_BC, bool EMIT>
__global__ void __launch_bounds__(F3_TX * F3_TY, min_blocks(F3_TX * F3_TY)) k_fused_d3q15(Params P, FusedArgs A) {
    step_dependency_wait();
    using L = D3Q15T;
    constexpr int EX = F3_TX + 2, EY = F3_TY + 2, NT = F3_TX * F3_TY, NRING = 2 * EX + 2 * F3_TY;
    extern __shared__ double dsm[];
    double(*s_psi)[EY][EX] = reinterpret_cast<double(*)[EY][EX]>(dsm);
    double* s_f = dsm + 3 * EY * EX;  // [2][15][NT]
    const int tid = threadIdx.x;
    const int tx = tid % F3_TX, ty = tid / F3_TX;
    const int tiles = A.tiles_x * A.tiles_y;
    const int col = blockIdx.x % tiles, chunk = blockIdx.x / tiles;
    const int bx = col % A.tiles_x, by = col / A.tiles_x;
    const int x0 = bx * F3_TX, y0 = by * F3_TY;
    const int z0 = chunk * A.zchunk;
    const int z1 = min(z0 + A.zchunk, A.nz);
    const int ox = slot_coord(x0, tx + 1, A.nx, A.px), oy = slot_coord(y0, ty + 1, A.ny, A.py);
    const bool own_xy = (x0 + tx) < A.nx && (y0 + ty) < A.ny;

    // Plane z: psi of every ext slot into the ring buffer; the own node's
    // pulled populations into s_f[buf]; returns whether the own slot exists.
    auto plane = [&](int z, int buf, double& rho, double& T, double& rr, uint32_t& id) -> bool {
        const int zs = slot_coord(z, 1, A.nz, A.pz);
        double g_unused[1];
        for (int r = tid; r < NRING; r += NT) {
            int ex, ey;
            ring_slot(r, F3_TX, F3_TY, ex, ey);
            const int x = slot_coord(x0, ex, A.nx, A.px);
            const int y = slot_coord(y0, ey, A.ny, A.py);
            if (x < 0 || y < 0 || zs < 0) continue;
            uint32_t rid = (uint32_t)x + (uint32_t)A.nx * ((uint32_t)y + (uint32_t)A.ny * (uint32_t)zs);
            double rf[15], rrho, rt;
            pull_node<L, true, false, HAS_BC>(P, A, x, y, zs, rid, rf, g_unused, rrho, rt);
            s_psi[(z + 3) % 3][ey][ex] = potential(P, rrho, rt);
        }
        if (ox < 0 || oy < 0 || zs < 0) return false;
        id = (uint32_t)ox + (uint32_t)A.nx * ((uint32_t)oy + (uint32_t)A.ny * (uint32_t)zs);
        double f[15];
        pull_node<L, true, false, HAS_BC>(P, A, ox, oy, zs, id, f, g_unused, rho, T);
        s_psi[(z + 3) % 3][ty + 1][tx + 1] = potential(P, rho, T);
        rr = rcp_rn(rho);
#pragma unroll
        for (int k = 0; k < 15; k++) s_f[(buf * 15 + k) * NT + tid] = f[k];
        return true;
    };

    double rc = 0, Tc = 0, rrc = 0, rn = 0, Tn = 0, rrn = 0;
    uint32_t idc = 0, idn = 0;
    {
        double dr, dt, drr;
        uint32_t did;
        plane(z0 - 1, 1, dr, dt, drr, did);  // psi only; its populations are never read
    }
    bool hc = plane(z0, z0 & 1, rc, Tc, rrc, idc);
    for (int z = z0; z < z1; z++) {
        bool hn = plane(z + 1, (z + 1) & 1, rn, Tn, rrn, idn);
        __syncthreads();
        if (own_xy && hc) {
            const bool onb = on_wall(A, ox, oy, z);
            const int ex = tx + 1, ey = ty + 1;
            double f[15], dum[1];
#pragma unroll
            for (int k = 0; k < 15; k++) f[k] = s_f[((z & 1) * 15 + k) * NT + tid];
            auto nbpsi = [&](int k) {
                return s_psi[(z + czk<L>(k) + 3) % 3][ey + cyk<L>(k)][ex + cxk<L>(k)];
            };
            finish_node<L, true, false, EMIT>(P, A, idc, onb, f, dum, rc, rrc, Tc, s_psi[z % 3][ey][ex], nbpsi, 0.0);
        }
        __syncthreads();
        rc = rn;
        rrc = rrn;
        Tc = Tn;
        idc = idn;
        hc = hn;
    }
}

// Pipelined variant: each node's pulled populations are fetched with cp.async two planes ahead
// into a three-slot shared-memory ring (k-major, thread fastest: conflict
// free), so their DRAM latency overlaps the collision of the current plane.
// psi lives in a three-plane ring (tile + one-node ring); the ring nodes'
// pulls are plain loads.  Isothermal: liTempMRT is D2Q9 only, so T is read,
// never written.
constexpr int F3_STAGES = 3;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int F3_TX, int F3_TY, bool HAS_BC, bool EMIT>
__global__ void __launch_bounds__(F3_TX * F3_TY, min_blocks(F3_TX * F3_TY)) k_fused_d3q15_pipe(Params P, FusedArgs A) {
    step_dependency_wait();
    using L = D3Q15T;
    constexpr int EX = F3_TX + 2, EY = F3_TY + 2, NT = F3_TX * F3_TY, NRING = 2 * EX + 2 * F3_TY;
    extern __shared__ double dsm[];
    double(*s_psi)[EY][EX] = reinterpret_cast<double(*)[EY][EX]>(dsm);
    double* s_f = dsm + 3 * EY * EX;  // [F3_STAGES][15][NT]
    const uint32_t n = P.n;
    const int tid = threadIdx.x;
    const int tx = tid % F3_TX, ty = tid / F3_TX;
    const int tiles = A.tiles_x * A.tiles_y;
    const int col = blockIdx.x % tiles, chunk = blockIdx.x / tiles;
    const int bx = col % A.tiles_x, by = col / A.tiles_x;
    const int x0 = bx * F3_TX, y0 = by * F3_TY;
    const int z0 = chunk * A.zchunk;
    const int z1 = min(z0 + A.zchunk, A.nz);
    const int ox = slot_coord(x0, tx + 1, A.nx, A.px), oy = slot_coord(y0, ty + 1, A.ny, A.py);
    const bool own_xy = (x0 + tx) < A.nx && (y0 + ty) < A.ny;

    // Plane z's own pulls -> stage (z+3)%3 (nothing when the slot is absent).
    auto prefetch = [&](int z) {
        const int zs = slot_coord(z, 1, A.nz, A.pz);
        if (ox >= 0 && oy >= 0 && zs >= 0) {
            const uint32_t id = (uint32_t)ox + (uint32_t)A.nx * ((uint32_t)oy + (uint32_t)A.ny * (uint32_t)zs);
            const NodeOffsets no = node_offsets(A, ox, oy, zs, 3);
            double* dst = s_f + ((z + 3) % F3_STAGES) * 15 * NT + tid;
            static_for<15>([&](auto kk) {
                constexpr int k = decltype(kk)::value;
                bool m;
                const uint32_t src = source_of(no, id, cxk<L>(k), cyk<L>(k), czk<L>(k), m);
                cp_async8(dst + k * NT, A.fin + (size_t)k * n + src);
            });
        }
        cp_async_commit();
    };
    // Plane z after its pulls landed: own boundary program, moments, psi; the
    // ring's psi from plain loads.  Returns whether the own slot exists.
    auto process = [&](int z, double& rho, double& T, double& rr, uint32_t& id) -> bool {
        const int zs = slot_coord(z, 1, A.nz, A.pz);
        double g_unused[1];
        bool have = false;
        if (ox >= 0 && oy >= 0 && zs >= 0) {
            id = (uint32_t)ox + (uint32_t)A.nx * ((uint32_t)oy + (uint32_t)A.ny * (uint32_t)zs);
            double* src = s_f + ((z + 3) % F3_STAGES) * 15 * NT + tid;
            double f[15];
#pragma unroll
            for (int k = 0; k < 15; k++) f[k] = src[k * NT];
            bool changed = false;
            if constexpr (HAS_BC) {
                if (A.bcmap[id]) {
                    const NodeOffsets no = node_offsets(A, ox, oy, zs, 3);
                    uint32_t miss = 0;
                    static_for<15>([&](auto kk) {
                        constexpr int k = decltype(kk)::value;
                        bool m;
                        source_of(no, id, cxk<L>(k), cyk<L>(k), czk<L>(k), m);
                        miss |= (uint32_t)m << k;
                    });
                    apply_flow_program<L>(A, id, miss, f);
                    changed = true;
                }
            }
            double s = 0;
#pragma unroll
            for (int k = 0; k < 15; k++) s += f[k];
            rho = s;
            T = A.Told[id];
            rr = rcp_rn(rho);
            s_psi[(z + 3) % 3][ty + 1][tx + 1] = potential(P, rho, T);
            if (changed) {
#pragma unroll
                for (int k = 0; k < 15; k++) src[k * NT] = f[k];
            }
            have = true;
        }
        for (int r = tid; r < NRING; r += NT) {
            int ex, ey;
            ring_slot(r, F3_TX, F3_TY, ex, ey);
            const int x = slot_coord(x0, ex, A.nx, A.px);
            const int y = slot_coord(y0, ey, A.ny, A.py);
            if (x < 0 || y < 0 || zs < 0) continue;
            uint32_t rid = (uint32_t)x + (uint32_t)A.nx * ((uint32_t)y + (uint32_t)A.ny * (uint32_t)zs);
            double rf[15], rrho, rt;
            pull_node<L, true, false, HAS_BC>(P, A, x, y, zs, rid, rf, g_unused, rrho, rt);
            s_psi[(z + 3) % 3][ey][ex] = potential(P, rrho, rt);
        }
        return have;
    };

    double rc = 0, Tc = 0, rrc = 0, rn = 0, Tn = 0, rrn = 0;
    uint32_t idc = 0, idn = 0;
    bool hc = false;
    prefetch(z0 - 1);
    prefetch(z0);
    for (int j = z0 - 1; j <= z1; j++) {
        cp_async_wait1();  // plane j's group is complete (only j+1's may be pending)
        const bool hn = process(j, rn, Tn, rrn, idn);
        __syncthreads();
        const int z = j - 1;
        if (z >= z0 && own_xy && hc) {
            const bool onb = on_wall(A, ox, oy, z);
            const int ex = tx + 1, ey = ty + 1;
            double f[15], dum[1];
            const double* src = s_f + ((z + 3) % F3_STAGES) * 15 * NT + tid;
#pragma unroll
            for (int k = 0; k < 15; k++) f[k] = src[k * NT];
            auto nbpsi = [&](int k) {
                return s_psi[(z + czk<L>(k) + 3) % 3][ey + cyk<L>(k)][ex + cxk<L>(k)];
            };
            finish_node<L, true, false, EMIT>(P, A, idc, onb, f, dum, rc, rrc, Tc, s_psi[(z + 3) % 3][ey][ex], nbpsi, 0.0);
        }
        __syncthreads();
        if (j + 2 <= z1) prefetch(j + 2);
        else cp_async_commit();  // empty group keeps the wait count uniform
        rc = rn;
        rrc = rrn;
        Tc = Tn;
        idc = idn;
        hc = hn;
    }
}

// ============================================================ launch geometry
// Candidate tile shapes.  The autotuner times each on the real state at the
// first fused step and keeps the fastest; results are identical for all.
struct TileCfg {
    int tx, ty;
    bool pipe;   // 3D only: cp.async-staged pulls
    int minb;    // resident blocks per SM asked of the register allocator (0 = default)
    bool inner;  // 2D only: the kernel variant whose inner tiles take the lean body (pays off
                 // on large lattices; a lattice of one wave prefers the smaller general kernel)
    bool tma;    // 3D only: planes staged by TMA (k_fused_d3q15_tma; fully periodic boxes)
    int ringw;   // 2D only: added warps that compute the ring (k_fused_d2q9 RINGW)
};
constexpr int N_CFG2 = 10, N_CFG3 = 10, N_CFG_MAX = 10;
constexpr TileCfg CFG2[N_CFG2] = {{32, 8, false, 0, false}, {32, 4, false, 0, false}, {64, 4, false, 0, false},
                                  {16, 8, false, 0, true},  {64, 4, false, 0, true},  {16, 8, false, 6, true},
                                  {32, 8, false, 3, true},  {32, 4, false, 8, true},
                                  {32, 8, false, 2, false, false, 3}, {16, 8, false, 4, false, false, 2}};
constexpr TileCfg CFG3[N_CFG3] = {{32, 8, false, 0, false}, {32, 8, true, 0, false}, {32, 4, false, 0, false},
                                  {64, 4, false, 0, false}, {32, 16, false, 0, false}, {64, 8, false, 0, false},
                                  {32, 4, false, 3, false, true}, {32, 8, false, 2, false, true},
                                  {32, 16, false, 1, false, true}, {64, 8, false, 1, false, true}};

struct Geom {
    int tiles_x, tiles_y, zchunk, nblocks;  // nblocks 0: the candidate does not take this lattice
};

// Launch geometry of a kernel whose blocks stay resident, minb per SM of a
// 148-SM part: the z chunk count that wastes the fewest block slots over
// the launch's waves (fewer chunks on a tie: each chunk re-reads two planes).
// Blocks are ordered column fastest, so the blocks running together hold
// neighbouring columns at the same planes and share their ring rows in L2.
inline Geom resident_geometry(const FusedArgs& A, int TX, int TY, int minb) {
    Geom g;
    g.tiles_x = A.nx / TX;
    g.tiles_y = A.ny / TY;
    const int cols = g.tiles_x * g.tiles_y, slots = 148 * std::max(1, minb);
    int best = 1;
    double best_t = 1e30;
    for (int c = 1; c <= std::max(1, A.nz / 4); c++) {
        const int zc = (A.nz + c - 1) / c;
        const int blocks = cols * ((A.nz + zc - 1) / zc);
        const double t = (double)((blocks + slots - 1) / slots) * (zc + 2);  // waves x planes per block
        if (t < best_t - 1e-9) {
            best_t = t;
            best = c;
        }
    }
    g.zchunk = (A.nz + best - 1) / best;
    g.nblocks = cols * ((A.nz + g.zchunk - 1) / g.zchunk);
    return g;
}

// Launch geometry for one tile shape: tiles per axis, z chunk (3D), blocks.
inline Geom fused_geometry(int lat, const FusedArgs& A, int TX, int TY) {
    Geom g;
    g.tiles_x = (A.nx + TX - 1) / TX;
    g.tiles_y = (A.ny + TY - 1) / TY;
    if (lat == MPLB_D2Q9) {
        g.zchunk = 1;
        g.nblocks = g.tiles_x * g.tiles_y;
        return g;
    }
    // z chunks: aim for >= 4 blocks of 256 threads per SM of a 148-SM part, chunks of >= 8 planes
    const int cols = g.tiles_x * g.tiles_y;
    const int per_sm = std::max(1, 4 * 256 / (TX * TY));
    const int want = (per_sm * 148 + cols - 1) / cols;
    int zc = (A.nz + want - 1) / want;
    zc = std::max(zc, std::min(8, A.nz));
    g.zchunk = zc;
    g.nblocks = cols * ((A.nz + zc - 1) / zc);
    return g;
}

inline void apply_geom(FusedArgs& A, const Geom& g) {
    A.tiles_x = g.tiles_x;
    A.tiles_y = g.tiles_y;
    A.zchunk = g.zchunk;
}

}  // namespace mplb

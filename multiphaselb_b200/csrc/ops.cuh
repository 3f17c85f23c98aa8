// ops.cuh -- one kernel per reference operator, driven by the neighbour table.
//
// Device layout (structure of arrays, node index fastest):
//   pdf[k*n + id]   populations        (reference: lbeField.value[id][k])
//   vec[j*n + id]   U, Fi, Ft          (reference: macroFields.U[id][j])
//   nb[k*n + id]    pull source of k   (reference: basicMesh.nb[id][k])
// Each kernel reproduces one function of src/lbEquation or src/boundary with
// the same per-node arithmetic; the launch order is the caller's.
#pragma once

#include "lattice.cuh"

namespace mplb {

struct PatchDev {
    uint32_t off, count;
    int32_t type;
    double val[3];
};

// ------------------------------------------------------------- equilibrium
// general/equilibrium.c:22-28 (liMRT, xuMRT)
template <class L>
__global__ void k_equilibrium_flow(Params P, double* __restrict__ f, const double* __restrict__ rho,
                                   const double* __restrict__ U) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double v[3] = {U[id], U[n + id], U[2 * n + id]};
    double r = rho[id];
    static_for<L::Q>([&](auto k) { f[(size_t)k * n + id] = eq_flow_k<L>(P, k, r, v); });
}

// general/equilibrium.c:37-55 (myMRT, liTempMRT)
template <class L>
__global__ void k_equilibrium_heat(Params P, double* __restrict__ g, const double* __restrict__ T,
                                   const double* __restrict__ U) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double v[L::Q];
    if (P.g_model == MPLB_MYMRT) {
        const double u[3] = {U[id], U[n + id], U[2 * n + id]};
        eq_mymrt<L>(P, T[id], u, v);
    } else {
        if constexpr (L::Q == 9) eq_heat(P, T[id], U[id], U[n + id], v);
    }
#pragma unroll
    for (int k = 0; k < L::Q; k++) g[(size_t)k * n + id] = v[k];
}

// --------------------------------------------------------------- collision
// liMRTCollision.c:43-109 / xuMRTCollision.c:42-92 over all nodes.
template <class L>
__global__ void k_collide_flow(Params P, double* __restrict__ f, const double* __restrict__ rho,
                               const double* __restrict__ U, const double* __restrict__ T,
                               const double* __restrict__ Fi, const double* __restrict__ Ft,
                               const int32_t* __restrict__ nb) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double v[L::Q];
#pragma unroll
    for (int k = 0; k < L::Q; k++) v[k] = f[(size_t)k * n + id];
    double u[3] = {U[id], U[n + id], U[2 * n + id]};
    double fi[3] = {Fi[id], Fi[n + id], Fi[2 * n + id]};
    const double ps = potential(P, rho[id], T[id]);
    // surface-tension term: zero on a node with any missing neighbour
    // (liMRTSurfaceTension.c:33-45), else from psi at x + c_k = nb[rev k]
    double C[L::Q];
    const double* Cp = nullptr;
    if (P.st_on) {
        bool interior = true;
#pragma unroll
        for (int k = 1; k < L::Q; k++) interior &= nb[(size_t)k * n + id] != -1;
        if (interior) {
            auto nbpsi = [&](int k) {
                const uint32_t m = (uint32_t)nb[(size_t)revk<L>(k) * n + id];
                return potential(P, rho[m], T[m]);
            };
            surface_tension<L>(P, ps, nbpsi, C);
        } else {
#pragma unroll
            for (int k = 0; k < L::Q; k++) C[k] = 0;
        }
        Cp = C;
    }
    if constexpr (L::Q == 9) {
        double ft[3] = {Ft[id], Ft[n + id], Ft[2 * n + id]};
        collide_limrt_psi(P, v, rho[id], u, ft, fi, ps, Cp);
    } else {
        collide_xumrt_psi(P, v, rho[id], u, fi, ps, Cp);
    }
#pragma unroll
    for (int k = 0; k < L::Q; k++) f[(size_t)k * n + id] = v[k];
}

// liTempMRTCollision.c:31-87 / myMRTCollision.c:141-212 over all nodes.
template <class L>
__global__ void k_collide_heat(Params P, double* __restrict__ g, const double* __restrict__ T,
                               const double* __restrict__ U, const double* __restrict__ S) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double v[L::Q];
#pragma unroll
    for (int k = 0; k < L::Q; k++) v[k] = g[(size_t)k * n + id];
    if (P.g_model == MPLB_MYMRT) {
        const double u[3] = {U[id], U[n + id], U[2 * n + id]};
        collide_mymrt<L>(P, v, T[id], u, S[id]);
    } else {
        if constexpr (L::Q == 9) collide_litemp(P, v, T[id], U[id], U[n + id], S[id]);
    }
#pragma unroll
    for (int k = 0; k < L::Q; k++) g[(size_t)k * n + id] = v[k];
}

// --------------------------------------------------------------- streaming
// lbstream.c:16-62: out = in pulled from nb where it exists, else in itself.
template <int Q>
__global__ void k_stream(uint32_t n, double* __restrict__ out, const double* __restrict__ in,
                         const int32_t* __restrict__ nb) {
    uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
#pragma unroll
    for (int k = 0; k < Q; k++) {
        int32_t s = nb[(size_t)k * n + id];
        out[(size_t)k * n + id] = in[(size_t)k * n + (s != -1 ? (uint32_t)s : id)];
    }
}

// ------------------------------------------------------------------ macros
// liMRTDensity.c:3-19 / xuMRTDensity.c:3-19 and liTempMRTTemperature.c:5-26:
// plain sum over k ascending.
template <int Q>
__global__ void k_moment0(uint32_t n, double* __restrict__ out, const double* __restrict__ pdf,
                          uint32_t start, uint32_t end) {
    uint32_t id = start + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= end) return;
    double s = 0;
#pragma unroll
    for (int k = 0; k < Q; k++) s += pdf[(size_t)k * n + id];
    out[id] = s;
}

// myMRTTemperature.c:5-37: sum over k ascending plus half the source.
template <int Q>
__global__ void k_temperature_my(uint32_t n, double* __restrict__ T, const double* __restrict__ g,
                                 const double* __restrict__ S, uint32_t start, uint32_t end) {
    uint32_t id = start + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= end) return;
    double s = 0;
#pragma unroll
    for (int k = 0; k < Q; k++) s += g[(size_t)k * n + id];
    T[id] = s + 0.5 * S[id];
}

// liMRTVelocity.c:6-55 (F = Ft) and xuMRTVelocity.c:6-55 (F = Fi + (rho - rho_0) g).
template <class L>
__global__ void k_velocity(Params P, double* __restrict__ U, const double* __restrict__ f,
                           const double* __restrict__ rho, const double* __restrict__ Fi,
                           const double* __restrict__ Ft, uint32_t start, uint32_t end) {
    uint32_t n = P.n, id = start + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= end) return;
    double v[L::Q];
#pragma unroll
    for (int k = 0; k < L::Q; k++) v[k] = f[(size_t)k * n + id];
    double r = rho[id];
    double F[3];
#pragma unroll
    for (int j = 0; j < 3; j++)
        F[j] = L::Q == 9 ? Ft[(size_t)j * n + id] : Fi[(size_t)j * n + id] + (r - P.rho_0) * P.g[j];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        double lv = 0;
#pragma unroll
        for (int k = 0; k < L::Q; k++) lv += ck<L>(k, j) * v[k];
        U[(size_t)j * n + id] = (lv + F[j] * 0.5) / r;
    }
}

// ------------------------------------------------------------ interForce
// interForce.c:16-47 with interactionForce.c:32-79.
template <class L>
__global__ void k_interforce(Params P, double* __restrict__ Fi, double* __restrict__ Ft,
                             const double* __restrict__ rho, const double* __restrict__ T,
                             const int32_t* __restrict__ nb, const uint8_t* __restrict__ onb) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double Ff[3] = {0, 0, 0};
    bool inner = onb[id] == 0;
    if (inner) {
        double F[3] = {0.0, 0.0, 0.0};
        static_for<L::Q - 1>([&](auto km1) {
            constexpr int k = decltype(km1)::value + 1;
            int32_t s = nb[(size_t)revk<L>(k) * n + id];
            double al = P.ppw[k] * potential(P, rho[s], T[s]);
            static_for<3>([&](auto i) {
                constexpr int c = ck<L>(k, decltype(i)::value);
                if constexpr (c == 1) F[i] = F[i] + al;
                else if constexpr (c == -1) F[i] = F[i] - al;
            });
        });
        double be = -P.G * potential(P, rho[id], T[id]);
#pragma unroll
        for (int i = 0; i < 3; i++) Ff[i] = F[i] * be;
    }
    double r = rho[id];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        Fi[(size_t)j * n + id] = Ff[j];
        double t = Ff[j] + (r - P.rho_0) * P.g[j];
        if (inner) t += P.fext[j];
        Ft[(size_t)j * n + id] = t;
    }
}

// ------------------------------------------------------------ heatSource
// finiteDifference/{scalarGradient,invScalarGradient,vectorDivergence}.c:
// central where both axis neighbours exist, one-sided where one is missing.
struct FD {
    double v;
    bool present;
};
__device__ __forceinline__ FD fd_pair(int32_t a, int32_t b, double fa, double fb, double fid) {
    if (a != -1 && b != -1) return {0.5 * (fa - fb), true};
    if (a == -1 && b != -1) return {fid - fb, true};
    if (a != -1 && b == -1) return {fa - fid, true};
    return {0.0, false};
}

// general/heatSource.c:28-166 (myMRT, liTempMRT): uses rho (new), T and U (old).
template <class L>
__global__ void k_heatsource(Params P, double* __restrict__ S, const double* __restrict__ rho,
                             const double* __restrict__ T, const double* __restrict__ U,
                             const int32_t* __restrict__ nb, int first) {
    uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    double gT[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, div = 0;
    double r = rho[id], t = T[id];
#pragma unroll
    for (int d = 0; d < L::D; d++) {
        int32_t a = nb[(size_t)fda<L>(d) * n + id];
        int32_t b = nb[(size_t)fdb<L>(d) * n + id];
        uint32_t ia = a != -1 ? (uint32_t)a : id, ib = b != -1 ? (uint32_t)b : id;
        gT[d] = fd_pair(a, b, T[ia], T[ib], t).v;
        gR[d] = fd_pair(a, b, 1.0 / rho[ia], 1.0 / rho[ib], 1.0 / r).v;
        FD dv = fd_pair(a, b, U[(size_t)d * n + ia], U[(size_t)d * n + ib], U[(size_t)d * n + id]);
        if (dv.present) div += dv.v;
    }
    double dot = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) dot += gT[k] * gR[k];
    if (P.g_model == MPLB_MYMRT) {
        S[id] = heat_source_value_my(P, r, t, dot, div);
    } else {
        double old = first ? 0.0 : S[id];
        S[id] = heat_source_value(P, r, t, dot, div, old);
    }
}

// ---------------------------------------------------------------- pressure
// macroPressure.c:8-69 with liMRTPressure.c:6-253 (D2Q9) and
// xuMRTPressure.c:6-22 (D3Q15, rho cs2 + G psi^2 / 2 only).
template <class L>
__global__ void k_pressure(Params P, double* __restrict__ p, const double* __restrict__ rho,
                           const double* __restrict__ T, const int32_t* __restrict__ nb) {
    const uint32_t n = P.n, id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    auto psi_at = [&](uint32_t i) { return potential(P, rho[i], T[i]); };
    const double ps = psi_at(id);
    double pr = rho[id] * P.cs2 + 0.5 * P.G * ps * ps;
    if constexpr (L::Q == 9) {
        // x term assigns lap, the y term adds to it left to right (liMRTPressure.c:27-110);
        // one-sided second differences reach two nodes into the lattice
        double lap = 0;
#pragma unroll
        for (int d = 0; d < 2; d++) {
            const int ka = fda<L>(d), kb = fdb<L>(d);
            const int32_t a = nb[(size_t)ka * n + id], b = nb[(size_t)kb * n + id];
            const double s0 = d == 0 ? 0.0 : lap;
            if (a != -1 && b != -1) {
                lap = d == 0 ? psi_at(a) + psi_at(b) - 2 * ps : s0 + psi_at(a) + psi_at(b) - 2 * ps;
            } else if (a == -1 && b != -1) {
                const int32_t c = nb[(size_t)kb * n + b];
                lap = d == 0 ? psi_at(c) - 2 * psi_at(b) + ps : s0 + psi_at(c) - 2 * psi_at(b) + ps;
            } else if (a != -1 && b == -1) {
                const int32_t c = nb[(size_t)ka * n + a];
                lap = d == 0 ? psi_at(c) - 2 * psi_at(a) + ps : s0 + psi_at(c) - 2 * psi_at(a) + ps;
            } else if (d == 0) {
                lap = 0;
            }
        }
        pr = pr + P.G * ps * lap / 12;
        double grad[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 2; d++) {
            const int32_t a = nb[(size_t)fda<L>(d) * n + id], b = nb[(size_t)fdb<L>(d) * n + id];
            if (a != -1 && b != -1) grad[d] = 0.5 * (psi_at(a) - psi_at(b));
            else if (a == -1 && b != -1) grad[d] = (ps - psi_at(b));
            else if (a != -1 && b == -1) grad[d] = (psi_at(a) - ps);
        }
        double g2 = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) g2 += grad[k] * grad[k];
        pr = pr + 2.0 * P.G * P.G * P.sigma_p * g2;
    }
    p[id] = pr;
}

// -------------------------------------------------------------- boundaries
// liTempMRTEquilibrium row k (fixedT.c:145,178): sum_j Mi[k][j] n_eq[j].
__device__ __forceinline__ double eq_heat_k(const Params& P, int k, double T, double u0, double u1) {
    double ne[9] = {T, -2.0 * T, 2.0 * T, T * u0, T * (-u0), T * u1, T * (-u1), 0, 0};
    double s = 0;
#pragma unroll
    for (int j = 0; j < 9; j++)
        if (Mint<D2Q9T>(j, k) != 0) s = s + P.Mi[k][j] * ne[j];
    return s;
}

// myMRTEquilibrium row k (fixedT.c:59-61,93-95, fixedRandomT.c:72-91).
template <class L>
__device__ __forceinline__ double eq_my_k(const Params& P, int k, double T, const double* u) {
    double ne[L::Q];
    neq_mymrt<L>(P, T, u, ne);
    double s = 0;
#pragma unroll
    for (int j = 0; j < L::Q; j++)
        if (Mint<L>(j, k) != 0) s = s + P.Mi[k][j] * ne[j];
    return s;
}

// One boundary node of one patch, in place (bounceBack.c:14-72,
// fixedT.c:33-134, fixedU.c:31-131, outflow.c:24-185, fixedRandomT.c:46-115).
// Remote reads go through pdf.  tab + slot*Q holds the node's host-made
// table: outflow [0..2] the normal, [3] the normal direction's index;
// fixedRandomT the perturbed wall temperature per direction, used while rnd.
template <class L>
__device__ void bc_node(const Params& P, const PatchDev& pt, int model, uint32_t id,
                        double* __restrict__ pdf, const int32_t* __restrict__ nb,
                        const double* __restrict__ rho, const double* __restrict__ T,
                        const double* __restrict__ U, const double* __restrict__ Fi,
                        const double* __restrict__ tab, uint32_t slot, bool rnd) {
    const uint32_t n = P.n;
    if (pt.type == MPLB_BC_BOUNCEBACK) {
        double v[L::Q];
        int32_t s[L::Q];
#pragma unroll
        for (int k = 0; k < L::Q; k++) {
            v[k] = pdf[(size_t)k * n + id];
            s[k] = nb[(size_t)k * n + id];
        }
#pragma unroll
        for (int k = 0; k < L::Q; k++) {
            const int r = revk<L>(k);
            if (s[k] == -1) {
                v[k] = v[r];
            } else if (s[r] != -1 && k >= 1 && k <= L::NAX) {
                v[k] = 0.5 * v[k] + 0.5 * v[r];
                v[r] = v[k];
            }
        }
#pragma unroll
        for (int k = 0; k < L::Q; k++) pdf[(size_t)k * n + id] = v[k];
    } else if (pt.type == MPLB_BC_FIXEDT) {
        for (int k = 0; k < L::Q; k++) {
            if (nb[(size_t)k * n + id] != -1) continue;
            int32_t m = nb[(size_t)revk<L>(k) * n + id];
            if (m == -1) continue;
            double eq_nb, eq_bnd;
            if (model == MPLB_MYMRT) {
                const double u[3] = {U[m], U[n + m], U[2 * n + m]};
                eq_nb = eq_my_k<L>(P, k, T[m], u);
                eq_bnd = eq_my_k<L>(P, k, pt.val[0], u);
            } else {
                double u0 = U[m], u1 = U[n + m];
                eq_nb = eq_heat_k(P, k, T[m], u0, u1);
                eq_bnd = eq_heat_k(P, k, pt.val[0], u0, u1);
            }
            pdf[(size_t)k * n + id] = eq_bnd + (pdf[(size_t)k * n + m] - eq_nb);
        }
    } else if (pt.type == MPLB_BC_FIXEDRANDOMT) {
        for (int k = 0; k < L::Q; k++) {
            if (nb[(size_t)k * n + id] != -1) continue;
            int32_t m = nb[(size_t)revk<L>(k) * n + id];
            if (m == -1) continue;
            const double u[3] = {U[m], U[n + m], U[2 * n + m]};
            const double eq_nb = eq_my_k<L>(P, k, T[m], u);
            const double Tb = rnd ? tab[(size_t)slot * L::Q + k] : pt.val[0];
            const double eq_bnd = eq_my_k<L>(P, k, Tb, u);
            pdf[(size_t)k * n + id] = eq_bnd + (pdf[(size_t)k * n + m] - eq_nb);
        }
    } else if (pt.type == MPLB_BC_OUTFLOW) {
        const double* t = tab + (size_t)slot * L::Q;
        const int32_t nbm = nb[(size_t)(int)t[3] * n + id];
        if (nbm != -1) {
            const uint32_t m = (uint32_t)nbm;
            double F[3], v[3] = {0, 0, 0}, nbrho = 0;
#pragma unroll
            for (int j = 0; j < 3; j++) F[j] = Fi[(size_t)j * n + m] + (rho[m] - P.rho_0) * P.g[j];
#pragma unroll
            for (int j = 0; j < 3; j++)
#pragma unroll
                for (int q = 0; q < L::Q; q++) v[j] += ck<L>(q, j) * pdf[(size_t)q * n + m];
#pragma unroll
            for (int q = 0; q < L::Q; q++) nbrho += pdf[(size_t)q * n + m];
#pragma unroll
            for (int j = 0; j < 3; j++) v[j] = (v[j] + F[j] * 0.5) / nbrho;
            double uadv = 0;
#pragma unroll
            for (int j = 0; j < 3; j++) uadv += t[j] * v[j];
            for (int k = 0; k < L::Q; k++)
                if (nb[(size_t)k * n + id] == -1)
                    pdf[(size_t)k * n + id] = (pdf[(size_t)k * n + id] + uadv * pdf[(size_t)k * n + m]) / (1 + uadv);
        }
    } else if (pt.type == MPLB_BC_FIXEDU && model == MPLB_LIMRT) {
        for (int k = 0; k < L::Q; k++) {
            if (nb[(size_t)k * n + id] != -1) continue;
            int32_t m = nb[(size_t)revk<L>(k) * n + id];
            if (m == -1) continue;
            double lv[3] = {0, 0, 0}, nbrho = 0, F[3];
#pragma unroll
            for (int j = 0; j < 3; j++) F[j] = Fi[(size_t)j * n + m] + (rho[m] - P.rho_0) * P.g[j];
#pragma unroll
            for (int j = 0; j < 3; j++)
#pragma unroll
                for (int q = 0; q < L::Q; q++) lv[j] += ck<L>(q, j) * pdf[(size_t)q * n + m];
#pragma unroll
            for (int q = 0; q < L::Q; q++) nbrho += pdf[(size_t)q * n + m];
#pragma unroll
            for (int j = 0; j < 3; j++) lv[j] = (lv[j] + F[j] * 0.5) / nbrho;
            double fn = eq_flow_k<L>(P, k, nbrho, lv);
            double fb = eq_flow_k<L>(P, k, nbrho, pt.val);
            pdf[(size_t)k * n + id] = fb + (pdf[(size_t)k * n + m] - fn);
        }
    }
}

// One patch, one thread per node (used when no node reads a population that
// another boundary node writes, checked on the host at create).
template <class L>
__global__ void k_bc_patch(Params P, PatchDev pt, int model, const uint32_t* __restrict__ nodes,
                           double* __restrict__ pdf, const int32_t* __restrict__ nb,
                           const double* __restrict__ rho, const double* __restrict__ T,
                           const double* __restrict__ U, const double* __restrict__ Fi,
                           const double* __restrict__ tab, int rnd) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pt.count) return;
    bc_node<L>(P, pt, model, nodes[pt.off + i], pdf, nb, rho, T, U, Fi, tab, pt.off + i, rnd != 0);
}

// All patches in file order, one node after another: the reference's exact
// serial semantics (updateBoundaries.c:16-71) for meshes where a boundary
// node reads what another one wrote.
template <class L>
__global__ void k_bc_serial(Params P, const PatchDev* __restrict__ pts, int npatch, int model,
                            const uint32_t* __restrict__ nodes, double* __restrict__ pdf,
                            const int32_t* __restrict__ nb, const double* __restrict__ rho,
                            const double* __restrict__ T, const double* __restrict__ U,
                            const double* __restrict__ Fi, const double* __restrict__ tab,
                            unsigned long long rnd_mask) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int p = 0; p < npatch; p++) {
        PatchDev pt = pts[p];
        const bool rnd = (rnd_mask >> p) & 1ull;
        for (uint32_t i = 0; i < pt.count; i++)
            bc_node<L>(P, pt, model, nodes[pt.off + i], pdf, nb, rho, T, U, Fi, tab, pt.off + i, rnd);
    }
}

// ----------------------------------------------------------------- layout
// [n][m] host order <-> [m][n] device order.
static __global__ void k_aos_to_soa(uint32_t n, int m, const double* __restrict__ aos, double* __restrict__ soa) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * m) return;
    uint32_t id = (uint32_t)(i / m);
    int j = (int)(i % m);
    soa[(size_t)j * n + id] = aos[i];
}
static __global__ void k_soa_to_aos(uint32_t n, int m, const double* __restrict__ soa, double* __restrict__ aos) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * m) return;
    uint32_t id = (uint32_t)(i / m);
    int j = (int)(i % m);
    aos[i] = soa[(size_t)j * n + id];
}

// ------------------------------------------------------------- reductions
// averageScalarField.c:28-32 order: one thread, node order.
static __global__ void k_sum_serial(uint32_t n, const double* __restrict__ x, double* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = 0;
    for (uint32_t i = 0; i < n; i++) s += x[i];
    out[0] = s;
}

// Block partial sums of two arrays with warp shuffles; partials[2*block+{0,1}].
static __global__ void k_sum2_partial(uint32_t n, const double* __restrict__ x, const double* __restrict__ y,
                               double* __restrict__ partials) {
    double a = 0, b = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a += x[i];
        if (y) b += y[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double sa[32], sb[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { partials[2 * blockIdx.x] = a; partials[2 * blockIdx.x + 1] = b; }
    }
}

// Final pass over the block partials (one block).
static __global__ void k_sum2_final(int nparts, const double* __restrict__ partials, double* __restrict__ out) {
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double sa[32], sb[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { out[0] = a; out[1] = b; }
    }
}

}  // namespace mplb

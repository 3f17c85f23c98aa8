// mplb_fp32.cu -- fused box kernels of the FP32-deviation form (fused32.cuh).
// Compiled with -fmad=true: this path is measured against FP64, not bitwise.
#include <cuda_runtime.h>

#include <algorithm>

#include "fused32.cuh"

namespace mplb {

// ------------------------------------------------------------- 2D tile
// Shared memory of one 2D tile (psi, 1/rho, T_{n-1}, U_{n-1} on tile + ring).
template <int TX, int TY, bool G_ON>
struct Smem32 {
    static constexpr int EX = TX + 2, EY = TY + 2, GY = G_ON ? EY : 1, GX = G_ON ? EX : 1;
    double psi[EY][EX];
    double inv[GY][GX];
    double To[GY][GX];
    double U0[GY][GX];
    double U1[GY][GX];
};

// One TX x TY tile (tile coordinates bx, by) of the lattice described by A.
// INNER: the tile, its ring and the ring's pull sources lie inside the box
// and away from every boundary program (see the FP64 kernel), so the wrap /
// missing-source / boundary bookkeeping is skipped.
template <int TX, int TY, bool F_ON, bool G_ON, bool HAS_BC, bool EMIT, bool INNER = false>
__device__ __forceinline__ void fused32_tile_d2q9(const Params& P, const FusedArgs32& A, Smem32<TX, TY, G_ON>& sm,
                                                  int bx, int by, double* emit_f, double* emit_g, double* rho_out,
                                                  double* Fi_out, double* Ft_out) {
    using L = D2Q9T;
    constexpr int NRING = 2 * (TX + 2) + 2 * TY;
    const uint32_t n = A.n;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int x0 = bx * TX, y0 = by * TY;

    auto slot = [&](int ex, int ey, float* f, float* g, double& rho, double& T, float& dr, float& dT, uint32_t& id,
                    bool mine, double& rr, EosRho& er) -> bool {
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
        if constexpr (INNER) pull_node32_inner<L, F_ON, G_ON>(P, A, id, f, g, rho, T, dr, dT);
        else pull_node32<L, F_ON, G_ON, HAS_BC>(P, A, x, y, 0, id, f, g, rho, T, dr, dT);
        if (mine) {
            rr = rcp_rn(rho);
            er = eos_rho(P, rho);
            if constexpr (F_ON) sm.psi[ey][ex] = potential_p(P, rho, p_eos_at(P, er, rho, T));
            if constexpr (G_ON) sm.inv[ey][ex] = rr;
        } else {
            if constexpr (F_ON) sm.psi[ey][ex] = potential(P, rho, T);
            if constexpr (G_ON) sm.inv[ey][ex] = 1.0 / rho;
        }
        if constexpr (G_ON) {
            sm.To[ey][ex] = A.Told[id];
            sm.U0[ey][ex] = A.Uold[id];
            sm.U1[ey][ex] = A.Uold[n + id];
        }
        return true;
    };
    if constexpr (INNER) {
        // the own node's loads start now; the ring work below overlaps them
        const int px = x0 + tx, py = y0 + ty;
        prefetch_node32<L, F_ON, G_ON>(A, px, py, (uint32_t)px + (uint32_t)A.nx * (uint32_t)py);
    }
    for (int r = threadIdx.x; r < NRING; r += blockDim.x) {
        int ex, ey;
        ring_slot(r, TX, TY, ex, ey);
        float rf[9], rg[9], rdr, rdt;
        double rrho, rt, rrr;
        EosRho rer;
        uint32_t rid;
        slot(ex, ey, rf, rg, rrho, rt, rdr, rdt, rid, false, rrr, rer);
    }
    float f[9], g[9], dr = 0.f, dT = 0.f;
    double rho = 0, T = 0, rr = 0;
    EosRho er{};
    uint32_t id = 0;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool own = INNER || (gx < A.nx && gy < A.ny);
    const bool have = slot(tx + 1, ty + 1, f, g, rho, T, dr, dT, id, own, rr, er);
    __syncthreads();
    if (own && have) {
        const int ex = tx + 1, ey = ty + 1;
        FusedArgs Gm{};
        Gm.nx = A.nx; Gm.ny = A.ny; Gm.nz = 1; Gm.px = A.px; Gm.py = A.py; Gm.pz = 1;
        const bool onb = INNER ? false : on_wall(Gm, gx, gy, 0);
        double heat = 0;
        if constexpr (G_ON && !EMIT) {
            double gT[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, div = 0;
            const double To = sm.To[ey][ex], iv = sm.inv[ey][ex];
            {
                const bool a = INNER || wrap1(gx + 1, A.nx, A.px) >= 0, b = INNER || wrap1(gx - 1, A.nx, A.px) >= 0;
                FD t = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.To[ey][ex + 1], sm.To[ey][ex - 1], To);
                FD r = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.inv[ey][ex + 1], sm.inv[ey][ex - 1], iv);
                FD u = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.U0[ey][ex + 1], sm.U0[ey][ex - 1], sm.U0[ey][ex]);
                gT[0] = t.v;
                gR[0] = r.v;
                if (u.present) div += u.v;
            }
            {
                const bool a = INNER || wrap1(gy + 1, A.ny, A.py) >= 0, b = INNER || wrap1(gy - 1, A.ny, A.py) >= 0;
                FD t = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.To[ey + 1][ex], sm.To[ey - 1][ex], To);
                FD r = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.inv[ey + 1][ex], sm.inv[ey - 1][ex], iv);
                FD u = fd_pair(a ? 0 : -1, b ? 0 : -1, sm.U1[ey + 1][ex], sm.U1[ey - 1][ex], sm.U1[ey][ex]);
                gT[1] = t.v;
                gR[1] = r.v;
                if (u.present) div += u.v;
            }
            const double dot = gT[0] * gR[0] + gT[1] * gR[1] + gT[2] * gR[2];
            heat = heat_source_value_er(P, er, rho, rr, To, dot, div, A.S[id]);
        }
        const double psi = F_ON ? sm.psi[ey][ex] : 0.0;
        auto nbpsi = [&](int k) { return sm.psi[ey + cyk<L>(k)][ex + cxk<L>(k)]; };
        finish_node32<L, F_ON, G_ON, EMIT>(P, A, id, onb, f, g, rho, dr, T, dT, psi, nbpsi, heat, emit_f, emit_g,
                                           rho_out, Fi_out, Ft_out);
    }
}

// ------------------------------------------------------------- 2D kernel
// MINB: resident blocks per SM asked of the register allocator (0 = default).
// TRY_INNER: inner tiles take the lean body (large lattices); otherwise the
// kernel holds the general body alone (a lattice of one wave prefers it).
template <int TX, int TY, bool F_ON, bool G_ON, bool HAS_BC, bool EMIT, int MINB = 0, bool TRY_INNER = false>
__global__ void __launch_bounds__(TX * TY, MINB ? MINB : min_blocks(TX * TY))
    k_fused32_d2q9(Params P, FusedArgs32 A, double* emit_f, double* emit_g, double* rho_out, double* Fi_out,
                   double* Ft_out) {
    step_dependency_wait();
    __shared__ Smem32<TX, TY, G_ON> sm;
    const int bx = blockIdx.x % A.tiles_x, by = blockIdx.x / A.tiles_x;
    if constexpr (TRY_INNER) {
        const int m = A.bc_margin > 0 ? A.bc_margin : 0;
        const int x0 = bx * TX, y0 = by * TY;
        if (x0 - 1 > m && x0 + TX < A.nx - 1 - m && y0 - 1 > m && y0 + TY < A.ny - 1 - m) {
            fused32_tile_d2q9<TX, TY, F_ON, G_ON, HAS_BC, EMIT, true>(P, A, sm, bx, by, emit_f, emit_g, rho_out,
                                                                      Fi_out, Ft_out);
            return;
        }
    }
    fused32_tile_d2q9<TX, TY, F_ON, G_ON, HAS_BC, EMIT, false>(P, A, sm, bx, by, emit_f, emit_g, rho_out, Fi_out,
                                                               Ft_out);
}

// Lattices of more tiles than this (32 x 8) take the register-capped
// inner-tile kernel: several waves, where it measured faster; fewer (one
// wave or so) keep the general kernel.
constexpr int F32_INNER_MIN_TILES = 4 * 148;

// ------------------------------------------------------------- 3D kernel
template <int TX, int TY>
constexpr size_t f3_smem32() {
    return (size_t)3 * (TY + 2) * (TX + 2) * sizeof(double) + (size_t)2 * 15 * TX * TY * sizeof(float);
}

template <int TX, int TY, bool HAS_BC, bool EMIT>
__global__ void __launch_bounds__(TX * TY, min_blocks(TX * TY))
    k_fused32_d3q15(Params P, FusedArgs32 A, double* emit_f, double* rho_out, double* Fi_out, double* Ft_out) {
    step_dependency_wait();
    using L = D3Q15T;
    constexpr int EX = TX + 2, EY = TY + 2, NT = TX * TY, NRING = 2 * EX + 2 * TY;
    extern __shared__ double dsm[];
    double(*s_psi)[EY][EX] = reinterpret_cast<double(*)[EY][EX]>(dsm);
    float* s_f = reinterpret_cast<float*>(dsm + 3 * EY * EX);  // [2][15][NT]
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int tiles = A.tiles_x * A.tiles_y;
    const int col = blockIdx.x % tiles, chunk = blockIdx.x / tiles;
    const int bx = col % A.tiles_x, by = col / A.tiles_x;
    const int x0 = bx * TX, y0 = by * TY;
    const int z0 = chunk * A.zchunk;
    const int z1 = min(z0 + A.zchunk, A.nz);
    const int ox = slot_coord(x0, tx + 1, A.nx, A.px), oy = slot_coord(y0, ty + 1, A.ny, A.py);
    const bool own_xy = (x0 + tx) < A.nx && (y0 + ty) < A.ny;
    FusedArgs Gm{};
    Gm.nx = A.nx; Gm.ny = A.ny; Gm.nz = A.nz; Gm.px = A.px; Gm.py = A.py; Gm.pz = A.pz;

    auto plane = [&](int z, int buf, double& rho, float& dr, double& T, uint32_t& id) -> bool {
        const int zs = slot_coord(z, 1, A.nz, A.pz);
        float g_unused[1];
        float dT_unused;
        for (int r = tid; r < NRING; r += NT) {
            int ex, ey;
            ring_slot(r, TX, TY, ex, ey);
            const int x = slot_coord(x0, ex, A.nx, A.px);
            const int y = slot_coord(y0, ey, A.ny, A.py);
            if (x < 0 || y < 0 || zs < 0) continue;
            const uint32_t rid = (uint32_t)x + (uint32_t)A.nx * ((uint32_t)y + (uint32_t)A.ny * (uint32_t)zs);
            float rf[15], rdr;
            double rrho, rt;
            pull_node32<L, true, false, HAS_BC>(P, A, x, y, zs, rid, rf, g_unused, rrho, rt, rdr, dT_unused);
            s_psi[(z + 3) % 3][ey][ex] = potential(P, rrho, rt);
        }
        if (ox < 0 || oy < 0 || zs < 0) return false;
        id = (uint32_t)ox + (uint32_t)A.nx * ((uint32_t)oy + (uint32_t)A.ny * (uint32_t)zs);
        float f[15];
        pull_node32<L, true, false, HAS_BC>(P, A, ox, oy, zs, id, f, g_unused, rho, T, dr, dT_unused);
        s_psi[(z + 3) % 3][ty + 1][tx + 1] = potential(P, rho, T);
#pragma unroll
        for (int k = 0; k < 15; k++) s_f[(buf * 15 + k) * NT + tid] = f[k];
        return true;
    };

    double rc = 0, Tc = 0, rn = 0, Tn = 0;
    float drc = 0.f, drn = 0.f;
    uint32_t idc = 0, idn = 0;
    {
        double a, b;
        float c;
        uint32_t d;
        plane(z0 - 1, 1, a, c, b, d);
    }
    bool hc = plane(z0, z0 & 1, rc, drc, Tc, idc);
    for (int z = z0; z < z1; z++) {
        const bool hn = plane(z + 1, (z + 1) & 1, rn, drn, Tn, idn);
        __syncthreads();
        if (own_xy && hc) {
            const bool onb = on_wall(Gm, ox, oy, z);
            const int ex = tx + 1, ey = ty + 1;
            float f[15], dum[1];
#pragma unroll
            for (int k = 0; k < 15; k++) f[k] = s_f[((z & 1) * 15 + k) * NT + tid];
            auto nbpsi = [&](int k) { return s_psi[(z + czk<L>(k) + 3) % 3][ey + cyk<L>(k)][ex + cxk<L>(k)]; };
            finish_node32<L, true, false, EMIT>(P, A, idc, onb, f, dum, rc, drc, Tc, 0.f, s_psi[(z + 3) % 3][ey][ex],
                                                nbpsi, 0.0, emit_f, nullptr, rho_out, Fi_out, Ft_out);
        }
        __syncthreads();
        rc = rn;
        drc = drn;
        Tc = Tn;
        idc = idn;
        hc = hn;
    }
}

template <int TX, int TY, bool BC, bool EMIT>
static cudaError_t set32() {
    return cudaFuncSetAttribute(k_fused32_d3q15<TX, TY, BC, EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)f3_smem32<TX, TY>());
}

}  // namespace mplb

using namespace mplb;

// FP32 constants and deviation weights from the FP64 parameter block.
FusedArgs32 mplb_make_args32(const FusedArgs& A, const Params& P, double rho_ref, double T_ref) {
    FusedArgs32 B{};
    B.nx = A.nx; B.ny = A.ny; B.nz = A.nz; B.px = A.px; B.py = A.py; B.pz = A.pz;
    B.tiles_x = A.tiles_x; B.tiles_y = A.tiles_y; B.zchunk = A.zchunk;
    B.n = P.n;
    B.bcmap = A.bcmap;
    B.bc_margin = A.bc_margin;
    for (int p = 0; p < MPLB_MAX_PATCHES; p++) B.Twall[p] = A.Twall[p];
    for (int q = 0; q < FUSED_MAX_PROGS; q++) B.prog[q] = A.prog[q];
    B.rho_ref = rho_ref;
    B.T_ref = T_ref;
    for (int k = 0; k < MPLB_MAX_Q; k++) {
        B.wf[k] = (float)P.w[k];
        B.Lf[k] = (float)P.Lf[k];
        B.relax_f[k] = (float)P.relax_f[k];
    }
    for (int k = 0; k < 9; k++) {
        B.Lg[k] = (float)P.Lg[k];
        // rest state of liTempMRT: M^-1 (1, -2, 2, 0, ...)
        B.wg[k] = (float)(P.Mi[k][0] - 2.0 * P.Mi[k][1] + 2.0 * P.Mi[k][2]);
    }
    B.s1_den = (float)P.s1_den;
    B.s2_den = (float)P.s2_den;
    B.sig12 = (float)P.sig12;
    B.sig6 = (float)P.sig6;
    B.corr3 = (float)P.corr3;
    B.corr5 = (float)P.corr5;
    return B;
}

int mplb_fused32_attributes() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    chk(set32<32, 8, true, true>());
    chk(set32<32, 8, false, true>());
    chk(set32<32, 4, true, false>());
    chk(set32<32, 4, false, false>());
    return e == cudaSuccess ? 0 : -1;
}

// One FP32-deviation fused step (EMIT: rebuild the FP64 reference state).
cudaError_t mplb_fused32_launch(int lat, bool has_bc, bool f_on, bool g_on, bool emit, FusedArgs32 B,
                                const Params& P, double* emit_f, double* emit_g, double* rho_out, double* Fi_out,
                                double* Ft_out, cudaStream_t s) {
    if (lat == MPLB_D2Q9) {
        FusedArgs tmp{};
        tmp.nx = B.nx; tmp.ny = B.ny; tmp.nz = 1;
        const Geom g = fused_geometry(MPLB_D2Q9, tmp, 32, 8);
        B.tiles_x = g.tiles_x;
        B.tiles_y = g.tiles_y;
        B.zchunk = 1;
        const bool big = !emit && g.nblocks > F32_INNER_MIN_TILES;
#define MPLB_L32(F, G, BC, E)                                                                              \
    (big ? (launch_step(k_fused32_d2q9<32, 8, F, G, BC, E, 3, true>, g.nblocks, 256, 0, s, P, B, emit_f, emit_g, \
                        rho_out, Fi_out, Ft_out), 0)                                                              \
         : (launch_step(k_fused32_d2q9<32, 8, F, G, BC, E>, g.nblocks, 256, 0, s, P, B, emit_f, emit_g, rho_out,  \
                        Fi_out, Ft_out), 0))
#define MPLB_L32_E(F, G, BC) (emit ? (MPLB_L32(F, G, BC, true), 0) : (MPLB_L32(F, G, BC, false), 0))
#define MPLB_L32_B(F, G) (has_bc ? MPLB_L32_E(F, G, true) : MPLB_L32_E(F, G, false))
        if (f_on && g_on) MPLB_L32_B(true, true);
        else if (f_on) MPLB_L32_B(true, false);
        else if (g_on) MPLB_L32_B(false, true);
#undef MPLB_L32
#undef MPLB_L32_E
#undef MPLB_L32_B
    } else {
        FusedArgs tmp{};
        tmp.nx = B.nx; tmp.ny = B.ny; tmp.nz = B.nz;
        if (emit) {
            const Geom g = fused_geometry(MPLB_D3Q15, tmp, 32, 8);
            B.tiles_x = g.tiles_x; B.tiles_y = g.tiles_y; B.zchunk = g.zchunk;
            if (has_bc) launch_step(k_fused32_d3q15<32, 8, true, true>, g.nblocks, 256, f3_smem32<32, 8>(), s, P, B, emit_f, rho_out, Fi_out, Ft_out);
            else launch_step(k_fused32_d3q15<32, 8, false, true>, g.nblocks, 256, f3_smem32<32, 8>(), s, P, B, emit_f, rho_out, Fi_out, Ft_out);
        } else {
            const Geom g = fused_geometry(MPLB_D3Q15, tmp, 32, 4);
            B.tiles_x = g.tiles_x; B.tiles_y = g.tiles_y; B.zchunk = g.zchunk;
            if (has_bc) launch_step(k_fused32_d3q15<32, 4, true, false>, g.nblocks, 128, f3_smem32<32, 4>(), s, P, B, emit_f, rho_out, Fi_out, Ft_out);
            else launch_step(k_fused32_d3q15<32, 4, false, false>, g.nblocks, 128, f3_smem32<32, 4>(), s, P, B, emit_f, rho_out, Fi_out, Ft_out);
        }
    }
    return cudaGetLastError();
}

// FP64 post-collision populations -> FP32 deviations (after the prologue).
__global__ void k_to_dev32(uint32_t n, int Q, const double* __restrict__ src, float* __restrict__ dst, FusedArgs32 B,
                           int heat) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * Q) return;
    const int k = (int)(i / n);
    const double ref = heat ? (double)B.wg[k] * B.T_ref : (double)B.wf[k] * B.rho_ref;
    (void)B.n;
    dst[i] = (float)(src[i] - ref);
}

cudaError_t mplb_to_dev32(uint32_t n, int Q, const double* src, float* dst, const FusedArgs32& B, int heat,
                          cudaStream_t s) {
    const size_t tot = (size_t)n * Q;
    k_to_dev32<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, Q, src, dst, B, heat);
    return cudaGetLastError();
}

// ============================================================ batched ensemble
// Many independent periodic D2Q9 lattices (isothermal, FP32 deviations) in one
// persistent launch: blocks stride over a table of (lattice, tile) pairs.
// Each lattice has its own parameter block and arguments (both parities of
// its ping-pong buffers) in device memory.
namespace mplb {

constexpr int N_BATCH_CFG = 4;
constexpr TileCfg BATCH_CFG[N_BATCH_CFG] = {{32, 8, false}, {32, 4, false}, {16, 8, false}, {64, 4, false}};

// The batch fills every SM with a persistent grid, so resident warps hide
// its memory latency: registers are capped for 24 warps per SM (3 blocks of
// 256 threads, 6 of 128) instead of the lone kernel's 16.
constexpr int batch_min_blocks(int threads) { return threads <= 128 ? 6 : 3; }

template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY, batch_min_blocks(TX * TY))
    k_batch32_d2q9(const Params* __restrict__ Ps, const FusedArgs32* __restrict__ As, const int2* __restrict__ tiles,
                   const int* __restrict__ ntiles, int parity) {
    __shared__ Smem32<TX, TY, false> sm;
    const int nt = *ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 w = tiles[t];
        const FusedArgs32& A = As[2 * w.x + parity];
        if (A.tiles_x <= 0 || w.y < 0 || w.y >= A.tiles_x * A.tiles_y) continue;  // block-uniform
        const int bx = w.y % A.tiles_x, by = w.y / A.tiles_x;
        const int x0 = bx * TX, y0 = by * TY;
        // fully periodic lattices without boundary programs: a tile whose
        // ring and its pull sources stay inside the box needs no wrap logic
        if (x0 >= 2 && x0 + TX + 1 <= A.nx - 1 && y0 >= 2 && y0 + TY + 1 <= A.ny - 1)
            fused32_tile_d2q9<TX, TY, true, false, false, false, true>(Ps[w.x], A, sm, bx, by, nullptr, nullptr,
                                                                        nullptr, nullptr, nullptr);
        else
            fused32_tile_d2q9<TX, TY, true, false, false, false>(Ps[w.x], A, sm, bx, by, nullptr, nullptr, nullptr,
                                                                  nullptr, nullptr);
        __syncthreads();
    }
}

// Per lattice: max over nodes of |rho_now - rho_snapshot|, then the snapshot
// becomes rho_now.  rho_now is what the next step's pull sums to.
template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
    k_batch32_check(const Params* __restrict__ Ps, const FusedArgs32* __restrict__ As,
                    const int2* __restrict__ tiles, const int* __restrict__ ntiles, int parity,
                    double* const* __restrict__ snaps, unsigned long long* __restrict__ dmax,
                    long long* __restrict__ jsum) {
    __shared__ double red[TX * TY / 32];
    const int nt = *ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 w = tiles[t];
        const FusedArgs32& A = As[2 * w.x + parity];
        if (A.tiles_x <= 0 || w.y < 0 || w.y >= A.tiles_x * A.tiles_y) continue;  // block-uniform
        const int bx = w.y % A.tiles_x, by = w.y / A.tiles_x;
        const int x = bx * TX + (int)threadIdx.x % TX, y = by * TY + (int)threadIdx.x / TX;
        double d = 0.0;
        long long m[2] = {0, 0};
        if (x < A.nx && y < A.ny) {
            const uint32_t id = (uint32_t)x + (uint32_t)A.nx * (uint32_t)y;
            float f[9], g[1], dr, dT;
            double rho, T;
            pull_node32<D2Q9T, true, false, false>(Ps[w.x], A, x, y, 0, id, f, g, rho, T, dr, dT);
            double* snap = snaps[w.x];
            d = isfinite(rho) ? fabs(rho - snap[id]) : INFINITY;  // +inf orders above every finite bit pattern
            snap[id] = rho;
            node_momentum_fx<D2Q9T>(A.fin, A.n, id, m);
        }
        warp_add_ll(m[0], jsum + 3 * w.x);
        warp_add_ll(m[1], jsum + 3 * w.x + 1);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_down_sync(0xffffffffu, d, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0.0;
            for (int i = 0; i < TX * TY / 32; i++) m = fmax(m, red[i]);
            // non-negative doubles order like their bit patterns
            atomicMax(dmax + w.x, (unsigned long long)__double_as_longlong(m));
        }
        __syncthreads();
    }
}

// Reset each flagged lattice's total momentum to J0 (see momentum_fix_node).
template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
    k_batch32_fix(const FusedArgs32* __restrict__ As, const int2* __restrict__ tiles, const int* __restrict__ ntiles,
                  int parity, const long long* __restrict__ jsum, const long long* __restrict__ j0,
                  const int* __restrict__ proj) {
    const int nt = *ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 w = tiles[t];
        if (!proj[w.x]) continue;
        const FusedArgs32& A = As[2 * w.x + parity];
        if (A.tiles_x <= 0 || w.y < 0 || w.y >= A.tiles_x * A.tiles_y) continue;
        const int bx = w.y % A.tiles_x, by = w.y / A.tiles_x;
        const int x = bx * TX + (int)threadIdx.x % TX, y = by * TY + (int)threadIdx.x / TX;
        if (x < A.nx && y < A.ny)
            momentum_fix_node<D2Q9T>(const_cast<float*>(A.fin), A.n, (uint32_t)x + (uint32_t)A.nx * (uint32_t)y,
                                     jsum + 3 * w.x, j0 + 3 * w.x);
    }
}

// Time-averaging filter.  A window is M steps; the launch after step s
// (0 <= s < last = M - 1) adds the state that step produced, and one more
// launch (finish = 1) before step `last` replaces the state that step reads
// by the mean; step `last` then runs from the mean, so both buffers hold
// filtered states (the one the reference state is emitted from, and the
// one the next step reads).  Lattice i, with a window of N = win[i] states
// (0: not filtered), sums the states after steps last-N .. last-1 into its
// FP64 accumulator (the first of them assigns).  An FP64 sum of at most
// 2^29 FP32 values is exact, so the mean is rounded once.  `parity` selects
// the buffer the next step reads, as in k_batch32_check.
template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
    k_batch32_average(const FusedArgs32* __restrict__ As, const int2* __restrict__ tiles,
                      const int* __restrict__ ntiles, int parity, double* const* __restrict__ acc,
                      const uint32_t* __restrict__ win, uint32_t s, uint32_t last, int finish) {
    const int nt = *ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int2 w = tiles[t];
        const uint32_t N = win[w.x];
        if (N == 0 || N > last || (!finish && s + N < last)) continue;  // block-uniform
        const FusedArgs32& A = As[2 * w.x + parity];
        if (A.tiles_x <= 0 || w.y < 0 || w.y >= A.tiles_x * A.tiles_y) continue;
        const int bx = w.y % A.tiles_x, by = w.y / A.tiles_x;
        const int x = bx * TX + (int)threadIdx.x % TX, y = by * TY + (int)threadIdx.x / TX;
        if (x >= A.nx || y >= A.ny) continue;
        const uint32_t id = (uint32_t)x + (uint32_t)A.nx * (uint32_t)y;
        double* a = acc[w.x];
        float* f = const_cast<float*>(A.fin);
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const size_t i = (size_t)k * A.n + id;
            if (finish) f[i] = (float)(a[i] / (double)N);
            else if (s + N == last) a[i] = (double)f[i];
            else a[i] += (double)f[i];
        }
    }
}

// Lone lattice: total momentum of the current FP32 buffer, and its reset.
template <class L>
__global__ void k_mom_sum32(uint32_t n, const float* __restrict__ f, long long* __restrict__ J) {
    long long m[3] = {0, 0, 0};
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) node_momentum_fx<L>(f, n, i, m);
#pragma unroll
    for (int d = 0; d < L::D; d++) warp_add_ll(m[d], J + d);
}

template <class L>
__global__ void k_mom_fix32(uint32_t n, float* __restrict__ f, const long long* __restrict__ J,
                            const long long* __restrict__ J0) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) momentum_fix_node<L>(f, n, i, J, J0);
}

}  // namespace mplb

cudaError_t mplb_mom_sum32(int lat, uint32_t n, const float* f, long long* J, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(J, 0, 3 * sizeof(long long), s);
    if (e != cudaSuccess) return e;
    const unsigned nb = (n + 255) / 256;
    if (lat == MPLB_D2Q9) k_mom_sum32<D2Q9T><<<nb, 256, 0, s>>>(n, f, J);
    else k_mom_sum32<D3Q15T><<<nb, 256, 0, s>>>(n, f, J);
    return cudaGetLastError();
}

cudaError_t mplb_mom_fix32(int lat, uint32_t n, float* f, const long long* J, const long long* J0, cudaStream_t s) {
    const unsigned nb = (n + 255) / 256;
    if (lat == MPLB_D2Q9) k_mom_fix32<D2Q9T><<<nb, 256, 0, s>>>(n, f, J, J0);
    else k_mom_fix32<D3Q15T><<<nb, 256, 0, s>>>(n, f, J, J0);
    return cudaGetLastError();
}

namespace {
template <int TX, int TY>
int batch_grid() {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch32_d2q9<TX, TY>, TX * TY, 0);
    return std::max(per, 1) * std::max(sms, 1);
}
}  // namespace

int mplb_batch_ncfg() { return N_BATCH_CFG; }
void mplb_batch_cfg(int c, int* tx, int* ty) {
    *tx = BATCH_CFG[c].tx;
    *ty = BATCH_CFG[c].ty;
}

// Resident blocks of the step kernel for candidate c on the current device
// (the persistent grid).
int mplb_batch_grid(int c) {
    switch (c) {
    case 0: return batch_grid<32, 8>();
    case 1: return batch_grid<32, 4>();
    case 2: return batch_grid<16, 8>();
    default: return batch_grid<64, 4>();
    }
}

cudaError_t mplb_batch32_launch(int cfg, const Params* dP, const FusedArgs32* dA, const int2* tiles,
                                const int* ntiles, int parity, int grid, cudaStream_t s) {
    switch (cfg) {
    case 0: k_batch32_d2q9<32, 8><<<grid, 256, 0, s>>>(dP, dA, tiles, ntiles, parity); break;
    case 1: k_batch32_d2q9<32, 4><<<grid, 128, 0, s>>>(dP, dA, tiles, ntiles, parity); break;
    case 2: k_batch32_d2q9<16, 8><<<grid, 128, 0, s>>>(dP, dA, tiles, ntiles, parity); break;
    default: k_batch32_d2q9<64, 4><<<grid, 256, 0, s>>>(dP, dA, tiles, ntiles, parity); break;
    }
    return cudaGetLastError();
}

cudaError_t mplb_batch32_check(int cfg, const Params* dP, const FusedArgs32* dA, const int2* tiles,
                               const int* ntiles, int parity, int grid, double* const* snaps,
                               unsigned long long* dmax, long long* jsum, cudaStream_t s) {
    switch (cfg) {
    case 0: k_batch32_check<32, 8><<<grid, 256, 0, s>>>(dP, dA, tiles, ntiles, parity, snaps, dmax, jsum); break;
    case 1: k_batch32_check<32, 4><<<grid, 128, 0, s>>>(dP, dA, tiles, ntiles, parity, snaps, dmax, jsum); break;
    case 2: k_batch32_check<16, 8><<<grid, 128, 0, s>>>(dP, dA, tiles, ntiles, parity, snaps, dmax, jsum); break;
    default: k_batch32_check<64, 4><<<grid, 256, 0, s>>>(dP, dA, tiles, ntiles, parity, snaps, dmax, jsum); break;
    }
    return cudaGetLastError();
}

cudaError_t mplb_batch32_average(int cfg, const FusedArgs32* dA, const int2* tiles, const int* ntiles, int parity,
                                 int grid, double* const* acc, const uint32_t* win, uint32_t s, uint32_t last,
                                 int finish, cudaStream_t st) {
    switch (cfg) {
    case 0: k_batch32_average<32, 8><<<grid, 256, 0, st>>>(dA, tiles, ntiles, parity, acc, win, s, last, finish); break;
    case 1: k_batch32_average<32, 4><<<grid, 128, 0, st>>>(dA, tiles, ntiles, parity, acc, win, s, last, finish); break;
    case 2: k_batch32_average<16, 8><<<grid, 128, 0, st>>>(dA, tiles, ntiles, parity, acc, win, s, last, finish); break;
    default: k_batch32_average<64, 4><<<grid, 256, 0, st>>>(dA, tiles, ntiles, parity, acc, win, s, last, finish); break;
    }
    return cudaGetLastError();
}

cudaError_t mplb_batch32_fix(int cfg, const FusedArgs32* dA, const int2* tiles, const int* ntiles, int parity,
                             int grid, const long long* jsum, const long long* j0, const int* proj,
                             cudaStream_t s) {
    switch (cfg) {
    case 0: k_batch32_fix<32, 8><<<grid, 256, 0, s>>>(dA, tiles, ntiles, parity, jsum, j0, proj); break;
    case 1: k_batch32_fix<32, 4><<<grid, 128, 0, s>>>(dA, tiles, ntiles, parity, jsum, j0, proj); break;
    case 2: k_batch32_fix<16, 8><<<grid, 128, 0, s>>>(dA, tiles, ntiles, parity, jsum, j0, proj); break;
    default: k_batch32_fix<64, 4><<<grid, 256, 0, s>>>(dA, tiles, ntiles, parity, jsum, j0, proj); break;
    }
    return cudaGetLastError();
}

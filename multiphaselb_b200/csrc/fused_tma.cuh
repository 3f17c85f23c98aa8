// fused_tma.cuh -- D3Q15 fused step with the plane neighbourhood staged by TMA.
//
// The same time step as k_fused_d3q15 (pull-stream, moments, psi on the tile
// and a one-node ring, force, velocity, xuMRT collision: lbstream.c:16-62,
// xuMRTDensity.c, potential.c:7-13, interactionForce.c:47-79,
// xuMRTVelocity.c:19-44, xuMRTCollision.c:46-89), for fully periodic boxes
// without boundary programs (the static-bubble workloads).  What differs is
// how a plane reaches the block:
//
//   * for every population k the tile's pull sources on plane z - c_kz form
//     one box of (TX+4) x (TY+2) nodes starting at x0-2, y0-1-c_ky (x0-2 is
//     even, so the box starts on a 16-byte boundary), and the temperature
//     plane one more box: 16 boxes per plane, each one TMA tensor copy
//     (cp.async.bulk.tensor, no multicast) into shared memory, completing on
//     the plane's mbarrier;
//   * tiles on a face of the box (their boxes would wrap around the periodic
//     faces, which a tensor copy cannot do) fill the same layout row by row
//     with bulk copies (cp.async.bulk), each row split where it wraps (x0-2
//     and the x extent are even, so every piece starts on a 16-byte boundary
//     and holds whole 16-byte units), completing on the same mbarrier;
//   * two stages: plane p+2 is requested as soon as plane p's stage has been
//     read (after the plane barrier), so its copies overlap two planes of
//     collisions.  The own node's pulled populations are carried in
//     registers from the plane they were read on to the collision one plane
//     later, so a stage is free once its psi pass is done.
//
// Per plane: wait for the stage, psi of every tile and ring slot (the sums
// in k order as pull_node), one barrier, request plane p+2, collide plane
// p-1 (finish_node, the shared node arithmetic).  psi lives in a four-plane
// ring so one barrier per plane suffices.  Results are bit-identical to the
// other fused kernels.
//
// Every wait on an mbarrier is bounded: on a timeout the kernel records
// MPLB_KERR_WAIT in A.kerr, waits (bounded again) for the copies it issued
// and returns; the host reports MPLB_E_TIMEOUT at the next synchronising
// call.
#pragma once

#include <cuda.h>

#include "fused.cuh"
#include "tma_util.cuh"

namespace mplb {

template <int TX, int TY>
struct TmaTile {
    static constexpr int BX = TX + 4, BY = TY + 2;  // box extent: x from x0-2, y from y0-1-c_y
    static constexpr int BOX_BYTES = BX * BY * 8;
    static constexpr int BOX_PITCH = (BOX_BYTES + 127) / 128 * 128;  // each box at a 128-byte boundary
    static constexpr int NBOX = 16;                                   // 15 populations + T
    static constexpr int STAGE_BYTES = NBOX * BOX_PITCH;
    static constexpr int NSTAGE = 2;
    static constexpr int EX = TX + 2, EY = TY + 2;  // tile + ring
    static constexpr int NPSI = 4;                  // psi planes kept
    static constexpr int HEAD = 128;                // mbarriers
    static constexpr size_t SMEM = 128 /* base alignment slack */ + HEAD + (size_t)NSTAGE * STAGE_BYTES +
                                   (size_t)NPSI * EY * EX * 8;
    static_assert(BX * 8 % 16 == 0, "box rows must be whole 16-byte units");
    static_assert(TX % 2 == 0, "x0 - 2 must be even");
};

template <int TX, int TY, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
    k_fused_d3q15_tma(Params P, FusedArgs A, const __grid_constant__ CUtensorMap tm_f,
                      const __grid_constant__ CUtensorMap tm_T) {
    step_dependency_wait();
    using L = D3Q15T;
    using G = TmaTile<TX, TY>;
    constexpr int NT = TX * TY, EX = G::EX, EY = G::EY, NRING = 2 * EX + 2 * TY;
    extern __shared__ unsigned char dsm_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);
    unsigned char* stage0 = base + G::HEAD;
    double(*s_psi)[EY][EX] = reinterpret_cast<double(*)[EY][EX]>(stage0 + G::NSTAGE * G::STAGE_BYTES);

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int tiles = A.tiles_x * A.tiles_y;
    const int col = blockIdx.x % tiles, chunk = blockIdx.x / tiles;
    const int x0 = (col % A.tiles_x) * TX, y0 = (col / A.tiles_x) * TY;
    const int z0 = chunk * A.zchunk, z1 = min(z0 + A.zchunk, A.nz);
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const uint32_t n = P.n;
    // boxes inside the box on x and y: tensor copies; else per-element copies with wrap
    const bool tma = x0 >= 2 && x0 + TX + 2 <= nx && y0 >= 2 && y0 + TY + 2 <= ny;

    // every thread arrives on a stage's mbarrier once per fill, announcing
    // the bytes of the copies it issues (none for most threads of an inner tile)
    if (tid == 0) {
        for (int s = 0; s < G::NSTAGE; s++) mbar_init(&bar[s], (uint32_t)NT);
        mbar_init_fence();
    }
    __syncthreads();

    auto box_ptr = [&](int s, int b) -> double* {
        return reinterpret_cast<double*>(stage0 + s * G::STAGE_BYTES + b * G::BOX_PITCH);
    };
    // Request plane p (z0-1 <= p <= z1) into stage s.
    auto fill = [&](int p, int s) {
        if (tma) {
            if (tid == 0) {
                mbar_arrive_expect_tx(&bar[s], (uint32_t)(G::NBOX * G::BOX_BYTES));
                static_for<15>([&](auto kk) {
                    constexpr int k = decltype(kk)::value;
                    tma_load_4d(box_ptr(s, k), &tm_f, x0 - 2, y0 - 1 - cyk<L>(k), wrap_any(p - czk<L>(k), nz), k,
                                &bar[s]);
                });
                tma_load_3d(box_ptr(s, 15), &tm_T, x0 - 2, y0 - 1, wrap_any(p, nz), &bar[s]);
            } else {
                mbar_arrive(&bar[s]);
            }
        } else {
            // rows (box b, row iy), one thread each; each row BX doubles
            constexpr int NROWS = G::NBOX * G::BY;
            const int mine = tid < NROWS ? (NROWS - 1 - tid) / NT + 1 : 0;
            mbar_arrive_expect_tx(&bar[s], (uint32_t)(mine * G::BX * 8));
            for (int r = tid; r < NROWS; r += NT) {
                const int b = r / G::BY, iy = r - b * G::BY;
                const int cy = b < 15 ? cyk<L>(b) : 0, cz = b < 15 ? czk<L>(b) : 0;
                const int y = wrap_any(y0 - 1 - cy + iy, ny), z = wrap_any(p - cz, nz);
                const double* row = (b < 15 ? A.fin + (size_t)b * n : A.Told) + (size_t)nx * ((size_t)y + (size_t)ny * z);
                double* dst = box_ptr(s, b) + iy * G::BX;
                // columns x0-2 .. x0+TX+1, split where they wrap (at most three pieces)
                for (int done = 0; done < G::BX;) {
                    const int x = wrap_any(x0 - 2 + done, nx);
                    const int len = min(G::BX - done, nx - x);
                    bulk_load(dst + done, row + x, (uint32_t)len * 8u, &bar[s]);
                    done += len;
                }
            }
        }
    };

    // per stage, bit s: the parity of its next wait, and whether a fill is outstanding
    uint32_t parity = 0, pending = 0;
    const int pfirst = z0 - 1, plast = z1;  // psi is needed on planes z0-1 .. z1
    for (int q = 0; q < G::NSTAGE && pfirst + q <= plast; q++) {
        fill(pfirst + q, q);
        pending |= 1u << q;
    }

    double fp[15], fc[15];  // own pulled populations: plane p-1 (collided now), plane p (next)
    double rp = 0, rrp = 0, Tp = 0, rc = 0, rrc = 0, Tcur = 0;
    bool failed = false;
    for (int p = pfirst; p <= plast; p++) {
        const int j = p - pfirst, s = j % G::NSTAGE;
        const bool landed = mbar_wait_bounded(&bar[s], (parity >> s) & 1u, TMA_WAIT_LIMIT);
        if (landed) {
            parity ^= 1u << s;
            pending &= ~(1u << s);
        }
        // psi of plane p: ring slots, then the own slot (whose populations
        // stay in registers).  Population k of ext slot (ex, ey) sits at
        // box k, row ey, column ex + 1 - c_kx; T at box 15, column ex + 1.
        const double* sb = box_ptr(s, 0);
        constexpr int BP = G::BOX_PITCH / 8;
        double(*psi_p)[EX] = s_psi[(p + G::NPSI) % G::NPSI];
        for (int r = tid; landed && r < NRING; r += NT) {
            int ex, ey;
            ring_slot(r, TX, TY, ex, ey);
            const double* sl = sb + ey * G::BX + ex + 1;
            double rho = 0;
            static_for<15>([&](auto kk) {
                constexpr int k = decltype(kk)::value;
                rho += sl[k * BP - cxk<L>(k)];
            });
            psi_p[ey][ex] = potential(P, rho, sl[15 * BP]);
        }
        if (landed) {
            const int ex = tx + 1, ey = ty + 1;
            const double* sl = sb + ey * G::BX + ex + 1;
            double rho = 0;
            static_for<15>([&](auto kk) {
                constexpr int k = decltype(kk)::value;
                fc[k] = sl[k * BP - cxk<L>(k)];
                rho += fc[k];
            });
            Tcur = sl[15 * BP];
            rc = rho;
            rrc = rcp_rn(rho);
            psi_p[ey][ex] = potential(P, rho, Tcur);
        }
        // one decision for the whole block: a wait that ran out in any thread ends the kernel
        if (__syncthreads_or(!landed)) {
            failed = true;
            break;
        }
        // stage s has been read: request plane p + NSTAGE into it
        if (p + G::NSTAGE <= plast) {
            fill(p + G::NSTAGE, s);
            pending |= 1u << s;
        }
        // collide plane p-1 with psi of planes p-2, p-1, p
        const int z = p - 1;
        if (z >= z0) {
            const uint32_t id = (uint32_t)(x0 + tx) + (uint32_t)nx * ((uint32_t)(y0 + ty) + (uint32_t)ny * (uint32_t)z);
            const int ex = tx + 1, ey = ty + 1;
            auto nbpsi = [&](int k) {
                return s_psi[(z + czk<L>(k) + G::NPSI) % G::NPSI][ey + cyk<L>(k)][ex + cxk<L>(k)];
            };
            double dum[1];
            finish_node<L, true, false, false>(P, A, id, false, fp, dum, rp, rrp, Tp,
                                               s_psi[(z + G::NPSI) % G::NPSI][ey][ex], nbpsi, 0.0);
        }
#pragma unroll
        for (int k = 0; k < 15; k++) fp[k] = fc[k];
        rp = rc;
        rrp = rrc;
        Tp = Tcur;
    }
    if (failed) {
        if (tid == 0) atomicExch(A.kerr, MPLB_KERR_WAIT);
        // let the copies this block issued land before its shared memory is released
        for (int s = 0; s < G::NSTAGE; s++)
            if ((pending >> s) & 1u) mbar_wait_bounded(&bar[s], (parity >> s) & 1u, TMA_WAIT_LIMIT);
    }
}

// Fully periodic D3Q15 box without boundary programs, tiles that divide
// the box, an even x extent: the lattices this kernel takes.
inline bool tma3_fits(const FusedArgs& A, bool has_bc, int TX, int TY) {
    return !has_bc && A.px && A.py && A.pz && A.nx % TX == 0 && A.ny % TY == 0 && A.nx % 2 == 0 && A.nz >= 2;
}

}  // namespace mplb

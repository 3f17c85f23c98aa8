// Host-only check of the fused kernels' index arithmetic (no GPU needed).
// Replays, for every block and thread of a launch, the slots, pull sources
// and neighbour indices the kernels compute, with the same helper functions,
// and checks that each index is inside its buffer and that every node is
// owned by exactly one thread.  Prints "OK <cases>" or the first violation.
#include <cstdio>
#include <vector>
#include "../multiphaselb_b200/csrc/fused.cuh"
#include "../multiphaselb_b200/csrc/fused_tma.cuh"

using namespace mplb;

static int fails = 0;
#define REQUIRE(c, ...) do { if (!(c)) { if (fails++ < 10) { printf("FAIL %s:%d ", __FILE__, __LINE__); printf(__VA_ARGS__); printf("\n"); } } } while (0)

template <class L>
void check_cfg(int nx, int ny, int nz, int px, int py, int pz, int TX, int TY) {
    FusedArgs A{};
    A.nx = nx; A.ny = ny; A.nz = L::D == 3 ? nz : 1;
    A.px = px; A.py = py; A.pz = L::D == 3 ? pz : 1;
    const Geom gm = fused_geometry(L::lattice, A, TX, TY);
    apply_geom(A, gm);
    const int nblocks = gm.nblocks;
    const int64_t n = (int64_t)A.nx * A.ny * A.nz;
    std::vector<int> owned(n, 0);
    const int EX = TX + 2, EY = TY + 2, NRING = 2 * EX + 2 * TY;
    auto check_node = [&](int x, int y, int z, const char* what) {
        REQUIRE(x >= 0 && x < A.nx && y >= 0 && y < A.ny && z >= 0 && z < A.nz, "%s node (%d,%d,%d)", what, x, y, z);
        int64_t id = (int64_t)x + (int64_t)A.nx * ((int64_t)y + (int64_t)A.ny * z);
        const NodeOffsets no = node_offsets(A, x, y, z, L::D);
        for (int k = 0; k < L::Q; k++) {
            int64_t s = pull_src(A.nx, A.ny, A.nz, A.px, A.py, A.pz, x, y, z, cxk<L>(k), cyk<L>(k), czk<L>(k));
            REQUIRE(s >= -1 && s < n, "pull src %lld of node %lld k %d", (long long)s, (long long)id, k);
            bool miss;
            uint32_t src = source_of(no, (uint32_t)id, cxk<L>(k), cyk<L>(k), czk<L>(k), miss);
            REQUIRE(miss == (s < 0), "missing flag of node %lld k %d", (long long)id, k);
            REQUIRE((int64_t)src == (s < 0 ? id : s), "offset source %u != %lld (node %lld k %d)", src, (long long)s,
                    (long long)id, k);
            // fixedT neighbour x + c_k (2D)
            int mx = wrap1(x + cxk<L>(k), A.nx, A.px), my = wrap1(y + cyk<L>(k), A.ny, A.py);
            if (mx >= 0 && my >= 0) REQUIRE((int64_t)mx + (int64_t)A.nx * my < n || L::D == 3, "fixedT nb");
        }
        return id;
    };
    for (int b = 0; b < nblocks; b++) {
        int x0, y0, z0 = 0, z1 = 1;
        if (L::D == 2) {
            x0 = (b % A.tiles_x) * TX; y0 = (b / A.tiles_x) * TY;
        } else {
            int tiles = A.tiles_x * A.tiles_y, col = b % tiles, chunk = b / tiles;
            x0 = (col % A.tiles_x) * TX; y0 = (col / A.tiles_x) * TY;
            z0 = chunk * A.zchunk; z1 = std::min(z0 + A.zchunk, A.nz);
            REQUIRE(z0 < A.nz, "empty z chunk %d", chunk);
        }
        for (int z = (L::D == 3 ? z0 - 1 : 0); z <= (L::D == 3 ? z1 : 0); z++) {
            int zs = L::D == 3 ? slot_coord(z, 1, A.nz, A.pz) : 0;
            if (zs < 0) continue;
            REQUIRE(zs < A.nz, "z slot");
            for (int t = 0; t < TX * TY; t++) {
                int tx = t % TX, ty = t / TX;
                int x = slot_coord(x0, tx + 1, A.nx, A.px), y = slot_coord(y0, ty + 1, A.ny, A.py);
                if (x >= 0 && y >= 0) check_node(x, y, zs, "interior slot");
                bool own = (x0 + tx) < A.nx && (y0 + ty) < A.ny;
                if (own) {
                    REQUIRE(x == x0 + tx && y == y0 + ty, "own slot moved");
                    if (L::D == 2 || (z >= z0 && z < z1)) owned[(size_t)(x + (int64_t)A.nx * (y + (int64_t)A.ny * zs))]++;
                    // psi / FD neighbours read from shared memory
                    for (int k = 0; k < L::Q; k++) {
                        int ex = tx + 1 + cxk<L>(k), ey = ty + 1 + cyk<L>(k);
                        REQUIRE(ex >= 0 && ex < EX && ey >= 0 && ey < EY, "smem neighbour");
                        bool onb = on_wall(A, x, y, zs);
                        if (!onb) {
                            int nxs = slot_coord(x0, ex, A.nx, A.px), nys = slot_coord(y0, ey, A.ny, A.py);
                            REQUIRE(nxs == wrap1(x + cxk<L>(k), A.nx, A.px) && nys == wrap1(y + cyk<L>(k), A.ny, A.py),
                                    "neighbour slot (%d,%d) holds (%d,%d), want (%d,%d)", ex, ey, nxs, nys,
                                    wrap1(x + cxk<L>(k), A.nx, A.px), wrap1(y + cyk<L>(k), A.ny, A.py));
                        }
                    }
                }
            }
            for (int r = 0; r < NRING; r++) {
                int ex, ey;
                ring_slot(r, TX, TY, ex, ey);
                REQUIRE(ex >= 0 && ex < EX && ey >= 0 && ey < EY, "ring slot %d -> (%d,%d)", r, ex, ey);
                REQUIRE(!(ex >= 1 && ex <= TX && ey >= 1 && ey <= TY), "ring slot %d inside tile", r);
                int x = slot_coord(x0, ex, A.nx, A.px), y = slot_coord(y0, ey, A.ny, A.py);
                if (x >= 0 && y >= 0) check_node(x, y, zs, "ring slot");
            }
        }
    }
    for (int64_t i = 0; i < n; i++) REQUIRE(owned[i] == 1, "node %lld owned %d times (dims %d %d %d)", (long long)i, owned[i], nx, ny, nz);
}

template <class L>
void check(int nx, int ny, int nz, int px, int py, int pz) {
    if (L::D == 2)
        for (int c = 0; c < N_CFG2; c++) check_cfg<L>(nx, ny, nz, px, py, pz, CFG2[c].tx, CFG2[c].ty);
    else
        for (int c = 0; c < N_CFG3; c++) check_cfg<L>(nx, ny, nz, px, py, pz, CFG3[c].tx, CFG3[c].ty);
}

// k_fused_d3q15_tma: geometry, tensor-copy boxes inside the tensor, per-element
// copies inside their buffers, shared-memory offsets inside the allocation,
// the pulled value of every ext slot taken from the node the pull reads, and
// every node collided by exactly one thread.
template <int TX, int TY, int MINB>
void check_tma(int nx, int ny, int nz) {
    using L = D3Q15T;
    using G = TmaTile<TX, TY>;
    FusedArgs A{};
    A.nx = nx; A.ny = ny; A.nz = nz; A.px = A.py = A.pz = 1;
    if (!tma3_fits(A, false, TX, TY)) return;
    const Geom gm = resident_geometry(A, TX, TY, MINB);
    apply_geom(A, gm);
    const int64_t n = (int64_t)nx * ny * nz;
    REQUIRE(gm.tiles_x * TX == nx && gm.tiles_y * TY == ny, "tma tiles");
    REQUIRE(gm.nblocks == gm.tiles_x * gm.tiles_y * ((nz + gm.zchunk - 1) / gm.zchunk), "tma block count");
    // shared memory: mbarriers, stages, psi ring, after the 128-byte alignment of the base
    const size_t used = (size_t)G::HEAD + (size_t)G::NSTAGE * G::STAGE_BYTES + (size_t)G::NPSI * G::EY * G::EX * 8;
    REQUIRE(used + 127 <= G::SMEM, "tma smem %zu of %zu", used, G::SMEM);
    REQUIRE(G::SMEM <= 227 * 1024, "tma smem over the per-block limit");
    REQUIRE(G::BOX_PITCH % 128 == 0 && G::BOX_PITCH >= G::BOX_BYTES && G::HEAD % 128 == 0 && G::STAGE_BYTES % 128 == 0,
            "tma box alignment");
    REQUIRE(G::NSTAGE * 8 <= G::HEAD, "mbarriers");
    std::vector<int> owned(n, 0);
    const int tiles = gm.tiles_x * gm.tiles_y;
    for (int b = 0; b < gm.nblocks; b++) {
        const int col = b % tiles, chunk = b / tiles;
        const int x0 = (col % gm.tiles_x) * TX, y0 = (col / gm.tiles_x) * TY;
        const int z0 = chunk * gm.zchunk, z1 = std::min(z0 + gm.zchunk, nz);
        REQUIRE(z0 < nz, "tma empty chunk");
        const bool tma = x0 >= 2 && x0 + TX + 2 <= nx && y0 >= 2 && y0 + TY + 2 <= ny;
        for (int p = z0 - 1; p <= z1; p++) {
            for (int bx = 0; bx < G::NBOX; bx++) {
                const int cy = bx < 15 ? cyk<L>(bx) : 0, cz = bx < 15 ? czk<L>(bx) : 0;
                if (tma) {
                    const int xs = x0 - 2, ys = y0 - 1 - cy, zs = wrap_any(p - cz, nz);
                    REQUIRE(xs >= 0 && xs + G::BX <= nx && xs % 2 == 0, "tma box x %d", xs);
                    REQUIRE(ys >= 0 && ys + G::BY <= ny, "tma box y %d", ys);
                    REQUIRE(zs >= 0 && zs < nz, "tma box z %d", zs);
                }
                if (!tma) {
                    // face tiles: rows of bulk copies, split where they wrap (the kernel's loop)
                    for (int iy = 0; iy < G::BY; iy++) {
                        const int y = wrap_any(y0 - 1 - cy + iy, ny), z = wrap_any(p - cz, nz);
                        REQUIRE(y >= 0 && y < ny && z >= 0 && z < nz, "bulk row node");
                        int pieces = 0;
                        for (int done = 0; done < G::BX;) {
                            const int x = wrap_any(x0 - 2 + done, nx);
                            const int len = std::min(G::BX - done, nx - x);
                            REQUIRE(x >= 0 && x < nx && len > 0 && x + len <= nx, "bulk piece x %d len %d", x, len);
                            REQUIRE(x % 2 == 0 && len % 2 == 0 && done % 2 == 0, "bulk piece alignment");
                            for (int i = 0; i < len; i++)  // each column of the piece is the wrapped x0-2+done+i
                                REQUIRE(x + i == wrap_any(x0 - 2 + done + i, nx), "bulk piece column");
                            done += len;
                            pieces++;
                        }
                        REQUIRE(pieces <= 3, "bulk pieces %d", pieces);
                    }
                }
            }
            // the value read for population k at ext slot (ex, ey): box k, row ey, column ex + 1 - c_kx
            for (int ey = 0; ey < G::EY; ey++)
                for (int ex = 0; ex < G::EX; ex++) {
                    const int sx = wrap_any(x0 - 1 + ex, nx), sy = wrap_any(y0 - 1 + ey, ny), sz = wrap_any(p, nz);
                    for (int k = 0; k < 15; k++) {
                        const int ix = ex + 1 - cxk<L>(k), iy = ey;
                        REQUIRE(ix >= 0 && ix < G::BX, "tma column");
                        const int x = wrap_any(x0 - 2 + ix, nx), y = wrap_any(y0 - 1 - cyk<L>(k) + iy, ny);
                        const int z = wrap_any(p - czk<L>(k), nz);
                        const int64_t got = (int64_t)x + (int64_t)nx * ((int64_t)y + (int64_t)ny * z);
                        const int64_t want = pull_src(nx, ny, nz, 1, 1, 1, sx, sy, sz, cxk<L>(k), cyk<L>(k), czk<L>(k));
                        REQUIRE(got == want, "tma pull of slot (%d,%d) plane %d k %d: %lld vs %lld", ex, ey, p, k,
                                (long long)got, (long long)want);
                    }
                    // T of the slot: box 15, column ex + 1
                    const int64_t tnode = (int64_t)wrap_any(x0 - 2 + ex + 1, nx) +
                                          (int64_t)nx * ((int64_t)wrap_any(y0 - 1 + ey, ny) + (int64_t)ny * sz);
                    REQUIRE(tnode == sx + (int64_t)nx * (sy + (int64_t)ny * sz), "tma T of slot");
                }
            const int z = p - 1;
            if (z >= z0)
                for (int t = 0; t < TX * TY; t++) {
                    const int64_t id = (int64_t)(x0 + t % TX) + (int64_t)nx * ((int64_t)(y0 + t / TX) + (int64_t)ny * z);
                    REQUIRE(id >= 0 && id < n, "tma own node");
                    owned[id]++;
                    for (int k = 1; k < 15; k++) {  // psi neighbour planes written at iterations p-2 .. p
                        const int q = z + czk<L>(k);
                        REQUIRE(q >= p - 2 && q <= p, "tma psi plane");
                    }
                }
        }
    }
    for (int64_t i = 0; i < n; i++) REQUIRE(owned[i] == 1, "tma node %lld collided %d times", (long long)i, owned[i]);
}

int main() {
    int cases = 0;
    int dims2[][2] = {{2, 2}, {3, 5}, {24, 20}, {12, 24}, {12, 16}, {32, 8}, {33, 9}, {128, 512}, {256, 256}, {100, 3}};
    for (auto& d : dims2)
        for (int px = 0; px < 2; px++)
            for (int py = 0; py < 2; py++) { check<D2Q9T>(d[0], d[1], 1, px, py, 1); cases++; }
    int dims3[][3] = {{2, 2, 2}, {10, 8, 6}, {8, 6, 7}, {33, 9, 17}, {40, 40, 40}, {70, 20, 30}, {40, 24, 100}};
    for (auto& d : dims3)
        for (int p = 0; p < 8; p++) { check<D3Q15T>(d[0], d[1], d[2], p & 1, (p >> 1) & 1, (p >> 2) & 1); cases++; }
    int dims_tma[][3] = {{32, 8, 2},      {64, 16, 9},     {96, 40, 33},   {192, 192, 12},
                         {128, 128, 128}, {64, 8, 64},     {192, 48, 6},   {192, 192, 192}, {128, 64, 5}};
    for (auto& d : dims_tma) {
        check_tma<32, 4, 3>(d[0], d[1], d[2]);
        check_tma<32, 8, 2>(d[0], d[1], d[2]);
        check_tma<32, 16, 1>(d[0], d[1], d[2]);
        check_tma<64, 8, 1>(d[0], d[1], d[2]);
        cases++;
    }
    if (fails) { printf("FAILED %d checks\n", fails); return 1; }
    printf("OK %d\n", cases);
    return 0;
}

// Host-only check of the fused kernels' index arithmetic (no GPU needed).
// Replays, for every block and thread of a launch, the slots, pull sources
// and neighbour indices the kernels compute, with the same helper functions,
// and checks that each index is inside its buffer and that every node is
// owned by exactly one thread.  Prints "OK <cases>" or the first violation.
#include <cstdio>
#include <vector>
#include "../multiphaselb_b200/csrc/fused.cuh"

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

int main() {
    int cases = 0;
    int dims2[][2] = {{2, 2}, {3, 5}, {24, 20}, {12, 24}, {12, 16}, {32, 8}, {33, 9}, {128, 512}, {256, 256}, {100, 3}};
    for (auto& d : dims2)
        for (int px = 0; px < 2; px++)
            for (int py = 0; py < 2; py++) { check<D2Q9T>(d[0], d[1], 1, px, py, 1); cases++; }
    int dims3[][3] = {{2, 2, 2}, {10, 8, 6}, {8, 6, 7}, {33, 9, 17}, {40, 40, 40}, {70, 20, 30}, {40, 24, 100}};
    for (auto& d : dims3)
        for (int p = 0; p < 8; p++) { check<D3Q15T>(d[0], d[1], d[2], p & 1, (p >> 1) & 1, (p >> 2) & 1); cases++; }
    if (fails) { printf("FAILED %d checks\n", fails); return 1; }
    printf("OK %d\n", cases);
    return 0;
}

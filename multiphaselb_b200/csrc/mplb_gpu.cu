// mplb_gpu.cu -- C-ABI of the B200 lattice update (include/mplb_gpu.h).
//
// One handle = one device-resident lattice.  The handle keeps the
// reference's state (f, g after streaming and boundaries; rho, U, T, Fi, Ft,
// scalarSource) in structure-of-arrays FP64 buffers and advances it either
// with one kernel per reference operator (any neighbour table) or with the
// fused box kernels of fused.cuh (structured boxes).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "mplb_io.h"
#include "ops.cuh"
#include "fused_host.cuh"
#include "fused32.cuh"

using namespace mplb;

// FP32-deviation kernels (mplb_fp32.cu, compiled with contraction on).
FusedArgs32 mplb_make_args32(const FusedArgs& A, const Params& P, double rho_ref, double T_ref);
int mplb_fused32_attributes();
cudaError_t mplb_fused32_launch(int lat, bool has_bc, bool f_on, bool g_on, bool emit, FusedArgs32 B, const Params& P,
                                double* emit_f, double* emit_g, double* rho_out, double* Fi_out, double* Ft_out,
                                cudaStream_t s);
cudaError_t mplb_to_dev32(uint32_t n, int Q, const double* src, float* dst, const FusedArgs32& B, int heat,
                          cudaStream_t s);
// Learned warm start (mplb_mlp.cu).
int mplb_mlp_bubble_launch(mplb_mlp* m, double* rho, uint32_t n, int nx, int ny, const double* c, double R,
                           double t_ratio, double a, double b, cudaStream_t s);
int mplb_mlp_column_launch(mplb_mlp* m, double* rho, uint32_t n, int nx, int ny, int axis, int ext, double c,
                           double height, double t_ratio, double a, double b, cudaStream_t s);
int mplb_mlp_device(const mplb_mlp* m);

// Batched ensemble kernels (mplb_fp32.cu).
int mplb_batch_ncfg();
void mplb_batch_cfg(int c, int* tx, int* ty);
int mplb_batch_grid(int c);
cudaError_t mplb_batch32_launch(int cfg, const Params* dP, const FusedArgs32* dA, const int2* tiles,
                                const int* ntiles, int parity, int grid, cudaStream_t s);
cudaError_t mplb_batch32_check(int cfg, const Params* dP, const FusedArgs32* dA, const int2* tiles,
                               const int* ntiles, int parity, int grid, double* const* snaps,
                               unsigned long long* dmax, long long* jsum, cudaStream_t s);
cudaError_t mplb_batch32_fix(int cfg, const FusedArgs32* dA, const int2* tiles, const int* ntiles, int parity,
                             int grid, const long long* jsum, const long long* j0, const int* proj,
                             cudaStream_t s);
cudaError_t mplb_batch32_average(int cfg, const FusedArgs32* dA, const int2* tiles, const int* ntiles, int parity,
                                 int grid, double* const* acc, const uint32_t* win, uint32_t s, uint32_t last,
                                 int finish, cudaStream_t st);
cudaError_t mplb_mom_sum32(int lat, uint32_t n, const float* f, long long* J, cudaStream_t s);
cudaError_t mplb_mom_fix32(int lat, uint32_t n, float* f, const long long* J, const long long* J0, cudaStream_t s);

#define MPLB_STR2(x) #x
#define MPLB_STR(x) MPLB_STR2(x)

namespace {

thread_local std::string g_err = "";

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(MPLB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int TPB = 256;

inline unsigned blocks(size_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

struct PatchHost {
    PatchDev d;
};

}  // namespace

struct mplb_gpu {
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Params P{};
    int lat = 0, Q = 0, D = 0;
    uint32_t n = 0;
    int path = MPLB_PATH_OPERATORS;
    // box description (when the neighbour table is a structured box)
    bool box = false;
    int dims[3] = {0, 0, 0}, per[3] = {0, 0, 0};
    // device state
    int32_t* nb = nullptr;
    uint8_t* onb = nullptr;
    double* pdf[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [field][buffer]
    int cur[2] = {0, 0};
    double *rho = nullptr, *T = nullptr, *S = nullptr, *U = nullptr, *Fi = nullptr, *Ft = nullptr;
    double* p = nullptr;                  // pressure (write-time output)
    double *T2 = nullptr, *U2 = nullptr;  // fused-path double buffers
    uint8_t* bcmap = nullptr;             // fused-path per-node boundary-program index
    uint32_t* pnodes = nullptr;
    // per field, [patch nodes][Q] tables made at create for outflow (normal,
    // normal direction) and fixedRandomT (perturbed wall temperatures)
    double* bctab[2] = {nullptr, nullptr};
    // fixedRandomT: boundary updates made on each field, and per patch how
    // many of the first ones are perturbed (psteps - localTStep)
    uint64_t bc_calls[2] = {0, 0};
    std::vector<int64_t> rnd_left[2];
    PatchDev* dpatches = nullptr;          // [field][patch] copies for the serial kernel
    std::vector<PatchDev> fpatch[2];       // per-field patch tables (type, values)
    std::vector<int32_t> bct[2];
    bool serial[2] = {false, false};
    int model[2] = {MPLB_NO_MODEL, MPLB_NO_MODEL};
    double* stage = nullptr;
    size_t stage_elems = 0;
    double* red = nullptr;  // reduction partials + results
    int red_parts = 0;
    FusedConfig fc{};
    int fstate = 0;  // 0: buffers hold the reference's state; 1: post-collision (fused)
    int precision = MPLB_FP64;
    float* p32[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // FP32 deviations [field][buffer]
    int cur32[2] = {0, 0};
    double rho_ref = 0, T_ref = 0;
    double* snap = nullptr;  // equilibrium monitor: density at the last check
    long long* mom = nullptr;  // FP32 equilibrium runs: total momentum now [0..2] and at the start [3..5]
    // write-step snapshot: device copy [rho | T | p | U as [node][3] | f, g
    // as [node][Q]], its pinned host image, the side stream that transfers
    // it, and events
    double* snap_dev = nullptr;
    double* snap_host = nullptr;
    size_t snap_cap = 0;  // doubles held by snap_dev and snap_host
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
    bool snap_pending = false, snap_has_p = false, snap_has_pdfs = false;
    uint32_t snap_time = 0;
    // host thread writing the last snapshot's files, and the first error of
    // the writes since the last join
    std::thread writer;
    int writer_rc = 0;
    std::string writer_err;
    int tile_request = 0;  // mplb_opts.tile_config
    uint32_t current = 0;
    // slabs on the fused path: the owned nodes (count 0 = every node), the
    // owned ranges whose step outputs also go into a neighbour's halo, and an
    // event that orders this handle's stream before a neighbour's next step
    uint32_t own_start = 0, own_count = 0;
    struct Mirror {
        uint32_t src_start, count, dst_start;
        mplb_gpu* dst;
    } mirrors[MPLB_MAX_MIRRORS] = {};
    int nmirror = 0;
    cudaEvent_t order_ev = nullptr;
    uint64_t launches = 0;
    uint64_t bytes = 0;
    bool initialized = false;

    double* F() { return pdf[0][cur[0]]; }
    double* G() { return pdf[1][cur[1]]; }
};

namespace {

template <class T>
int dalloc(mplb_gpu* h, T** p, size_t count) {
    size_t b = std::max<size_t>(count, 1) * sizeof(T);
    CK(cudaMalloc((void**)p, b));
    CK(cudaMemsetAsync(*p, 0, b, h->stream));
    h->bytes += b;
    return 0;
}

void free_all(mplb_gpu* h) {
    void* ps[] = {h->p, h->nb, h->onb, h->pdf[0][0], h->pdf[0][1], h->pdf[1][0], h->pdf[1][1], h->rho, h->T,
                  h->S, h->U, h->Fi, h->Ft, h->T2, h->U2, h->bcmap, h->pnodes, h->dpatches, h->stage,
                  h->red};
    for (void* p : ps)
        if (p) cudaFree(p);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (h->p32[i][j]) cudaFree(h->p32[i][j]);
    if (h->snap) cudaFree(h->snap);
    if (h->mom) cudaFree(h->mom);
    for (int i = 0; i < 2; i++)
        if (h->bctab[i]) cudaFree(h->bctab[i]);
}

// Does the FP32 form's momentum reset apply?  Fully periodic box without
// boundary patches and without net body force (gravity, external force).
bool momentum_conserved(const mplb_gpu* h) {
    if (h->precision != MPLB_FP32_DEV || h->path != MPLB_PATH_FUSED || !h->box || h->fc.has_bc) return false;
    for (int d = 0; d < h->D; d++)
        if (!h->per[d]) return false;
    for (int j = 0; j < 3; j++)
        if (h->P.g[j] != 0.0 || h->P.fext[j] != 0.0) return false;
    return h->P.f_update != 0;
}

// x = (1 - w) a + w x
__global__ void k_blend(uint32_t n, double w, const double* __restrict__ a, double* __restrict__ x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (1.0 - w) * a[i] + w * x[i];
}

__global__ void k_add(uint32_t n, double v, double* __restrict__ x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += v;
}

__global__ void k_fill(uint32_t n, double v, double* __restrict__ x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}

// Equilibrium monitor.  Per node the mass of the current populations, sum
// over k: after a fused step these are post-collision (the collision
// conserves mass, so the sum is the node's density), on the operator path
// post-streaming (the sum is what macroDensity computes).  Per block: the
// largest change against the snapshot of the previous call and the block's
// mass; the snapshot is refreshed.  Fixed grid and order: deterministic.
template <class T>
__global__ void k_monitor_partial(uint32_t n, int Q, const T* __restrict__ f, double ref, double* __restrict__ snap,
                                  int first, double* __restrict__ partials) {
    double m = 0.0, mass = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T s = 0;
        for (int k = 0; k < Q; k++) s += f[(size_t)k * n + i];
        const double r = ref + (double)s;
        // fmax drops NaN: a non-finite density must show as an infinite change
        if (!first) m = isfinite(r) ? fmax(m, fabs(r - snap[i])) : INFINITY;
        snap[i] = r;
        mass += r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        mass += __shfl_down_sync(0xffffffffu, mass, o);
    }
    __shared__ double sm[32], ss[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sm[w] = m;
        ss[w] = mass;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 1; j < (int)((blockDim.x + 31) >> 5); j++) {
            m = fmax(m, sm[j]);
            mass += ss[j];
        }
        partials[2 * blockIdx.x] = m;
        partials[2 * blockIdx.x + 1] = mass;
    }
}

__global__ void k_monitor_final(int nparts, const double* __restrict__ partials, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double m = 0.0, mass = 0.0;
    for (int b = 0; b < nparts; b++) {
        m = fmax(m, partials[2 * b]);
        mass += partials[2 * b + 1];
    }
    out[0] = m;
    out[1] = mass;
}

// Lattice tables on the host, the same way the reference defines them
// (D2Q9_omega.c, D2Q9_ppw.c, D3Q15_omega.c, D3Q15_ppw.c, D*_MRTInv.c).
template <class L>
void fill_tables(Params& P) {
    P.Q = L::Q;
    P.cs2 = 1.0 / 3.0;
    for (int k = 0; k < L::Q; k++) {
        int c2 = cxk<L>(k) * cxk<L>(k) + cyk<L>(k) * cyk<L>(k) + czk<L>(k) * czk<L>(k);
        if (L::Q == 9) {
            P.w[k] = c2 == 0 ? 4.0 / 9.0 : (c2 == 1 ? 1.0 / 9.0 : 1.0 / 36.0);
            P.ppw[k] = c2 == 0 ? 0.0 : (c2 == 1 ? 1.0 / 3 : 1.0 / 12);
        } else {
            P.w[k] = c2 == 0 ? 2.0 / 9.0 : (c2 == 1 ? 1.0 / 9.0 : 1.0 / 72.0);
            P.ppw[k] = c2 == 0 ? 0.0 : (c2 == 1 ? 1.0 / 3.0 : 1.0 / 24.0);
        }
    }
    for (int r = 0; r < L::Q; r++) {
        int norm = 0;
        for (int k = 0; k < L::Q; k++) norm += Mint<L>(r, k) * Mint<L>(r, k);
        for (int k = 0; k < L::Q; k++) P.Mi[k][r] = (double)Mint<L>(r, k) / (double)norm;
    }
}

int check_field(const mplb_field_desc* d, int lat, int which, uint32_t npatch, std::string& why) {
    if (!d || d->model == MPLB_NO_MODEL) return 0;
    // A frozen field is never touched by the reference (every operator checks
    // field->update first), so any model and boundary set is accepted for it.
    if (!d->update) return 0;
    if (d->surface_tension != 0 && (which != 0 || (d->model != MPLB_LIMRT && d->model != MPLB_XUMRT))) {
        why = "surface tension is a liMRT / xuMRT flow-field option";
        return MPLB_E_UNSUPPORTED;
    }
    if (which == 0) {
        if (d->model == MPLB_LIMRT && lat != MPLB_D2Q9) { why = "liMRT is D2Q9 only (liMRTForce.c:13)"; return MPLB_E_UNSUPPORTED; }
        if (d->model == MPLB_XUMRT && lat != MPLB_D3Q15) { why = "xuMRT is D3Q15 only (xuMRTForce.c:9)"; return MPLB_E_UNSUPPORTED; }
        if (d->model != MPLB_LIMRT && d->model != MPLB_XUMRT) { why = "f model must be liMRT or xuMRT"; return MPLB_E_UNSUPPORTED; }
    } else {
        if (d->model != MPLB_LITEMPMRT && d->model != MPLB_MYMRT) { why = "g model must be liTempMRT or myMRT"; return MPLB_E_UNSUPPORTED; }
        if (d->model == MPLB_LITEMPMRT && lat != MPLB_D2Q9) { why = "liTempMRT is D2Q9 only (liTempMRTEquilibriumMS.c:45-49)"; return MPLB_E_UNSUPPORTED; }
    }
    for (uint32_t p = 0; p < npatch; p++) {
        int t = d->bc_type ? d->bc_type[p] : MPLB_BC_PERIODIC;
        switch (t) {
        case MPLB_BC_PERIODIC:
        case MPLB_BC_BOUNCEBACK: break;
        case MPLB_BC_FIXEDT:
            if (d->model != MPLB_LITEMPMRT && d->model != MPLB_MYMRT) { why = "fixedT needs a liTempMRT or myMRT field (fixedT.c:57-73)"; return MPLB_E_UNSUPPORTED; }
            break;
        case MPLB_BC_FIXEDRANDOMT:
            if (d->model != MPLB_MYMRT) { why = "fixedRandomT needs the myMRT field (fixedRandomT.c:20,125)"; return MPLB_E_UNSUPPORTED; }
            break;
        case MPLB_BC_OUTFLOW: break;
        case MPLB_BC_FIXEDU: break;  // a no-op for models other than liMRT (fixedU.c:10)
        default:
            why = "boundary type " + std::to_string(t) + " is outside this path (bounceBack, fixedT, fixedU, fixedRandomT, outflow, periodic)";
            return MPLB_E_UNSUPPORTED;
        }
        if ((t == MPLB_BC_FIXEDT || t == MPLB_BC_FIXEDU || t == MPLB_BC_FIXEDRANDOMT) && !d->bc_value) { why = "bc_value missing"; return MPLB_E_ARG; }
    }
    return 0;
}

// Does the neighbour table describe an Nx x Ny x Nz box in x-fastest node
// order, each axis either wrapping or walled?  Needs coordinates.
bool detect_box(mplb_gpu* h, const mplb_mesh_desc* m) {
    if (!m->points) return false;
    int lo[3], hi[3];
    for (int j = 0; j < 3; j++) lo[j] = hi[j] = m->points[j];
    for (uint32_t i = 0; i < h->n; i++)
        for (int j = 0; j < 3; j++) {
            lo[j] = std::min(lo[j], m->points[3 * (size_t)i + j]);
            hi[j] = std::max(hi[j], m->points[3 * (size_t)i + j]);
        }
    long long d[3];
    for (int j = 0; j < 3; j++) d[j] = (long long)hi[j] - lo[j] + 1;
    if (d[0] * d[1] * d[2] != (long long)h->n) return false;
    if (h->lat == MPLB_D2Q9 && d[2] != 1) return false;
    for (uint32_t i = 0; i < h->n; i++) {
        long long x = m->points[3 * (size_t)i] - lo[0], y = m->points[3 * (size_t)i + 1] - lo[1],
                  z = m->points[3 * (size_t)i + 2] - lo[2];
        if (x + d[0] * (y + d[1] * z) != (long long)i) return false;
    }
    // Decide each axis from the first node's neighbours, then verify all.
    int per[3] = {1, 1, 1};
    for (int ax = 0; ax < 3; ax++) {
        if (d[ax] == 1) { per[ax] = 1; continue; }
        // node at coordinate 0 along ax, others 0; direction with c_ax = +1 pulls from -1.
        int k = -1;
        for (int q = 0; q < h->Q; q++) {
            int c[3] = {h->lat == MPLB_D2Q9 ? cxk<D2Q9T>(q) : cxk<D3Q15T>(q),
                        h->lat == MPLB_D2Q9 ? cyk<D2Q9T>(q) : cyk<D3Q15T>(q),
                        h->lat == MPLB_D2Q9 ? czk<D2Q9T>(q) : czk<D3Q15T>(q)};
            int ok = c[ax] == 1;
            for (int j = 0; j < 3; j++) if (j != ax && c[j] != 0) ok = 0;
            if (ok) k = q;
        }
        per[ax] = m->nb[0 * (size_t)h->Q + k] != -1;
    }
    for (uint32_t i = 0; i < h->n; i++) {
        long long x = i % d[0], y = (i / d[0]) % d[1], z = i / (d[0] * d[1]);
        for (int q = 0; q < h->Q; q++) {
            int c[3] = {h->lat == MPLB_D2Q9 ? cxk<D2Q9T>(q) : cxk<D3Q15T>(q),
                        h->lat == MPLB_D2Q9 ? cyk<D2Q9T>(q) : cyk<D3Q15T>(q),
                        h->lat == MPLB_D2Q9 ? czk<D2Q9T>(q) : czk<D3Q15T>(q)};
            long long s[3] = {x - c[0], y - c[1], z - c[2]};
            bool ok = true;
            for (int j = 0; j < 3; j++) {
                if (per[j]) s[j] = ((s[j] % d[j]) + d[j]) % d[j];
                else if (s[j] < 0 || s[j] >= d[j]) ok = false;
            }
            long long want = ok ? s[0] + d[0] * (s[1] + d[1] * s[2]) : -1;
            if (m->nb[(size_t)i * h->Q + q] != want) return false;
        }
    }
    for (int j = 0; j < 3; j++) { h->dims[j] = (int)d[j]; h->per[j] = per[j]; }
    return true;
}

// outflow.c:29-90 for one boundary node: the normal, sum of the velocities
// whose node x + c_k is missing, normalised in float as the reference does,
// and ln, the last direction equal to the normal truncated to int.  Returns
// false where no normal exists ("Unable to detect normal in outflow boundary").
bool outflow_normal(int Q, const int32_t* nb, float* normal, int* ln) {
    auto rev = [&](int k) { return Q == 9 ? revk<D2Q9T>(k) : revk<D3Q15T>(k); };
    auto c = [&](int k, int j) { return Q == 9 ? ck<D2Q9T>(k, j) : ck<D3Q15T>(k, j); };
    normal[0] = normal[1] = normal[2] = 0;
    for (int k = 0; k < Q; k++)
        if (nb[rev(k)] == -1)
            for (int j = 0; j < 3; j++) normal[j] += c(k, j);
    float nmag = 0;
    for (int j = 0; j < 3; j++) nmag += normal[j] * normal[j];
    if (nmag == 0) return false;
    nmag = (float)std::sqrt((double)nmag);
    for (int j = 0; j < 3; j++) normal[j] = normal[j] / nmag;
    *ln = 0;
    for (int k = 0; k < Q; k++)
        if (c(k, 0) == (int)normal[0] && c(k, 1) == (int)normal[1] && c(k, 2) == (int)normal[2]) *ln = k;
    return true;
}

// rand() of the GNU C library after srand(seed), which fixedRandomT calls at
// every application (fixedRandomT.c:37,81): the additive feedback generator
// r_i = r_{i-3} + r_{i-31} (mod 2^32) over 31 words seeded by the Park-Miller
// generator r_i = 16807 r_{i-1} mod (2^31 - 1) (seed 0 taken as 1), the
// first 310 outputs discarded, each output r_i >> 1 (P. Selinger, "The GLIBC
// pseudo-random number generator", 2007).
class GnuRand {
public:
    explicit GnuRand(uint32_t seed) {
        int64_t w = seed == 0 ? 1 : seed;
        r_[0] = (uint32_t)w;
        for (int i = 1; i < 31; i++) {
            w = (16807 * w) % 2147483647;
            if (w < 0) w += 2147483647;
            r_[i] = (uint32_t)w;
        }
        for (int i = 31; i < 34; i++) r_[i] = r_[i - 31];
        i_ = 34;
        for (int i = 0; i < 310; i++) next();
    }
    int next() {
        uint32_t v = r_[(i_ - 31) % 34] + r_[(i_ - 3) % 34];
        r_[i_ % 34] = v;
        i_++;
        return (int)(v >> 1);
    }

private:
    uint32_t r_[34];
    uint64_t i_;
};

// Can a field's boundary patches run one thread per node?  Not if a node
// reads a population that any boundary op writes (the reference's serial
// order would then be observable) or if a patch lists a node twice.
bool needs_serial(const mplb_gpu* h, const mplb_mesh_desc* m, int fi) {
    if (!(fi == 0 ? h->P.f_update : h->P.g_update)) return false;
    const int Q = h->Q;
    const int nax = Q == 9 ? 4 : 6;
    auto rev = [&](int k) { return Q == 9 ? revk<D2Q9T>(k) : revk<D3Q15T>(k); };
    std::unordered_set<uint64_t> writes;
    std::vector<uint64_t> reads;
    size_t off = 0;
    for (uint32_t p = 0; p < m->n_patches; p++) {
        int t = h->bct[fi][p];
        std::unordered_set<uint32_t> seen;
        for (uint32_t i = 0; i < m->patch_count[p]; i++) {
            uint32_t id = m->patch_nodes[off + i];
            if (t == MPLB_BC_PERIODIC || (t == MPLB_BC_FIXEDU && h->model[fi] != MPLB_LIMRT)) continue;
            if (!seen.insert(id).second) return true;
            const int32_t* nb = m->nb + (size_t)id * Q;
            for (int k = 0; k < Q; k++) {
                if (t == MPLB_BC_BOUNCEBACK) {
                    if (nb[k] == -1) writes.insert((uint64_t)id * Q + k);
                    else if (nb[rev(k)] != -1 && k >= 1 && k <= nax) {
                        writes.insert((uint64_t)id * Q + k);
                        writes.insert((uint64_t)id * Q + rev(k));
                    }
                } else if (t == MPLB_BC_OUTFLOW) {
                    if (nb[k] == -1) writes.insert((uint64_t)id * Q + k);
                } else if (nb[k] == -1 && nb[rev(k)] != -1) {
                    uint32_t nbid = (uint32_t)nb[rev(k)];
                    writes.insert((uint64_t)id * Q + k);
                    if (t == MPLB_BC_FIXEDT || t == MPLB_BC_FIXEDRANDOMT) reads.push_back((uint64_t)nbid * Q + k);
                    else
                        for (int q = 0; q < Q; q++) reads.push_back((uint64_t)nbid * Q + q);
                }
            }
            if (t == MPLB_BC_OUTFLOW) {
                // outflow.c:93-175: every population of the inner neighbour along the normal
                int ln;
                float nrm[3];
                if (outflow_normal(Q, nb, nrm, &ln)) {
                    int32_t m = nb[ln];
                    if (m != -1)
                        for (int q = 0; q < Q; q++) reads.push_back((uint64_t)m * Q + q);
                }
            }
        }
        off += m->patch_count[p];
    }
    for (uint64_t r : reads)
        if (writes.count(r)) return true;
    return false;
}

int launch_check(mplb_gpu* h) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return 0;
}

#define LAUNCH(kernel, grid, ...)                                    \
    do {                                                             \
        kernel<<<(grid), TPB, 0, h->stream>>>(__VA_ARGS__);          \
        h->launches++;                                               \
        if (int rc_ = launch_check(h)) return rc_;                   \
    } while (0)

// --------------------------------------------------------------- operators
template <class L>
int op_equilibrium(mplb_gpu* h, int fi) {
    if (h->model[fi] == MPLB_NO_MODEL || !(fi == 0 ? h->P.f_update : h->P.g_update)) return 0;
    if (fi == 0) LAUNCH(k_equilibrium_flow<L>, blocks(h->n), h->P, h->F(), h->rho, h->U);
    else LAUNCH(k_equilibrium_heat<L>, blocks(h->n), h->P, h->G(), h->T, h->U);
    return 0;
}

template <class L>
int op_collision(mplb_gpu* h, int fi) {
    if (h->model[fi] == MPLB_NO_MODEL || !(fi == 0 ? h->P.f_update : h->P.g_update)) return 0;
    if (fi == 0) LAUNCH(k_collide_flow<L>, blocks(h->n), h->P, h->F(), h->rho, h->U, h->T, h->Fi, h->Ft, h->nb);
    else LAUNCH(k_collide_heat<L>, blocks(h->n), h->P, h->G(), h->T, h->U, h->S);
    return 0;
}

template <class L>
int op_stream(mplb_gpu* h, int fi) {
    if (h->model[fi] == MPLB_NO_MODEL || !(fi == 0 ? h->P.f_update : h->P.g_update)) return 0;
    double* in = h->pdf[fi][h->cur[fi]];
    double* out = h->pdf[fi][h->cur[fi] ^ 1];
    LAUNCH(k_stream<L::Q>, blocks(h->n), h->n, out, in, h->nb);
    h->cur[fi] ^= 1;
    return 0;
}

template <class L>
int op_boundaries(mplb_gpu* h, int fi) {
    if (h->model[fi] == MPLB_NO_MODEL || !(fi == 0 ? h->P.f_update : h->P.g_update)) return 0;
    double* pdf = h->pdf[fi][h->cur[fi]];
    const std::vector<PatchDev>& pts = h->fpatch[fi];
    bool any = false;
    for (const PatchDev& pt : pts) {
        if (pt.type == MPLB_BC_PERIODIC || (pt.type == MPLB_BC_FIXEDU && h->model[fi] != MPLB_LIMRT)) continue;
        any = true;
    }
    if (!any) return 0;
    // fixedRandomT: the first psteps - localTStep updates are perturbed
    // (fixedRandomT.c:79,117); one update per call, as updateBoundaries
    unsigned long long rnd = 0;
    for (size_t p = 0; p < pts.size(); p++)
        if (pts[p].type == MPLB_BC_FIXEDRANDOMT && (int64_t)h->bc_calls[fi] < h->rnd_left[fi][p]) rnd |= 1ull << p;
    h->bc_calls[fi]++;
    if (h->serial[fi]) {
        LAUNCH(k_bc_serial<L>, 1, h->P, h->dpatches + fi * pts.size(), (int)pts.size(), h->model[fi],
               h->pnodes, pdf, h->nb, h->rho, h->T, h->U, h->Fi, h->bctab[fi], rnd);
        return 0;
    }
    for (size_t p = 0; p < pts.size(); p++) {
        const PatchDev& pt = pts[p];
        if (pt.type == MPLB_BC_PERIODIC || pt.count == 0) continue;
        if (pt.type == MPLB_BC_FIXEDU && h->model[fi] != MPLB_LIMRT) continue;
        LAUNCH(k_bc_patch<L>, blocks(pt.count), h->P, pt, h->model[fi], h->pnodes, pdf, h->nb, h->rho,
               h->T, h->U, h->Fi, h->bctab[fi], (int)((rnd >> p) & 1ull));
    }
    return 0;
}

template <class L>
int op_density(mplb_gpu* h, uint32_t s, uint32_t e) {
    if (h->model[0] == MPLB_NO_MODEL || !h->P.f_update || e <= s) return 0;
    LAUNCH(k_moment0<L::Q>, blocks(e - s), h->n, h->rho, h->F(), s, e);
    return 0;
}

template <class L>
int op_temperature(mplb_gpu* h, uint32_t s, uint32_t e) {
    if (h->model[1] == MPLB_NO_MODEL || !h->P.g_update || e <= s) return 0;
    if (h->model[1] == MPLB_MYMRT) LAUNCH(k_temperature_my<L::Q>, blocks(e - s), h->n, h->T, h->G(), h->S, s, e);
    else LAUNCH(k_moment0<L::Q>, blocks(e - s), h->n, h->T, h->G(), s, e);
    return 0;
}

template <class L>
int op_velocity(mplb_gpu* h, uint32_t s, uint32_t e) {
    if (h->model[0] == MPLB_NO_MODEL || !h->P.f_update || e <= s) return 0;
    LAUNCH(k_velocity<L>, blocks(e - s), h->P, h->U, h->F(), h->rho, h->Fi, h->Ft, s, e);
    return 0;
}

template <class L>
int op_interforce(mplb_gpu* h) {
    LAUNCH(k_interforce<L>, blocks(h->n), h->P, h->Fi, h->Ft, h->rho, h->T, h->nb, h->onb);
    return 0;
}

template <class L>
int op_heatsource(mplb_gpu* h) {
    if (h->model[1] == MPLB_NO_MODEL || !h->P.g_update) return 0;
    LAUNCH(k_heatsource<L>, blocks(h->n), h->P, h->S, h->rho, h->T, h->U, h->nb, h->current == 0 ? 1 : 0);
    return 0;
}

#define RET(x) do { if (int rc_ = (x)) return rc_; } while (0)

template <class L>
int op_pressure(mplb_gpu* h) {
    if (!h->P.f_update) return 0;
    LAUNCH(k_pressure<L>, blocks(h->n), h->P, h->p, h->rho, h->T, h->nb);
    return 0;
}

// multiPhasePP.c:157-240, one operator after another.
template <class L>
int step_operators(mplb_gpu* h) {
    ++h->current;
    RET(op_collision<L>(h, 0));
    RET(op_stream<L>(h, 0));
    RET(op_boundaries<L>(h, 0));
    RET(op_collision<L>(h, 1));
    RET(op_stream<L>(h, 1));
    RET(op_boundaries<L>(h, 1));
    RET(op_density<L>(h, 0, h->n));
    if (h->P.g_update) RET(op_heatsource<L>(h));
    RET(op_temperature<L>(h, 0, h->n));
    if (h->P.f_update) RET(op_interforce<L>(h));
    RET(op_velocity<L>(h, 0, h->n));
    return 0;
}

template <class L>
int initialize_impl(mplb_gpu* h) {
    RET(op_equilibrium<L>(h, 0));
    RET(op_equilibrium<L>(h, 1));
    RET(op_interforce<L>(h));
    RET(op_heatsource<L>(h));
    h->initialized = true;
    return 0;
}

#define DISPATCH(h, fn, ...) \
    ((h)->lat == MPLB_D2Q9 ? fn<D2Q9T>(__VA_ARGS__) : fn<D3Q15T>(__VA_ARGS__))

int staging(mplb_gpu* h, size_t elems) {
    if (h->stage_elems >= elems) return 0;
    if (h->stage) { cudaFree(h->stage); h->bytes -= h->stage_elems * sizeof(double); }
    h->stage = nullptr;
    h->stage_elems = 0;
    CK(cudaMalloc((void**)&h->stage, elems * sizeof(double)));
    h->stage_elems = elems;
    h->bytes += elems * sizeof(double);
    return 0;
}

int put_aos(mplb_gpu* h, const double* host, double* dev, int m) {
    if (!host) return 0;
    size_t e = (size_t)h->n * m;
    RET(staging(h, e));
    CK(cudaMemcpyAsync(h->stage, host, e * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    LAUNCH(k_aos_to_soa, blocks(e), h->n, m, h->stage, dev);
    return 0;
}

// Device-to-host copies of one field, queued on the handle's stream (the
// caller synchronises once after the last one).  get_aos transposes through
// the staging buffer, which the caller has sized for the largest field so
// that no reallocation happens between queued copies; stream order keeps the
// next transpose behind the previous copy out of it.
int get_aos(mplb_gpu* h, double* host, const double* dev, int m, bool sync = true) {
    if (!host) return 0;
    size_t e = (size_t)h->n * m;
    RET(staging(h, e));
    LAUNCH(k_soa_to_aos, blocks(e), h->n, m, dev, h->stage);
    CK(cudaMemcpyAsync(host, h->stage, e * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (sync) CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int get_scalar(mplb_gpu* h, double* host, const double* dev, bool sync = true) {
    if (!host) return 0;
    CK(cudaMemcpyAsync(host, dev, (size_t)h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (sync) CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int put_scalar(mplb_gpu* h, const double* host, double* dev) {
    if (!host) return 0;
    CK(cudaMemcpyAsync(dev, host, (size_t)h->n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return 0;
}

// Waits for the snapshot writer thread, if one runs; its status stays in
// writer_rc for the next join.
void writer_wait(mplb_gpu* h) {
    if (h->writer.joinable()) h->writer.join();
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

// A bounded wait inside a fused kernel that ran out leaves MPLB_KERR_WAIT in
// the handle's kernel flag; the steps before the check are not valid.
// queue_kernel_flag() queues the flag's read on the stream; after the
// caller has synchronised the stream, kernel_flag_status() reports it.
int queue_kernel_flag(mplb_gpu* h) {
    if (h->path != MPLB_PATH_FUSED) return 0;
    if (!fused_queue_kerr(h->fc, h->stream)) return fail(MPLB_E_CUDA, "queueing the kernel flag read failed");
    return 0;
}
int kernel_flag_status(mplb_gpu* h) {
    if (h->path != MPLB_PATH_FUSED || !fused_kerr_value(h->fc)) return 0;
    *h->fc.kerr_host = 0;
    return fail(MPLB_E_TIMEOUT, "a bounded wait inside a fused step kernel ran out (TMA plane copy not "
                                "complete); the steps before this call are not valid");
}

// Order `waiter`'s stream after the work queued so far on `h`'s stream (no
// host wait; nothing to do on one stream).
int order_streams(mplb_gpu* h, mplb_gpu* waiter) {
    if (h->dev == waiter->dev && h->stream == waiter->stream) return 0;
    {
        DeviceGuard guard(h->dev);
        if (!h->order_ev) CK(cudaEventCreateWithFlags(&h->order_ev, cudaEventDisableTiming));
        CK(cudaEventRecord(h->order_ev, h->stream));
    }
    DeviceGuard guard(waiter->dev);
    CK(cudaStreamWaitEvent(waiter->stream, h->order_ev, 0));
    return 0;
}

// Slabs: the mirrored ranges of this step.  A neighbour that has not yet
// taken this step (same time) receives into the buffers its step writes and
// the step after reads; one that has (one step ahead) into its current
// buffers.  This handle's step is queued after the neighbours' queued work:
// their last step reads and writes the buffers this step writes into, and
// wrote this handle's halo.
int mirror_args(mplb_gpu* h, FusedArgs& A, bool fon, bool gon) {
    const bool udb = fon && gon;
    A.nmirror = h->nmirror;
    for (int m = 0; m < h->nmirror; m++) {
        const mplb_gpu::Mirror& M = h->mirrors[m];
        mplb_gpu* d = M.dst;
        if (d->path != MPLB_PATH_FUSED || d->fstate == 0)
            return fail(MPLB_E_STATE, "a mirror's neighbour is not in the fused state (exchange its state once, "
                                      "mplb_gpu_copy_state, before the first mirrored step)");
        if (d->current != h->current && d->current != h->current + 1)
            return fail(MPLB_E_STATE, "a mirror's neighbour is not at this step's time or one step ahead (linked "
                                      "slabs take one step each, in turn)");
        const uint64_t dlo = d->own_start, dhi = dlo + (d->own_count ? d->own_count : d->n);
        if ((uint64_t)M.dst_start < dhi && dlo < (uint64_t)M.dst_start + M.count)
            return fail(MPLB_E_STATE, "a mirror's target overlaps the neighbour's owned range");
        const int nx = d->current == h->current ? 1 : 0;  // 1: the buffers its coming step writes
        MirrorRange& R = A.mirror[m];
        R.lo = M.src_start;
        R.cnt = M.count;
        R.dst = M.dst_start;
        R.n_dst = d->n;
        R.f = fon ? d->pdf[0][d->cur[0] ^ nx] : nullptr;
        R.g = gon ? d->pdf[1][d->cur[1] ^ nx] : nullptr;
        R.T = gon ? (nx ? d->T2 : d->T) : nullptr;
        R.U = udb ? (nx ? d->U2 : d->U) : nullptr;
        RET(order_streams(d, h));
    }
    return 0;
}

// ... and the neighbours' next steps after this one (it wrote their halos).
int mirror_order_after(mplb_gpu* h) {
    for (int m = 0; m < h->nmirror; m++) RET(order_streams(h, h->mirrors[m].dst));
    return 0;
}

// One fused time step, or (emit) the rebuild of the reference state after
// the last step from that step's retained input buffers.
int fused_step(mplb_gpu* h, bool emit) {
    const bool fon = h->P.f_update != 0, gon = h->P.g_update != 0;
    FusedArgs A = h->fc.args;
    const int c0 = h->cur[0], c1 = h->cur[1];
    if (fon) {
        A.fin = emit ? h->pdf[0][c0 ^ 1] : h->pdf[0][c0];
        A.fout = emit ? h->pdf[0][c0] : h->pdf[0][c0 ^ 1];
    }
    if (gon) {
        A.gin = emit ? h->pdf[1][c1 ^ 1] : h->pdf[1][c1];
        A.gout = emit ? h->pdf[1][c1] : h->pdf[1][c1 ^ 1];
    }
    const bool udb = fon && gon;  // U double-buffered (the heat source reads U_{n-1})
    A.Told = gon ? (emit ? h->T2 : h->T) : h->T;
    A.Tnew = gon ? h->T2 : nullptr;
    A.Uold = udb ? (emit ? h->U2 : h->U) : h->U;
    A.Unew = udb ? (emit ? h->U : h->U2) : h->U;
    A.S = h->S;
    A.rho_c = h->rho;
    A.rho_out = h->rho;
    A.Fi_out = h->Fi;
    A.Ft_out = h->Ft;
    if (!emit && h->own_count) {
        A.own_lo = h->own_start;
        A.own_cnt = h->own_count;
    }
    if (!emit && h->nmirror) RET(mirror_args(h, A, fon, gon));
    if (!emit && !h->fc.tuned) {
        if (h->tile_request == 0) {
            RET(staging(h, h->n));
            if (int rc = fused_autotune(h->fc, h->P, A, fon, gon, h->S, h->stage, h->n, h->stream))
                return fail(rc, h->fc.err);
        } else {
            int c = h->tile_request > 0 ? h->tile_request - 1 : 0;
            if (c >= h->fc.ncfg) return fail(MPLB_E_ARG, "tile_config out of range");
            if (h->fc.geom[c].nblocks == 0)
                return fail(MPLB_E_ARG, "tile_config " + std::to_string(h->tile_request) + " does not take this lattice");
            h->fc.cfg = c;
            h->fc.tuned = true;
        }
    }
    cudaError_t e = fused_launch(h->fc, h->P, A, h->lat, fon, gon, emit, h->stream);
    h->launches++;
    if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("fused kernel launch: ") + cudaGetErrorString(e));
    if (!emit && h->nmirror) RET(mirror_order_after(h));
    if (!emit) {
        if (fon) h->cur[0] ^= 1;
        if (gon) {
            h->cur[1] ^= 1;
            std::swap(h->T, h->T2);
        }
        if (udb) std::swap(h->U, h->U2);
    }
    return 0;
}

// FP32-deviation step (or emit: rebuild the FP64 reference state).
int fused32_step(mplb_gpu* h, bool emit) {
    const bool fon = h->P.f_update != 0, gon = h->P.g_update != 0;
    FusedArgs32 B = mplb_make_args32(h->fc.args, h->P, h->rho_ref, h->T_ref);
    const int c0 = h->cur32[0], c1 = h->cur32[1];
    if (fon) {
        B.fin = emit ? h->p32[0][c0 ^ 1] : h->p32[0][c0];
        B.fout = emit ? nullptr : h->p32[0][c0 ^ 1];
    }
    if (gon) {
        B.gin = emit ? h->p32[1][c1 ^ 1] : h->p32[1][c1];
        B.gout = emit ? nullptr : h->p32[1][c1 ^ 1];
    }
    const bool udb = fon && gon;
    B.Told = gon ? (emit ? h->T2 : h->T) : h->T;
    B.Tnew = gon ? (emit ? h->T : h->T2) : nullptr;
    B.Uold = udb ? (emit ? h->U2 : h->U) : h->U;
    B.Unew = udb ? (emit ? h->U : h->U2) : h->U;
    B.S = h->S;
    B.rho_c = h->rho;
    cudaError_t e = mplb_fused32_launch(h->lat, h->fc.has_bc, fon, gon, emit, B, h->P, fon ? h->F() : nullptr,
                                        gon ? h->G() : nullptr, h->rho, h->Fi, h->Ft, h->stream);
    h->launches++;
    if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("FP32 fused kernel launch: ") + cudaGetErrorString(e));
    if (!emit) {
        if (fon) h->cur32[0] ^= 1;
        if (gon) {
            h->cur32[1] ^= 1;
            std::swap(h->T, h->T2);
        }
        if (udb) std::swap(h->U, h->U2);
    }
    return 0;
}

// FP64 reference state -> FP32 post-collision deviations.  The reference
// values are the lattice means of rho and T (any value is valid; the mean
// keeps deviations small).
int prologue32(mplb_gpu* h) {
    const int parts = std::min<int>(h->red_parts, (int)blocks(h->n));
    k_sum2_partial<<<parts, TPB, 0, h->stream>>>(h->n, h->rho, h->T, h->red);
    k_sum2_final<<<1, TPB, 0, h->stream>>>(parts, h->red, h->red + 2 * h->red_parts);
    h->launches += 2;
    RET(launch_check(h));
    double r[2] = {0, 0};
    CK(cudaMemcpyAsync(r, h->red + 2 * h->red_parts, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->rho_ref = r[0] / h->n;
    h->T_ref = r[1] / h->n;
    RET(DISPATCH(h, op_collision, h, 0));
    RET(DISPATCH(h, op_collision, h, 1));
    FusedArgs32 B = mplb_make_args32(h->fc.args, h->P, h->rho_ref, h->T_ref);
    for (int fi = 0; fi < 2; fi++) {
        if (!(fi == 0 ? h->P.f_update : h->P.g_update)) continue;
        cudaError_t e = mplb_to_dev32(h->n, h->Q, h->pdf[fi][h->cur[fi]], h->p32[fi][h->cur32[fi]], B, fi, h->stream);
        h->launches++;
        if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("FP32 conversion: ") + cudaGetErrorString(e));
    }
    h->fstate = 1;
    return 0;
}

// Bring the buffers back to the reference's state (after the last step).
// Enter the fused path's state (post-collision populations) from the
// reference's: the first collision of the loop (multiPhasePP.c:163,194).
int enter_fused(mplb_gpu* h) {
    if (h->path != MPLB_PATH_FUSED || h->precision != MPLB_FP64 || h->fstate == 1) return 0;
    RET(DISPATCH(h, op_collision, h, 0));
    RET(DISPATCH(h, op_collision, h, 1));
    h->fstate = 1;
    return 0;
}

// One strided node copy: `rows` component rows of a [component][node] array.
struct NodeCopy {
    double* d;
    const double* s;
    int rows;
};
int copy_node_rows(mplb_gpu* dst, uint32_t dst_start, mplb_gpu* src, uint32_t src_start, uint32_t count,
                   const NodeCopy* parts, int np);

int materialize(mplb_gpu* h) {
    if (h->fstate == 0) return 0;
    if (h->precision == MPLB_FP32_DEV) RET(fused32_step(h, true));
    else RET(fused_step(h, true));
    h->fstate = 0;
    return 0;
}

}  // namespace

// Error text for the library's other translation units.
int mplb_internal_fail(int code, const std::string& msg) { return fail(code, msg); }

// ================================================================= C-ABI
extern "C" {

const char* mplb_gpu_version(void) { return "multiphaselb-b200 ABI " MPLB_STR(MPLB_ABI_VERSION) " (sm_100a, FP64)"; }
const char* mplb_gpu_last_error(void) { return g_err.c_str(); }

int mplb_gpu_create(const mplb_mesh_desc* mesh, const mplb_eos_desc* eos, const mplb_field_desc* f,
                    const mplb_field_desc* g, const mplb_opts* opts, mplb_gpu_t** out) {
    if (!out) return fail(MPLB_E_ARG, "out is NULL");
    *out = nullptr;
    if (!mesh || !eos) return fail(MPLB_E_ARG, "mesh and eos descriptors are required");
    if (mesh->lattice != MPLB_D2Q9 && mesh->lattice != MPLB_D3Q15) return fail(MPLB_E_ARG, "unknown lattice");
    if (mesh->n_points == 0 || !mesh->nb) return fail(MPLB_E_ARG, "empty mesh");
    if (mesh->n_patches > MPLB_MAX_PATCHES) return fail(MPLB_E_ARG, "too many boundary patches");
    if (mesh->n_patches && (!mesh->patch_count || !mesh->patch_nodes)) return fail(MPLB_E_ARG, "patch lists missing");
    if (eos->type < MPLB_EOS_IDEAL || eos->type > MPLB_EOS_VDW) return fail(MPLB_E_ARG, "unknown EOS");
    if (opts && opts->precision != MPLB_FP64 && opts->precision != MPLB_FP32_DEV)
        return fail(MPLB_E_ARG, "unknown precision");
    const int Q = mesh->lattice == MPLB_D2Q9 ? 9 : 15;
    const size_t nq = (size_t)mesh->n_points * Q;
    for (size_t i = 0; i < nq; i++)
        if (mesh->nb[i] < -1 || mesh->nb[i] >= (int64_t)mesh->n_points)
            return fail(MPLB_E_ARG, "neighbour index out of range at entry " + std::to_string(i));
    size_t tot = 0;
    for (uint32_t p = 0; p < mesh->n_patches; p++) tot += mesh->patch_count[p];
    for (size_t i = 0; i < tot; i++)
        if (mesh->patch_nodes[i] >= mesh->n_points) return fail(MPLB_E_ARG, "boundary node out of range");
    std::string why;
    if (int rc = check_field(f, mesh->lattice, 0, mesh->n_patches, why)) return fail(rc, why);
    if (int rc = check_field(g, mesh->lattice, 1, mesh->n_patches, why)) return fail(rc, why);

    mplb_gpu* h = new mplb_gpu();
    h->lat = mesh->lattice;
    h->Q = Q;
    h->D = Q == 9 ? 2 : 3;
    h->n = mesh->n_points;
    h->current = opts ? opts->start_time : 0;
    h->tile_request = opts ? opts->tile_config : 0;
    h->precision = opts ? opts->precision : MPLB_FP64;
    int want_path = opts ? opts->path : MPLB_PATH_AUTO;
    int dev = opts ? opts->device : -1;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) { delete h; return fail(MPLB_E_CUDA, "no CUDA device"); }
    }
    h->dev = dev;
    DeviceGuard guard(dev);
    if (cudaSetDevice(dev) != cudaSuccess) { delete h; return fail(MPLB_E_CUDA, "cudaSetDevice failed"); }
    if (opts && opts->stream) {
        h->stream = (cudaStream_t)opts->stream;
    } else {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete h;
            return fail(MPLB_E_CUDA, "stream creation failed");
        }
        h->own_stream = true;
    }

    // Parameter block.
    Params& P = h->P;
    P.lat = h->lat;
    P.n = h->n;
    if (h->lat == MPLB_D2Q9) fill_tables<D2Q9T>(P);
    else fill_tables<D3Q15T>(P);
    h->model[0] = f ? f->model : MPLB_NO_MODEL;
    h->model[1] = g ? g->model : MPLB_NO_MODEL;
    P.f_model = h->model[0];
    P.g_model = h->model[1];
    P.f_update = (f && f->model != MPLB_NO_MODEL && f->update) ? 1 : 0;
    P.g_update = (g && g->model != MPLB_NO_MODEL && g->update) ? 1 : 0;
    if (f && f->model != MPLB_NO_MODEL) {
        for (int k = 0; k < MPLB_MAX_Q; k++) {
            P.Lf[k] = f->Lambda[k];
            P.relax_f[k] = (1 - 0.5 * f->Lambda[k]);
        }
        P.s1_den = ((1 / f->Lambda[1]) - 0.5);
        P.s2_den = ((1 / f->Lambda[2]) - 0.5);
        P.sig12 = 12 * f->sigma;
        P.sig6 = 6.0 * f->sigma;
        P.sigma_p = f->sigma;
        P.st_on = (f->update && f->surface_tension) ? 1 : 0;
        P.kappa_st = f->kappa_st;
    }
    if (g && g->model != MPLB_NO_MODEL) {
        for (int k = 0; k < MPLB_MAX_Q; k++) P.Lg[k] = g->Lambda[k];
        P.corr3 = (1 - g->Lambda[3] / 2) * g->Lambda[4];
        P.corr5 = (1 - g->Lambda[5] / 2) * g->Lambda[6];
        P.lam_fac = (1 / g->Lambda[3] - 0.5);
        if (g->model == MPLB_MYMRT) {
            // myMRTCollision.c:47-140 and heatSource.c:36-48, evaluated as there
            P.my_a1 = g->alpha_1;
            P.my_a2 = g->alpha_2;
            P.my_qo[0] = g->Lambda[4] * (g->Lambda[3] / 2.0 - 1.0);
            P.my_qo[1] = g->Lambda[6] * (g->Lambda[5] / 2.0 - 1.0);
            P.my_qo[2] = h->lat == MPLB_D3Q15 ? g->Lambda[8] * (g->Lambda[7] / 2.0 - 1.0) : 0.0;
            P.my_qa0 = 1.0 + -0.5 * g->Lambda[0];
            if (h->lat == MPLB_D2Q9) {
                P.my_lgeo = 4.0 + 3.0 * g->alpha_1 + 2.0 * g->alpha_2;
                P.my_ldiv = 6.0;
            } else {
                P.my_lgeo = 6.0 + 11.0 * g->alpha_1 + g->alpha_2;
                P.my_ldiv = 9.0;
            }
        }
    }
    P.eos = eos->type;
    P.a = eos->a;
    P.b = eos->b;
    P.R = eos->R;
    P.G = eos->G;
    P.M = eos->M;
    P.Cv = eos->Cv;
    P.rho_0 = eos->rho_0;
    for (int j = 0; j < 3; j++) { P.g[j] = eos->g[j]; P.fext[j] = eos->fext[j]; }
    P.g_neg1 = eos->G == -1.0;
    P.cv_one = eos->Cv == 1.0;
    P.m2_one = eos->M * eos->M == 1.0;
    if (eos->type == MPLB_EOS_PR) {
        P.pr_tc = 0.170151343 * eos->a / (eos->b * eos->R);
        P.pr_kappa = 0.37464 + 1.5422 * eos->w - 0.26992 * eos->w * eos->w;
    }

    // Boundary tables per field.
    const mplb_field_desc* fds[2] = {f, g};
    for (int fi = 0; fi < 2; fi++) {
        h->bct[fi].assign(mesh->n_patches, MPLB_BC_PERIODIC);
        if (fds[fi] && fds[fi]->model != MPLB_NO_MODEL && fds[fi]->bc_type)
            for (uint32_t p = 0; p < mesh->n_patches; p++) h->bct[fi][p] = fds[fi]->bc_type[p];
    }
    for (int fi = 0; fi < 2; fi++) {
        uint32_t off = 0;
        for (uint32_t p = 0; p < mesh->n_patches; p++) {
            PatchDev d{};
            d.off = off;
            d.count = mesh->patch_count[p];
            d.type = h->bct[fi][p];
            if (fds[fi] && fds[fi]->model != MPLB_NO_MODEL && fds[fi]->bc_value)
                for (int j = 0; j < 3; j++) d.val[j] = fds[fi]->bc_value[3 * p + j];
            h->fpatch[fi].push_back(d);
            off += mesh->patch_count[p];
        }
    }
    // outflow normals and fixedRandomT wall temperatures, per field
    std::vector<double> tabs[2];
    const int32_t rank = opts ? opts->rank : 0;
    for (int fi = 0; fi < 2; fi++) {
        h->rnd_left[fi].assign(mesh->n_patches, 0);
        if (!fds[fi] || fds[fi]->model == MPLB_NO_MODEL || !fds[fi]->update) continue;
        for (uint32_t p = 0; p < mesh->n_patches; p++) {
            const int t = h->bct[fi][p];
            if (t != MPLB_BC_OUTFLOW && t != MPLB_BC_FIXEDRANDOMT) continue;
            if (tabs[fi].empty()) tabs[fi].assign(std::max<size_t>(tot, 1) * Q, 0.0);
            const PatchDev& pt = h->fpatch[fi][p];
            if (t == MPLB_BC_OUTFLOW) {
                for (uint32_t i = 0; i < pt.count; i++) {
                    const uint32_t id = mesh->patch_nodes[pt.off + i];
                    float nrm[3];
                    int ln;
                    if (!outflow_normal(Q, mesh->nb + (size_t)id * Q, nrm, &ln)) {
                        if (h->own_stream) cudaStreamDestroy(h->stream);
                        delete h;
                        return fail(MPLB_E_ARG, "Unable to detect normal in outflow boundary (node " +
                                                    std::to_string(id) + ", outflow.c:67-71)");
                    }
                    double* row = tabs[fi].data() + (size_t)(pt.off + i) * Q;
                    for (int j = 0; j < 3; j++) row[j] = (double)nrm[j];
                    row[3] = ln;
                }
            } else {
                // fixedRandomT.c:37-41,79-85: srand(pid) at every call, so
                // every perturbed update draws the same sequence, one value
                // per (node, missing direction with an inner neighbour)
                const double T0 = pt.val[0], pc = pt.val[1];
                const double minT = T0 * (100.0 - pc) / 100.0, maxT = T0 * (100.0 + pc) / 100.0;
                h->rnd_left[fi][p] = (int64_t)pt.val[2];
                GnuRand rng((uint32_t)rank);
                for (uint32_t i = 0; i < pt.count; i++) {
                    const uint32_t id = mesh->patch_nodes[pt.off + i];
                    const int32_t* nbi = mesh->nb + (size_t)id * Q;
                    double* row = tabs[fi].data() + (size_t)(pt.off + i) * Q;
                    for (int k = 0; k < Q; k++) {
                        if (nbi[k] != -1) continue;
                        const int r = Q == 9 ? revk<D2Q9T>(k) : revk<D3Q15T>(k);
                        if (nbi[r] == -1) continue;
                        const double u = (double)rng.next() / 2147483647;
                        row[k] = minT + (maxT - minT) * u;
                    }
                }
            }
        }
    }
    for (int fi = 0; fi < 2; fi++) h->serial[fi] = needs_serial(h, mesh, fi);
    h->box = detect_box(h, mesh);

    // Device buffers.
    int rc = 0;
    auto bail = [&](int code) {
        std::string keep = g_err;
        free_all(h);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        delete h;
        g_err = keep;
        return code;
    };
    if ((rc = dalloc(h, &h->nb, nq)) || (rc = dalloc(h, &h->onb, h->n)) || (rc = dalloc(h, &h->rho, h->n)) ||
        (rc = dalloc(h, &h->T, h->n)) || (rc = dalloc(h, &h->S, h->n)) || (rc = dalloc(h, &h->p, h->n)) || (rc = dalloc(h, &h->U, 3 * (size_t)h->n)) ||
        (rc = dalloc(h, &h->Fi, 3 * (size_t)h->n)) || (rc = dalloc(h, &h->Ft, 3 * (size_t)h->n)) ||
        (rc = dalloc(h, &h->pnodes, tot)) || (rc = dalloc(h, &h->dpatches, 2 * std::max<size_t>(1, mesh->n_patches))))
        return bail(rc);
    for (int fi = 0; fi < 2; fi++) {
        if (h->model[fi] == MPLB_NO_MODEL) continue;
        if ((rc = dalloc(h, &h->pdf[fi][0], nq)) || (rc = dalloc(h, &h->pdf[fi][1], nq))) return bail(rc);
    }
    // Create-time tables go to the device on the handle's own stream, which
    // does not wait for the legacy default stream: a synchronous cudaMemcpy
    // from pageable memory may return before its DMA lands, and a kernel on a
    // non-blocking stream could then read the old contents.  Stream order plus
    // one synchronisation before create returns.
    auto to_dev = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream) == cudaSuccess;
    };
    for (int fi = 0; fi < 2; fi++) {
        if (tabs[fi].empty()) continue;
        if ((rc = dalloc(h, &h->bctab[fi], tabs[fi].size()))) return bail(rc);
        if (!to_dev(h->bctab[fi], tabs[fi].data(), tabs[fi].size() * sizeof(double)))
            return bail(fail(MPLB_E_CUDA, "copying the boundary tables failed"));
    }
    {
        // neighbour table to [k][n], boundary flags
        std::vector<int32_t> nbs(nq);
        std::vector<uint8_t> onb(h->n, 0);
        for (uint32_t i = 0; i < h->n; i++)
            for (int k = 0; k < Q; k++) {
                int32_t s = mesh->nb[(size_t)i * Q + k];
                nbs[(size_t)k * h->n + i] = s;
                if (s == -1) onb[i] = 1;  // readLatticeMesh.c:171-203
            }
        if (!to_dev(h->nb, nbs.data(), nq * sizeof(int32_t)) || !to_dev(h->onb, onb.data(), h->n) ||
            (tot && !to_dev(h->pnodes, mesh->patch_nodes, tot * sizeof(uint32_t))))
            return bail(fail(MPLB_E_CUDA, "copying the mesh failed"));
        std::vector<PatchDev> both(h->fpatch[0]);
        both.insert(both.end(), h->fpatch[1].begin(), h->fpatch[1].end());
        if (!both.empty() && !to_dev(h->dpatches, both.data(), both.size() * sizeof(PatchDev)))
            return bail(fail(MPLB_E_CUDA, "copying the patches failed"));
        // the host vectors above go out of scope here
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bail(fail(MPLB_E_CUDA, "copying the mesh failed"));
    }
    // Execution path.
    std::string fwhy;
    bool fusable = h->box && fused_supported(h->lat, h->model, h->P, h->fpatch, h->serial, mesh, h->dims, h->per, fwhy);
    if ((want_path == MPLB_PATH_FUSED || h->precision == MPLB_FP32_DEV) && !fusable)
        return bail(fail(MPLB_E_UNSUPPORTED, std::string(h->precision == MPLB_FP32_DEV ? "FP32-deviation storage needs the fused box path; " : "") +
                                                 "fused path unavailable: " + (h->box ? fwhy : std::string("mesh is not a box"))));
    if (h->precision == MPLB_FP32_DEV && h->P.st_on)
        return bail(fail(MPLB_E_UNSUPPORTED, "FP32-deviation storage has no surface-tension term"));
    if (h->precision == MPLB_FP32_DEV && h->model[1] == MPLB_MYMRT && h->P.g_update)
        return bail(fail(MPLB_E_UNSUPPORTED, "FP32-deviation storage has no myMRT thermal collision"));
    if (h->precision == MPLB_FP32_DEV && want_path == MPLB_PATH_OPERATORS)
        return bail(fail(MPLB_E_UNSUPPORTED, "FP32-deviation storage runs on the fused path only"));
    h->path = (want_path == MPLB_PATH_OPERATORS || !fusable) ? MPLB_PATH_OPERATORS : MPLB_PATH_FUSED;
    if (h->path == MPLB_PATH_FUSED) {
        if ((rc = fused_setup(h->fc, h->lat, h->model, h->P, h->fpatch, mesh, h->dims, h->per, h->stream, &h->bytes)))
            return bail(fail(rc, "fused setup: " + h->fc.err));
        if ((rc = dalloc(h, &h->T2, h->n)) || (rc = dalloc(h, &h->U2, 3 * (size_t)h->n))) return bail(rc);
        if (h->precision == MPLB_FP32_DEV) {
            for (int fi = 0; fi < 2; fi++) {
                if (h->model[fi] == MPLB_NO_MODEL) continue;
                if ((rc = dalloc(h, &h->p32[fi][0], nq)) || (rc = dalloc(h, &h->p32[fi][1], nq))) return bail(rc);
            }
            if (mplb_fused32_attributes()) return bail(fail(MPLB_E_CUDA, "cannot raise the shared memory limit (FP32 kernels)"));
        }
    }
    h->red_parts = 2 * 148;
    if ((rc = dalloc(h, &h->red, 2 * (size_t)h->red_parts + 8))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(MPLB_E_CUDA, "device set-up failed"));
    *out = h;
    return 0;
}

int mplb_gpu_destroy(mplb_gpu_t* h) {
    if (!h) return 0;
    DeviceGuard guard(h->dev);
    writer_wait(h);
    cudaStreamSynchronize(h->stream);
    if (h->snap_stream) {
        cudaStreamSynchronize(h->snap_stream);
        cudaStreamDestroy(h->snap_stream);
    }
    if (h->order_ev) cudaEventDestroy(h->order_ev);
    if (h->snap_ready) cudaEventDestroy(h->snap_ready);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->snap_dev) cudaFree(h->snap_dev);
    if (h->snap_host) cudaFreeHost(h->snap_host);
    fused_free(h->fc);
    free_all(h);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

int mplb_gpu_info(mplb_gpu_t* h, mplb_info* info) {
    if (!h || !info) return fail(MPLB_E_ARG, "NULL argument");
    info->path = h->path;
    for (int j = 0; j < 3; j++) { info->box_dims[j] = h->box ? h->dims[j] : 0; info->box_periodic[j] = h->box ? h->per[j] : 0; }
    info->bc_sequential = (h->serial[0] ? 1 : 0) | (h->serial[1] ? 2 : 0);
    info->current_time = h->current;
    info->device_bytes = h->bytes;
    info->kernel_launches = h->launches;
    info->tile_config = (h->path == MPLB_PATH_FUSED && h->fc.tuned) ? h->fc.cfg : -1;
    for (int c = 0; c < 16; c++) info->tile_ms[c] = c < h->fc.ncfg ? h->fc.tune_ms[c] : 0.0f;
    return 0;
}

int mplb_gpu_upload(mplb_gpu_t* h, const double* rho, const double* U, const double* T, const double* f,
                    const double* g, const double* S, const double* Fi, const double* Ft) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    RET(put_scalar(h, rho, h->rho));
    RET(put_scalar(h, T, h->T));
    RET(put_scalar(h, S, h->S));
    RET(put_aos(h, U, h->U, 3));
    RET(put_aos(h, Fi, h->Fi, 3));
    RET(put_aos(h, Ft, h->Ft, 3));
    if (f && h->model[0] != MPLB_NO_MODEL) RET(put_aos(h, f, h->F(), h->Q));
    if (g && h->model[1] != MPLB_NO_MODEL) RET(put_aos(h, g, h->G(), h->Q));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int mplb_gpu_download(mplb_gpu_t* h, double* rho, double* U, double* T, double* Fi, double* Ft, double* S,
                      double* f, double* g) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(queue_kernel_flag(h));
    RET(materialize(h));
    // every copy queued behind the last, one wait at the end
    const bool pdfs = (f && h->model[0] != MPLB_NO_MODEL) || (g && h->model[1] != MPLB_NO_MODEL);
    RET(staging(h, (size_t)h->n * (pdfs ? std::max(3, h->Q) : 3)));
    RET(get_scalar(h, rho, h->rho, false));
    RET(get_scalar(h, T, h->T, false));
    RET(get_scalar(h, S, h->S, false));
    RET(get_aos(h, U, h->U, 3, false));
    RET(get_aos(h, Fi, h->Fi, 3, false));
    RET(get_aos(h, Ft, h->Ft, 3, false));
    if (f) {
        if (h->model[0] == MPLB_NO_MODEL) std::memset(f, 0, (size_t)h->n * h->Q * sizeof(double));
        else RET(get_aos(h, f, h->F(), h->Q, false));
    }
    if (g) {
        if (h->model[1] == MPLB_NO_MODEL) std::memset(g, 0, (size_t)h->n * h->Q * sizeof(double));
        else RET(get_aos(h, g, h->G(), h->Q, false));
    }
    CK(cudaStreamSynchronize(h->stream));
    return kernel_flag_status(h);
}

int mplb_gpu_initialize(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, initialize_impl, h);
}

int mplb_gpu_step(mplb_gpu_t* h, uint32_t nsteps) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (nsteps == 0) return 0;
    DeviceGuard guard(h->dev);
    if (h->path == MPLB_PATH_FUSED && h->precision == MPLB_FP32_DEV) {
        if (h->fstate == 0) RET(prologue32(h));
        for (uint32_t s = 0; s < nsteps; s++) RET(fused32_step(h, false));
        h->current += nsteps;
        return 0;
    }
    if (h->path == MPLB_PATH_FUSED) {
        if (h->nmirror && nsteps > 1)
            return fail(MPLB_E_STATE, "a handle with mirrored ranges takes one step per call (its neighbours "
                                      "step in between)");
        RET(enter_fused(h));  // prologue: the first collision of the loop, on the reference state
        for (uint32_t s = 0; s < nsteps; s++) RET(fused_step(h, false));
        h->current += nsteps;
        return 0;
    }
    for (uint32_t s = 0; s < nsteps; s++) RET(DISPATCH(h, step_operators, h));
    return 0;
}

int mplb_gpu_equilibrium(mplb_gpu_t* h, int32_t field) {
    if (!h || (field != MPLB_FIELD_F && field != MPLB_FIELD_G)) return fail(MPLB_E_ARG, "bad handle or field");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_equilibrium, h, field);
}
int mplb_gpu_collision(mplb_gpu_t* h, int32_t field) {
    if (!h || (field != MPLB_FIELD_F && field != MPLB_FIELD_G)) return fail(MPLB_E_ARG, "bad handle or field");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_collision, h, field);
}
int mplb_gpu_lbstream(mplb_gpu_t* h, int32_t field) {
    if (!h || (field != MPLB_FIELD_F && field != MPLB_FIELD_G)) return fail(MPLB_E_ARG, "bad handle or field");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_stream, h, field);
}
int mplb_gpu_update_boundaries(mplb_gpu_t* h, int32_t field) {
    if (!h || (field != MPLB_FIELD_F && field != MPLB_FIELD_G)) return fail(MPLB_E_ARG, "bad handle or field");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_boundaries, h, field);
}
int mplb_gpu_macro_density(mplb_gpu_t* h, uint32_t start, uint32_t end) {
    if (!h || start > end || end > h->n) return fail(MPLB_E_ARG, "bad handle or node range");
    if (h->model[0] != MPLB_LIMRT && h->model[0] != MPLB_XUMRT && h->P.f_update)
        return fail(MPLB_E_UNSUPPORTED, "Density update not available (macroDensity.c:65-67)");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_density, h, start, end);
}
int mplb_gpu_macro_velocity(mplb_gpu_t* h, uint32_t start, uint32_t end) {
    if (!h || start > end || end > h->n) return fail(MPLB_E_ARG, "bad handle or node range");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_velocity, h, start, end);
}
int mplb_gpu_macro_temperature(mplb_gpu_t* h, uint32_t start, uint32_t end) {
    if (!h || start > end || end > h->n) return fail(MPLB_E_ARG, "bad handle or node range");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_temperature, h, start, end);
}
int mplb_gpu_inter_force(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_interforce, h);
}
int mplb_gpu_heat_source(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_heatsource, h);
}

int mplb_gpu_macro_pressure(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (h->P.f_update && h->model[0] != MPLB_LIMRT && h->model[0] != MPLB_XUMRT)
        return fail(MPLB_E_UNSUPPORTED, "Pressure update not available (macroPressure.c:60-64)");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    return DISPATCH(h, op_pressure, h);
}

int mplb_gpu_snapshot(mplb_gpu_t* h, int32_t flags) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (flags & ~(MPLB_SNAP_PRESSURE | MPLB_SNAP_PDFS)) return fail(MPLB_E_ARG, "unknown snapshot flags");
    const bool with_p = flags & MPLB_SNAP_PRESSURE, with_pdfs = flags & MPLB_SNAP_PDFS;
    if (with_p && h->P.f_update && h->model[0] != MPLB_LIMRT && h->model[0] != MPLB_XUMRT)
        return fail(MPLB_E_UNSUPPORTED, "Pressure update not available (macroPressure.c:60-64)");
    DeviceGuard guard(h->dev);
    const size_t n = h->n, Q = h->Q;
    const size_t need = 6 * n + (with_pdfs ? 2 * Q * n : 0);
    // the host image must not be rewritten while a writer reads it
    writer_wait(h);
    if (need > h->snap_cap) {
        if (h->snap_pending) CK(cudaEventSynchronize(h->snap_done));
        if (h->snap_dev) {
            CK(cudaStreamSynchronize(h->stream));
            cudaFree(h->snap_dev);
            h->bytes -= h->snap_cap * sizeof(double);
            h->snap_dev = nullptr;
        }
        if (h->snap_host) cudaFreeHost(h->snap_host);
        h->snap_host = nullptr;
        h->snap_cap = 0;
        h->snap_pending = false;
        CK(cudaMalloc((void**)&h->snap_dev, need * sizeof(double)));
        h->bytes += need * sizeof(double);
        CK(cudaMallocHost((void**)&h->snap_host, need * sizeof(double)));
        h->snap_cap = need;
    }
    if (!h->snap_stream) {
        CK(cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
    }
    // the device copy must not be rewritten while the previous one is in flight
    if (h->snap_pending) CK(cudaStreamWaitEvent(h->stream, h->snap_done, 0));
    RET(materialize(h));
    if (with_p) RET(DISPATCH(h, op_pressure, h));
    CK(cudaMemcpyAsync(h->snap_dev, h->rho, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->snap_dev + n, h->T, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (with_p)
        CK(cudaMemcpyAsync(h->snap_dev + 2 * n, h->p, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    LAUNCH(k_soa_to_aos, blocks(3 * n), h->n, 3, h->U, h->snap_dev + 3 * n);
    if (with_pdfs) {
        for (int fi = 0; fi < 2; fi++) {
            double* dst = h->snap_dev + 6 * n + fi * Q * n;
            if (h->model[fi] == MPLB_NO_MODEL) CK(cudaMemsetAsync(dst, 0, Q * n * sizeof(double), h->stream));
            else LAUNCH(k_soa_to_aos, blocks(Q * n), h->n, h->Q, fi ? h->G() : h->F(), dst);
        }
    }
    CK(cudaEventRecord(h->snap_ready, h->stream));
    CK(cudaStreamWaitEvent(h->snap_stream, h->snap_ready, 0));
    CK(cudaMemcpyAsync(h->snap_host, h->snap_dev, need * sizeof(double), cudaMemcpyDeviceToHost, h->snap_stream));
    CK(cudaEventRecord(h->snap_done, h->snap_stream));
    h->snap_pending = true;
    h->snap_has_p = with_p;
    h->snap_has_pdfs = with_pdfs;
    h->snap_time = h->current;
    return 0;
}

int mplb_gpu_snapshot_wait(mplb_gpu_t* h, double* rho, double* U, double* T, double* p) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (!h->snap_pending) return fail(MPLB_E_STATE, "no snapshot was taken");
    if (p && !h->snap_has_p) return fail(MPLB_E_STATE, "the snapshot was taken without the pressure");
    DeviceGuard guard(h->dev);
    CK(cudaEventSynchronize(h->snap_done));
    const size_t n = h->n;
    if (rho) std::memcpy(rho, h->snap_host, n * sizeof(double));
    if (T) std::memcpy(T, h->snap_host + n, n * sizeof(double));
    if (p) std::memcpy(p, h->snap_host + 2 * n, n * sizeof(double));
    if (U) std::memcpy(U, h->snap_host + 3 * n, 3 * n * sizeof(double));
    return 0;
}

int mplb_gpu_snapshot_write(mplb_gpu_t* h, const char* root, int32_t pid, int32_t format) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (!h->snap_pending) return fail(MPLB_E_STATE, "no snapshot was taken");
    if (format == MPLB_FMT_ENSIGHT) return fail(MPLB_E_UNSUPPORTED, "EnSight output (MPI-IO) is not provided");
    if (format != MPLB_FMT_ASCII_RAW && format != MPLB_FMT_BINARY_RAW && format != MPLB_FMT_PVTU)
        return fail(MPLB_E_ARG, "unknown data format");
    writer_wait(h);
    std::string dir = root ? root : "";
    auto job = [h, dir, pid, format]() {
        int rc = 0;
        std::string err;
        cudaSetDevice(h->dev);
        cudaError_t e = cudaEventSynchronize(h->snap_done);
        if (e != cudaSuccess) {
            rc = MPLB_E_CUDA;
            err = std::string("snapshot transfer: ") + cudaGetErrorString(e);
        }
        const size_t n = h->n, Q = h->Q;
        const double* s = h->snap_host;
        struct Item { const char* name; const double* v; uint32_t vs; bool scalar; bool on; };
        const Item items[] = {{"rho", s, 1, true, true},
                              {"T", s + n, 1, true, true},
                              {"p", s + 2 * n, 1, true, h->snap_has_p},
                              {"U", s + 3 * n, 3, false, true},
                              {"f", s + 6 * n, (uint32_t)Q, false, h->snap_has_pdfs},
                              {"g", s + 6 * n + Q * n, (uint32_t)Q, false, h->snap_has_pdfs}};
        for (const Item& it : items) {
            if (rc) break;
            if (!it.on) continue;
            rc = mplb_io_write(dir.c_str(), pid, h->snap_time, format, it.name, it.v, n, it.vs, it.scalar, &err);
        }
        if (rc && !h->writer_rc) {
            h->writer_rc = rc;
            h->writer_err = err;
        }
    };
    try {
        h->writer = std::thread(job);
    } catch (const std::exception& e) {
        return fail(MPLB_E_STATE, std::string("cannot start the writer thread: ") + e.what());
    }
    return 0;
}

int mplb_gpu_snapshot_join(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    writer_wait(h);
    const int rc = h->writer_rc;
    h->writer_rc = 0;
    return rc ? fail(rc, h->writer_err) : 0;
}

int mplb_gpu_download_pressure(mplb_gpu_t* h, double* p) {
    if (!h || !p) return fail(MPLB_E_ARG, "NULL argument");
    DeviceGuard guard(h->dev);
    return get_scalar(h, p, h->p);
}

int mplb_gpu_set_time(mplb_gpu_t* h, uint32_t current) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    h->current = current;
    return 0;
}

int mplb_gpu_set_rho0(mplb_gpu_t* h, double rho_0) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    // the post-collision buffers were made with the old rho_0
    RET(materialize(h));
    h->P.rho_0 = rho_0;
    return 0;
}

int mplb_gpu_average_rho0(mplb_gpu_t* h, double* rho_0) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    double avg = 0;
    if (!(h->P.rho_0 <= 0)) {
        LAUNCH(k_sum_serial, 1, h->n, h->rho, h->red);
        double s = 0;
        CK(cudaMemcpyAsync(&s, h->red, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        avg = s / (int)h->n;
    }
    h->P.rho_0 = avg;
    if (rho_0) *rho_0 = avg;
    return 0;
}

int mplb_gpu_mass_energy(mplb_gpu_t* h, double* mass, double* energy) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    int parts = std::min<int>(h->red_parts, (int)blocks(h->n));
    k_sum2_partial<<<parts, TPB, 0, h->stream>>>(h->n, h->rho, h->T, h->red);
    h->launches++;
    RET(launch_check(h));
    k_sum2_final<<<1, TPB, 0, h->stream>>>(parts, h->red, h->red + 2 * h->red_parts);
    h->launches++;
    RET(launch_check(h));
    double r[2] = {0, 0};
    CK(cudaMemcpyAsync(r, h->red + 2 * h->red_parts, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (mass) *mass = r[0];
    if (energy) *energy = r[1];
    return 0;
}

int mplb_gpu_monitor(mplb_gpu_t* h, int32_t reset, double* max_drho, double* mass) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (!h->P.f_update || h->model[0] == MPLB_NO_MODEL)
        return fail(MPLB_E_UNSUPPORTED, "the monitor needs an updated flow field");
    DeviceGuard guard(h->dev);
    if (!h->snap) {
        RET(dalloc(h, &h->snap, h->n));
        reset = 1;
    }
    const int parts = std::min<int>(h->red_parts, (int)blocks(h->n));
    double* out = h->red + 2 * (size_t)h->red_parts + 4;
    if (h->path == MPLB_PATH_FUSED && h->precision == MPLB_FP32_DEV) {
        if (h->fstate == 0) RET(prologue32(h));
        k_monitor_partial<float><<<parts, TPB, 0, h->stream>>>(h->n, h->Q, h->p32[0][h->cur32[0]], h->rho_ref,
                                                               h->snap, reset, h->red);
    } else {
        if (h->path == MPLB_PATH_FUSED && h->fstate == 0) {
            RET(DISPATCH(h, op_collision, h, 0));
            RET(DISPATCH(h, op_collision, h, 1));
            h->fstate = 1;
        }
        k_monitor_partial<double><<<parts, TPB, 0, h->stream>>>(h->n, h->Q, h->F(), 0.0, h->snap, reset, h->red);
    }
    h->launches++;
    RET(launch_check(h));
    k_monitor_final<<<1, 32, 0, h->stream>>>(parts, h->red, out);
    h->launches++;
    RET(launch_check(h));
    double r[2] = {0, 0};
    CK(cudaMemcpyAsync(r, out, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (max_drho) *max_drho = reset ? 0.0 : r[0];
    if (mass) *mass = r[1];
    return 0;
}

int mplb_gpu_run_to_equilibrium(mplb_gpu_t* h, uint32_t max_steps, uint32_t check_interval, double tol,
                                uint32_t* steps, double* rate) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (check_interval == 0) return fail(MPLB_E_ARG, "check_interval must be >= 1");
    DeviceGuard guard(h->dev);
    double d = 0;
    RET(mplb_gpu_monitor(h, 1, &d, nullptr));
    // FP32 form: reset the total momentum to its starting value at every check
    const bool fix = momentum_conserved(h);
    auto momentum = [&](long long* J) -> int {
        cudaError_t e = mplb_mom_sum32(h->lat, h->n, h->p32[0][h->cur32[0]], J, h->stream);
        h->launches++;
        if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("momentum sum: ") + cudaGetErrorString(e));
        return 0;
    };
    if (fix) {
        if (!h->mom) CK(cudaMalloc((void**)&h->mom, 6 * sizeof(long long)));
        RET(momentum(h->mom + 3));
    }
    uint32_t done = 0;
    double r = -1.0;
    while (done < max_steps) {
        RET(mplb_gpu_step(h, check_interval));
        done += check_interval;
        RET(mplb_gpu_monitor(h, 0, &d, nullptr));
        if (!std::isfinite(d)) {
            if (steps) *steps = done;
            if (rate) *rate = d;
            return fail(MPLB_E_NONFINITE, "non-finite density after " + std::to_string(done) + " steps");
        }
        if (fix) {
            RET(momentum(h->mom));
            cudaError_t e = mplb_mom_fix32(h->lat, h->n, h->p32[0][h->cur32[0]], h->mom, h->mom + 3, h->stream);
            h->launches++;
            if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("momentum reset: ") + cudaGetErrorString(e));
        }
        r = d / check_interval;
        if (r < tol) break;
    }
    if (steps) *steps = done;
    if (rate) *rate = r;
    return 0;
}

int mplb_mlp_init_bubble(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, const double* center, double radius,
                         double T) {
    if (!m || !h || !center) return fail(MPLB_E_ARG, "NULL argument");
    if (!(radius > 0.0)) return fail(MPLB_E_ARG, "radius must be positive");
    if (!h->box) return fail(MPLB_E_UNSUPPORTED, "warm start needs a box lattice");
    if (h->P.eos != MPLB_EOS_CS) return fail(MPLB_E_UNSUPPORTED, "warm start is trained on the Carnahan-Starling EOS");
    if (mplb_mlp_device(m) != h->dev) return fail(MPLB_E_ARG, "network and lattice on different devices");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    RET(mplb_mlp_bubble_launch(m, h->rho, h->n, h->dims[0], h->dims[1], center, radius, t_ratio, h->P.a, h->P.b,
                               h->stream));
    h->launches++;
    CK(cudaMemsetAsync(h->U, 0, 3 * (size_t)h->n * sizeof(double), h->stream));
    k_fill<<<blocks(h->n), TPB, 0, h->stream>>>(h->n, T, h->T);
    h->launches++;
    RET(launch_check(h));
    h->initialized = false;
    return 0;
}

// Common part of the *_mass warm starts: place_at(p) writes the network's
// density for the shape parameter p (bubble radius, band height); the
// lattice mass is monotonic in p, falling as p grows for dir = -1 (a bubble)
// and rising for dir = +1 (a liquid band).  The network's inputs are BF16,
// so the mass is a step function of p: secant steps to get close, a bracket
// [pa, pb] with g(pa) >= 0 >= g(pb) (g = the mass excess, signed so that it
// falls with p), bisection down to one step, then the two fields blended so
// that the lattice holds the target mass exactly.  *used = the effective p.
int place_with_mass(mplb_gpu* h, const std::function<int(double)>& place_at, double p0, int dir, double target_mass,
                    double* used) {
    const int parts = std::min<int>(h->red_parts, (int)blocks(h->n));
    auto total = [&](double* M) -> int {
        k_sum2_partial<<<parts, TPB, 0, h->stream>>>(h->n, h->rho, nullptr, h->red);
        k_sum2_final<<<1, TPB, 0, h->stream>>>(parts, h->red, h->red + 2 * h->red_parts);
        h->launches += 2;
        RET(launch_check(h));
        CK(cudaMemcpyAsync(M, h->red + 2 * h->red_parts, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return 0;
    };
    // mass excess of the network's field at p, signed to fall as p grows
    auto g_at = [&](double p, double* f) -> int {
        RET(place_at(p));
        RET(total(f));
        *f = (*f - target_mass) * (double)(-dir);
        return 0;
    };
    double r0 = p0, r1 = p0 * 1.02, f0 = 0, f1 = 0;
    RET(g_at(r0, &f0));
    RET(g_at(r1, &f1));
    for (int it = 0; it < 8 && f1 != f0 && f1 != 0.0; it++) {
        const double r2 = std::min(2.0 * p0, std::max(0.5 * p0, r1 - f1 * (r1 - r0) / (f1 - f0)));
        r0 = r1;
        f0 = f1;
        r1 = r2;
        RET(g_at(r1, &f1));
    }
    double ra = r1, fa = f1, rb = r1, fb = f1, step = 0.01 * r1;
    for (int it = 0; it < 40 && !(fa >= 0.0 && fb <= 0.0); it++, step *= 2.0) {
        if (fa < 0.0) {
            ra = std::max(1e-3, ra - step);
            RET(g_at(ra, &fa));
        }
        if (fb > 0.0) {
            rb += step;
            RET(g_at(rb, &fb));
        }
    }
    double w = 0.0;  // weight of the rb field
    if (fa >= 0.0 && fb <= 0.0) {
        for (int it = 0; it < 40 && rb - ra > 1e-9 * p0 && fa != 0.0 && fb != 0.0; it++) {
            const double rm = 0.5 * (ra + rb);
            double fm = 0;
            RET(g_at(rm, &fm));
            if (fm >= 0.0) {
                ra = rm;
                fa = fm;
            } else {
                rb = rm;
                fb = fm;
            }
        }
        w = (fa == fb) ? 0.0 : fa / (fa - fb);
    }
    double* tmp = nullptr;
    CK(cudaMalloc((void**)&tmp, (size_t)h->n * sizeof(double)));
    auto blend = [&]() -> int {
        RET(g_at(ra, &fa));
        CK(cudaMemcpyAsync(tmp, h->rho, (size_t)h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        RET(g_at(rb, &fb));
        k_blend<<<blocks(h->n), TPB, 0, h->stream>>>(h->n, w, tmp, h->rho);
        h->launches++;
        RET(launch_check(h));
        // the blend's rounding (far below the network's error) goes uniformly
        double M = 0;
        RET(total(&M));
        k_add<<<blocks(h->n), TPB, 0, h->stream>>>(h->n, (target_mass - M) / (double)h->n, h->rho);
        h->launches++;
        RET(launch_check(h));
        CK(cudaStreamSynchronize(h->stream));
        return 0;
    };
    const int rc = blend();
    cudaFree(tmp);
    if (rc) return rc;
    if (used) *used = ra + w * (rb - ra);
    return 0;
}

int mplb_mlp_init_bubble_mass(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, const double* center, double radius,
                              double T, double target_mass, double* radius_used) {
    if (!m || !h || !center) return fail(MPLB_E_ARG, "NULL argument");
    if (!(radius > 0.0) || !(target_mass > 0.0)) return fail(MPLB_E_ARG, "radius and mass must be positive");
    DeviceGuard guard(h->dev);
    return place_with_mass(
        h, [&](double R) { return mplb_mlp_init_bubble(m, h, t_ratio, center, R, T); }, radius, -1, target_mass,
        radius_used);
}

int mplb_mlp_init_column(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, int32_t axis, double center, double height,
                         double T) {
    if (!m || !h) return fail(MPLB_E_ARG, "NULL argument");
    if (!(height > 0.0)) return fail(MPLB_E_ARG, "height must be positive");
    if (!h->box) return fail(MPLB_E_UNSUPPORTED, "warm start needs a box lattice");
    const int D = h->lat == MPLB_D2Q9 ? 2 : 3;
    if (axis < 0 || axis >= D) return fail(MPLB_E_ARG, "axis must be 0 .. dimensions - 1");
    if (h->P.eos != MPLB_EOS_CS) return fail(MPLB_E_UNSUPPORTED, "warm start is trained on the Carnahan-Starling EOS");
    if (mplb_mlp_device(m) != h->dev) return fail(MPLB_E_ARG, "network and lattice on different devices");
    DeviceGuard guard(h->dev);
    RET(materialize(h));
    RET(mplb_mlp_column_launch(m, h->rho, h->n, h->dims[0], h->dims[1], axis, h->dims[axis], center, height, t_ratio,
                               h->P.a, h->P.b, h->stream));
    h->launches++;
    CK(cudaMemsetAsync(h->U, 0, 3 * (size_t)h->n * sizeof(double), h->stream));
    k_fill<<<blocks(h->n), TPB, 0, h->stream>>>(h->n, T, h->T);
    h->launches++;
    RET(launch_check(h));
    h->initialized = false;
    return 0;
}

int mplb_mlp_init_column_mass(mplb_mlp_t* m, mplb_gpu_t* h, double t_ratio, int32_t axis, double center,
                              double height, double T, double target_mass, double* height_used) {
    if (!m || !h) return fail(MPLB_E_ARG, "NULL argument");
    if (!(height > 0.0) || !(target_mass > 0.0)) return fail(MPLB_E_ARG, "height and mass must be positive");
    DeviceGuard guard(h->dev);
    return place_with_mass(
        h, [&](double H) { return mplb_mlp_init_column(m, h, t_ratio, axis, center, H, T); }, height, +1,
        target_mass, height_used);
}

int mplb_gpu_sync(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    DeviceGuard guard(h->dev);
    RET(queue_kernel_flag(h));
    CK(cudaStreamSynchronize(h->stream));
    return kernel_flag_status(h);
}

int mplb_gpu_copy_nodes(mplb_gpu_t* dst, uint32_t dst_start, mplb_gpu_t* src, uint32_t src_start,
                        uint32_t count, int32_t fields) {
    if (!dst || !src) return fail(MPLB_E_ARG, "NULL handle");
    const int32_t all = MPLB_NODES_RHO | MPLB_NODES_U | MPLB_NODES_T | MPLB_NODES_FI | MPLB_NODES_FT |
                        MPLB_NODES_S | MPLB_NODES_F | MPLB_NODES_G;
    if (fields & ~all) return fail(MPLB_E_ARG, "unknown field bits");
    if (dst->Q != src->Q) return fail(MPLB_E_ARG, "the lattices differ");
    if (dst->precision != MPLB_FP64 || src->precision != MPLB_FP64)
        return fail(MPLB_E_UNSUPPORTED, "node copies need FP64 storage");
    if ((uint64_t)dst_start + count > dst->n || (uint64_t)src_start + count > src->n)
        return fail(MPLB_E_ARG, "node range out of bounds");
    for (int fi = 0; fi < 2; fi++)
        if ((fields & (fi ? MPLB_NODES_G : MPLB_NODES_F)) &&
            (dst->model[fi] == MPLB_NO_MODEL || src->model[fi] == MPLB_NO_MODEL))
            return fail(MPLB_E_ARG, fi ? "no g field" : "no f field");
    if (dst == src && (uint64_t)dst_start < (uint64_t)src_start + count &&
        (uint64_t)src_start < (uint64_t)dst_start + count)
        return fail(MPLB_E_ARG, "overlapping ranges on one handle");
    if (count == 0 || fields == 0) return 0;
    {
        DeviceGuard guard(src->dev);
        RET(materialize(src));
    }
    {
        DeviceGuard guard(dst->dev);
        RET(materialize(dst));
    }
    // every field is [component][node] on the device: one strided copy each
    NodeCopy parts[8];
    int np = 0;
    auto add = [&](int32_t bit, double* d, const double* s, int rows) {
        if (fields & bit) parts[np++] = NodeCopy{d, s, rows};
    };
    add(MPLB_NODES_RHO, dst->rho, src->rho, 1);
    add(MPLB_NODES_U, dst->U, src->U, 3);
    add(MPLB_NODES_T, dst->T, src->T, 1);
    add(MPLB_NODES_FI, dst->Fi, src->Fi, 3);
    add(MPLB_NODES_FT, dst->Ft, src->Ft, 3);
    add(MPLB_NODES_S, dst->S, src->S, 1);
    if (fields & MPLB_NODES_F) add(MPLB_NODES_F, dst->F(), src->F(), dst->Q);
    if (fields & MPLB_NODES_G) add(MPLB_NODES_G, dst->G(), src->G(), dst->Q);
    return copy_node_rows(dst, dst_start, src, src_start, count, parts, np);
}

int mplb_gpu_copy_state(mplb_gpu_t* dst, uint32_t dst_start, mplb_gpu_t* src, uint32_t src_start, uint32_t count) {
    if (!dst || !src) return fail(MPLB_E_ARG, "NULL handle");
    if (dst->path != MPLB_PATH_FUSED || src->path != MPLB_PATH_FUSED || dst->precision != MPLB_FP64 ||
        src->precision != MPLB_FP64)
        return fail(MPLB_E_UNSUPPORTED, "state copies need two handles on the fused FP64 path");
    if (dst->lat != src->lat || dst->model[0] != src->model[0] || dst->model[1] != src->model[1] ||
        dst->P.f_update != src->P.f_update || dst->P.g_update != src->P.g_update)
        return fail(MPLB_E_ARG, "the lattices or field options differ");
    if ((uint64_t)dst_start + count > dst->n || (uint64_t)src_start + count > src->n)
        return fail(MPLB_E_ARG, "node range out of bounds");
    if (dst == src && (uint64_t)dst_start < (uint64_t)src_start + count &&
        (uint64_t)src_start < (uint64_t)dst_start + count)
        return fail(MPLB_E_ARG, "overlapping ranges on one handle");
    if (count == 0) return 0;
    for (mplb_gpu* h : {src, dst}) {
        DeviceGuard guard(h->dev);
        RET(enter_fused(h));
    }
    // the input buffers of the next fused step: post-collision populations of
    // every updated field, T and U of the last step
    NodeCopy parts[4];
    int np = 0;
    for (int fi = 0; fi < 2; fi++)
        if (dst->model[fi] != MPLB_NO_MODEL && (fi == 0 ? dst->P.f_update : dst->P.g_update))
            parts[np++] = NodeCopy{dst->pdf[fi][dst->cur[fi]], src->pdf[fi][src->cur[fi]], dst->Q};
    parts[np++] = NodeCopy{dst->T, src->T, 1};
    parts[np++] = NodeCopy{dst->U, src->U, 3};
    return copy_node_rows(dst, dst_start, src, src_start, count, parts, np);
}

int mplb_gpu_set_owned(mplb_gpu_t* h, uint32_t start, uint32_t count) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    if (h->path != MPLB_PATH_FUSED || h->precision != MPLB_FP64)
        return fail(MPLB_E_UNSUPPORTED, "an owned range needs a handle on the fused FP64 path");
    if ((uint64_t)start + count > h->n) return fail(MPLB_E_ARG, "node range out of bounds");
    for (int m = 0; m < h->nmirror; m++)
        if (h->mirrors[m].src_start < start || (uint64_t)h->mirrors[m].src_start + h->mirrors[m].count >
                                                   (uint64_t)start + (count ? count : h->n))
            return fail(MPLB_E_ARG, "a mirrored range lies outside the owned range");
    h->own_start = count ? start : 0;
    h->own_count = count;
    return 0;
}

int mplb_gpu_add_mirror(mplb_gpu_t* h, uint32_t src_start, uint32_t count, mplb_gpu_t* dst, uint32_t dst_start) {
    if (!h || !dst) return fail(MPLB_E_ARG, "NULL handle");
    if (h == dst) return fail(MPLB_E_ARG, "a handle cannot mirror into itself");
    if (h->path != MPLB_PATH_FUSED || dst->path != MPLB_PATH_FUSED || h->precision != MPLB_FP64 ||
        dst->precision != MPLB_FP64)
        return fail(MPLB_E_UNSUPPORTED, "mirrors need two handles on the fused FP64 path");
    if (dst->lat != h->lat || dst->model[0] != h->model[0] || dst->model[1] != h->model[1] ||
        dst->P.f_update != h->P.f_update || dst->P.g_update != h->P.g_update)
        return fail(MPLB_E_ARG, "the lattices or field options differ");
    if (h->nmirror >= MPLB_MAX_MIRRORS) return fail(MPLB_E_ARG, "at most two mirrored ranges per handle");
    if (count == 0) return fail(MPLB_E_ARG, "empty range");
    if ((uint64_t)src_start + count > h->n || (uint64_t)dst_start + count > dst->n)
        return fail(MPLB_E_ARG, "node range out of bounds");
    const uint64_t olo = h->own_start, ohi = olo + (h->own_count ? h->own_count : h->n);
    if (src_start < olo || (uint64_t)src_start + count > ohi)
        return fail(MPLB_E_ARG, "the mirrored range lies outside this handle's owned range");
    const uint64_t dlo = dst->own_start, dhi = dlo + (dst->own_count ? dst->own_count : dst->n);
    if ((uint64_t)dst_start < dhi && dlo < (uint64_t)dst_start + count)
        return fail(MPLB_E_ARG, "the target range overlaps the neighbour's owned range (set it first)");
    if (dst->dev != h->dev) {
        DeviceGuard guard(h->dev);
        int can = 0;
        CK(cudaDeviceCanAccessPeer(&can, h->dev, dst->dev));
        if (!can) return fail(MPLB_E_UNSUPPORTED, "the neighbour's GPU is not reachable from this one");
        cudaError_t e = cudaDeviceEnablePeerAccess(dst->dev, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
        else CK(e);
    }
    h->mirrors[h->nmirror++] = mplb_gpu::Mirror{src_start, count, dst_start, dst};
    return 0;
}

int mplb_gpu_clear_mirrors(mplb_gpu_t* h) {
    if (!h) return fail(MPLB_E_ARG, "NULL handle");
    h->nmirror = 0;
    return 0;
}

}  // extern "C"

namespace {

// Rows of [component][node] device arrays, `count` nodes from src_start of
// src to dst_start of dst: one strided copy per part, queued on the source
// handle's stream after the destination's queued work, and the destination's
// stream made to wait for it (nothing blocks the host; between GPUs the copy
// goes peer to peer, peer access enabled on first use).
int copy_node_rows(mplb_gpu* dst, uint32_t dst_start, mplb_gpu* src, uint32_t src_start, uint32_t count,
                   const NodeCopy* parts, int np) {
    const bool same_queue = dst->dev == src->dev && dst->stream == src->stream;
    struct Events {
        cudaEvent_t dst_ready = nullptr, copied = nullptr;
        ~Events() {
            if (dst_ready) cudaEventDestroy(dst_ready);
            if (copied) cudaEventDestroy(copied);
        }
    } ev;
    if (!same_queue) {
        DeviceGuard guard(dst->dev);
        CK(cudaEventCreateWithFlags(&ev.dst_ready, cudaEventDisableTiming));
        CK(cudaEventRecord(ev.dst_ready, dst->stream));
    }
    DeviceGuard guard(src->dev);
    if (dst->dev != src->dev) {
        int can = 0;
        CK(cudaDeviceCanAccessPeer(&can, src->dev, dst->dev));
        if (can) {
            cudaError_t e = cudaDeviceEnablePeerAccess(dst->dev, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            else CK(e);
        }
    }
    if (!same_queue) CK(cudaStreamWaitEvent(src->stream, ev.dst_ready, 0));
    const size_t dpitch = (size_t)dst->n * sizeof(double), spitch = (size_t)src->n * sizeof(double);
    const size_t width = (size_t)count * sizeof(double);
    for (int i = 0; i < np; i++) {
        const NodeCopy& p = parts[i];
        CK(cudaMemcpy2DAsync(p.d + dst_start, dpitch, p.s + src_start, spitch, width, p.rows, cudaMemcpyDefault,
                             src->stream));
    }
    if (!same_queue) {
        CK(cudaEventCreateWithFlags(&ev.copied, cudaEventDisableTiming));
        CK(cudaEventRecord(ev.copied, src->stream));
        DeviceGuard dguard(dst->dev);
        CK(cudaStreamWaitEvent(dst->stream, ev.copied, 0));
    }
    return 0;
}

// The ranks of one process: every handle must hold the same lattice and
// field options, and every run must name handles of the list.
int ranks_check(mplb_gpu_t* const* h, uint32_t count, const mplb_ghost_run* runs, uint32_t nruns) {
    if (!h || count == 0) return fail(MPLB_E_ARG, "no handles");
    if (nruns && !runs) return fail(MPLB_E_ARG, "runs missing");
    for (uint32_t r = 0; r < count; r++) {
        if (!h[r]) return fail(MPLB_E_ARG, "NULL handle");
        const mplb_gpu* a = h[0];
        const mplb_gpu* b = h[r];
        if (b->Q != a->Q || b->model[0] != a->model[0] || b->model[1] != a->model[1] ||
            b->P.f_update != a->P.f_update || b->P.g_update != a->P.g_update || b->P.st_on != a->P.st_on)
            return fail(MPLB_E_ARG, "the ranks' lattices or field options differ");
    }
    for (uint32_t i = 0; i < nruns; i++)
        if (runs[i].dst >= count || runs[i].src >= count) return fail(MPLB_E_ARG, "run names a handle outside the list");
    return 0;
}

int ranks_exchange(mplb_gpu_t* const* h, const mplb_ghost_run* runs, uint32_t nruns, int32_t fields) {
    for (uint32_t i = 0; i < nruns; i++) {
        const mplb_ghost_run& g = runs[i];
        RET(mplb_gpu_copy_nodes(h[g.dst], g.dst_start, h[g.src], g.src_start, g.count, fields));
    }
    return 0;
}

}  // namespace

extern "C" {

int mplb_ranks_initialize(mplb_gpu_t* const* h, uint32_t count, const mplb_ghost_run* runs, uint32_t nruns) {
    RET(ranks_check(h, count, runs, nruns));
    RET(ranks_exchange(h, runs, nruns, MPLB_NODES_RHO | MPLB_NODES_U | MPLB_NODES_T));
    for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_equilibrium(h[r], MPLB_FIELD_F));
    if (h[0]->model[1] != MPLB_NO_MODEL)
        for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_equilibrium(h[r], MPLB_FIELD_G));
    for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_inter_force(h[r]));
    RET(ranks_exchange(h, runs, nruns, MPLB_NODES_FI | MPLB_NODES_FT));
    if (h[0]->model[1] != MPLB_NO_MODEL && h[0]->P.g_update) {
        for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_heat_source(h[r]));
        RET(ranks_exchange(h, runs, nruns, MPLB_NODES_S));
    }
    for (uint32_t r = 0; r < count; r++) h[r]->initialized = true;
    return 0;
}

int mplb_ranks_step(mplb_gpu_t* const* h, uint32_t count, const mplb_ghost_run* runs, uint32_t nruns,
                    uint32_t nsteps) {
    RET(ranks_check(h, count, runs, nruns));
    const bool f_on = h[0]->model[0] != MPLB_NO_MODEL && h[0]->P.f_update;
    const bool g_on = h[0]->model[1] != MPLB_NO_MODEL && h[0]->P.g_update;
    const bool f_st = f_on && h[0]->P.st_on;
    for (uint32_t s = 0; s < nsteps; s++) {
        for (uint32_t r = 0; r < count; r++) h[r]->current++;
        for (int fi = 0; fi < 2; fi++) {
            if (!(fi ? g_on : f_on)) continue;
            const int32_t bit = fi ? MPLB_NODES_G : MPLB_NODES_F;
            for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_collision(h[r], fi));
            if (fi == 0 && f_st) RET(ranks_exchange(h, runs, nruns, bit));
            for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_lbstream(h[r], fi));
            for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_update_boundaries(h[r], fi));
            RET(ranks_exchange(h, runs, nruns, bit));
        }
        for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_macro_density(h[r], 0, h[r]->n));
        if (g_on) {
            for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_heat_source(h[r]));
            RET(ranks_exchange(h, runs, nruns, MPLB_NODES_S));
        }
        for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_macro_temperature(h[r], 0, h[r]->n));
        if (f_on) {
            for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_inter_force(h[r]));
            RET(ranks_exchange(h, runs, nruns, MPLB_NODES_FI | MPLB_NODES_FT));
        }
        for (uint32_t r = 0; r < count; r++) RET(mplb_gpu_macro_velocity(h[r], 0, h[r]->n));
    }
    return 0;
}

}  // extern "C"

// ================================================================= batch
struct mplb_batch {
    int dev = 0;
    cudaStream_t stream = nullptr;
    std::vector<mplb_gpu*> lat;
    uint64_t nodes = 0;
    uint32_t K = 0;
    double tol = 0;
    int tile_request = 0;
    int cfg = -1;
    int grid = 0;
    float tile_ms[8] = {};
    Params* dP = nullptr;
    FusedArgs32* dA = nullptr;  // [lattice][parity]
    int2* dtiles = nullptr;
    int* dnt = nullptr;
    size_t tile_cap = 0;
    double** dsnap = nullptr;   // per-lattice pointers into snap
    double* snap = nullptr;
    unsigned long long* dmax = nullptr;
    unsigned long long* hmax = nullptr;  // pinned
    long long* jsum = nullptr;  // per lattice total momentum (fixed point), now
    long long* j0 = nullptr;    // ... and at the start of the run
    int* proj = nullptr;        // per lattice: momentum reset applies
    cudaGraphExec_t graph = nullptr;
    int graph_cfg = -1;
    uint32_t graph_K = 0;
    uint64_t launches = 0, graph_launches = 0;
    // time-averaging filter (mplb_batch_filter)
    std::vector<uint32_t> win;  // per lattice: window in steps, 0 = not filtered
    uint32_t* dwin = nullptr;
    double* acc = nullptr;      // 9 n doubles per filtered lattice
    double** dacc = nullptr;    // per-lattice pointers into acc (null when not filtered)
    uint32_t filter_first = 0, filter_every = 0;
    uint64_t windows = 0;       // filter windows run
};

namespace {

void batch_free(mplb_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    void* ps[] = {b->dP,   b->dA, b->dtiles, b->dnt,  b->dsnap, b->snap, b->dmax,
                  b->jsum, b->j0, b->proj,   b->dwin, b->acc,   b->dacc};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (b->hmax) cudaFreeHost(b->hmax);
}

// Order the batch stream after every handle's queued work.
int batch_enter(mplb_batch* b) {
    for (mplb_gpu* h : b->lat)
        if (h->stream != b->stream) CK(cudaStreamSynchronize(h->stream));
    for (mplb_gpu* h : b->lat) {
        if (h->fstate == 0) {
            RET(prologue32(h));
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    return 0;
}

// ... and every handle's later work after the batch.
int batch_leave(mplb_batch* b) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, b->stream);
    for (mplb_gpu* h : b->lat)
        if (e == cudaSuccess && h->stream != b->stream) e = cudaStreamWaitEvent(h->stream, ev, 0);
    cudaEventDestroy(ev);
    CK(e);
    return 0;
}

// Kernel arguments of every lattice for candidate c: [2i] steps from the
// handle's current buffer, [2i+1] back.
int batch_args(mplb_batch* b, int c) {
    int tx = 0, ty = 0;
    mplb_batch_cfg(c, &tx, &ty);
    std::vector<FusedArgs32> A(2 * b->lat.size());
    for (size_t i = 0; i < b->lat.size(); i++) {
        mplb_gpu* h = b->lat[i];
        FusedArgs a = h->fc.args;
        a.tiles_x = (a.nx + tx - 1) / tx;
        a.tiles_y = (a.ny + ty - 1) / ty;
        FusedArgs32 B = mplb_make_args32(a, h->P, h->rho_ref, h->T_ref);
        if (B.tiles_x != a.tiles_x || B.tiles_y != a.tiles_y || B.tiles_x <= 0 || B.tiles_y <= 0 || B.n != h->n)
            return fail(MPLB_E_STATE, "batch: inconsistent tile geometry");
        B.Told = h->T;  // the frozen temperature field, read by every pull
        B.Tnew = nullptr;
        B.Uold = B.Unew = h->U;
        B.S = h->S;
        B.rho_c = h->rho;
        const int c0 = h->cur32[0];
        for (int par = 0; par < 2; par++) {
            FusedArgs32 Bp = B;
            Bp.fin = h->p32[0][c0 ^ par];
            Bp.fout = h->p32[0][c0 ^ par ^ 1];
            if (!Bp.fin || !Bp.fout || !Bp.Told || !Bp.Uold || !Bp.S || !Bp.rho_c)
                return fail(MPLB_E_STATE, "batch: lattice buffers missing");
            A[2 * i + par] = Bp;
        }
    }
    CK(cudaMemcpyAsync(b->dA, A.data(), A.size() * sizeof(FusedArgs32), cudaMemcpyHostToDevice, b->stream));
    return 0;
}

// Work table of the lattices flagged in `active` for candidate c.
int batch_table(mplb_batch* b, int c, const std::vector<char>& active, int* count) {
    int tx = 0, ty = 0;
    mplb_batch_cfg(c, &tx, &ty);
    std::vector<int2> t;
    for (size_t i = 0; i < b->lat.size(); i++) {
        if (!active[i]) continue;
        const FusedArgs& a = b->lat[i]->fc.args;
        const int nt = ((a.nx + tx - 1) / tx) * ((a.ny + ty - 1) / ty);
        for (int k = 0; k < nt; k++) t.push_back(make_int2((int)i, k));
    }
    if (t.size() > b->tile_cap) return fail(MPLB_E_STATE, "batch work table overflow");
    const int nt = (int)t.size();
    if (nt) CK(cudaMemcpyAsync(b->dtiles, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->dnt, &nt, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    // the host vector and nt leave scope: finish the copies first
    CK(cudaStreamSynchronize(b->stream));
    if (count) *count = nt;
    return 0;
}

int batch_launch(mplb_batch* b, int c, int grid, int parity) {
    cudaError_t e = mplb_batch32_launch(c, b->dP, b->dA, b->dtiles, b->dnt, parity, grid, b->stream);
    b->launches++;
    if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("batch step launch: ") + cudaGetErrorString(e));
    return 0;
}

// Convergence check (max |drho| per lattice, density snapshot, total
// momentum), then the FP32 momentum reset; dmax and jsum are cleared first.
int batch_check(mplb_batch* b, int parity, bool fix) {
    const size_t N = b->lat.size();
    CK(cudaMemsetAsync(b->dmax, 0, N * sizeof(unsigned long long), b->stream));
    CK(cudaMemsetAsync(b->jsum, 0, 3 * N * sizeof(long long), b->stream));
    cudaError_t e = mplb_batch32_check(b->cfg, b->dP, b->dA, b->dtiles, b->dnt, parity, b->grid, b->dsnap, b->dmax,
                                       b->jsum, b->stream);
    b->launches++;
    if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("batch check launch: ") + cudaGetErrorString(e));
    if (fix) {
        e = mplb_batch32_fix(b->cfg, b->dA, b->dtiles, b->dnt, parity, b->grid, b->jsum, b->j0, b->proj, b->stream);
        b->launches++;
        if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("batch fix launch: ") + cudaGetErrorString(e));
    }
    return 0;
}

// Autotuner: each candidate re-runs the first step from the current state
// (parity 0 only, so the state does not advance: the step reads the current
// buffers and rewrites the spare ones), best of a few timed launches.
int batch_tune(mplb_batch* b) {
    const std::vector<char> all(b->lat.size(), 1);
    if (b->tile_request > 0) {
        b->cfg = std::min(b->tile_request - 1, mplb_batch_ncfg() - 1);
    } else {
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 1e30f;
        int pick = 0;
        for (int c = 0; c < mplb_batch_ncfg(); c++) {
            RET(batch_args(b, c));
            int nt = 0;
            RET(batch_table(b, c, all, &nt));
            const int grid = std::max(1, std::min(mplb_batch_grid(c), nt));
            RET(batch_launch(b, c, grid, 0));
            float ms = 1e30f;
            for (int r = 0; r < 3; r++) {
                CK(cudaEventRecord(e0, b->stream));
                RET(batch_launch(b, c, grid, 0));
                CK(cudaEventRecord(e1, b->stream));
                CK(cudaEventSynchronize(e1));
                float t = 0;
                CK(cudaEventElapsedTime(&t, e0, e1));
                ms = std::min(ms, t);
            }
            b->tile_ms[c] = ms;
            if (ms < best) {
                best = ms;
                pick = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->cfg = pick;
    }
    return 0;
}

// Arguments and full work table for the chosen candidate.
int batch_ready(mplb_batch* b, const std::vector<char>& active, int* nt) {
    if (b->cfg < 0) RET(batch_tune(b));
    RET(batch_args(b, b->cfg));
    RET(batch_table(b, b->cfg, active, nt));
    int tiles = 0;
    for (size_t i = 0; i < b->lat.size(); i++) {
        int tx = 0, ty = 0;
        mplb_batch_cfg(b->cfg, &tx, &ty);
        const FusedArgs& a = b->lat[i]->fc.args;
        tiles += ((a.nx + tx - 1) / tx) * ((a.ny + ty - 1) / ty);
    }
    b->grid = std::max(1, std::min(mplb_batch_grid(b->cfg), tiles));
    return 0;
}

// One check interval as a graph: K step launches (parity alternating, K is
// even so every lattice ends on the buffer it started from), then the check
// and the momentum reset.
int batch_graph(mplb_batch* b) {
    if (b->graph && b->graph_cfg == b->cfg && b->graph_K == b->K) return 0;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    for (uint32_t s = 0; s < b->K && !rc; s++) rc = batch_launch(b, b->cfg, b->grid, (int)(s & 1));
    if (!rc) rc = batch_check(b, 0, true);
    cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
    b->launches -= b->K + 2;  // counted when replayed
    if (rc) {
        if (ee == cudaSuccess) cudaGraphDestroy(g);
        return rc;
    }
    CK(ee);
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    b->graph_cfg = b->cfg;
    b->graph_K = b->K;
    return 0;
}

// One filter window over the lattices in the work table: M steps, M the
// smallest even count above the longest window among `active` (even, so
// every lattice ends on the buffer it started from).  Lattice i sums the
// states after steps last-win[i] .. last-1 (last = M - 1); their mean
// replaces the state step `last` reads, and step `last` runs from it.
// *M_out = 0 when no active lattice is filtered (nothing launched).
int batch_window(mplb_batch* b, const std::vector<char>& active, uint32_t* M_out) {
    uint32_t W = 0;
    for (size_t i = 0; i < b->lat.size(); i++)
        if (active[i] && !b->win.empty()) W = std::max(W, b->win[i]);
    const uint32_t M = W ? (W + 2u) & ~1u : 0u, last = M - 1u;
    *M_out = M;
    if (!M) return 0;
    auto avg = [&](int parity, uint32_t s, int finish) -> int {
        cudaError_t e = mplb_batch32_average(b->cfg, b->dA, b->dtiles, b->dnt, parity, b->grid, b->dacc, b->dwin, s,
                                             last, finish, b->stream);
        b->launches++;
        if (e != cudaSuccess) return fail(MPLB_E_CUDA, std::string("batch filter launch: ") + cudaGetErrorString(e));
        return 0;
    };
    for (uint32_t s = 0; s < last; s++) {
        RET(batch_launch(b, b->cfg, b->grid, (int)(s & 1)));
        RET(avg((int)((s + 1) & 1), s, 0));
    }
    RET(avg((int)(last & 1), last, 1));
    RET(batch_launch(b, b->cfg, b->grid, (int)(last & 1)));
    b->windows++;
    return 0;
}

}  // namespace

extern "C" {

int mplb_batch_create(mplb_gpu_t* const* lattices, uint32_t count, const mplb_batch_opts* opts, mplb_batch_t** out) {
    if (!out) return fail(MPLB_E_ARG, "out is NULL");
    *out = nullptr;
    if (!lattices || count == 0) return fail(MPLB_E_ARG, "no lattices");
    const uint32_t K = opts ? opts->check_interval : 1000;
    if (K < 2 || (K & 1)) return fail(MPLB_E_ARG, "check_interval must be even and >= 2");
    std::unordered_set<const mplb_gpu*> seen;
    for (uint32_t i = 0; i < count; i++) {
        const mplb_gpu* h = lattices[i];
        if (!h) return fail(MPLB_E_ARG, "NULL handle in batch");
        if (!seen.insert(h).second) return fail(MPLB_E_ARG, "handle listed twice in batch");
        const std::string at = "lattice " + std::to_string(i) + ": ";
        if (h->dev != lattices[0]->dev) return fail(MPLB_E_ARG, at + "batch lattices must share one device");
        if (h->lat != MPLB_D2Q9) return fail(MPLB_E_UNSUPPORTED, at + "batch needs D2Q9");
        if (h->precision != MPLB_FP32_DEV) return fail(MPLB_E_UNSUPPORTED, at + "batch needs MPLB_FP32_DEV");
        if (h->path != MPLB_PATH_FUSED) return fail(MPLB_E_UNSUPPORTED, at + "batch needs the fused path");
        if (h->fc.has_bc || !h->per[0] || !h->per[1])
            return fail(MPLB_E_UNSUPPORTED, at + "batch needs a fully periodic box without boundary patches");
        if (!h->P.f_update || h->P.g_update) return fail(MPLB_E_UNSUPPORTED, at + "batch needs f updated, g frozen");
    }
    mplb_batch* b = new mplb_batch();
    b->dev = lattices[0]->dev;
    b->stream = lattices[0]->stream;
    b->lat.assign(lattices, lattices + count);
    b->K = K;
    b->tol = opts ? opts->tol : 1e-9;
    b->tile_request = opts ? opts->tile_config : 0;
    DeviceGuard guard(b->dev);
    size_t cap = 0;
    for (int c = 0; c < mplb_batch_ncfg(); c++) {
        int tx = 0, ty = 0;
        mplb_batch_cfg(c, &tx, &ty);
        size_t t = 0;
        for (mplb_gpu* h : b->lat) t += (size_t)((h->fc.args.nx + tx - 1) / tx) * ((h->fc.args.ny + ty - 1) / ty);
        cap = std::max(cap, t);
    }
    b->tile_cap = cap;
    std::vector<Params> P(count);
    std::vector<double*> snaps(count);
    for (uint32_t i = 0; i < count; i++) {
        P[i] = b->lat[i]->P;
        b->nodes += b->lat[i]->n;
    }
    auto setup = [&]() -> int {
        CK(cudaMalloc((void**)&b->dP, count * sizeof(Params)));
        CK(cudaMalloc((void**)&b->dA, 2 * count * sizeof(FusedArgs32)));
        CK(cudaMalloc((void**)&b->dtiles, std::max<size_t>(cap, 1) * sizeof(int2)));
        CK(cudaMalloc((void**)&b->dnt, sizeof(int)));
        CK(cudaMalloc((void**)&b->dsnap, count * sizeof(double*)));
        CK(cudaMalloc((void**)&b->snap, b->nodes * sizeof(double)));
        CK(cudaMalloc((void**)&b->dmax, count * sizeof(unsigned long long)));
        CK(cudaMallocHost((void**)&b->hmax, count * sizeof(unsigned long long)));
        CK(cudaMalloc((void**)&b->jsum, 3 * count * sizeof(long long)));
        CK(cudaMalloc((void**)&b->j0, 3 * count * sizeof(long long)));
        CK(cudaMalloc((void**)&b->proj, count * sizeof(int)));
        std::vector<int> pr(count);
        for (uint32_t i = 0; i < count; i++) pr[i] = momentum_conserved(b->lat[i]) ? 1 : 0;
        CK(cudaMemcpyAsync(b->proj, pr.data(), count * sizeof(int), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        size_t off = 0;
        for (uint32_t i = 0; i < count; i++) {
            snaps[i] = b->snap + off;
            off += b->lat[i]->n;
        }
        CK(cudaMemcpyAsync(b->dP, P.data(), count * sizeof(Params), cudaMemcpyHostToDevice, b->stream));
        CK(cudaMemcpyAsync(b->dsnap, snaps.data(), count * sizeof(double*), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        return 0;
    };
    if (int rc = setup()) {
        batch_free(b);
        delete b;
        return rc;
    }
    *out = b;
    return 0;
}

int mplb_batch_destroy(mplb_batch_t* b) {
    if (!b) return 0;
    DeviceGuard guard(b->dev);
    cudaStreamSynchronize(b->stream);
    batch_free(b);
    delete b;
    return 0;
}

int mplb_batch_info_get(mplb_batch_t* b, mplb_batch_info* info) {
    if (!b || !info) return fail(MPLB_E_ARG, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->n_lattices = (uint32_t)b->lat.size();
    info->nodes = b->nodes;
    info->tile_config = b->cfg;
    info->n_candidates = mplb_batch_ncfg();
    for (int c = 0; c < mplb_batch_ncfg() && c < 8; c++) {
        int tx = 0, ty = 0;
        mplb_batch_cfg(c, &tx, &ty);
        info->tile_x[c] = tx;
        info->tile_y[c] = ty;
        info->tile_ms[c] = b->tile_ms[c];
    }
    info->grid = b->grid;
    info->kernel_launches = b->launches;
    info->graph_launches = b->graph_launches;
    return 0;
}

int mplb_batch_step(mplb_batch_t* b, uint32_t nsteps) {
    if (!b) return fail(MPLB_E_ARG, "NULL batch");
    if (nsteps == 0) return 0;
    DeviceGuard guard(b->dev);
    RET(batch_enter(b));
    const std::vector<char> all(b->lat.size(), 1);
    int nt = 0;
    RET(batch_ready(b, all, &nt));
    for (uint32_t s = 0; s < nsteps; s++) RET(batch_launch(b, b->cfg, b->grid, (int)(s & 1)));
    for (mplb_gpu* h : b->lat) {
        if (nsteps & 1) h->cur32[0] ^= 1;
        h->current += nsteps;
    }
    return batch_leave(b);
}

int mplb_batch_run(mplb_batch_t* b, uint32_t max_steps, uint32_t* steps_out, double* rate_out,
                   uint32_t* n_converged) {
    if (!b) return fail(MPLB_E_ARG, "NULL batch");
    DeviceGuard guard(b->dev);
    const size_t N = b->lat.size();
    RET(batch_enter(b));
    std::vector<char> active(N, 1);
    std::vector<uint32_t> steps(N, 0);
    std::vector<double> rate(N, -1.0);
    int nt = 0;
    RET(batch_ready(b, active, &nt));
    RET(batch_graph(b));
    RET(batch_check(b, 0, false));  // snapshot of the starting rho and momentum
    CK(cudaMemcpyAsync(b->j0, b->jsum, 3 * N * sizeof(long long), cudaMemcpyDeviceToDevice, b->stream));
    size_t left = N;
    uint32_t done = 0, conv = 0;
    // the check of an interval of `len` steps has been queued: read it, retire lattices
    auto account = [&](uint32_t len) -> int {
        CK(cudaMemcpyAsync(b->hmax, b->dmax, N * sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        done += len;
        bool retired = false;
        for (size_t i = 0; i < N; i++) {
            if (!active[i]) continue;
            steps[i] += len;
            double d;
            std::memcpy(&d, &b->hmax[i], sizeof(double));
            rate[i] = d / len;
            if (rate[i] < b->tol || !std::isfinite(rate[i])) {  // converged, or failed (non-finite)
                active[i] = 0;
                left--;
                if (std::isfinite(rate[i])) conv++;
                retired = true;
            }
        }
        if (retired && left) RET(batch_table(b, b->cfg, active, &nt));
        return 0;
    };
    // filter windows: the first once `filter_first` steps are done, then one
    // `filter_every` steps after the end of the previous, each at the end of
    // a check interval and followed by a check of its own
    uint64_t next_window = b->filter_every && !b->win.empty() ? b->filter_first : UINT64_MAX;
    while (left && done < max_steps) {
        if (done >= next_window) {
            uint32_t M = 0;
            RET(batch_window(b, active, &M));
            if (M) {
                RET(batch_check(b, 0, true));
                RET(account(M));
                next_window = (uint64_t)done + b->filter_every;
                continue;
            }
            next_window = UINT64_MAX;  // no active lattice is filtered
        }
        CK(cudaGraphLaunch(b->graph, b->stream));
        b->graph_launches++;
        b->launches += b->K + 2;
        RET(account(b->K));
    }
    for (size_t i = 0; i < N; i++) {
        b->lat[i]->current += steps[i];
        if (steps_out) steps_out[i] = steps[i];
        if (rate_out) rate_out[i] = rate[i];
    }
    if (n_converged) *n_converged = conv;
    return batch_leave(b);
}

int mplb_batch_filter(mplb_batch_t* b, const uint32_t* window, uint32_t first, uint32_t every) {
    if (!b) return fail(MPLB_E_ARG, "NULL batch");
    DeviceGuard guard(b->dev);
    const size_t N = b->lat.size();
    // finish queued work before the accumulators change
    CK(cudaStreamSynchronize(b->stream));
    for (void* p : {(void*)b->dwin, (void*)b->acc, (void*)b->dacc})
        if (p) cudaFree(p);
    b->dwin = nullptr;
    b->acc = nullptr;
    b->dacc = nullptr;
    b->win.clear();
    b->filter_first = b->filter_every = 0;
    if (!window) return 0;  // filter off
    size_t tot = 0;
    for (size_t i = 0; i < N; i++) {
        if (window[i] > MPLB_BATCH_MAX_WINDOW)
            return fail(MPLB_E_ARG, "lattice " + std::to_string(i) + ": window longer than MPLB_BATCH_MAX_WINDOW");
        if (window[i]) tot += (size_t)b->lat[i]->Q * b->lat[i]->n;
    }
    std::vector<double*> ptr(N, nullptr);
    auto setup = [&]() -> int {
        if (tot) CK(cudaMalloc((void**)&b->acc, tot * sizeof(double)));
        CK(cudaMalloc((void**)&b->dacc, N * sizeof(double*)));
        CK(cudaMalloc((void**)&b->dwin, N * sizeof(uint32_t)));
        size_t off = 0;
        for (size_t i = 0; i < N; i++) {
            if (!window[i]) continue;
            ptr[i] = b->acc + off;
            off += (size_t)b->lat[i]->Q * b->lat[i]->n;
        }
        CK(cudaMemcpyAsync(b->dacc, ptr.data(), N * sizeof(double*), cudaMemcpyHostToDevice, b->stream));
        CK(cudaMemcpyAsync(b->dwin, window, N * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        return 0;
    };
    if (int rc = setup()) {
        for (void* p : {(void*)b->dwin, (void*)b->acc, (void*)b->dacc})
            if (p) cudaFree(p);
        b->dwin = nullptr;
        b->acc = nullptr;
        b->dacc = nullptr;
        return rc;
    }
    b->win.assign(window, window + N);
    b->filter_first = first;
    b->filter_every = every;
    return 0;
}

int mplb_batch_average(mplb_batch_t* b, uint32_t* steps_out) {
    if (!b) return fail(MPLB_E_ARG, "NULL batch");
    if (steps_out) *steps_out = 0;
    if (b->win.empty()) return fail(MPLB_E_STATE, "no filter windows set (mplb_batch_filter)");
    DeviceGuard guard(b->dev);
    RET(batch_enter(b));
    const std::vector<char> all(b->lat.size(), 1);
    int nt = 0;
    RET(batch_ready(b, all, &nt));
    uint32_t M = 0;
    RET(batch_window(b, all, &M));
    for (mplb_gpu* h : b->lat) h->current += M;
    if (steps_out) *steps_out = M;
    return batch_leave(b);
}

}  // extern "C"

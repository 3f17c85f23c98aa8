// fused_host.cuh -- host side of the fused box path: boundary-program
// tables, candidate launches, the tile autotuner.  Included only by the FP64
// translation unit, so the FP64 kernels are instantiated in exactly one
// object (compiled without multiply-add contraction).
#pragma once

#include <cudaTypedefs.h>

#include "fused.cuh"
#include "fused_tma.cuh"

namespace mplb {

// Tensor maps of one TMA candidate over one input population buffer and the
// temperature field (a map holds its box shape, so each candidate has its own).
struct TmaMaps {
    int cfg = -1;
    const void* f = nullptr;
    const void* T = nullptr;
    alignas(64) CUtensorMap mf;
    alignas(64) CUtensorMap mT;
};

struct FusedConfig {
    std::string err;
    FusedArgs args{};
    uint8_t* bcmap = nullptr;
    bool has_bc = false;
    int lat = 0;
    int cfg = 0;           // chosen candidate
    bool tuned = false;    // autotuner has run (or a candidate was forced)
    Geom geom[N_CFG_MAX];
    float tune_ms[N_CFG_MAX] = {};
    int ncfg = 0;
    int nblocks = 0;
    double* my_scratch = nullptr;  // myMRT: rho_a and gsum_a, 2 n doubles
    int* kerr = nullptr;           // kernel error flag (bounded waits), one int
    int* kerr_host = nullptr;      // its pinned host copy
    TmaMaps tmaps[4];              // two TMA candidates x two population buffers
    int tmaps_next = 0;
};

// cuTensorMapEncodeTiled from the driver, found through the runtime (the
// library does not link the driver API).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The maps of TMA candidate `cfg` for the step's input buffers: the
// populations as a 4D tensor (x, y, z, k) and T as a 3D one (x, y, z), FP64,
// boxes of (TX+4) x (TY+2) x 1 (x 1), no swizzle, zero fill (never read: the
// kernel takes tensor copies only for boxes inside the lattice).
inline const TmaMaps* tma_maps(FusedConfig& fc, int cfg, const FusedArgs& A, uint32_t n) {
    for (const TmaMaps& m : fc.tmaps)
        if (m.cfg == cfg && m.f == A.fin && m.T == A.Told) return &m;
    auto enc = tensor_map_encoder();
    if (!enc) {
        fc.err = "cuTensorMapEncodeTiled is not available from the driver";
        return nullptr;
    }
    TmaMaps& m = fc.tmaps[fc.tmaps_next];
    const TileCfg t = CFG3[cfg];
    const cuuint64_t dims[4] = {(cuuint64_t)A.nx, (cuuint64_t)A.ny, (cuuint64_t)A.nz, 15};
    const cuuint64_t strides[3] = {(cuuint64_t)A.nx * 8, (cuuint64_t)A.nx * A.ny * 8, (cuuint64_t)n * 8};
    const cuuint32_t box[4] = {(cuuint32_t)(t.tx + 4), (cuuint32_t)(t.ty + 2), 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(&m.mf, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(A.fin), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = enc(&m.mT, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(A.Told), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fc.err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        m.cfg = -1;
        return nullptr;
    }
    m.cfg = cfg;
    m.f = A.fin;
    m.T = A.Told;
    fc.tmaps_next = (fc.tmaps_next + 1) % 4;
    return &m;
}

template <int TX, int TY, bool PIPE, bool HAS_BC, bool EMIT>
cudaError_t set_smem3() {
    if constexpr (PIPE)
        return cudaFuncSetAttribute(k_fused_d3q15_pipe<TX, TY, HAS_BC, EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)f3_smem<TX, TY, PIPE>());
    else
        return cudaFuncSetAttribute(k_fused_d3q15<TX, TY, HAS_BC, EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)f3_smem<TX, TY, PIPE>());
}

// The 3D kernels use more than the 48 KB of static shared memory.
inline cudaError_t fused_attributes() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    chk(set_smem3<32, 8, false, true, true>());
    chk(set_smem3<32, 8, false, false, true>());
#define MPLB_SET3(TX, TY, PIPE) chk(set_smem3<TX, TY, PIPE, true, false>()); chk(set_smem3<TX, TY, PIPE, false, false>());
    MPLB_SET3(32, 8, false)
    MPLB_SET3(32, 8, true)
    MPLB_SET3(32, 4, false)
    MPLB_SET3(64, 4, false)
    MPLB_SET3(32, 16, false)
    MPLB_SET3(64, 8, false)
#undef MPLB_SET3
    chk(cudaFuncSetAttribute(k_fused_d3q15_tma<32, 4, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TmaTile<32, 4>::SMEM));
    chk(cudaFuncSetAttribute(k_fused_d3q15_tma<32, 8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TmaTile<32, 8>::SMEM));
    chk(cudaFuncSetAttribute(k_fused_d3q15_tma<32, 16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TmaTile<32, 16>::SMEM));
    chk(cudaFuncSetAttribute(k_fused_d3q15_tma<64, 8, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TmaTile<64, 8>::SMEM));
    return e;
}

template <int TX, int TY, int MINB>
cudaError_t launch3_tma(FusedConfig& fc, int cfg, int nb, const Params& P, const FusedArgs& A, cudaStream_t s) {
    const TmaMaps* m = tma_maps(fc, cfg, A, P.n);
    if (!m) return cudaErrorInvalidValue;
    launch_step(k_fused_d3q15_tma<TX, TY, MINB>, nb, TX * TY, TmaTile<TX, TY>::SMEM, s, P, A, m->mf, m->mT);
    return cudaSuccess;
}

template <int TX, int TY, int MINB, bool F_ON, bool G_ON, bool EMIT, bool INNER, bool MY = false, int RINGW = 0>
void launch2(bool bc, int nb, const Params& P, const FusedArgs& A, cudaStream_t s) {
    constexpr int nt = TX * TY + 32 * RINGW;
    if (bc) launch_step(k_fused_d2q9<TX, TY, MINB, F_ON, G_ON, true, EMIT, INNER, MY, RINGW>, nb, nt, 0, s, P, A);
    else launch_step(k_fused_d2q9<TX, TY, MINB, F_ON, G_ON, false, EMIT, INNER, MY, RINGW>, nb, nt, 0, s, P, A);
}

// myMRT steps first fill rho_a, gsum_a (k_pullsum_d2q9).
template <bool F_ON>
void launch_pullsum(bool bc, const Params& P, const FusedArgs& A, cudaStream_t s) {
    const unsigned nb = (P.n + 255) / 256;
    if (bc) launch_step(k_pullsum_d2q9<F_ON, true>, nb, 256, 0, s, P, A);
    else launch_step(k_pullsum_d2q9<F_ON, false>, nb, 256, 0, s, P, A);
}

template <int TX, int TY, bool EMIT, int MINB = 0, bool INNER = false, int RINGW = 0>
void launch2_fg(bool fon, bool gon, bool bc, int nb, const Params& P, const FusedArgs& A, cudaStream_t s) {
    const bool my = gon && P.g_model == MPLB_MYMRT;
    if (my) {
        if constexpr (!EMIT) {
            if (fon) launch_pullsum<true>(bc, P, A, s);
            else launch_pullsum<false>(bc, P, A, s);
        }
        if (fon) launch2<TX, TY, MINB, true, true, EMIT, INNER, true, RINGW>(bc, nb, P, A, s);
        else launch2<TX, TY, MINB, false, true, EMIT, INNER, true, RINGW>(bc, nb, P, A, s);
        return;
    }
    if (fon && gon) launch2<TX, TY, MINB, true, true, EMIT, INNER, false, RINGW>(bc, nb, P, A, s);
    else if (fon) launch2<TX, TY, MINB, true, false, EMIT, INNER, false, RINGW>(bc, nb, P, A, s);
    else if (gon) launch2<TX, TY, MINB, false, true, EMIT, INNER, false, RINGW>(bc, nb, P, A, s);
}

template <int TX, int TY, bool PIPE, bool EMIT>
void launch3(bool bc, int nb, const Params& P, const FusedArgs& A, cudaStream_t s) {
    constexpr size_t sm = f3_smem<TX, TY, PIPE>();
    if constexpr (PIPE) {
        if (bc) launch_step(k_fused_d3q15_pipe<TX, TY, true, EMIT>, nb, TX * TY, sm, s, P, A);
        else launch_step(k_fused_d3q15_pipe<TX, TY, false, EMIT>, nb, TX * TY, sm, s, P, A);
    } else {
        if (bc) launch_step(k_fused_d3q15<TX, TY, true, EMIT>, nb, TX * TY, sm, s, P, A);
        else launch_step(k_fused_d3q15<TX, TY, false, EMIT>, nb, TX * TY, sm, s, P, A);
    }
}

// Launch one fused step with candidate `cfg` (EMIT always uses candidate 0).
inline cudaError_t fused_launch_cfg(FusedConfig& fc, int cfg, const Params& P, FusedArgs A, bool f_on, bool g_on,
                                    bool emit, cudaStream_t s) {
    if (emit) cfg = 0;
    apply_geom(A, fc.geom[cfg]);
    const int nb = fc.geom[cfg].nblocks;
    if (nb == 0) return cudaErrorInvalidConfiguration;  // the candidate does not take this lattice
    const bool bc = fc.has_bc;
    if (fc.lat == MPLB_D2Q9) {
        if (emit) {
            launch2_fg<32, 8, true>(f_on, g_on, bc, nb, P, A, s);
        } else {
            switch (cfg) {
            case 0: launch2_fg<32, 8, false>(f_on, g_on, bc, nb, P, A, s); break;
            case 1: launch2_fg<32, 4, false>(f_on, g_on, bc, nb, P, A, s); break;
            case 2: launch2_fg<64, 4, false>(f_on, g_on, bc, nb, P, A, s); break;
            case 3: launch2_fg<16, 8, false, 0, true>(f_on, g_on, bc, nb, P, A, s); break;
            case 4: launch2_fg<64, 4, false, 0, true>(f_on, g_on, bc, nb, P, A, s); break;
            case 5: launch2_fg<16, 8, false, 6, true>(f_on, g_on, bc, nb, P, A, s); break;
            case 6: launch2_fg<32, 8, false, 3, true>(f_on, g_on, bc, nb, P, A, s); break;
            case 7: launch2_fg<32, 4, false, 8, true>(f_on, g_on, bc, nb, P, A, s); break;
            case 8: launch2_fg<32, 8, false, 2, false, 3>(f_on, g_on, bc, nb, P, A, s); break;
            default: launch2_fg<16, 8, false, 4, false, 2>(f_on, g_on, bc, nb, P, A, s); break;
            }
        }
    } else {
        if (emit) {
            launch3<32, 8, false, true>(bc, nb, P, A, s);
        } else {
            switch (cfg) {
            case 0: launch3<32, 8, false, false>(bc, nb, P, A, s); break;
            case 1: launch3<32, 8, true, false>(bc, nb, P, A, s); break;
            case 2: launch3<32, 4, false, false>(bc, nb, P, A, s); break;
            case 3: launch3<64, 4, false, false>(bc, nb, P, A, s); break;
            case 4: launch3<32, 16, false, false>(bc, nb, P, A, s); break;
            case 5: launch3<64, 8, false, false>(bc, nb, P, A, s); break;
            case 6: if (cudaError_t e = launch3_tma<32, 4, 3>(fc, cfg, nb, P, A, s)) return e; break;
            case 7: if (cudaError_t e = launch3_tma<32, 8, 2>(fc, cfg, nb, P, A, s)) return e; break;
            case 8: if (cudaError_t e = launch3_tma<32, 16, 1>(fc, cfg, nb, P, A, s)) return e; break;
            default: if (cudaError_t e = launch3_tma<64, 8, 1>(fc, cfg, nb, P, A, s)) return e; break;
            }
        }
    }
    return cudaGetLastError();
}

inline cudaError_t fused_launch(FusedConfig& fc, const Params& P, const FusedArgs& A, int lat, bool f_on,
                                bool g_on, bool emit, cudaStream_t s) {
    (void)lat;
    return fused_launch_cfg(fc, fc.cfg, P, A, f_on, g_on, emit, s);
}

// Time every candidate on the current state and keep the fastest.  Three
// sweeps over the candidates (so a transient -- clocks settling, another
// process -- does not favour the candidates timed during it); in each, a
// candidate's warm-up launch and 8 timed launches are queued back to back
// with an event between consecutive launches and one host wait at the end,
// so a launch's interval holds its device time only (a host wait between
// launches would add the host's launch latency, several microseconds, to
// every interval: on a lattice of one wave that is as large as the
// differences between candidates).  A candidate's time is the median of its
// 24 intervals.  The step's outputs are rewritten by the real launch that
// follows; the heat-source history S, updated in place, is saved to `save`
// before and restored after every candidate's launches.
inline int fused_autotune(FusedConfig& fc, const Params& P, const FusedArgs& A, bool f_on, bool g_on, double* S,
                          double* save, size_t n, cudaStream_t s) {
    constexpr int SWEEPS = 3, WARM = 1, TIMED = 8;
    cudaEvent_t ev[TIMED + 1];
    int made = 0;
    for (; made < TIMED + 1; made++)
        if (cudaEventCreate(&ev[made]) != cudaSuccess) break;
    if (made < TIMED + 1) {
        for (int i = 0; i < made; i++) cudaEventDestroy(ev[i]);
        fc.err = "autotune: event creation failed";
        return MPLB_E_CUDA;
    }
    const bool keep_s = g_on && S && save;
    if (keep_s && cudaMemcpyAsync(save, S, n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        for (int i = 0; i < TIMED + 1; i++) cudaEventDestroy(ev[i]);
        fc.err = "autotune: saving S failed";
        return MPLB_E_CUDA;
    }
    float ms_all[N_CFG_MAX][SWEEPS * TIMED];
    bool ok_c[N_CFG_MAX];
    for (int c = 0; c < fc.ncfg; c++) ok_c[c] = fc.geom[c].nblocks > 0;
    for (int sw = 0; sw < SWEEPS; sw++) {
        for (int c = 0; c < fc.ncfg; c++) {
            bool ok = ok_c[c];
            for (int r = 0; r < WARM + TIMED && ok; r++) {
                if (r >= WARM) cudaEventRecord(ev[r - WARM], s);
                ok = fused_launch_cfg(fc, c, P, A, f_on, g_on, false, s) == cudaSuccess;
            }
            if (ok) cudaEventRecord(ev[TIMED], s);
            if (ok && cudaEventSynchronize(ev[TIMED]) == cudaSuccess) {
                for (int r = 0; r < TIMED; r++) {
                    float ms = 0;
                    cudaEventElapsedTime(&ms, ev[r], ev[r + 1]);
                    ms_all[c][sw * TIMED + r] = ms;
                }
            } else {
                ok = false;
            }
            if (keep_s) cudaMemcpyAsync(S, save, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
            ok_c[c] = ok;
        }
    }
    float best = 1e30f;
    int best_cfg = 0;
    for (int c = 0; c < fc.ncfg; c++) {
        float med = -1.0f;
        if (ok_c[c]) {
            float* m = ms_all[c];
            std::sort(m, m + SWEEPS * TIMED);
            med = 0.5f * (m[SWEEPS * TIMED / 2 - 1] + m[SWEEPS * TIMED / 2]);
        }
        fc.tune_ms[c] = ok_c[c] ? med : -1.0f;
        if (ok_c[c] && med >= 0 && med < best) {
            best = med;
            best_cfg = c;
        }
    }
    cudaGetLastError();
    for (int i = 0; i < TIMED + 1; i++) cudaEventDestroy(ev[i]);
    fc.cfg = best_cfg;
    fc.nblocks = fc.geom[best_cfg].nblocks;
    fc.tuned = true;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : MPLB_E_CUDA;
}

// Fused path preconditions: box mesh, no serial boundary dependence, only
// bounceBack / fixedT / periodic patches, at most FUSED_MAX_OPS ops per node
// and field, at most FUSED_MAX_PROGS distinct node programs.
inline bool fused_supported(int lat, const int* model, const Params& P, const std::vector<PatchDev>* fp,
                            const bool* serial, const mplb_mesh_desc* mesh, const int* dims, const int* per,
                            std::string& why) {
    (void)per;
    const bool active[2] = {model[0] != MPLB_NO_MODEL && P.f_update != 0, model[1] != MPLB_NO_MODEL && P.g_update != 0};
    if (serial[0] || serial[1]) { why = "boundary updates depend on the serial order"; return false; }
    if (!active[0] && !active[1]) { why = "no field is updated"; return false; }
    if (!active[0] && model[0] == MPLB_NO_MODEL) { why = "no flow field"; return false; }
    if (lat == MPLB_D3Q15 && active[1]) { why = "thermal field on D3Q15"; return false; }
    for (int fi = 0; fi < 2; fi++) {
        if (!active[fi]) continue;
        for (const PatchDev& pt : fp[fi]) {
            if (pt.type == MPLB_BC_PERIODIC) continue;
            if (pt.type == MPLB_BC_BOUNCEBACK) continue;
            if (pt.type == MPLB_BC_FIXEDT && fi == 1) continue;
            if (pt.type == MPLB_BC_FIXEDU && model[fi] != MPLB_LIMRT) continue;  // no-op
            why = "boundary type " + std::to_string(pt.type) + " is handled by the operator path only";
            return false;
        }
    }
    if (dims[0] < 2 || dims[1] < 2 || (lat == MPLB_D3Q15 && dims[2] < 2)) { why = "box thinner than 2 nodes"; return false; }
    (void)mesh;
    return true;
}

inline int fused_setup(FusedConfig& fc, int lat, const int* model, const Params& P, const std::vector<PatchDev>* fp,
                       const mplb_mesh_desc* mesh, const int* dims, const int* per, cudaStream_t stream,
                       uint64_t* bytes) {
    (void)model;
    FusedArgs& A = fc.args;
    A.nx = dims[0];
    A.ny = dims[1];
    A.nz = lat == MPLB_D3Q15 ? dims[2] : 1;
    A.px = per[0];
    A.py = per[1];
    A.pz = lat == MPLB_D3Q15 ? per[2] : 1;
    A.own_lo = 0;
    A.own_cnt = P.n;  // every node's outputs stored; slabs narrow it (mplb_gpu_set_owned)
    A.nmirror = 0;
    // Node programs: for every node, the ops of every patch holding it, in
    // patch order, per field.  Identical programs share one table entry.
    const uint32_t n = P.n;
    std::vector<uint8_t> map(n, 0);
    std::vector<BCProg> progs(1, BCProg{});
    std::vector<BCProg> per_node;
    bool any = false;
    {
        std::vector<BCProg> node(n, BCProg{});
        size_t off = 0;
        for (size_t p = 0; p < fp[0].size(); p++) {
            for (uint32_t i = 0; i < fp[0][p].count; i++) {
                uint32_t id = mesh->patch_nodes[off + i];
                for (int fi = 0; fi < 2; fi++) {
                    if (!(fi == 0 ? P.f_update : P.g_update)) continue;
                    int t = fp[fi][p].type;
                    if (t != MPLB_BC_BOUNCEBACK && t != MPLB_BC_FIXEDT) continue;
                    BCProg& b = node[id];
                    if (fi == 0) {
                        if (b.nf >= FUSED_MAX_OPS) { fc.err = "too many boundary ops on one node"; return MPLB_E_UNSUPPORTED; }
                        b.ft[b.nf++] = (uint8_t)t;
                    } else {
                        if (b.ng >= FUSED_MAX_OPS) { fc.err = "too many boundary ops on one node"; return MPLB_E_UNSUPPORTED; }
                        b.gp[b.ng] = (uint8_t)p;
                        b.gt[b.ng++] = (uint8_t)t;
                    }
                    any = true;
                }
            }
            off += fp[0][p].count;
        }
        for (uint32_t id = 0; id < n; id++) {
            const BCProg& b = node[id];
            if (b.nf == 0 && b.ng == 0) continue;
            int found = -1;
            for (size_t q = 1; q < progs.size(); q++)
                if (std::memcmp(&progs[q], &b, sizeof(BCProg)) == 0) { found = (int)q; break; }
            if (found < 0) {
                if (progs.size() >= FUSED_MAX_PROGS) { fc.err = "too many distinct boundary programs"; return MPLB_E_UNSUPPORTED; }
                progs.push_back(b);
                found = (int)progs.size() - 1;
            }
            map[id] = (uint8_t)found;
        }
    }
    // farthest distance of a node with a boundary program from its nearest
    // box face (-1: none); tiles whose ring lies farther in hold none
    A.bc_margin = -1;
    for (uint32_t id = 0; id < n; id++) {
        if (!map[id]) continue;
        const int x = (int)(id % (uint32_t)A.nx), y = (int)((id / (uint32_t)A.nx) % (uint32_t)A.ny);
        const int z = (int)(id / ((uint32_t)A.nx * (uint32_t)A.ny));
        int d = std::min(std::min(x, A.nx - 1 - x), std::min(y, A.ny - 1 - y));
        if (lat == MPLB_D3Q15) d = std::min(d, std::min(z, A.nz - 1 - z));
        A.bc_margin = std::max(A.bc_margin, d);
    }
    for (size_t q = 0; q < progs.size(); q++) A.prog[q] = progs[q];
    for (size_t p = 0; p < fp[1].size() && p < MPLB_MAX_PATCHES; p++) A.Twall[p] = fp[1][p].val[0];
    fc.has_bc = any;
    if (any) {
        if (cudaMalloc((void**)&fc.bcmap, n) != cudaSuccess) { fc.err = "cudaMalloc bcmap"; return MPLB_E_CUDA; }
        if (cudaMemcpyAsync(fc.bcmap, map.data(), n, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
            fc.err = "copy bcmap";
            return MPLB_E_CUDA;
        }
        if (cudaStreamSynchronize(stream) != cudaSuccess) { fc.err = "copy bcmap"; return MPLB_E_CUDA; }
        *bytes += n;
    }
    A.bcmap = fc.bcmap;
    A.rho_a = A.gsum_a = nullptr;
    if (lat == MPLB_D2Q9 && model[1] == MPLB_MYMRT && P.g_update) {
        if (cudaMalloc((void**)&fc.my_scratch, 2 * (size_t)n * sizeof(double)) != cudaSuccess) {
            fc.err = "cudaMalloc myMRT scratch";
            return MPLB_E_CUDA;
        }
        *bytes += 2 * (size_t)n * sizeof(double);
        A.rho_a = fc.my_scratch;
        A.gsum_a = fc.my_scratch + n;
    }
    fc.lat = lat;
    fc.ncfg = lat == MPLB_D2Q9 ? N_CFG2 : N_CFG3;
    for (int c = 0; c < fc.ncfg; c++) {
        const TileCfg t = lat == MPLB_D2Q9 ? CFG2[c] : CFG3[c];
        if (t.tma) {
            fc.geom[c] = tma3_fits(A, any, t.tx, t.ty) ? resident_geometry(A, t.tx, t.ty, t.minb) : Geom{0, 0, 0, 0};
        } else {
            fc.geom[c] = fused_geometry(lat, A, t.tx, t.ty);
        }
    }
    if (cudaMalloc((void**)&fc.kerr, sizeof(int)) != cudaSuccess) { fc.err = "cudaMalloc kernel flag"; return MPLB_E_CUDA; }
    if (cudaMallocHost((void**)&fc.kerr_host, sizeof(int)) != cudaSuccess) { fc.err = "cudaMallocHost kernel flag"; return MPLB_E_CUDA; }
    *fc.kerr_host = 0;
    if (cudaMemsetAsync(fc.kerr, 0, sizeof(int), stream) != cudaSuccess) { fc.err = "clear kernel flag"; return MPLB_E_CUDA; }
    *bytes += sizeof(int);
    A.kerr = fc.kerr;
    fc.cfg = 0;
    apply_geom(A, fc.geom[0]);
    fc.nblocks = fc.geom[0].nblocks;
    if (lat == MPLB_D3Q15 && fused_attributes() != cudaSuccess) {
        fc.err = "cannot raise the dynamic shared memory limit";
        return MPLB_E_CUDA;
    }
    return 0;
}

// The kernel error flag (0, or MPLB_KERR_WAIT after a bounded wait ran
// out): queue its copy to the pinned host int and its reset on the stream;
// after the caller's next synchronisation fused_kerr_value() holds it.
inline bool fused_queue_kerr(FusedConfig& fc, cudaStream_t s) {
    if (!fc.kerr) return true;
    return cudaMemcpyAsync(fc.kerr_host, fc.kerr, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
           cudaMemsetAsync(fc.kerr, 0, sizeof(int), s) == cudaSuccess;
}
inline int fused_kerr_value(const FusedConfig& fc) { return fc.kerr_host ? *fc.kerr_host : 0; }

inline void fused_free(FusedConfig& fc) {
    if (fc.kerr) cudaFree(fc.kerr);
    fc.kerr = nullptr;
    if (fc.kerr_host) cudaFreeHost(fc.kerr_host);
    fc.kerr_host = nullptr;
    if (fc.bcmap) cudaFree(fc.bcmap);
    fc.bcmap = nullptr;
    if (fc.my_scratch) cudaFree(fc.my_scratch);
    fc.my_scratch = nullptr;
}


}  // namespace mplb

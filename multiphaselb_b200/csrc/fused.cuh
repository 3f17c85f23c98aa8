// fused.cuh -- fused box kernels (placeholder until the fused path lands).
#pragma once
#include <string>
#include <vector>
#include "ops.cuh"

namespace mplb {

struct FusedConfig {
    std::string err;
};

inline bool fused_supported(int, const int*, const Params&, const std::vector<PatchDev>*, const bool*,
                            const mplb_mesh_desc*, const int*, const int*, std::string& why) {
    why = "fused kernels not built";
    return false;
}
inline int fused_setup(FusedConfig& fc, int, const int*, const Params&, const std::vector<PatchDev>*,
                       const mplb_mesh_desc*, const int*, const int*, cudaStream_t, uint64_t*) {
    fc.err = "fused kernels not built";
    return MPLB_E_UNSUPPORTED;
}
inline int fused_run(FusedConfig& fc, const Params&, uint32_t, uint32_t, double* (*)[2], int*, double*,
                     double*&, double*&, double*, double*&, double*&, double*, double*, cudaStream_t,
                     uint64_t*) {
    fc.err = "fused kernels not built";
    return MPLB_E_UNSUPPORTED;
}
inline void fused_free(FusedConfig&) {}

}  // namespace mplb

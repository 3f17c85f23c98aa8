// mplb_noalloc.cu -- mass / energy sums that allocate no device memory.
//
// Who needs this: a caller that is not allowed to call cudaMalloc at the
// point where it wants the conservation check.  Examples are host code that
// runs inside a framework whose caching allocator owns all device memory and
// forbids raw allocations, a production time loop with a no-allocation
// policy (allocation can block or fail when memory is nearly full, and that
// must not happen mid-run), and code that must stay asynchronous (cudaMalloc
// may synchronise the device).  mplb_gpu_mass_energy() needs a handle, whose
// creation allocates; this entry point takes plain device arrays instead and
// keeps its scratch in a fixed array inside the library.
//
// Scratch: g_noalloc_scratch, 2 * NA_MAX_BLOCKS doubles (64 KiB), a file-scope
// __device__ array.  Every GPU that loads the library holds one copy until
// the process exits.  All calls on a device share it, so two calls whose
// kernels overlap on the GPU (different streams, no ordering between them)
// race on it and may return wrong sums; calls ordered on one stream are safe.
// Every block writes its own slot before the final pass reads it, so nothing
// has to be cleared between calls (the array keeps the last call's partials).
#include <cuda_runtime.h>

#include <string>

#include "../../include/mplb_gpu.h"

// error text shared with the rest of the library (mplb_gpu.cu)
int mplb_internal_fail(int code, const std::string& msg);

namespace {

constexpr int NA_TPB = 256;
constexpr int NA_ITEMS = 16;  // elements per thread
constexpr int NA_MAX_BLOCKS = 4096;
constexpr uint64_t NA_MAX_N = (uint64_t)NA_MAX_BLOCKS * NA_TPB * NA_ITEMS;  // 16,777,216

// In host code this name is only a host-side stand-in, never a device
// address: every call asks the runtime for the array's address on the
// current device (cudaGetSymbolAddress), so a module loaded again after a
// device reset is found where it now lies.
static __device__ __align__(256) double g_noalloc_scratch[2 * NA_MAX_BLOCKS];

__device__ __forceinline__ void block_sum2(double& a, double& b, double* sa, double* sb) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

// Block b sums elements [b*NA_TPB*NA_ITEMS, (b+1)*NA_TPB*NA_ITEMS) of x and y
// into part[2b], part[2b+1].  part is the scratch array's device address.
__global__ void __launch_bounds__(NA_TPB) na_partial(const double* __restrict__ x, const double* __restrict__ y,
                                                     uint32_t n, double* __restrict__ part) {
    __shared__ double sa[32], sb[32];
    const size_t base = (size_t)blockIdx.x * NA_TPB * NA_ITEMS;
    double a = 0, b = 0;
#pragma unroll 4
    for (int i = 0; i < NA_ITEMS; i++) {
        const size_t j = base + (size_t)i * NA_TPB + threadIdx.x;
        if (j < n) {
            a += x[j];
            if (y) b += y[j];
        }
    }
    block_sum2(a, b, sa, sb);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

__global__ void __launch_bounds__(NA_TPB) na_final(const double* __restrict__ part, int nparts, double* __restrict__ out) {
    __shared__ double sa[32], sb[32];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < nparts; i += NA_TPB) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    block_sum2(a, b, sa, sb);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
    }
}

}  // namespace

extern "C" int mplb_mass_energy_noalloc(const double* rho, const double* T, uint32_t n, double* out, void* stream) {
    if (!rho || !out) return mplb_internal_fail(MPLB_E_ARG, "mplb_mass_energy_noalloc: rho and out are required");
    if ((uint64_t)n > NA_MAX_N)
        return mplb_internal_fail(MPLB_E_ARG, "mplb_mass_energy_noalloc: n = " + std::to_string(n) +
                                                  " exceeds the fixed scratch limit of " + std::to_string(NA_MAX_N) +
                                                  " nodes; use mplb_gpu_mass_energy for larger lattices");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return mplb_internal_fail(MPLB_E_CUDA, std::string("mplb_mass_energy_noalloc: no current device: ") +
                                                   cudaGetErrorString(e));
    // An error left pending by earlier work would otherwise be read back after
    // the launches below and reported as theirs.
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return mplb_internal_fail(MPLB_E_CUDA, std::string("mplb_mass_energy_noalloc: an error from earlier CUDA "
                                                           "work was pending (now cleared), nothing was queued: ") +
                                                   cudaGetErrorString(e));
    // The first call on a device loads the library's module there; later
    // calls only look the address up.
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return mplb_internal_fail(MPLB_E_CUDA, std::string("mplb_mass_energy_noalloc: scratch lookup failed on device ") +
                                                   std::to_string(dev) + ": " + cudaGetErrorString(e));
    double* scratch = static_cast<double*>(p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nblocks = (int)(((uint64_t)n + (uint64_t)NA_TPB * NA_ITEMS - 1) / ((uint64_t)NA_TPB * NA_ITEMS));
    if (nblocks > 0) na_partial<<<nblocks, NA_TPB, 0, s>>>(rho, T, n, scratch);
    na_final<<<1, NA_TPB, 0, s>>>(scratch, nblocks, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return mplb_internal_fail(MPLB_E_CUDA, std::string("mplb_mass_energy_noalloc: launch failed: ") + cudaGetErrorString(e));
    return 0;
}

// mplb_mlp.cu -- learned warm start: a 5-64-64-64-1 tanh network that maps
// (T/Tc, a, b, r/R, R) to the equilibrium density of a static bubble, trained
// on the GPU on density profiles the solver itself converged.
//
// Precision: weights and activations are BF16 (round-to-nearest-even of the
// FP32 value), every dot product accumulates in FP32 with fmaf in a fixed
// order, biases, gradients and the Adam state are FP32.  The master weights
// are FP32; the BF16 copy is refreshed after every update.
//
// Kernels.  Inference (mplb_mlp_predict, mplb_mlp_init_bubble) runs the two
// 64 x 64 layers on the tensor cores, 128 samples per CTA (tcgen05.mma from
// shared memory into tensor memory, see k_mlp_predict).  Training runs on
// the CUDA cores: one block of 64 threads (thread j = unit j) carries SB
// samples through all layers with the weights in shared memory, forward and
// backward, and writes per-block gradient partials that a second kernel sums
// in a fixed order (deterministic) and feeds to Adam.
//
// This translation unit is compiled without FMA contraction: the feature
// normalisation below runs on host and device and must agree bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mplb_gpu.h"
#include "umma.cuh"

int mplb_internal_fail(int code, const std::string& msg);

namespace {

constexpr int NIN = 5, NH = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH * NH, OFF_W4 = OFF_B3 + NH, OFF_B4 = OFF_W4 + NH,
              NPARAM = OFF_B4 + 1;
static_assert(NPARAM == MPLB_MLP_PARAMS, "parameter layout");
constexpr int SB = 32;        // samples per block
constexpr int WS = NH + 1;    // padded row stride of the weight tiles (bank-conflict free)

// ---------------------------------------------------------------- features
__host__ __device__ inline uint32_t f2u(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}
__host__ __device__ inline float u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}
// Round to the nearest BF16 value, ties to even (finite inputs).
__host__ __device__ inline float bf16_round(float f) {
    uint32_t u = f2u(f);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return u2f(u & 0xFFFF0000u);
}
__host__ __device__ inline uint16_t bf16_bits(float f) { return (uint16_t)(f2u(bf16_round(f)) >> 16); }
__device__ inline float bf16_float(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Network inputs.  T/Tc centred on the trained range [0.6, 0.95]; the CS
// constants relative to a = 1, b = 4; the node position r/R and the radius R
// as the pair d = (r - R)/W and k = W/R (W = 5 lattice units, the initial
// interface width; r/R = 1 + d k), so the interface sits at d = 0 with a
// width independent of R and the curvature k carries the Laplace shift of
// the bulk densities.  A flat interface (a liquid column or band) is the
// limit R -> infinity: R = +inf, and r is then the signed distance to the
// interface, positive on the liquid side (k = 0).  d is clamped to [-6, 6]
// (bulk beyond).  Rounded to BF16 (GEMM operands).  Output: b * rho.
constexpr double W_IFACE = 5.0;
__host__ __device__ inline void features(double t_ratio, double a, double b, double r, double R, float* x) {
    const bool flat = R > 1.0e300;
    double d = (flat ? r : r - R) / W_IFACE;
    d = d < -6.0 ? -6.0 : (d > 6.0 ? 6.0 : d);
    x[0] = bf16_round((float)((t_ratio - 0.775) / 0.175));
    x[1] = bf16_round((float)(a - 1.0));
    x[2] = bf16_round((float)(b * 0.25 - 1.0));
    x[3] = bf16_round((float)(d / 6.0));
    x[4] = bf16_round((float)((W_IFACE / R - 0.3) / 0.3));
}

// ------------------------------------------------------------ block state
struct Block {
    float W1[NH * NIN], b1[NH], W2[NH * WS], b2[NH], W3[NH * WS], b3[NH], W4[NH], b4;
    float x[SB][NIN], h1[SB][NH], h2[SB][NH], h3[SB][NH], out[SB], dout[SB];
    float dzA[SB][NH], dzB[SB][NH];
};

__device__ void load_weights(Block& s, const float* __restrict__ P, const uint16_t* __restrict__ Wb) {
    const int t = threadIdx.x;
    for (int i = t; i < NH * NIN; i += blockDim.x) s.W1[i] = bf16_float(Wb[OFF_W1 + i]);
    for (int i = t; i < NH * NH; i += blockDim.x) {
        const int r = i / NH, c = i % NH;
        s.W2[r * WS + c] = bf16_float(Wb[OFF_W2 + i]);
        s.W3[r * WS + c] = bf16_float(Wb[OFF_W3 + i]);
    }
    for (int i = t; i < NH; i += blockDim.x) {
        s.b1[i] = P[OFF_B1 + i];
        s.b2[i] = P[OFF_B2 + i];
        s.b3[i] = P[OFF_B3 + i];
        s.W4[i] = bf16_float(Wb[OFF_W4 + i]);
    }
    if (t == 0) s.b4 = P[OFF_B4];
}

// Forward pass of the block's samples; thread j = hidden unit j, then
// thread s < SB = sample s for the output unit.
__device__ void forward(Block& s) {
    const int j = threadIdx.x;
    for (int q = 0; q < SB; q++) {
        float z = s.b1[j];
#pragma unroll
        for (int i = 0; i < NIN; i++) z = fmaf(s.W1[j * NIN + i], s.x[q][i], z);
        s.h1[q][j] = bf16_round(tanhf(z));
    }
    __syncthreads();
    for (int q = 0; q < SB; q++) {
        float z = s.b2[j];
#pragma unroll 16
        for (int i = 0; i < NH; i++) z = fmaf(s.W2[j * WS + i], s.h1[q][i], z);
        s.h2[q][j] = bf16_round(tanhf(z));
    }
    __syncthreads();
    for (int q = 0; q < SB; q++) {
        float z = s.b3[j];
#pragma unroll 16
        for (int i = 0; i < NH; i++) z = fmaf(s.W3[j * WS + i], s.h2[q][i], z);
        s.h3[q][j] = bf16_round(tanhf(z));
    }
    __syncthreads();
    if (j < SB) {
        float z = s.b4;
#pragma unroll 16
        for (int i = 0; i < NH; i++) z = fmaf(s.W4[i], s.h3[j][i], z);
        s.out[j] = z;
    }
    __syncthreads();
}

__device__ inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Sample q of this block: batch entry `e`, drawn from the data set by a
// counter-based hash of (seed, step, e), or entry e itself (full pass).
__device__ inline uint32_t pick(uint32_t e, uint32_t ndata, uint32_t seed, uint32_t step, int draw) {
    if (!draw) return e;
    return mix32(mix32(seed ^ 0x9e3779b9u * (step + 1)) ^ (e * 0x85ebca6bu)) % ndata;
}

// Forward + backward of one batch; per-block gradient partials.
__global__ void __launch_bounds__(NH) k_mlp_grad(const float* __restrict__ P, const uint16_t* __restrict__ Wb,
                                                 const float* __restrict__ X, const float* __restrict__ Y,
                                                 uint32_t ndata, uint32_t nbatch, int draw, uint32_t seed,
                                                 uint32_t step, float inv_n, float* __restrict__ partial,
                                                 double* __restrict__ loss_partial) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Block& s = *reinterpret_cast<Block*>(smem_raw);
    const int j = threadIdx.x;
    load_weights(s, P, Wb);
    const uint32_t base = blockIdx.x * SB;
    __shared__ float ys[SB];
    __shared__ int valid[SB];
    if (j < SB) {
        const uint32_t e = base + j;
        valid[j] = e < nbatch;
        const uint32_t id = e < nbatch ? pick(e, ndata, seed, step, draw) : 0;
#pragma unroll
        for (int i = 0; i < NIN; i++) s.x[j][i] = e < nbatch ? X[(size_t)id * NIN + i] : 0.f;
        ys[j] = e < nbatch ? Y[id] : 0.f;
    }
    __syncthreads();
    forward(s);
    // loss and output gradient: L = (1/n) sum (out - y)^2
    if (j < SB) {
        const float d = valid[j] ? s.out[j] - ys[j] : 0.f;
        s.dout[j] = 2.f * d * inv_n;
        s.out[j] = d * d;
    }
    __syncthreads();
    float* g = partial + (size_t)blockIdx.x * NPARAM;
    if (j == 0) {
        double l = 0.0, db4 = 0.0;
        for (int q = 0; q < SB; q++) {
            l += (double)s.out[q];
            db4 += (double)s.dout[q];
        }
        loss_partial[blockIdx.x] = l;
        g[OFF_B4] = (float)db4;
    }
    // layer 4
    {
        float acc = 0.f;
        for (int q = 0; q < SB; q++) acc = fmaf(s.dout[q], s.h3[q][j], acc);
        g[OFF_W4 + j] = acc;
        for (int q = 0; q < SB; q++) {
            const float h = s.h3[q][j];
            s.dzA[q][j] = s.dout[q] * s.W4[j] * (1.f - h * h);
        }
    }
    __syncthreads();
    // layer 3: dW3 row j, db3, then dz2 = (W3^T dz3) * (1 - h2^2) (column j)
    {
        float acc[NH];
#pragma unroll
        for (int i = 0; i < NH; i++) acc[i] = 0.f;
        float bacc = 0.f;
        for (int q = 0; q < SB; q++) {
            const float d = s.dzA[q][j];
            bacc += d;
#pragma unroll
            for (int i = 0; i < NH; i++) acc[i] = fmaf(d, s.h2[q][i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < NH; i++) g[OFF_W3 + j * NH + i] = acc[i];
        g[OFF_B3 + j] = bacc;
        for (int q = 0; q < SB; q++) {
            float t = 0.f;
#pragma unroll 16
            for (int r = 0; r < NH; r++) t = fmaf(s.W3[r * WS + j], s.dzA[q][r], t);
            const float h = s.h2[q][j];
            s.dzB[q][j] = t * (1.f - h * h);
        }
    }
    __syncthreads();
    // layer 2
    {
        float acc[NH];
#pragma unroll
        for (int i = 0; i < NH; i++) acc[i] = 0.f;
        float bacc = 0.f;
        for (int q = 0; q < SB; q++) {
            const float d = s.dzB[q][j];
            bacc += d;
#pragma unroll
            for (int i = 0; i < NH; i++) acc[i] = fmaf(d, s.h1[q][i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < NH; i++) g[OFF_W2 + j * NH + i] = acc[i];
        g[OFF_B2 + j] = bacc;
        for (int q = 0; q < SB; q++) {
            float t = 0.f;
#pragma unroll 16
            for (int r = 0; r < NH; r++) t = fmaf(s.W2[r * WS + j], s.dzB[q][r], t);
            const float h = s.h1[q][j];
            s.dzA[q][j] = t * (1.f - h * h);
        }
    }
    __syncthreads();
    // layer 1
    {
        float acc[NIN];
#pragma unroll
        for (int i = 0; i < NIN; i++) acc[i] = 0.f;
        float bacc = 0.f;
        for (int q = 0; q < SB; q++) {
            const float d = s.dzA[q][j];
            bacc += d;
#pragma unroll
            for (int i = 0; i < NIN; i++) acc[i] = fmaf(d, s.x[q][i], acc[i]);
        }
#pragma unroll
        for (int i = 0; i < NIN; i++) g[OFF_W1 + j * NIN + i] = acc[i];
        g[OFF_B1 + j] = bacc;
    }
}

// Sum of the block partials in block order; optionally one Adam step on the
// FP32 master weights and a fresh BF16 copy.
__global__ void k_mlp_reduce(const float* __restrict__ partial, int nblk, const double* __restrict__ loss_partial,
                             float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
                             uint16_t* __restrict__ Wb, float lr, float c1, float c2, int update,
                             float* __restrict__ grad_out, double* __restrict__ loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        double l = 0.0;
        for (int b = 0; b < nblk; b++) l += loss_partial[b];
        *loss_out = l;
    }
    if (p >= NPARAM) return;
    float gsum = 0.f;
    for (int b = 0; b < nblk; b++) gsum += partial[(size_t)b * NPARAM + p];
    if (grad_out) grad_out[p] = gsum;
    if (!update) return;
    constexpr float B1 = 0.9f, B2 = 0.999f, EPS = 1e-8f;
    const float m = B1 * M[p] + (1.f - B1) * gsum;
    const float v = B2 * V[p] + (1.f - B2) * gsum * gsum;
    M[p] = m;
    V[p] = v;
    const float w = P[p] - lr * (m * c1) / (sqrtf(v * c2) + EPS);
    P[p] = w;
    Wb[p] = bf16_bits(w);
}

// ------------------------------------------------- inference on tcgen05
// 128 samples per CTA, one per thread and tensor-memory lane.  Layer 1
// (5 -> 64) runs on the CUDA cores; layers 2 and 3 (64 x 64) are each one
// 128 x 64 x 64 BF16 product on the tensor core (activations and weights in
// shared memory in the core-matrix layout of umma.cuh, FP32 accumulators in
// tensor memory, four K = 16 instructions issued by one thread); bias, tanh
// and the BF16 rounding of each activation happen in the epilogue after
// tcgen05.ld; layer 4 (64 -> 1) is a per-thread dot product.  The FP32 sums
// of layers 2 and 3 are the tensor core's (their order and rounding differ
// from the CUDA-core fmaf chain of training), so an activation on a BF16
// rounding boundary can land one BF16 step away.
constexpr int TC_M = 128;
constexpr uint32_t TC_COLS = 128;  // two 64-column accumulators
struct TcBlock {
    uint16_t A[TC_M * NH];  // activations (16 KB; first, at the aligned base)
    uint16_t W2[NH * NH];   // weights [out][in] (8 KB each)
    uint16_t W3[NH * NH];
    float W1[NH * NIN], b1[NH], b2[NH], b3[NH], W4[NH], b4;
    uint64_t bar;
    uint32_t tmem;
};
// 1 KB alignment slack; at least 48 KB so that at most four CTAs share an
// SM and their tensor-memory allocations (4 x 128 of 512 columns) all fit
constexpr size_t TC_SMEM = sizeof(TcBlock) + 1024 > 48 * 1024 ? sizeof(TcBlock) + 1024 : 48 * 1024;

__device__ inline TcBlock& tc_block() {
    extern __shared__ unsigned char tc_raw[];
    return *reinterpret_cast<TcBlock*>(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
}

// Weights into shared memory, mbarrier, tensor memory.
__device__ void tc_setup(TcBlock& s, const float* __restrict__ P, const uint16_t* __restrict__ Wb) {
    const int t = threadIdx.x;
    for (int i = t; i < NH * NH; i += blockDim.x) {
        const int o = i / NH, k = i % NH;
        s.W2[mplb::umma_core_index(o, k, NH)] = Wb[OFF_W2 + i];
        s.W3[mplb::umma_core_index(o, k, NH)] = Wb[OFF_W3 + i];
    }
    for (int i = t; i < NH * NIN; i += blockDim.x) s.W1[i] = bf16_float(Wb[OFF_W1 + i]);
    for (int i = t; i < NH; i += blockDim.x) {
        s.b1[i] = P[OFF_B1 + i];
        s.b2[i] = P[OFF_B2 + i];
        s.b3[i] = P[OFF_B3 + i];
        s.W4[i] = bf16_float(Wb[OFF_W4 + i]);
    }
    if (t == 0) {
        s.b4 = P[OFF_B4];
        mplb::mbar_init(&s.bar, 1);
        mplb::mbar_init_fence();
    }
    if (t < 32) mplb::tmem_alloc(&s.tmem, TC_COLS);
    mplb::tc_fence_before();
    __syncthreads();
    mplb::tc_fence_after();
}

// This thread's row of activations h[0..63] into the A operand.
__device__ inline void tc_store_row(TcBlock& s, const float* h) {
    const int r = threadIdx.x;
#pragma unroll
    for (int c = 0; c < NH / 8; c++) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
            w[q] = (uint32_t)bf16_bits(h[8 * c + 2 * q]) | ((uint32_t)bf16_bits(h[8 * c + 2 * q + 1]) << 16);
        *reinterpret_cast<uint4*>(&s.A[mplb::umma_core_index(r, 8 * c, NH)]) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    mplb::fence_async_smem();
}

// One thread issues A x W^T into tensor-memory columns col .. col+63.
__device__ inline void tc_layer(TcBlock& s, const uint16_t* W, uint32_t col) {
    if (threadIdx.x != 0) return;
    constexpr uint32_t IDESC = mplb::umma_idesc_bf16(TC_M, NH), LBO = 128, SBO = NH / 8 * 128;
    const uint32_t a0 = mplb::smem_u32(s.A), b0 = mplb::smem_u32(W);
#pragma unroll
    for (int kk = 0; kk < NH / 16; kk++)
        mplb::umma_bf16(s.tmem + col, mplb::umma_smem_desc(a0 + 256 * kk, LBO, SBO),
                        mplb::umma_smem_desc(b0 + 256 * kk, LBO, SBO), IDESC, kk > 0);
    mplb::umma_commit(&s.bar);
}

// Epilogue: bias, tanh and BF16 rounding of this thread's row of columns col .. col+63.
__device__ inline void tc_epilogue(TcBlock& s, uint32_t col, const float* bias, float* h) {
    const uint32_t lane0 = (uint32_t)(threadIdx.x & ~31) << 16;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float v[32];
        mplb::tmem_ld32(s.tmem + lane0 + col + 32 * half, v);
#pragma unroll
        for (int c = 0; c < 32; c++) h[32 * half + c] = bf16_round(tanhf(v[c] + bias[32 * half + c]));
    }
}

// The network on this thread's features x (all 128 threads of the CTA
// call it together); false when a bounded wait for the tensor core ran out
// (the CTA then records the error and its outputs are not valid).
__device__ bool tc_forward(TcBlock& s, const float* x, float& out, int* kerr) {
    float h[NH];
#pragma unroll
    for (int j = 0; j < NH; j++) {
        float z = s.b1[j];
#pragma unroll
        for (int i = 0; i < NIN; i++) z = fmaf(s.W1[j * NIN + i], x[i], z);
        h[j] = bf16_round(tanhf(z));
    }
    bool good = true;
    uint32_t phase = 0;
#pragma unroll
    for (int layer = 0; layer < 2; layer++) {
        tc_store_row(s, h);
        mplb::tc_fence_before();
        __syncthreads();
        mplb::tc_fence_after();
        tc_layer(s, layer == 0 ? s.W2 : s.W3, 64u * layer);
        const bool landed = mplb::mbar_wait_bounded(&s.bar, phase, mplb::TMA_WAIT_LIMIT);
        mplb::tc_fence_after();
        if (__syncthreads_or(!landed)) {
            good = false;
            // let the products in flight finish before the tensor memory is released
            mplb::mbar_wait_bounded(&s.bar, phase, mplb::TMA_WAIT_LIMIT);
            break;
        }
        phase ^= 1u;
        tc_epilogue(s, 64u * layer, layer == 0 ? s.b2 : s.b3, h);
    }
    if (good) {
        float z = s.b4;
#pragma unroll
        for (int i = 0; i < NH; i++) z = fmaf(s.W4[i], h[i], z);
        out = z;
    } else if (threadIdx.x == 0) {
        atomicExch(kerr, mplb::MPLB_KERR_WAIT);
    }
    mplb::tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) mplb::tmem_dealloc(s.tmem, TC_COLS);
    return good;
}

// Forward pass over arbitrary samples (features already normalised).
__global__ void __launch_bounds__(TC_M) k_mlp_predict(const float* __restrict__ P, const uint16_t* __restrict__ Wb,
                                                      const float* __restrict__ X, uint32_t n, float* __restrict__ Y,
                                                      int* __restrict__ kerr) {
    TcBlock& s = tc_block();
    tc_setup(s, P, Wb);
    const uint32_t e = blockIdx.x * TC_M + threadIdx.x;
    float x[NIN];
#pragma unroll
    for (int i = 0; i < NIN; i++) x[i] = e < n ? X[(size_t)e * NIN + i] : 0.f;
    float out = 0.f;
    if (tc_forward(s, x, out, kerr) && e < n) Y[e] = out;
}

// Initial density of a liquid band of a box lattice: along `axis`, nodes
// within height/2 of `c` (periodic distance over the axis length `ext`) are
// liquid; the feature distance is height/2 - |s - c|, a flat interface.
__global__ void __launch_bounds__(TC_M) k_mlp_column(const float* __restrict__ P, const uint16_t* __restrict__ Wb,
                                                     uint32_t n, int nx, int ny, int axis, int ext, double c,
                                                     double height, double t_ratio, double a, double b,
                                                     double* __restrict__ rho, int* __restrict__ kerr) {
    TcBlock& s = tc_block();
    tc_setup(s, P, Wb);
    const uint32_t e = blockIdx.x * TC_M + threadIdx.x;
    const uint32_t i = e < n ? e : 0;
    const uint32_t coord = axis == 0 ? i % (uint32_t)nx
                                     : (axis == 1 ? (i / (uint32_t)nx) % (uint32_t)ny : i / ((uint32_t)nx * (uint32_t)ny));
    double ds = (double)coord - c;
    if (ds > 0.5 * ext) ds -= ext;
    if (ds < -0.5 * ext) ds += ext;
    float f[NIN];
    features(t_ratio, a, b, 0.5 * height - fabs(ds), INFINITY, f);
    float out = 0.f;
    if (tc_forward(s, f, out, kerr) && e < n) rho[e] = (double)out / b;
}

// Initial density of a box lattice: node i at (i % nx, i / nx % ny, i / (nx ny)),
// r = distance to the bubble centre, rho = network(T/Tc, a, b, r/R) / b.
__global__ void __launch_bounds__(TC_M) k_mlp_bubble(const float* __restrict__ P, const uint16_t* __restrict__ Wb,
                                                     uint32_t n, int nx, int ny, double cx, double cy, double cz,
                                                     double R, double t_ratio, double a, double b,
                                                     double* __restrict__ rho, int* __restrict__ kerr) {
    TcBlock& s = tc_block();
    tc_setup(s, P, Wb);
    const uint32_t e = blockIdx.x * TC_M + threadIdx.x;
    const uint32_t i = e < n ? e : 0;
    const double x = (double)(i % (uint32_t)nx) - cx, y = (double)((i / (uint32_t)nx) % (uint32_t)ny) - cy,
                 z = (double)(i / ((uint32_t)nx * (uint32_t)ny)) - cz;
    float f[NIN];
    features(t_ratio, a, b, sqrt(x * x + y * y + z * z), R, f);
    float out = 0.f;
    if (tc_forward(s, f, out, kerr) && e < n) rho[e] = (double)out / b;
}

constexpr size_t SMEM = sizeof(Block);

int set_attrs() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        err = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(k_mlp_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(k_mlp_bubble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(k_mlp_column, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    });
    return err == cudaSuccess ? 0 : mplb_internal_fail(MPLB_E_CUDA, std::string("MLP kernel attributes: ") +
                                                                       cudaGetErrorString(err));
}

#define CKM(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return mplb_internal_fail(MPLB_E_CUDA, std::string(#call) + ": " +   \
                                                                          cudaGetErrorString(e_));  \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

struct mplb_mlp {
    int dev = 0;
    cudaStream_t stream = nullptr;
    float *P = nullptr, *M = nullptr, *V = nullptr;
    uint16_t* Wb = nullptr;
    float *X = nullptr, *Y = nullptr;
    uint32_t ndata = 0, cap = 0;
    float* partial = nullptr;
    double* loss_partial = nullptr;
    int nblk_cap = 0;
    double* loss = nullptr;
    float* grad = nullptr;
    int* kerr = nullptr;  // inference kernels: a bounded wait for the tensor core ran out
    uint32_t seed = 0;
    uint64_t step = 0;
};

namespace {

void mlp_free(mplb_mlp* m) {
    void* ps[] = {m->P, m->M, m->V, m->Wb, m->X, m->Y, m->partial, m->loss_partial, m->loss, m->grad, m->kerr};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
}

int ensure_blocks(mplb_mlp* m, int nblk) {
    if (nblk <= m->nblk_cap) return 0;
    if (m->partial) cudaFree(m->partial);
    if (m->loss_partial) cudaFree(m->loss_partial);
    m->partial = nullptr;
    m->loss_partial = nullptr;
    m->nblk_cap = 0;
    CKM(cudaMalloc((void**)&m->partial, (size_t)nblk * NPARAM * sizeof(float)));
    CKM(cudaMalloc((void**)&m->loss_partial, (size_t)nblk * sizeof(double)));
    m->nblk_cap = nblk;
    return 0;
}

int upload_params(mplb_mlp* m, const float* host) {
    std::vector<uint16_t> b(NPARAM);
    for (int i = 0; i < NPARAM; i++) b[i] = bf16_bits(host[i]);
    CKM(cudaMemcpyAsync(m->P, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CKM(cudaMemcpyAsync(m->Wb, b.data(), NPARAM * sizeof(uint16_t), cudaMemcpyHostToDevice, m->stream));
    CKM(cudaMemsetAsync(m->M, 0, NPARAM * sizeof(float), m->stream));
    CKM(cudaMemsetAsync(m->V, 0, NPARAM * sizeof(float), m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    m->step = 0;
    return 0;
}

// After an inference launch on stream s: wait for it and report a tensor-core
// wait that ran out (the flag is cleared for the next call).
int inference_status(mplb_mlp* m, cudaStream_t s) {
    int v = 0;
    CKM(cudaMemcpyAsync(&v, m->kerr, sizeof(int), cudaMemcpyDeviceToHost, s));
    CKM(cudaStreamSynchronize(s));
    if (!v) return 0;
    CKM(cudaMemsetAsync(m->kerr, 0, sizeof(int), s));
    CKM(cudaStreamSynchronize(s));
    return mplb_internal_fail(MPLB_E_TIMEOUT, "MLP inference: a bounded wait for the tensor core ran out");
}

// One pass: gradient over `nbatch` samples (drawn, or the first nbatch in
// order), optionally followed by an Adam step.
int pass(mplb_mlp* m, uint32_t nbatch, int draw, int update, float lr, float* grad_host, double* loss_host) {
    const int nblk = (int)((nbatch + SB - 1) / SB);
    if (int rc = ensure_blocks(m, nblk)) return rc;
    k_mlp_grad<<<nblk, NH, SMEM, m->stream>>>(m->P, m->Wb, m->X, m->Y, m->ndata, nbatch, draw, m->seed,
                                             (uint32_t)m->step, 1.f / (float)nbatch, m->partial, m->loss_partial);
    CKM(cudaGetLastError());
    const double t = (double)(m->step + 1);
    const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, t))), c2 = (float)(1.0 / (1.0 - std::pow(0.999, t)));
    k_mlp_reduce<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->partial, nblk, m->loss_partial, m->P, m->M, m->V,
                                                              m->Wb, lr, c1, c2, update,
                                                              grad_host ? m->grad : nullptr, m->loss);
    CKM(cudaGetLastError());
    if (update) m->step++;
    if (grad_host) CKM(cudaMemcpyAsync(grad_host, m->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (loss_host) {
        double l = 0;
        CKM(cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        CKM(cudaStreamSynchronize(m->stream));
        *loss_host = l / nbatch;
    }
    return 0;
}

}  // namespace

// Used by mplb_gpu.cu for mplb_mlp_init_bubble.
int mplb_mlp_bubble_launch(mplb_mlp* m, double* rho, uint32_t n, int nx, int ny, const double* c, double R,
                           double t_ratio, double a, double b, cudaStream_t s) {
    DevGuard g(m->dev);
    if (int rc = set_attrs()) return rc;
    // order the handle's stream after the network's last update
    cudaEvent_t ev;
    CKM(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, m->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    cudaEventDestroy(ev);
    CKM(e);
    k_mlp_bubble<<<(n + TC_M - 1) / TC_M, TC_M, TC_SMEM, s>>>(m->P, m->Wb, n, nx, ny, c[0], c[1], c[2], R, t_ratio,
                                                               a, b, rho, m->kerr);
    CKM(cudaGetLastError());
    return inference_status(m, s);
}

// Used by mplb_gpu.cu for mplb_mlp_init_column.
int mplb_mlp_column_launch(mplb_mlp* m, double* rho, uint32_t n, int nx, int ny, int axis, int ext, double c,
                           double height, double t_ratio, double a, double b, cudaStream_t s) {
    DevGuard g(m->dev);
    if (int rc = set_attrs()) return rc;
    cudaEvent_t ev;
    CKM(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, m->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    cudaEventDestroy(ev);
    CKM(e);
    k_mlp_column<<<(n + TC_M - 1) / TC_M, TC_M, TC_SMEM, s>>>(m->P, m->Wb, n, nx, ny, axis, ext, c, height, t_ratio,
                                                               a, b, rho, m->kerr);
    CKM(cudaGetLastError());
    return inference_status(m, s);
}

int mplb_mlp_device(const mplb_mlp* m) { return m->dev; }

extern "C" {

void mplb_mlp_features(double t_ratio, double a, double b, double r, double R, float* out) {
    features(t_ratio, a, b, r, R, out);
}

int mplb_mlp_create(int32_t device, uint64_t seed, mplb_mlp_t** out) {
    if (!out) return mplb_internal_fail(MPLB_E_ARG, "out is NULL");
    *out = nullptr;
    int dev = device;
    if (dev < 0) CKM(cudaGetDevice(&dev));
    DevGuard g(dev);
    if (int rc = set_attrs()) return rc;
    mplb_mlp* m = new mplb_mlp();
    m->dev = dev;
    m->seed = (uint32_t)(seed ^ (seed >> 32));
    auto setup = [&]() -> int {
        CKM(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        CKM(cudaMalloc((void**)&m->P, NPARAM * sizeof(float)));
        CKM(cudaMalloc((void**)&m->M, NPARAM * sizeof(float)));
        CKM(cudaMalloc((void**)&m->V, NPARAM * sizeof(float)));
        CKM(cudaMalloc((void**)&m->Wb, NPARAM * sizeof(uint16_t)));
        CKM(cudaMalloc((void**)&m->grad, NPARAM * sizeof(float)));
        CKM(cudaMalloc((void**)&m->loss, sizeof(double)));
        CKM(cudaMalloc((void**)&m->kerr, sizeof(int)));
        CKM(cudaMemsetAsync(m->kerr, 0, sizeof(int), m->stream));
        // Glorot-uniform weights from a seeded xorshift generator, zero biases.
        std::vector<float> p(NPARAM, 0.f);
        uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
        auto uni = [&]() {
            st ^= st << 13;
            st ^= st >> 7;
            st ^= st << 17;
            return (double)(st >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
        };
        auto fill = [&](int off, int fan_out, int fan_in) {
            const double lim = std::sqrt(6.0 / (fan_in + fan_out));
            for (int i = 0; i < fan_out * fan_in; i++) p[off + i] = (float)(lim * uni());
        };
        fill(OFF_W1, NH, NIN);
        fill(OFF_W2, NH, NH);
        fill(OFF_W3, NH, NH);
        fill(OFF_W4, 1, NH);
        return upload_params(m, p.data());
    };
    if (int rc = setup()) {
        mlp_free(m);
        delete m;
        return rc;
    }
    *out = m;
    return 0;
}

int mplb_mlp_destroy(mplb_mlp_t* m) {
    if (!m) return 0;
    DevGuard g(m->dev);
    cudaStreamSynchronize(m->stream);
    mlp_free(m);
    delete m;
    return 0;
}

int mplb_mlp_get_params(mplb_mlp_t* m, float* out) {
    if (!m || !out) return mplb_internal_fail(MPLB_E_ARG, "NULL argument");
    DevGuard g(m->dev);
    CKM(cudaMemcpyAsync(out, m->P, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    return 0;
}

int mplb_mlp_set_params(mplb_mlp_t* m, const float* in) {
    if (!m || !in) return mplb_internal_fail(MPLB_E_ARG, "NULL argument");
    for (int i = 0; i < NPARAM; i++)
        if (!std::isfinite(in[i])) return mplb_internal_fail(MPLB_E_NONFINITE, "non-finite parameter");
    DevGuard g(m->dev);
    return upload_params(m, in);
}

int mplb_mlp_set_samples(mplb_mlp_t* m, const double* t_ratio, const double* a, const double* b, const double* r,
                         const double* R, const double* rho, uint32_t n) {
    if (!m || !t_ratio || !a || !b || !r || !R || !rho || n == 0)
        return mplb_internal_fail(MPLB_E_ARG, "samples missing");
    std::vector<float> x((size_t)n * NIN), y(n);
    for (uint32_t i = 0; i < n; i++) {
        if (!(b[i] > 0.0) || !(R[i] > 0.0)) return mplb_internal_fail(MPLB_E_ARG, "b and R must be positive");
        features(t_ratio[i], a[i], b[i], r[i], R[i], &x[(size_t)i * NIN]);
        y[i] = (float)(b[i] * rho[i]);
    }
    DevGuard g(m->dev);
    if (n > m->cap) {
        if (m->X) cudaFree(m->X);
        if (m->Y) cudaFree(m->Y);
        m->X = m->Y = nullptr;
        m->cap = 0;
        CKM(cudaMalloc((void**)&m->X, (size_t)n * NIN * sizeof(float)));
        CKM(cudaMalloc((void**)&m->Y, (size_t)n * sizeof(float)));
        m->cap = n;
    }
    CKM(cudaMemcpyAsync(m->X, x.data(), x.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CKM(cudaMemcpyAsync(m->Y, y.data(), y.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CKM(cudaStreamSynchronize(m->stream));
    m->ndata = n;
    return 0;
}

int mplb_mlp_gradient(mplb_mlp_t* m, float* grad, double* loss) {
    if (!m || !grad) return mplb_internal_fail(MPLB_E_ARG, "NULL argument");
    if (!m->ndata) return mplb_internal_fail(MPLB_E_STATE, "no samples");
    DevGuard g(m->dev);
    if (int rc = pass(m, m->ndata, 0, 0, 0.f, grad, loss)) return rc;
    CKM(cudaStreamSynchronize(m->stream));
    return 0;
}

int mplb_mlp_train(mplb_mlp_t* m, uint32_t steps, uint32_t batch, float lr, double* loss) {
    if (!m || batch == 0) return mplb_internal_fail(MPLB_E_ARG, "bad argument");
    if (!m->ndata) return mplb_internal_fail(MPLB_E_STATE, "no samples");
    DevGuard g(m->dev);
    for (uint32_t s = 0; s < steps; s++)
        if (int rc = pass(m, batch, 1, 1, lr, nullptr, (loss && s + 1 == steps) ? loss : nullptr)) return rc;
    CKM(cudaStreamSynchronize(m->stream));
    return 0;
}

int mplb_mlp_predict(mplb_mlp_t* m, const double* t_ratio, const double* a, const double* b, const double* r,
                     const double* R, uint32_t n, double* rho) {
    if (!m || !t_ratio || !a || !b || !r || !R || !rho) return mplb_internal_fail(MPLB_E_ARG, "NULL argument");
    if (n == 0) return 0;
    std::vector<float> x((size_t)n * NIN), y(n);
    for (uint32_t i = 0; i < n; i++) {
        if (!(b[i] > 0.0) || !(R[i] > 0.0)) return mplb_internal_fail(MPLB_E_ARG, "b and R must be positive");
        features(t_ratio[i], a[i], b[i], r[i], R[i], &x[(size_t)i * NIN]);
    }
    DevGuard g(m->dev);
    float *dx = nullptr, *dy = nullptr;
    auto run = [&]() -> int {
        CKM(cudaMalloc((void**)&dx, x.size() * sizeof(float)));
        CKM(cudaMalloc((void**)&dy, y.size() * sizeof(float)));
        CKM(cudaMemcpyAsync(dx, x.data(), x.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
        k_mlp_predict<<<(n + TC_M - 1) / TC_M, TC_M, TC_SMEM, m->stream>>>(m->P, m->Wb, dx, n, dy, m->kerr);
        CKM(cudaGetLastError());
        if (int rc = inference_status(m, m->stream)) return rc;
        CKM(cudaMemcpyAsync(y.data(), dy, y.size() * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        CKM(cudaStreamSynchronize(m->stream));
        return 0;
    };
    const int rc = run();
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    if (rc) return rc;
    for (uint32_t i = 0; i < n; i++) rho[i] = (double)y[i] / b[i];
    return 0;
}

}  // extern "C"

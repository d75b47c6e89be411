// sph_mlp.cuh -- the Johnson-Cook return-map surrogate: a 4 -> 64 -> 64 -> 64 -> 1 SiLU
// MLP.  No counterpart in the reference (its return map is the Newton-bisection of
// MAT002_johnson_cook.py:251-354, called from SOLID.py:2889-2913); the network proposes
// the plastic increment and the exact residual decides whether it is kept.
//
//   * training: float32 forward / backward on CUDA cores (k_mlp_grad, one thread per
//     sample, gradients reduced per warp, then per block in shared memory) and Adam;
//   * inference: BF16 operands on the 5th-generation tensor cores with FP32 accumulators
//     in TMEM (k_mlp_tc): 128-row tiles, the two 64x64 hidden layers as
//     tcgen05.mma kind::f16 (M 128, N 64, K 4 x 16), the 4-wide input layer and the
//     64-wide output dot on CUDA cores inside the same kernel.
//
// Features of a return (jc_features): f0 = ln(max(vm_trial / sigma_y0 - 1, 1e-8)) / 10,
// f1 = eps_p,
// f2 = ln(max(eps_dot_eq / eps0_dot, 1)) / 10, f3 = ln(max(d_hi / (dt eps0_dot), 1)) / 10,
// with d_hi = (vm_trial - sigma_y0) / (3 G) the upper bracket of the plastic increment.
// The output is u = 10 (1 - d / d_hi): the hardening share of the overstress, O(1), so
// the BF16 rounding of the hidden layers costs a relative error of u, not of d / d_hi,
// which sits close to 1.
#pragma once
#include <cuda_bf16.h>
#include "sph_device.cuh"

namespace sph {

constexpr int kMlpIn = 4, kMlpH = 64;
constexpr int kOffW1 = 0;                          // [64][4]  (out, in)
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;    // [64]
constexpr int kOffW2 = kOffB1 + kMlpH;             // [64][64]
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;             // [64]
constexpr int kOffB4 = kOffW4 + kMlpH;             // [1]
constexpr int kMlpParams = kOffB4 + 1;             // 8705
// BF16 hidden-layer weights in the tensor cores' canonical K-major layout, W2 then W3.
constexpr int kMlpPackedHalf = kMlpH * kMlpH;      // bf16 elements per matrix
constexpr int kMlpPackedBytes = 2 * kMlpPackedHalf * 2;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
// Inference SiLU from the identity z sigma(z) = z (1 + tanh(z / 2)) / 2 with the hardware
// tanh approximation (one SFU op; its ~2^-11 relative error is below the BF16 rounding
// of the activations it feeds).
__device__ __forceinline__ float silu_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Float32 forward of one sample (the training reference; inference runs k_mlp_tc).
__device__ __forceinline__ float mlp_forward_f32(const float* __restrict__ W, const float x[kMlpIn]) {
    float h1[kMlpH], h2[kMlpH];
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB1 + j);
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) z += __ldg(W + kOffW1 + kMlpIn * j + k) * x[k];
        h1[j] = silu(z);
    }
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB2 + j);
        for (int k = 0; k < kMlpH; ++k) z += __ldg(W + kOffW2 + kMlpH * j + k) * h1[k];
        h2[j] = silu(z);
    }
    float y = __ldg(W + kOffB4);
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB3 + j);
        for (int k = 0; k < kMlpH; ++k) z += __ldg(W + kOffW3 + kMlpH * j + k) * h2[k];
        y += __ldg(W + kOffW4 + j) * silu(z);
    }
    return y;
}

__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ W, const float4* __restrict__ X,
                                                     int n, float* __restrict__ Y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float4 f = X[r];
    const float x[kMlpIn] = {f.x, f.y, f.z, f.w};
    Y[r] = mlp_forward_f32(W, x);
}

// Gradient of the mean squared error over n samples, added into G (zeroed by the caller);
// the loss sum(e^2) / n goes to *loss in FP64.  One thread per sample: forward with the
// pre-activations kept, then backward; every parameter's contribution is summed over the
// warp by shuffles and over the block in shared memory before one global atomic.
constexpr int kMlpGradThreads = 128;
__device__ __forceinline__ void grad_add(float* sg, int idx, float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sg + idx, v);
}

__global__ void __launch_bounds__(kMlpGradThreads) k_mlp_grad(const float* __restrict__ W, const float4* __restrict__ X,
                                                              const float* __restrict__ T, int n, float inv_n,
                                                              float* __restrict__ G, double* __restrict__ loss) {
    extern __shared__ float sg[];                  // kMlpParams floats
    for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) sg[q] = 0.0f;
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = r < n;                          // off lanes carry zero gradients
    float x[kMlpIn] = {0.0f, 0.0f, 0.0f, 0.0f};
    float t = 0.0f;
    if (on) { const float4 f = X[r]; x[0] = f.x; x[1] = f.y; x[2] = f.z; x[3] = f.w; t = T[r]; }
    float z1[kMlpH], z2[kMlpH], z3[kMlpH];
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB1 + j);
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) z += __ldg(W + kOffW1 + kMlpIn * j + k) * x[k];
        z1[j] = z;
    }
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB2 + j);
        for (int k = 0; k < kMlpH; ++k) z += __ldg(W + kOffW2 + kMlpH * j + k) * silu(z1[k]);
        z2[j] = z;
    }
    float y = __ldg(W + kOffB4);
    for (int j = 0; j < kMlpH; ++j) {
        float z = __ldg(W + kOffB3 + j);
        for (int k = 0; k < kMlpH; ++k) z += __ldg(W + kOffW3 + kMlpH * j + k) * silu(z2[k]);
        z3[j] = z;
        y += __ldg(W + kOffW4 + j) * silu(z);
    }
    const float e = on ? y - t : 0.0f;
    const float dy = 2.0f * e * inv_n;
    // output layer; z3 becomes dL/dz3
    grad_add(sg, kOffB4, dy);
    for (int j = 0; j < kMlpH; ++j) {
        grad_add(sg, kOffW4 + j, dy * silu(z3[j]));
        z3[j] = dy * __ldg(W + kOffW4 + j) * silu_grad(z3[j]);
    }
    // layer 3: z2 becomes dL/dz2
    for (int j = 0; j < kMlpH; ++j) {
        grad_add(sg, kOffB3 + j, z3[j]);
        for (int k = 0; k < kMlpH; ++k) grad_add(sg, kOffW3 + kMlpH * j + k, z3[j] * silu(z2[k]));
    }
    for (int k = 0; k < kMlpH; ++k) {
        float s = 0.0f;
        for (int j = 0; j < kMlpH; ++j) s += __ldg(W + kOffW3 + kMlpH * j + k) * z3[j];
        z2[k] = s * silu_grad(z2[k]);
    }
    // layer 2: z1 becomes dL/dz1
    for (int j = 0; j < kMlpH; ++j) {
        grad_add(sg, kOffB2 + j, z2[j]);
        for (int k = 0; k < kMlpH; ++k) grad_add(sg, kOffW2 + kMlpH * j + k, z2[j] * silu(z1[k]));
    }
    for (int k = 0; k < kMlpH; ++k) {
        float s = 0.0f;
        for (int j = 0; j < kMlpH; ++j) s += __ldg(W + kOffW2 + kMlpH * j + k) * z2[j];
        z1[k] = s * silu_grad(z1[k]);
    }
    // layer 1
    for (int j = 0; j < kMlpH; ++j) {
        grad_add(sg, kOffB1 + j, z1[j]);
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) grad_add(sg, kOffW1 + kMlpIn * j + k, z1[j] * x[k]);
    }
    double l = (double)e * (double)e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * (double)inv_n);
    __syncthreads();
    for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x)
        if (sg[q] != 0.0f) atomicAdd(G + q, sg[q]);
}

// Adam (Kingma & Ba 2015) with bias correction; step counts from 1.
__global__ void k_mlp_adam(float* __restrict__ W, const float* __restrict__ G, float* __restrict__ M,
                           float* __restrict__ V, int np, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np) return;
    const float g = G[q];
    const float m = b1 * M[q] + (1.0f - b1) * g;
    const float v = b2 * V[q] + (1.0f - b2) * g * g;
    M[q] = m;
    V[q] = v;
    W[q] -= lr * (m * c1) / (sqrtf(v * c2) + eps);
}

// Byte offset of element (row, k) of a K-major BF16 operand with `rows` rows in the
// canonical no-swizzle layout: 8x8 core matrices (8 rows x 16 bytes, rows 16 bytes apart),
// the 8-row groups of one 8-wide K chunk 128 bytes apart, the K chunks rows*16 bytes apart.
__host__ __device__ __forceinline__ int kmajor_offset(int row, int k, int rows) {
    return ((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// W2 and W3 (float32, [out][in]) to BF16 in the B-operand layout (N = out rows, K = in).
__global__ void k_mlp_pack(const float* __restrict__ W, __nv_bfloat16* __restrict__ packed) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 2 * kMlpPackedHalf) return;
    const int m = q / kMlpPackedHalf, e = q % kMlpPackedHalf;
    const int row = e / kMlpH, k = e % kMlpH;
    const float w = W[(m == 0 ? kOffW2 : kOffW3) + e];
    packed[m * kMlpPackedHalf + kmajor_offset(row, k, kMlpH) / 2] = __float2bfloat16_rn(w);
}

// ------------------------------------------------------------------ tcgen05 primitives
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {     // one warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_addr(slot)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {   // same warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase with the given parity to complete; gives up after `tries` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long tries) {
    const uint32_t a = smem_addr(bar);
    for (long t = 0; t < tries; ++t) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P;\n\t}"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}
// Shared-memory matrix descriptor, K-major, no swizzle: start, leading-dimension byte
// offset (between the two 8-element K chunks of one K = 16 step), stride byte offset
// (between 8-row groups), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N = 64, M = 128.
constexpr uint32_t kMlpIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMlpH >> 3) << 17) |
                               ((uint32_t)(128 >> 4) << 24);
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(kMlpIdesc), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_addr(bar)) : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (32 lanes per warp).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// ------------------------------------------------------------------ tensor-core inference
// Persistent: CTAs of 128 threads (thread t = row t of a 128-row tile = TMEM lane t) loop
// over tiles of the n input rows (n read from *n_dev when given).  Per tile: layer 1 on
// CUDA cores -> BF16 A tile in shared memory -> 4 MMAs (K 16 each) with W2 -> TMEM ->
// bias + SiLU -> BF16 A tile -> 4 MMAs with W3 -> TMEM -> bias + SiLU + output dot.
// Every wait is bounded: a phase that does not complete sets MLP_ERR in *err, the kernel
// waits once more (bounded), frees its TMEM and returns.
constexpr int kMlpTcThreads = 128;
constexpr int kMlpCtasPerSm = 6;       // 34 KB shared memory and 64 TMEM columns each
constexpr int kMlpTileRows = 128;
constexpr uint32_t kMlpTmemCols = 64;
constexpr long kMlpWaitTries = 1L << 22;
constexpr int kMlpErrTimeout = SPH_EW_MLP_TIMEOUT;

__global__ void __launch_bounds__(kMlpTcThreads) k_mlp_tc(const float* __restrict__ W,
                                                          const __nv_bfloat16* __restrict__ packed,
                                                          const float4* __restrict__ X, int n,
                                                          const int* __restrict__ n_dev,
                                                          float* __restrict__ Y, int* __restrict__ err) {
    __shared__ __align__(128) unsigned char sA[kMlpTileRows * kMlpH * 2];   // 16 KB
    __shared__ __align__(128) unsigned char sB[kMlpPackedBytes];            // W2 | W3, 16 KB
    __shared__ float sW1[kMlpH * kMlpIn], sB1[kMlpH], sB2[kMlpH], sB3[kMlpH], sW4[kMlpH];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;
    const int rows = n_dev ? min(*n_dev, n) : n;
    const int ntiles = (rows + kMlpTileRows - 1) / kMlpTileRows;
    if ((int)blockIdx.x >= ntiles) return;          // whole CTA leaves: nothing allocated yet
    // weights to shared memory (16-byte copies of the packed BF16 matrices)
    for (int q = t; q < kMlpPackedBytes / 16; q += blockDim.x)
        reinterpret_cast<uint4*>(sB)[q] = __ldg(reinterpret_cast<const uint4*>(packed) + q);
    for (int q = t; q < kMlpH * kMlpIn; q += blockDim.x) sW1[q] = W[kOffW1 + q];
    for (int q = t; q < kMlpH; q += blockDim.x) {
        sB1[q] = W[kOffB1 + q]; sB2[q] = W[kOffB2 + q]; sB3[q] = W[kOffB3 + q]; sW4[q] = W[kOffW4 + q];
    }
    const float b4 = W[kOffB4];
    if (t == 0) mbar_init(&bar, 1);
    if (warp == 0) tmem_alloc(&tmem_slot, kMlpTmemCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);   // this warp's 32 lanes
    const uint32_t aA = smem_addr(sA), aB = smem_addr(sB);
    const uint32_t lboA = (kMlpTileRows / 8) * 128, lboB = (kMlpH / 8) * 128, sbo = 128;
    uint32_t phase = 0;
    bool ok = true;
    auto a_store16 = [&](int k0, const float* h) {      // h[0..15] -> row t, columns k0..k0+15
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            uint4 v;
            __nv_bfloat162 p0 = __floats2bfloat162_rn(h[8 * half + 0], h[8 * half + 1]);
            __nv_bfloat162 p1 = __floats2bfloat162_rn(h[8 * half + 2], h[8 * half + 3]);
            __nv_bfloat162 p2 = __floats2bfloat162_rn(h[8 * half + 4], h[8 * half + 5]);
            __nv_bfloat162 p3 = __floats2bfloat162_rn(h[8 * half + 6], h[8 * half + 7]);
            v.x = *reinterpret_cast<uint32_t*>(&p0); v.y = *reinterpret_cast<uint32_t*>(&p1);
            v.z = *reinterpret_cast<uint32_t*>(&p2); v.w = *reinterpret_cast<uint32_t*>(&p3);
            *reinterpret_cast<uint4*>(sA + kmajor_offset(t, k0 + 8 * half, kMlpTileRows)) = v;
        }
    };
    auto mma_layer = [&](int layer) {                   // all threads; one issues
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (t == 0) {
            const uint32_t bbase = aB + (uint32_t)(layer * kMlpPackedHalf * 2);
#pragma unroll
            for (int s = 0; s < kMlpH / 16; ++s) {
                const uint64_t da = umma_desc(aA + (uint32_t)(2 * s) * lboA, lboA, sbo);
                const uint64_t db = umma_desc(bbase + (uint32_t)(2 * s) * lboB, lboB, sbo);
                umma_bf16(tmem, da, db, s > 0 ? 1u : 0u);
            }
            umma_commit(&bar);
        }
        bool mine = mbar_wait(&bar, phase & 1u, kMlpWaitTries);
        ok = __syncthreads_and(mine) != 0;          // one verdict for the whole CTA
        if (!ok && t == 0) atomicOr(err, kMlpErrTimeout);
        ++phase;
        tc_fence_after();
    };
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int r = tile * kMlpTileRows + t;
        float x[kMlpIn] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (r < rows) { const float4 f = X[r]; x[0] = f.x; x[1] = f.y; x[2] = f.z; x[3] = f.w; }
        // layer 1 (4 -> 64) on CUDA cores
#pragma unroll
        for (int k0 = 0; k0 < kMlpH; k0 += 16) {
            float h[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = k0 + q;
                float z = sB1[j];
#pragma unroll
                for (int k = 0; k < kMlpIn; ++k) z += sW1[kMlpIn * j + k] * x[k];
                h[q] = silu_fast(z);
            }
            a_store16(k0, h);
        }
        // layer 2 (64 -> 64) on the tensor cores
        mma_layer(0);
        if (!ok) break;
#pragma unroll
        for (int k0 = 0; k0 < kMlpH; k0 += 16) {
            float h[16];
            tmem_ld16(tlane + (uint32_t)k0, h);
#pragma unroll
            for (int q = 0; q < 16; ++q) h[q] = silu_fast(h[q] + sB2[k0 + q]);
            a_store16(k0, h);
        }
        // layer 3 (64 -> 64) on the tensor cores, then the output dot (64 -> 1)
        mma_layer(1);
        if (!ok) break;
        float y = b4;
#pragma unroll
        for (int k0 = 0; k0 < kMlpH; k0 += 16) {
            float h[16];
            tmem_ld16(tlane + (uint32_t)k0, h);
#pragma unroll
            for (int q = 0; q < 16; ++q) y += sW4[k0 + q] * silu_fast(h[q] + sB3[k0 + q]);
        }
        if (r < rows) Y[r] = y;
    }
    if (!ok) mbar_wait(&bar, (phase - 1u) & 1u, kMlpWaitTries);   // the MMAs in flight
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kMlpTmemCols);
    }
}

}  // namespace sph

// sph_noalloc.cu -- the FP64 energy/momentum reductions without a handle and without
// any device allocation, for callers that cannot allocate GPU memory.
//
// Who needs it: a host that runs inside another framework's fixed device-memory pool
// (cudaMalloc would fail or fragment that pool), code that records a CUDA graph and may
// not allocate while capturing, and FFI callers (a JVM, a Go runtime) that hold only raw
// device pointers handed to them and no right to create a library handle, which
// allocates its scratch in sph_create.  They pass the particle buffers and an output
// buffer they already own; the scratch lives in a fixed array compiled into this file.
//
// The scratch is g_partials below: one row of SPH_RED_COUNT doubles per thread block of
// the first pass, kNoAllocMaxBlocks rows, so at most kNoAllocMaxParticles particles
// (4,194,304) per call, 1.44 MB of device memory that every GPU which loads the library
// holds until the process exits.  Every call shares that one array and overwrites the
// rows it uses (nothing in it has to start at zero: each block writes its whole row
// before the second pass reads it).  Two calls whose work overlaps on the GPU (on
// different streams, or from several host threads) race on it; serialise them.  The
// array's address is looked up once per device and kept, so a cudaDeviceReset between
// calls is not supported.  A solid is refused (SPH_ERR_UNSUPPORTED): its elastic energy
// needs the stress and material rows, which this entry point is not given.
#include <cuda_runtime.h>

#include <mutex>

#include "sph_host.cuh"

namespace {

using namespace sph;

constexpr int kNoAllocMaxBlocks = 16384;
constexpr int64_t kNoAllocMaxParticles = (int64_t)kNoAllocMaxBlocks * kBlock;
static_assert(kNoAllocMaxParticles == SPH_NOALLOC_MAX_PARTICLES,
              "the public cap in sph_b200.h must equal the scratch array's real capacity");
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kNoAllocMaxBlocks * SPH_RED_COUNT];

// Device addresses of g_partials, found once per device with that device current.
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SPH_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_partials) != cudaSuccess || !p) return SPH_ERR_CUDA;
        g_addr[dev] = p;
    }
    *out = static_cast<double*>(g_addr[dev]);
    return SPH_OK;
}

// First pass: each block writes its block sums, no atomics (so the result does not
// depend on the order blocks finish in).
__global__ void __launch_bounds__(kBlock) k_reduce_partials(Cst c, const float4* __restrict__ pos,
                                                            const float4* __restrict__ vel,
                                                            const float4* __restrict__ shift,
                                                            double* __restrict__ partials) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double r[SPH_RED_COUNT];
#pragma unroll
    for (int k = 0; k < SPH_RED_COUNT; ++k) r[k] = 0.0;
    if (i < c.n) reduce_terms(c, pos[i], vel[i], shift ? shift[i].w : 0.0f, r);
    __shared__ double red[SPH_RED_COUNT][kBlock / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < SPH_RED_COUNT; ++k) {
        double v = warp_sum(r[k]);
        if (lane == 0) red[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < SPH_RED_COUNT) {
        double s = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) s += red[threadIdx.x][w];
        partials[(size_t)blockIdx.x * SPH_RED_COUNT + threadIdx.x] = s;
    }
}

// Second pass: one block sums the rows in a fixed order.
__global__ void __launch_bounds__(256) k_reduce_final(const double* __restrict__ partials, int nblocks,
                                                      double* __restrict__ out) {
    __shared__ double red[SPH_RED_COUNT][8];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < SPH_RED_COUNT; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * SPH_RED_COUNT + k];
        s = warp_sum(s);
        if (lane == 0) red[k][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < SPH_RED_COUNT) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

}  // namespace

extern "C" int sph_reduce_noalloc(const SphParams* p, const float* pos, const float* vel,
                                  const float* shift, int64_t n, double* out, void* stream) {
    if (!p || !out || n < 0) return SPH_ERR_ARG;
    if (p->struct_size != (int32_t)sizeof(SphParams)) return SPH_ERR_ARG;
    // a solid's elastic energy needs each particle's stress and material row, which this
    // entry point is not given: refused rather than returned as a silent zero
    if (p->is_solid) return SPH_ERR_UNSUPPORTED;
    if (n > kNoAllocMaxParticles) return SPH_ERR_SCRATCH_CAP;
    if (n > 0 && (!pos || !vel)) return SPH_ERR_ARG;
    auto misaligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) != 0; };
    if ((pos && misaligned(pos)) || (vel && misaligned(vel)) || (shift && misaligned(shift)) ||
        (reinterpret_cast<uintptr_t>(out) & 7u) != 0)
        return SPH_ERR_ARG;
    double* partials = nullptr;
    int r = scratch_address(&partials);
    if (r != SPH_OK) return r;
    Cst c;
    fill_constants_from(*p, n, c);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int nb = (int)((n + kBlock - 1) / kBlock);
    if (nb == 0) nb = 1;
    k_reduce_partials<<<nb, kBlock, 0, st>>>(c, reinterpret_cast<const float4*>(pos),
                                             reinterpret_cast<const float4*>(vel),
                                             reinterpret_cast<const float4*>(shift), partials);
    k_reduce_final<<<1, 256, 0, st>>>(partials, nb, out);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

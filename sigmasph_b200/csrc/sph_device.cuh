// sph_device.cuh -- launch-parameter structs and device helpers shared by every kernel
// of libsph_b200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sph_b200.h"

namespace sph {

constexpr int kBlock = 256;          // threads per block of the particle-parallel kernels
// Pair-loop kernels whose live state fits 64 registers with little spilling run four
// 256-thread blocks per SM (50% occupancy): their gathers are latency-bound, so the extra
// resident warps pay more than the spills cost.  Kernels that keep a 3x3 stress and
// velocity gradient per pair live keep the compiler's default budget.
#define SPH_PAIR_BOUNDS_OCC4 __launch_bounds__(kBlock, 4)
// The solid sweeps that keep a stress and a velocity gradient live (110+ registers at the
// default budget) run three blocks per SM: 80 registers and a few spills measured 6%
// faster per step than two blocks without spills.
#define SPH_PAIR_BOUNDS_OCC3 __launch_bounds__(kBlock, 3)
// Resident 256-thread blocks per SM of each pass over the lists (the register budget
// follows: 64, 40 and 32 registers at 4, 6 and 8), as measured best on the 1M dam break
// and the 2.38M bar: the passes are latency-bound, so resident warps pay until spills
// grow (the shift pass: 5 -> 6 blocks 0.75 -> 0.70 ms, 7 and 8 slower; lambda 4 -> 6,
// 0.30 -> 0.26 ms; the filter 8; the force and gradient passes spill heavily below 64
// registers and stay at 4; the solid sweeps slow down at 4).  A build may override one
// with -DSPH_OCC_<PASS>=n to time another.
#ifndef SPH_OCC_LAM
#define SPH_OCC_LAM 7
#endif
#ifndef SPH_OCC_LAMGRAD
#define SPH_OCC_LAMGRAD 4
#endif
#ifndef SPH_OCC_FORCE
#define SPH_OCC_FORCE 5
#endif
#ifndef SPH_OCC_PST
#define SPH_OCC_PST 6
#endif
#ifndef SPH_OCC_FILTER
#define SPH_OCC_FILTER 8
#endif
#ifndef SPH_OCC_SOLID_A
#define SPH_OCC_SOLID_A 3
#endif
#ifndef SPH_OCC_SOLID_B
#define SPH_OCC_SOLID_B 3
#endif
#ifndef SPH_OCC_SOLID_FORCE
#define SPH_OCC_SOLID_FORCE 3
#endif
#define SPH_BOUNDS(occ) __launch_bounds__(kBlock, occ)
constexpr int kMirShift = 30;        // neighbour entry = j | mirror code << 30
constexpr int kIdxMask = (1 << 29) - 1;

// Cell layout of the current rebuild, written by k_layout on the device.
struct GridLayout {
    int mode;          // 0 dense Morton table over the occupied cell box, 1 hashed table
    int nbuckets;      // buckets in use; the off-grid bucket is index nbuckets
    int cmin[3];
    int cmax[3];
    int bits[3];       // Morton bits per axis (dense mode)
    int total_bits;
    unsigned mask[3];  // the key bits each axis occupies (dense mode)
};

// Device copy of SphScalars (identical layout, so one memcpy returns it).
typedef SphScalars DevScalars;

// Per-step accumulators that are not part of the user-visible scalars.
struct DevAccum {
    double w_diff_step;      // sum_i -V_i p_i rate1_i of the continuity pass
    double red[SPH_RED_COUNT];
    unsigned int max_c_sq_bits;
    unsigned int max_accel_bits;
    unsigned int max_v_bits;
    unsigned int max_disp_bits;  // max position change of this step's advect (float bits)
    unsigned int max_grip_disp_bits;  // max position change of the grips' overwrite
    unsigned int d_start_bits;   // max |x - x_build| at this step's start (0 after a build)
    int rebuild;                 // 1: this step builds the candidate lists
    int force_build;             // set by the host: the next step builds
    int off_grid_build;          // off-grid count at the last build
    unsigned int ovf_used;       // overflow-pool entries taken this step
    unsigned int near_m_bits;    // margin M of this step's near lists (0: none)
    unsigned int relax_max_bits; // the initial relaxation's residual (float bits)
    unsigned int m_min_bits, m_max_bits;   // this step's particle masses, as bit patterns
                                           // (equal: every particle has that mass)
    double hg_power;         // sum_i mw_i de_hg_i of the in-loop damper (solid)
    double visc_power;       // sum_i m_i de_visc_i, Morris + Monaghan (solid)
    unsigned int visc_c_bits;    // max signal speed of the viscosities' CFL limits (solid)
    unsigned long long n_steps, n_builds, n_shift_search;   // list statistics
};

// Constants of one handle, passed by value to every kernel.
struct Cst {
    SphParams p;
    int n;               // active particles
    int K;               // neighbour-list capacity per particle
    int mcap;            // bucket capacity of the coarse cell table (power of two)
    int mcap_log2;
    float h;             // support radius == cell size of the reference's bins
    float inv_h;         // 1 / h
    float alpha;         // Wendland prefactor
    float kgrad;         // 20 alpha / h
    float eta2;          // 0.01 h^2
    float W_dx0;         // W(dx0)
    float d2_lt;         // |r| < h  <=>  d2 < d2_lt, with d2 = (dx^2 + dy^2) + dz^2 (RN)
    float visc_coef;     // 2 (dim + 2) nu = 10 nu
    float delta_coef;    // delta h c0
    float cfl_h;         // CFL h
    float wall_hi[3];    // domain_size - padding
    float rest_1p;       // 1 + c_f
    float rest_loss;     // 1 - c_f^2
    float max_shift;     // pst_max_shift dx0
    float colle_coef;    // -2 h
    float sun_coef;      // -CFL
    int mirror_y, mirror_z;
    // solid material table (device) and ensemble mode
    int n_inst;          // 0: one scene; > 0: instances, instance = material row
    int any_plastic;     // some material row has a yield stress
    int all_gamma_one;   // every EOS is linear (exponent 1)
    int any_jc;          // some material row is Johnson-Cook (return statistics kept)
    int one_material;    // one material row and no ensemble: every pair is same-material
    int block;           // threads per block of the solid particle kernels
    // candidate lists with a skin: every pair within h + skin at the last build, binned
    // in coarse cells of h + skin; complete while no particle moved more than dlim since
    int Kv;              // candidate-list capacity per particle
    unsigned int ovf_cap;  // overflow-pool capacity (entries)
    float skin;          // skin width (h / 10)
    float hc;            // coarse cell size h + skin
    float dlim;          // displacement bound of the lists: skin / 2, less a margin
    float d2_skin;       // |r| < h + skin (conservative) in dist2_rn units
    float d2_deep;       // |r| < h - skin (conservative): stays within h under the bound
};

// Johnson-Cook return-map surrogate and sample log (solid only; null when unused).
struct JcPtr {
    int* count;                    // queued returns this step
    int* idx;                      // [n] particle of each queued return
    float4* feat;                  // [n] its features
    float* fpred;                  // [n] network output u = 10 (1 - d / d_hi)
    const float* W;                // [8705] float32 parameters
    const void* packed;            // BF16 hidden-layer weights, tensor-core layout
    unsigned long long* stats;     // Newton solves, Newton iterations, queued, accepted
    float* log;                    // [log_cap][8] exact returns of the plain path
    unsigned long long* log_count;
    long long log_cap;
};

// Device pointers of one launch.
struct Ptr {
    SphFieldSet cur, nxt;
    float4* acc;
    float* lam;
    float4* lsym;        // two float4 per particle
    float4* lgrad;
    float4* div;
    float* gradv;
    float4* aux;
    float4* gsym;        // [n][2] solid: the symmetric part of grad v (S00 S11 S22 S01 | S02 S12)
                         // with the pressure p and the bulk viscosity q in the last two words
    // scratch
    int4* cell;          // coarse cell at the last build, current order: x, y, z, bucket
                         // (w = -1 off-grid)
    int4* fcell;         // cell of size h at this step's start: x, y, z, 0 (w = -1 off-grid)
    float4* xb;          // positions at the last build

    int* key;            // bucket of each pre-sort particle
    int* rank;           // slot within its bucket (arbitrary before the stabilise pass)
    int* perm;           // new index -> old index
    int* hist;           // [mcap + 2] bucket counts
    int* start;          // [mcap + 2] exclusive scan of hist
    int* bsum;           // block sums of the scan
    int* bbox;           // [6] cell box min/max
    GridLayout* layout;
    int* nbr;            // [K][n] this step's neighbours, k-major
    int* nbr_cnt;        // [n] true count; entries past K sit in the overflow pool
    int* ovf;            // [ovf_cap] overflow pool, one run per overflowing particle
    int* ovf_off;        // [n] start of the particle's run
    int* vl;             // [Kv][n] candidates within h + skin at the last build, k-major
    int* vl_cnt;         // [n]
    int* nl_cnt;         // [n] this step's near candidates (edge, h <= |r| < h + M), kept in
                         // the neighbour list's last rows
    DevScalars* sc;
    DevAccum* ac;
    JcPtr jc;
    const SphMatRow* mat;      // [rows] solid material rows
    const SphInstRow* irow;    // [n_inst] ensemble instance constants
    SphInstState* inst;        // [n_inst] ensemble instance state
};

// ------------------------------------------------------------------ small vector ops
struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ void operator+=(F3& a, F3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float norm3(F3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ F3 mirror3(int code, F3 a) {
    return {a.x, (code & 1) ? -a.y : a.y, (code & 2) ? -a.z : a.z};
}

// Squared distance in the pinned order (dx^2 + dy^2) + dz^2, every operation rounded to
// nearest with no contraction: the neighbour test must decide exactly as the reference's
// float32 (x_i - x_j).norm() < h does.
__device__ __forceinline__ float dist2_rn(F3 a, F3 b) {
    float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Cell of a position: floor(x / h) with a correctly rounded division
// (particle_system.py:1220-1222).  Clamped far outside any grid so the integer
// conversion stays defined.
__device__ __forceinline__ int cell_of(float x, float h) {
    float q = floorf(__fdiv_rn(x, h));
    q = fminf(fmaxf(q, -1.0e9f), 1.0e9f);
    return (int)q;
}

// cell_of from a product with the rounded reciprocal when that cannot change the floor:
// x * inv_h is within 2.5e-7 relative of x / h, so a quotient more than 1e-6 (relative)
// from the nearest integer floors the same; otherwise the correctly rounded division.
__device__ __forceinline__ int cell_of_fast(float x, float h, float inv_h) {
    const float q = x * inv_h;
    if (fabsf(q - rintf(q)) > 1.0e-6f * fmaxf(fabsf(q), 1.0f) && fabsf(q) < 1.0e9f) return (int)floorf(q);
    return cell_of(x, h);
}

// Spatial hash of the reference (particle_system.py:1283-1293), the fallback table.
__device__ __forceinline__ int hash_cell(int cx, int cy, int cz, int mcap) {
    unsigned h = (unsigned)cx * 73856093u;
    h ^= (unsigned)cy * 19349663u;
    h ^= (unsigned)cz * 83492791u;
    return (int)(h & (unsigned)(mcap - 1));
}

// Compact Morton code of a cell offset inside the occupied box: bits are interleaved
// from the least significant end, x then y then z, each axis contributing only the
// bits its extent needs.  The key is the OR of the three axes' dilated offsets: each
// offset's bits deposited, lowest first, at the key bits its axis occupies (mask[a]).
__device__ __forceinline__ unsigned dilate(unsigned v, unsigned mask) {
    unsigned r = 0u;
    for (unsigned m = mask; m != 0u && v != 0u; m &= m - 1u, v >>= 1) r |= (v & 1u) ? (m & (0u - m)) : 0u;
    return r;
}
// The dilated offset one step further along the same axis: the carry skips the other
// axes' bits (which the OR with ~mask fills).
__device__ __forceinline__ unsigned dilated_next(unsigned d, unsigned mask) { return ((d | ~mask) + 1u) & mask; }
__device__ __forceinline__ int morton_key(int ox, int oy, int oz, const GridLayout& L) {
    return (int)(dilate((unsigned)ox, L.mask[0]) | dilate((unsigned)oy, L.mask[1]) |
                 dilate((unsigned)oz, L.mask[2]));
}

// Bucket of a cell, or -1 if no particle can be binned there (outside the dense box).
__device__ __forceinline__ int bucket_of(int cx, int cy, int cz, const GridLayout& L, int mcap) {
    if (L.mode == 0) {
        int ox = cx - L.cmin[0], oy = cy - L.cmin[1], oz = cz - L.cmin[2];
        if (ox < 0 || oy < 0 || oz < 0 || cx > L.cmax[0] || cy > L.cmax[1] || cz > L.cmax[2])
            return -1;
        return morton_key(ox, oy, oz, L);
    }
    return hash_cell(cx, cy, cz, mcap);
}

// ------------------------------------------------------------------ Wendland C2 (sph_base.py:42-92)
__device__ __forceinline__ float wendland_W(float r, const Cst& c) {
    float q = r * c.inv_h;
    if (q < 1.0f) {
        float t = 1.0f - q;
        float t2 = t * t;
        return c.alpha * (t2 * t2) * (4.0f * q + 1.0f);
    }
    return 0.0f;
}
// grad_i W for r = x_i - x_j given |r| (the caller has it already).
__device__ __forceinline__ F3 wendland_dW(F3 r, float rn, const Cst& c) {
    float q = rn * c.inv_h;
    if (q < 1.0f && rn > 1.0e-5f) {
        float t = 1.0f - q;
        float cc = -(c.kgrad * q * (t * t * t));
        float f = __fdividef(cc, rn);
        return f * r;
    }
    return {0.0f, 0.0f, 0.0f};
}
// |r| and grad_i W from the squared separation, one reciprocal square root.
__device__ __forceinline__ F3 wendland_dW2(F3 r, float d2, float& rn, const Cst& c) {
    rn = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;   // coincident pair: |r| = 0, grad W = 0
    float q = rn * c.inv_h;
    if (q < 1.0f && rn > 1.0e-5f) {
        float t = 1.0f - q;
        float f = -(c.kgrad * c.inv_h * (t * t * t));   // (-kgrad q (1-q)^3) / |r|
        return f * r;
    }
    return {0.0f, 0.0f, 0.0f};
}

// The factor f of grad_i W = f r (r = x_i - x_j) from the squared separation: the
// arithmetic of wendland_dW2 without the vector.
__device__ __forceinline__ float wendland_dW_factor(float d2, const Cst& c) {
    const float rn = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;
    const float q = rn * c.inv_h;
    if (q < 1.0f && rn > 1.0e-5f) {
        const float t = 1.0f - q;
        return -(c.kgrad * c.inv_h * (t * t * t));
    }
    return 0.0f;
}

// W and grad_i W from the squared separation in one evaluation: the same arithmetic as
// wendland_dW2 followed by wendland_W(rn).
__device__ __forceinline__ F3 wendland_W_dW2(F3 r, float d2, float& W, const Cst& c) {
    const float rn = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;
    const float q = rn * c.inv_h;
    W = 0.0f;
    if (q < 1.0f) {
        const float t = 1.0f - q;
        const float t2 = t * t;
        W = c.alpha * (t2 * t2) * (4.0f * q + 1.0f);
        if (rn > 1.0e-5f) {
            const float f = -(c.kgrad * c.inv_h * (t2 * t));
            return f * r;
        }
    }
    return {0.0f, 0.0f, 0.0f};
}

// x^n for the Monaghan tensile-correction exponent (an integer in every deck; any other
// value goes through powf).  Repeated products in the order ((x x) x) ..., unrolled.
__device__ __forceinline__ float ipow_or_pow(float x, int n) {
    float r;
    switch (n) {
        case 0: return 1.0f;
        case 1: return x;
        case 2: return x * x;
        case 3: r = x * x; return r * x;
        case 4: r = x * x; r = r * x; return r * x;
        default: break;
    }
    if (n > 4 && n <= 8) {
        r = 1.0f;
        for (int k = 0; k < n; ++k) r *= x;
        return r;
    }
    return powf(x, (float)n);
}

// SPH quadrature weight and its mass (particle_system.py:990-1004).
__device__ __forceinline__ float w_of(float4 pos, const Cst& c) {
    return c.p.axisymmetric ? pos.w / fmaxf(pos.y, c.p.axi_r_min) : pos.w;
}
__device__ __forceinline__ float mw_of(float m, float4 pos, const Cst& c) {
    return c.p.axisymmetric ? m / fmaxf(pos.y, c.p.axi_r_min) : m;
}

// The deck as the pair passes see it, fixed when a pass is compiled (Shape<kShape>):
//  0  every switch read from the parameters;
//  1  plain: a 3D deck with no mirror plane and no axisymmetry (neighbour entries carry
//     no mirror code; the weights are the stored volumes);
//  2  plain and standard: also every term of the default step on -- delta+-SPH with the
//     shift, its ALE terms, the gradient-lambda surface normal, delta diffusion and the dt
//     pair limit; for a solid also one material, the in-loop hourglass damper, Morris
//     viscosity, plasticity and the ALE transport of the history and of e -- no ensemble;
//  3  plain 2D: a single-layer (plane-strain or 2D) deck with no mirror plane and no
//     axisymmetry (the strip ensembles).
// A uniform switch inside a pair loop costs issue slots and splits the loop body the
// compiler schedules; the dam break and the round bar run instance 2.
__host__ __device__ __forceinline__ bool plain_shape(const Cst& c) {
    return !c.mirror_y && !c.mirror_z && !c.p.axisymmetric && !c.p.two_d;
}
__host__ __device__ __forceinline__ bool std_form(const Cst& c) {
    const SphParams& p = c.p;
    const bool fluid = p.pst_enabled && p.pst_ale_momentum && !p.pst_normal_eigvec && p.delta_sph > 0.0f &&
                       p.dt_pair_mode != 0 && c.n_inst == 0 && !p.delta_pairs_all && !p.c0_mixed &&
                       !p.hg_mixed_impedance;
    if (!p.is_solid) return fluid;
    return fluid && p.hourglass_alpha > 0.0f && !p.hourglass_sts && p.viscosity > 0.0f && c.one_material &&
           c.any_plastic && p.ale_history && p.transport_e && p.ale_diffusion > 0.0f;
}
__host__ __device__ __forceinline__ bool plain2d_shape(const Cst& c) {
    return !c.mirror_y && !c.mirror_z && !c.p.axisymmetric && c.p.two_d;
}
__host__ __device__ __forceinline__ int shape_of(const Cst& c) {
    return plain_shape(c) ? (std_form(c) ? 2 : 1) : (plain2d_shape(c) ? 3 : 0);
}
template <int kShape>
struct Shape {
    static constexpr bool kPlain = kShape >= 1, kStd = kShape == 2, k2D = kShape == 3;
    __device__ static __forceinline__ bool two_d(const Cst& c) { return k2D || (!kPlain && c.p.two_d); }
    __device__ static __forceinline__ bool axi(const Cst& c) { return !kPlain && c.p.axisymmetric; }
    __device__ static __forceinline__ float w(float4 pos, const Cst& c) { return kPlain ? pos.w : w_of(pos, c); }
    __device__ static __forceinline__ float mw(float m, float4 pos, const Cst& c) {
        return kPlain ? m : mw_of(m, pos, c);
    }
    __device__ static __forceinline__ int idx(int e) { return kPlain ? e : (e & kIdxMask); }
    __device__ static __forceinline__ int mir(int e) { return kPlain ? 0 : (int)((unsigned)e >> kMirShift); }
    // the step's terms
    __device__ static __forceinline__ bool pst(const Cst& c) { return kStd || c.p.pst_enabled; }
    __device__ static __forceinline__ bool lgrad(const Cst& c) { return kStd || !c.p.pst_normal_eigvec; }
    __device__ static __forceinline__ bool delta(const Cst& c) { return kStd || c.p.delta_sph > 0.0f; }
    __device__ static __forceinline__ bool ale_mom(const Cst& c) {
        return kStd || (c.p.pst_enabled && c.p.pst_ale_momentum);
    }
    __device__ static __forceinline__ bool dt_pairs(const Cst& c) { return kStd || c.p.dt_pair_mode != 0; }
    __device__ static __forceinline__ bool ensemble(const Cst& c) { return !kStd && c.n_inst > 0; }
    __device__ static __forceinline__ bool pairs_all(const Cst& c) { return !kStd && c.p.delta_pairs_all; }
    __device__ static __forceinline__ bool c0_mixed(const Cst& c) { return !kStd && c.p.c0_mixed; }
    // the solid's
    __device__ static __forceinline__ bool hg_inloop(const Cst& c) {
        return kStd || (c.p.hourglass_alpha > 0.0f && !c.p.hourglass_sts);
    }
    __device__ static __forceinline__ bool hg_mixed(const Cst& c) { return !kStd && c.p.hg_mixed_impedance; }
    __device__ static __forceinline__ bool visc(const Cst& c) { return kStd || c.p.viscosity > 0.0f; }
    __device__ static __forceinline__ bool one(const Cst& c) { return kStd || c.one_material; }
    __device__ static __forceinline__ bool plastic(const Cst& c) { return kStd || c.any_plastic; }
    __device__ static __forceinline__ bool ale_hist(const Cst& c) { return kStd || c.p.ale_history; }
    __device__ static __forceinline__ bool transport_e(const Cst& c) { return kStd || c.p.transport_e; }
    __device__ static __forceinline__ bool ale_diff(const Cst& c) { return kStd || c.p.ale_diffusion > 0.0f; }
};
// Launches the instance of a shape-templated pass for the deck (shape_of).
#define SHAPED(shape, kernel, ...)                   \
    do {                                             \
        const int shape_ = (shape);                  \
        if (shape_ == 2) kernel<2> __VA_ARGS__;      \
        else if (shape_ == 1) kernel<1> __VA_ARGS__; \
        else if (shape_ == 3) kernel<3> __VA_ARGS__; \
        else kernel<0> __VA_ARGS__;                  \
    } while (0)

// One particle's terms of every FP64 reduction.
__device__ __forceinline__ void reduce_terms(const Cst& c, float4 p, float4 v, float e_int,
                                             double r[SPH_RED_COUNT]) {
    {
        double m = (double)v.w;
        float vv = v.x * v.x + v.y * v.y + v.z * v.z;
        double ke = (double)(0.5f * v.w * vv);
        bool ongrid = !(isnan(p.x) || isnan(p.y) || isnan(p.z));
        r[SPH_RED_KE] = ke;
        r[SPH_RED_KE_OFFGRID] = ongrid ? 0.0 : ke;
        float gdx = c.p.gravity[0] * p.x + c.p.gravity[1] * p.y + c.p.gravity[2] * p.z;
        r[SPH_RED_PE] = -m * (double)gdx;
        // DSPHSolver.compute_elastic_energy: Tait compression energy in float64
        double rho = m / (double)p.w, rho0 = (double)c.p.density0;
        double S = (double)c.p.stiffness, gam = (double)c.p.exponent;
        double x = rho / rho0, e;
        if (fabs(gam - 1.0) < 1.0e-6) e = (S / rho0) * (log(x) + 1.0 / x - 1.0);
        else e = (S / rho0) * ((pow(x, gam - 1.0) - 1.0) / (gam - 1.0) + 1.0 / x - 1.0);
        if (!c.p.allow_negative_pressure && rho < rho0) e = 0.0;
        r[SPH_RED_SE] = c.p.is_solid ? 0.0 : m * e;
        r[SPH_RED_IE] = c.p.is_solid ? m * (double)e_int : 0.0;
        r[SPH_RED_MASS] = m;
        r[SPH_RED_PX] = m * (double)v.x;
        r[SPH_RED_PY] = m * (double)v.y;
        r[SPH_RED_PZ] = m * (double)v.z;
        double vx = v.x, vy = v.y, vz = v.z;
        r[SPH_RED_GROSS_P] = m * sqrt(vx * vx + vy * vy + vz * vz);
        r[SPH_RED_ELASTIC] = 0.0;
    }
}

// ------------------------------------------------------------------ reductions
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Block sum of a double, atomically added to *dst by one thread per block.
__device__ __forceinline__ void block_sum_atomic(double v, double* dst) {
    __shared__ double red[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double s = lane < nw ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0 && s != 0.0) atomicAdd(dst, s);
    }
    __syncthreads();
}
// Block minimum and maximum of 32-bit patterns, atomically folded into *dmin and *dmax.
__device__ __forceinline__ void block_minmax_bits(unsigned int lo, unsigned int hi,
                                                  unsigned int* dmin, unsigned int* dmax) {
    __shared__ unsigned int red[2][32];
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { red[0][wid] = lo; red[1][wid] = hi; }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        unsigned int a = lane < nw ? red[0][lane] : 0xffffffffu, b = lane < nw ? red[1][lane] : 0u;
        a = __reduce_min_sync(0xffffffffu, a);
        b = __reduce_max_sync(0xffffffffu, b);
        if (lane == 0) { atomicMin(dmin, a); atomicMax(dmax, b); }
    }
    __syncthreads();
}
// Block max of a non-negative float, atomically maxed into the bit pattern *dst
// (order-preserving for non-negative IEEE floats).
__device__ __forceinline__ void block_max_atomic(float v, unsigned int* dst) {
    __shared__ float red[32];
    v = warp_max(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        float s = lane < nw ? red[lane] : 0.0f;
        s = warp_max(s);
        if (lane == 0) atomicMax(dst, __float_as_uint(fmaxf(s, 0.0f)));
    }
    __syncthreads();
}

// ------------------------------------------------------------------ 3x3 symmetric eigen
// Cyclic Jacobi (the same published method the oracle restates for ti.sym_eig).
// A is overwritten; Q receives the eigenvectors as columns; ev the eigenvalues.
template <class T>
__device__ __forceinline__ void sym_eig3(T A[3][3], T ev[3], T Q[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Q[i][j] = (i == j) ? T(1) : T(0);
    const T eps = sizeof(T) == 4 ? T(1e-14) : T(1e-30);
    for (int sweep = 0; sweep < 12; ++sweep) {
        T off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        T diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (!(off > eps * diag) || off == T(0)) break;
#pragma unroll
        for (int p = 0; p < 2; ++p) {
#pragma unroll
            for (int q = p + 1; q < 3; ++q) {
                T apq = A[p][q];
                if (apq == T(0)) continue;
                T theta = (A[q][q] - A[p][p]) / (T(2) * apq);
                T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
                T cs = T(1) / sqrt(t * t + T(1));
                T s = t * cs;
                T tau = s / (T(1) + cs);
                A[p][p] -= t * apq;
                A[q][q] += t * apq;
                A[p][q] = A[q][p] = T(0);
                const int r = 3 - p - q;
                T arp = A[r][p], arq = A[r][q];
                A[r][p] = A[p][r] = arp - s * (arq + tau * arp);
                A[r][q] = A[q][r] = arq + s * (arp - tau * arq);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    T qkp = Q[k][p], qkq = Q[k][q];
                    Q[k][p] = qkp - s * (qkq + tau * qkp);
                    Q[k][q] = qkq + s * (qkp - tau * qkq);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) ev[k] = A[k][k];
}

// spd_inverse.py:45-50
template <class T>
__device__ __forceinline__ T spd_weight(T e, T tol) {
    T u = fmin(T(1), fmax(T(0), (e - tol) / tol));
    T beta = u * u * (T(3) - T(2) * u);
    return beta / fmax(e, tol) + (T(1) - beta);
}

}  // namespace sph

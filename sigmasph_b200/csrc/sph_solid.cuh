// sph_solid.cuh -- the hypoelastic tensile-solid step (SOLID.py HypoElasticSolver.substep,
// :5060-5196, and step, :5227-5231) as sm_100a kernels over the neighbour lists.
//
//   k_solid_load     update_load_factor (SOLID.py:5001-5017), on the device clock
//   (rebuild, k_lam as for the fluid; k_lam also forms the kernel-correction inverse)
//   k_solid_a        grad lambda + continuity + grad v, one sweep      (DSPH.py:683-702,
//                    :1208-1338, SOLID.py:1721-1794)
//   k_solid_b        ALE transport of s, eps_p, e (one sweep); epilogue: Jaumann update,
//                    J2 / Johnson-Cook return, energy and temperature  (SOLID.py:1799-2293,
//                    :2691-3004)
//   k_solid_commit   the updated history, volume update, per-material EOS, the bulk
//                    viscosity q, gravity; banks the previous step's damper, viscous
//                    and diffusion work                            (SOLID.py:2182-2207)
//   k_solid_force    stress divergence (p + q) + Morris + Monaghan + in-loop hourglass
//                    + ALE momentum, the work conjugate de_int, the dt pair estimate
//                                                                  (SOLID.py:3204-3852)
//   k_solid_dt       CFL limits incl. the viscosities', the damper cap or sub-step
//                    count                       (SOLID.py:3939-4009, :4116-4161, :4510-4539)
//   k_half_kick, k_gradv, k_hg_stage x32, k_sts_finish   the sub-cycled damper between
//                    the half kicks, with a device-side stage count (SOLID.py:4485-4615)
//   k_solid_advect   plain advect when the damper is in-loop
//   k_constraints    grip kinematics and FP64 grip force          (SOLID.py:5019-5055)
//   (k_pst, k_finish as for the fluid)
//
// Per-step scratch in aux ([n][24] floats = 6 float4):
//   aux[0]  s_new xx yy zz xy     aux[1]  s_new xz yz, eps_p_new, e_new
//   aux[2]  T_new, -, -, -        aux[3]  kernel-correction inverse L00 L11 L22 L01
//   aux[4]  L02 L12 | v_sync.xy   aux[5]  v_sync.z | -
// The damper's sub-stepped velocity ping-pongs between aux[0..1] and aux[2..3]-free
// slots: y_a = aux float4 slot 0 (xyz), y_b = slot 2 (xyz), used only after the history
// has been committed.
#pragma once
#include "sph_fluid.cuh"
#include "sph_mlp.cuh"

namespace sph {

constexpr int kStsMaxStages = 32;

// Library-owned buffers of the Johnson-Cook surrogate, allocated on its first use
// (sph_jc_surrogate); the sample log is caller-owned (sph_jc_log).
struct SolidScratch {
    int* q_count = nullptr;
    int* q_idx = nullptr;
    float4* q_feat = nullptr;
    float* q_pred = nullptr;
    float* W = nullptr;
    void* packed = nullptr;
    unsigned long long* stats = nullptr;
    int* mlp_err = nullptr;
    float* log = nullptr;
    unsigned long long* log_count = nullptr;
    long long log_cap = 0;
    // material rows (ordinary scene: from SphParams) and ensemble instances
    SphMatRow* mat = nullptr;
    SphInstRow* irow = nullptr;
    SphInstState* inst = nullptr;
    float4* gsym = nullptr;          // [n][2] symmetric grad v, p, q (the damper's pair record)
    int n_inst = 0;
    bool any_plastic = false, all_gamma_one = true, any_jc = false;
};
constexpr int kMaxInstances = 1024;

inline void solid_fill_constants(Cst&) {}
inline int solid_alloc(SolidScratch& s, const SphParams& p, int64_t n) {
    if (!p.is_solid) return SPH_OK;
    if (cudaMalloc(&s.stats, 4 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&s.gsym, (size_t)(n > 0 ? n : 1) * 2 * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&s.mat, kMaxInstances * sizeof(SphMatRow)) != cudaSuccess ||
        cudaMalloc(&s.irow, kMaxInstances * sizeof(SphInstRow)) != cudaSuccess ||
        cudaMalloc(&s.inst, kMaxInstances * sizeof(SphInstState)) != cudaSuccess)
        return SPH_ERR_NOMEM;
    if (cudaMemset(s.stats, 0, 4 * sizeof(unsigned long long)) != cudaSuccess) return SPH_ERR_CUDA;
    return SPH_OK;
}
// The rows of an ordinary scene, from SphParams' per-material tables.
inline void solid_rows_from_params(const SphParams& p, SphMatRow* rows) {
    for (int k = 0; k < p.n_materials && k < 4; ++k) {
        SphMatRow& r = rows[k];
        r.rho0 = p.mat_rho0[k]; r.K = p.mat_K[k]; r.G = p.mat_G[k]; r.cp = p.mat_cp[k];
        r.c0 = p.mat_c0[k]; r.delta = p.mat_delta[k];
        r.plastic_kind = p.plastic_kind[k]; r.sy0 = p.plastic_sy0[k]; r.H = p.plastic_H[k];
        r.jc_A = p.jc_A[k]; r.jc_B = p.jc_B[k]; r.jc_n = p.jc_n[k]; r.jc_C = p.jc_C[k];
        r.jc_eps0_dot = p.jc_eps0_dot[k]; r.jc_T0 = p.jc_T0[k]; r.jc_Tm = p.jc_Tm[k];
        r.jc_m = p.jc_m[k]; r.jc_chi = p.jc_chi[k];
        r.cv = p.mat_cv[k]; r.stiff = p.mat_stiff[k]; r.gamma = p.mat_gamma[k]; r.T0 = p.mat_T0[k];
    }
}
inline void solid_row_flags(const SphMatRow* rows, int n, bool& any_plastic, bool& all_gamma_one,
                            bool& any_jc) {
    any_plastic = false;
    all_gamma_one = true;
    any_jc = false;
    for (int k = 0; k < n; ++k) {
        any_plastic = any_plastic || rows[k].sy0 > 0.0f;
        all_gamma_one = all_gamma_one && rows[k].gamma == 1.0f;
        any_jc = any_jc || rows[k].plastic_kind == 2;
    }
}
// Uploads the scene's own rows (single-scene mode) and sets the table flags in c.
inline int solid_sync_rows(SolidScratch& s, const SphParams& p, Cst& c) {
    if (!p.is_solid || !s.mat) return SPH_OK;
    if (s.n_inst > 0) {                      // an ensemble keeps its rows
        c.n_inst = s.n_inst;
        c.any_plastic = s.any_plastic;
        c.all_gamma_one = s.all_gamma_one;
        c.any_jc = s.any_jc;
        c.one_material = 0;
        return SPH_OK;
    }
    SphMatRow rows[4] = {};
    solid_rows_from_params(p, rows);
    solid_row_flags(rows, p.n_materials, s.any_plastic, s.all_gamma_one, s.any_jc);
    c.n_inst = 0;
    c.any_plastic = s.any_plastic;
    c.all_gamma_one = s.all_gamma_one;
    c.any_jc = s.any_jc;
    c.one_material = p.n_materials <= 1;
    if (cudaMemcpy(s.mat, rows, sizeof(rows), cudaMemcpyHostToDevice) != cudaSuccess) return SPH_ERR_CUDA;
    return SPH_OK;
}
inline int solid_jc_alloc(SolidScratch& s, int64_t n) {
    if (s.q_count) return SPH_OK;
    const size_t m = (size_t)(n > 0 ? n : 1);
    if (cudaMalloc(&s.q_count, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&s.q_idx, m * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&s.q_feat, m * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&s.q_pred, m * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s.W, kMlpParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s.packed, kMlpPackedBytes) != cudaSuccess ||
        cudaMalloc(&s.mlp_err, sizeof(int)) != cudaSuccess)
        return SPH_ERR_NOMEM;
    if (cudaMemset(s.q_count, 0, sizeof(int)) != cudaSuccess ||
        cudaMemset(s.mlp_err, 0, sizeof(int)) != cudaSuccess)
        return SPH_ERR_CUDA;
    return SPH_OK;
}
inline void solid_free(SolidScratch& s) {
    void* ps[] = {s.q_count, s.q_idx, s.q_feat, s.q_pred, s.W, s.packed, s.stats, s.mlp_err,
                  s.mat, s.irow, s.inst, s.gsym};
    for (void* q : ps) if (q) cudaFree(q);
    s = SolidScratch();
}
inline JcPtr solid_jc_ptr(const SolidScratch& s) {
    JcPtr j;
    j.count = s.q_count; j.idx = s.q_idx; j.feat = s.q_feat; j.fpred = s.q_pred;
    j.W = s.W; j.packed = s.packed; j.stats = s.stats;
    j.log = s.log; j.log_count = s.log_count; j.log_cap = s.log_cap;
    return j;
}

// ------------------------------------------------------------------ helpers
struct Sym { float xx, yy, zz, xy, xz, yz; };
__device__ __forceinline__ Sym load_s(const float* sdev, int i) {
    const float4* s = reinterpret_cast<const float4*>(sdev) + 2 * i;
    float4 a = __ldg(s), b = __ldg(s + 1);
    return {a.x, a.y, a.z, a.w, b.x, b.y};
}
// load_s and the plastic strain, which shares the record's second float4.
__device__ __forceinline__ Sym load_s_ep(const float* sdev, int i, float& ep) {
    const float4* s = reinterpret_cast<const float4*>(sdev) + 2 * i;
    float4 a = __ldg(s), b = __ldg(s + 1);
    ep = b.z;
    return {a.x, a.y, a.z, a.w, b.x, b.y};
}
__device__ __forceinline__ Sym mirror_sym(int code, Sym s) {
    // M s M with M = diag(1, sy, sz): s_xy *= sy, s_xz *= sz, s_yz *= sy sz
    float sy = (code & 1) ? -1.0f : 1.0f, sz = (code & 2) ? -1.0f : 1.0f;
    return {s.xx, s.yy, s.zz, s.xy * sy, s.xz * sz, s.yz * sy * sz};
}
__device__ __forceinline__ float vm_sym(const Sym& s) {
    float t = s.xx * s.xx + s.yy * s.yy + s.zz * s.zz + 2.0f * (s.xy * s.xy + s.xz * s.xz + s.yz * s.yz);
    return sqrtf(1.5f * t);
}
__device__ __forceinline__ int eos_of(const Ptr& P, int i) {
    return (int)__ldg(P.cur.bcdisp + 4 * i + 3);
}
// Whether particle j has material row k (always, with one material and no ensemble).
__device__ __forceinline__ bool same_material(const Cst& c, const Ptr& P, int j, int k) {
    return c.one_material || eos_of(P, j) == k;
}
// Ensemble mode: a particle's material row is its instance, whose step state is
// per instance; an ordinary scene keeps one state in the device scalars.
__device__ __forceinline__ float dt_at(const Cst& c, const Ptr& P, int k) {
    return c.n_inst > 0 ? P.inst[k].dt : P.sc->dt;
}
__device__ __forceinline__ float visc_at(const Cst& c, const Ptr& P, int k) {
    return c.n_inst > 0 ? P.irow[k].visc_coef : c.visc_coef;
}
// atomicMax of a non-negative float (as its bits) into a field of each lane's instance:
// one pass per distinct instance in the warp (usually one), all lanes reducing together.
__device__ __forceinline__ void inst_max_atomic(float v, int k, bool on, unsigned int SphInstState::*field,
                                                SphInstState* inst) {
    const unsigned full = 0xffffffffu;
    unsigned pending = __ballot_sync(full, on);
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const int kl = __shfl_sync(full, k, leader);
        const bool mine = on && k == kl;
        const unsigned bits = __reduce_max_sync(full, mine ? __float_as_uint(v) : 0u);
        if ((int)(threadIdx.x & 31) == leader) atomicMax(&(inst[kl].*field), bits);
        pending &= ~__ballot_sync(full, mine);
    }
}
// atomicAdd of v into *addr, one atomic per distinct address in the warp.
__device__ __forceinline__ void addr_add_atomic(double v, double* addr, bool on) {
    const unsigned full = 0xffffffffu;
    const unsigned long long a = (unsigned long long)addr;
    unsigned pending = __ballot_sync(full, on);
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const unsigned long long al = __shfl_sync(full, a, leader);
        const bool mine = on && a == al;
        double t = mine ? v : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(full, t, o);
        if ((int)(threadIdx.x & 31) == leader) atomicAdd(reinterpret_cast<double*>(al), t);
        pending &= ~__ballot_sync(full, mine);
    }
}
__device__ __forceinline__ float r_axi_of(float y, const Cst& c) { return fmaxf(y, c.p.axi_r_min); }

// Per-material pressure: S((rho/rho0)^gamma - 1), exactly linear when every material's
// gamma is 1 (SOLID.py:3009-3038).
__device__ __forceinline__ float solid_pressure(const Cst& c, const Ptr& P, int k, float rho) {
    const SphMatRow& M = P.mat[k];
    float rho0 = M.rho0, S = M.stiff;
    float p = c.all_gamma_one ? S * (rho / rho0 - 1.0f) : S * (powf(rho / rho0, M.gamma) - 1.0f);
    if (!c.p.allow_negative_pressure) p = fmaxf(p, 0.0f);
    return p;
}

// _hg_impedance_ratio (SOLID.py:4184-4239): the damper's pair force carries particle i's
// acoustic impedance Z = rho0 c_p; 2 Z_j / (Z_i + Z_j) turns it into the pair's harmonic
// mean, so the force is antisymmetric across a material interface (exactly 1 when the two
// impedances are equal).
__device__ __forceinline__ float hg_impedance_ratio(const Ptr& P, int ki, int j) {
    const int kj = eos_of(P, j);
    const float zi = P.mat[ki].rho0 * P.mat[ki].cp, zj = P.mat[kj].rho0 * P.mat[kj].cp;
    const float den = zi + zj;
    return den > 0.0f ? 2.0f * zj / den : 1.0f;
}

// ------------------------------------------------------------------ load factor
__global__ void k_solid_load(Cst c, Ptr P) {
    if (c.n_inst > 0) {
        // per instance: its smoothstep from its own clock, and a fresh dt maximum
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.n_inst; k += gridDim.x * blockDim.x) {
            SphInstState& S = P.inst[k];
            const double T = P.irow[k].ramp_time;
            if (T <= 0.0) { S.load_s = 1.0f; S.load_sdot = 0.0f; }
            else {
                const double u = fmin(1.0, fmax(0.0, S.sim_time / T));
                S.load_s = (float)(u * u * (3.0 - 2.0 * u));
                S.load_sdot = (float)(6.0 * u * (1.0 - u) / T);
            }
            const float cs = P.irow[k].c_signal;
            S.max_c_sq_bits = __float_as_uint(cs * cs);
            S.max_accel_bits = __float_as_uint(1e-10f);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (P.jc.count) *P.jc.count = 0;
            P.sc->sts_stages = 0;   // the largest instance's stage count, from k_solid_dt
        }
        return;
    }
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (P.jc.count) *P.jc.count = 0;            // the surrogate queue of this step
    double T = c.p.ramp_time;
    if (T <= 0.0) { P.sc->load_s = 1.0f; P.sc->load_sdot = 0.0f; return; }
    double u = fmin(1.0, fmax(0.0, P.sc->sim_time / T));
    P.sc->load_s = (float)(u * u * (3.0 - 2.0 * u));
    P.sc->load_sdot = (float)(6.0 * u * (1.0 - u) / T);
}

// Velocity gradient sum G = sum_j w_j (v_j - v_i) (x) grad W (SOLID.py:1721-1794) with
// the optional correction G L, single-layer zeroing and the axisymmetric hoop rate.
template <class Extra>
__device__ __forceinline__ void grad_v_finish(const Cst& c, const Ptr& P, int i, float G[3][3],
                                              float4 pi, float vy) {
    if (c.p.kernel_correction) {
        float4 a = P.aux[6 * i + 3], b = P.aux[6 * i + 4];
        float L[3][3] = {{a.x, a.w, b.x}, {a.w, a.y, b.y}, {b.x, b.y, a.z}};
        float R[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) R[r][q] = G[r][0] * L[0][q] + G[r][1] * L[1][q] + G[r][2] * L[2][q];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) G[r][q] = R[r][q];
    }
    if (c.p.two_d) {
#pragma unroll
        for (int d = 0; d < 3; ++d) { G[2][d] = 0.0f; G[d][2] = 0.0f; }
    }
    if (c.p.axisymmetric) G[2][2] = vy / r_axi_of(pi.y, c);
    float* g = P.gradv + 12 * i;
    reinterpret_cast<float4*>(g)[0] = make_float4(G[0][0], G[0][1], G[0][2], G[1][0]);
    reinterpret_cast<float4*>(g)[1] = make_float4(G[1][1], G[1][2], G[2][0], G[2][1]);
    reinterpret_cast<float4*>(g)[2] = make_float4(G[2][2], 0.0f, 0.0f, 0.0f);
    // the damper's pair term reads only r^T (G_i + G_j) r, i.e. the symmetric parts (the
    // record's last two words, p and q, are k_solid_commit's)
    P.gsym[2 * i] = make_float4(G[0][0], G[1][1], G[2][2], 0.5f * (G[0][1] + G[1][0]));
    reinterpret_cast<float2*>(P.gsym + 2 * i + 1)[0] =
        make_float2(0.5f * (G[0][2] + G[2][0]), 0.5f * (G[1][2] + G[2][1]));
}
struct SymG { float xx, yy, zz, xy, xz, yz; };
// r^T S r for a symmetric S.
__device__ __forceinline__ float quad_sym(const SymG& S, F3 r) {
    return r.x * (S.xx * r.x + 2.0f * (S.xy * r.y + S.xz * r.z)) + r.y * (S.yy * r.y + 2.0f * S.yz * r.z) +
           S.zz * (r.z * r.z);
}
// Particle j's symmetric grad v (and p, q in the last two words) as a mirror image: M S M
// with M = diag(1, sy, sz) flips S_xy by sy, S_xz by sz, S_yz by sy sz.
__device__ __forceinline__ SymG load_gsym(const Ptr& P, int j, int mir, float& pj, float& qj) {
    const float4 a = __ldg(P.gsym + 2 * j), b = __ldg(P.gsym + 2 * j + 1);
    pj = b.z;
    qj = b.w;
    SymG S = {a.x, a.y, a.z, a.w, b.x, b.y};
    if (mir) {
        const float sy = (mir & 1) ? -1.0f : 1.0f, sz = (mir & 2) ? -1.0f : 1.0f;
        S.xy *= sy; S.xz *= sz; S.yz *= sy * sz;
    }
    return S;
}
__device__ __forceinline__ SymG own_gsym(const Ptr& P, int i) {
    const float4 a = P.gsym[2 * i], b = P.gsym[2 * i + 1];
    return {a.x, a.y, a.z, a.w, b.x, b.y};
}
struct NoExtra {};
__device__ __forceinline__ void load_gradv(const Ptr& P, int j, float G[3][3]) {
    const float4* g = reinterpret_cast<const float4*>(P.gradv + 12 * j);
    float4 a = __ldg(g), b = __ldg(g + 1), d = __ldg(g + 2);
    G[0][0] = a.x; G[0][1] = a.y; G[0][2] = a.z; G[1][0] = a.w;
    G[1][1] = b.x; G[1][2] = b.y; G[2][0] = b.z; G[2][1] = b.w; G[2][2] = d.x;
}


// ------------------------------------------------------------------ kernel-correction inverse
// The regularised inverse of E at the consumer's tolerance (spd_inverse.py:86-101), formed
// from the lambda pass's E.  Near a free surface (lambda below 0.75) the eigen-problem is
// solved in float64: there the smallest eigenvalues approach the tolerance and decide the
// correction.
__device__ __forceinline__ void store_kc_inverse(const Cst& c, const Ptr& P, int i, const float E[3][3],
                                                 float lam) {
    const float tol = c.p.l_eig_tol;
    float L00, L11, L22, L01, L02, L12;
    if (c.p.two_d) {
        float a = E[0][0], b = 0.5f * (E[0][1] + E[1][0]), dd = E[1][1];
        float disc = sqrtf(fmaxf((a - dd) * (a - dd) + 4.0f * b * b, 0.0f));
        float e1 = 0.5f * (a + dd + disc), e2 = 0.5f * (a + dd - disc);
        float n1x = 1.0f, n1y = 0.0f;
        float scale = fabsf(a) + fabsf(dd) + 1e-30f;
        if (disc > 1e-9f * scale) {
            float v1x = b, v1y = e1 - a, v2x = e1 - dd, v2y = b;
            float l1 = sqrtf(v1x * v1x + v1y * v1y), l2 = sqrtf(v2x * v2x + v2y * v2y);
            if (l1 >= l2) { n1x = v1x / l1; n1y = v1y / l1; } else { n1x = v2x / l2; n1y = v2y / l2; }
        }
        float n2x = -n1y, n2y = n1x;
        float w1 = spd_weight(e1, tol), w2 = spd_weight(e2, tol);
        L00 = w1 * (n1x * n1x) + w2 * (n2x * n2x);
        L01 = w1 * (n1x * n1y) + w2 * (n2x * n2y);
        L11 = w1 * (n1y * n1y) + w2 * (n2y * n2y);
        L22 = 1.0f; L02 = 0.0f; L12 = 0.0f;
    } else if (lam < 0.75f) {
        double A[3][3], ev[3], Q[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) A[a][b] = 0.5 * ((double)E[a][b] + (double)E[b][a]);
        sym_eig3(A, ev, Q);
        double w[3];
        for (int k = 0; k < 3; ++k) w[k] = spd_weight(ev[k], (double)tol);
        double M[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) M[a][b] = w[0] * Q[a][0] * Q[b][0] + w[1] * Q[a][1] * Q[b][1] + w[2] * Q[a][2] * Q[b][2];
        L00 = (float)M[0][0]; L11 = (float)M[1][1]; L22 = (float)M[2][2];
        L01 = (float)M[0][1]; L02 = (float)M[0][2]; L12 = (float)M[1][2];
    } else {
        float A[3][3], ev[3], Q[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) A[a][b] = 0.5f * (E[a][b] + E[b][a]);
        sym_eig3(A, ev, Q);
        float w[3];
        for (int k = 0; k < 3; ++k) w[k] = spd_weight(ev[k], tol);
        L00 = w[0] * Q[0][0] * Q[0][0] + w[1] * Q[0][1] * Q[0][1] + w[2] * Q[0][2] * Q[0][2];
        L11 = w[0] * Q[1][0] * Q[1][0] + w[1] * Q[1][1] * Q[1][1] + w[2] * Q[1][2] * Q[1][2];
        L22 = w[0] * Q[2][0] * Q[2][0] + w[1] * Q[2][1] * Q[2][1] + w[2] * Q[2][2] * Q[2][2];
        L01 = w[0] * Q[0][0] * Q[1][0] + w[1] * Q[0][1] * Q[1][1] + w[2] * Q[0][2] * Q[1][2];
        L02 = w[0] * Q[0][0] * Q[2][0] + w[1] * Q[0][1] * Q[2][1] + w[2] * Q[0][2] * Q[2][2];
        L12 = w[0] * Q[1][0] * Q[2][0] + w[1] * Q[1][1] * Q[2][1] + w[2] * Q[1][2] * Q[2][2];
    }
    P.aux[6 * i + 3] = make_float4(L00, L11, L22, L01);
    float4 b = P.aux[6 * i + 4];
    b.x = L02; b.y = L12;
    P.aux[6 * i + 4] = b;
}

template <int kShape>
__global__ void __launch_bounds__(kBlock) k_kc_inverse(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    F3 xi = f3(pos[i]);
    // E = sum V_j (x_j - x_i) (x) grad W, symmetric (grad W = f r): six entries
    float e00 = 0.f, e11 = 0.f, e22 = 0.f, e01 = 0.f, e02 = 0.f, e12 = 0.f;
    for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
        float4 pj = __ldg(pos + j);
        F3 xj = f3(pj);
        if (mir) xj = mirror3(mir, xj);
        const F3 r = xi - xj;
        const F3 sr = (-(S::w(pj, c) * wendland_dW_factor(dot3(r, r), c))) * r;
        e00 += sr.x * r.x; e01 += sr.x * r.y; e02 += sr.x * r.z;
        e11 += sr.y * r.y; e12 += sr.y * r.z; e22 += sr.z * r.z;
    });
    const float E[3][3] = {{e00, e01, e02}, {e01, e11, e12}, {e02, e12, e22}};
    store_kc_inverse(c, P, i, E, P.lam[i]);
}

// ------------------------------------------------------------------ pass A
template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_SOLID_A) k_solid_a(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double wdiff = 0.0;
    unsigned int mlo = 0xffffffffu, mhi = 0u;   // this particle's mass bits, for the range
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4* __restrict__ shf = as4c(P.cur.shift);
        const float* __restrict__ lam = P.lam;
        float4 pi = pos[i], vi4 = vel[i];
        F3 xi = f3(pi), vi = f3(vi4);
        mlo = mhi = __float_as_uint(vi4.w);
        float4 l0 = P.lsym[2 * i], l1 = P.lsym[2 * i + 1];
        const float L00 = l0.x, L11 = l0.y, L22 = l0.z, L01 = l0.w, L02 = l1.x, L12 = l1.y;
        const float lam_i = lam[i];
        const float rho_i = vi4.w / pi.w, inv_rho_i = 1.0f / rho_i;
        const bool pst = S::pst(c);
        const int ki = eos_of(P, i);
        const float dt = dt_at(c, P, ki), inv_dt = 1.0f / dt;
        const float di = P.mat[ki].delta;
        const float c0i = S::ensemble(c) ? P.irow[ki].c0 : c.p.c0;
        F3 lg = {0, 0, 0};
        float r0 = 0.0f, r1 = 0.0f;
        float G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
            float4 pj = __ldg(pos + j), vj4 = __ldg(vel + j);
            F3 xj = f3(pj), vj = f3(vj4);
            if (mir) { xj = mirror3(mir, xj); vj = mirror3(mir, vj); }
            F3 r = xi - xj;
            float rn2 = dot3(r, r), rn;
            F3 g = wendland_dW2(r, rn2, rn, c);
            float Vj = S::w(pj, c);
            float ld = __ldg(lam + j) - lam_i;
            F3 Lg = {L00 * g.x + L01 * g.y + L02 * g.z, L01 * g.x + L11 * g.y + L12 * g.z,
                     L02 * g.x + L12 * g.y + L22 * g.z};
            lg += (Vj * ld) * Lg;
            F3 dv = vj - vi;
            const F3 vd = Vj * dv;
            G[0][0] += vd.x * g.x; G[0][1] += vd.x * g.y; G[0][2] += vd.x * g.z;
            G[1][0] += vd.y * g.x; G[1][1] += vd.y * g.y; G[1][2] += vd.y * g.z;
            G[2][0] += vd.z * g.x; G[2][1] += vd.z * g.y; G[2][2] += vd.z * g.z;
            float rho_j = vj4.w / pj.w;
            // velocity divergence with the shift's mass flux, its du_i terms cancelled
            // (DSPH.py:1240-1262): V_j [(v_i - v_j) . gW + (rho_j - rho_i) / rho_i du_j . gW]
            float rr = -dot3(dv, g);
            if (pst) {
                float4 s = __ldg(shf + j);
                F3 du_j = {s.x * inv_dt, s.y * inv_dt, s.z * inv_dt};
                if (mir) du_j = mirror3(mir, du_j);
                rr += (rho_j - rho_i) * inv_rho_i * dot3(du_j, g);
            }
            r0 += Vj * rr;
            // pair_delta and pair_c0 (SOLID.py:4102-4114, DSPH.py:483-511) on same-material
            // pairs, or on every pair under Diffusion.pairs "all" (DSPH.py:1271-1282)
            const int kj = S::one(c) ? ki : eos_of(P, j);
            if (kj == ki || S::pairs_all(c)) {
                const float dj = kj == ki ? di : P.mat[kj].delta;
                float den = di + dj;
                float dl = den > 1e-12f ? 2.0f * di * dj / den : 0.0f;
                if (dl > 0.0f) {
                    const float c0p = S::c0_mixed(c) ? 0.5f * (P.mat[ki].c0 + P.mat[kj].c0) : c0i;
                    float psig = __fdividef(2.0f * (rho_j - rho_i) * (-dot3(r, g)), rn2 + c.eta2);
                    float rate = dl * c.h * c0p * Vj * psig * inv_rho_i;
                    r0 += rate;
                    r1 += rate;
                }
            }
        });
        if (S::two_d(c)) lg.z = 0.0f;
        P.lgrad[i] = make_float4(lg.x, lg.y, lg.z, 0.0f);
        float dvg = r0;
        if (S::axi(c)) dvg -= vi.y / r_axi_of(pi.y, c);
        P.div[i] = make_float4(dvg, r1, 0.0f, 0.0f);
        wdiff = -(double)pi.w * (double)__ldg(P.cur.disp + 4 * i + 3) * (double)r1;
        grad_v_finish<NoExtra>(c, P, i, G, pi, vi.y);
    }
    block_sum_atomic(wdiff, &P.ac->w_diff_step);
    // the range of this step's masses (equal bits: every particle has that mass), for the
    // stress pass's sweep
    block_minmax_bits(mlo, mhi, &P.ac->m_min_bits, &P.ac->m_max_bits);
}

// ------------------------------------------------------------------ grad v alone (damper refresh)
template <int kShape>
__global__ void SPH_PAIR_BOUNDS_OCC4 k_gradv(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    const float4* __restrict__ vel = as4c(P.cur.vel);
    float4 pi = pos[i];
    F3 xi = f3(pi), vi = f3(vel[i]);
    float G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
        float4 pj = __ldg(pos + j);
        F3 xj = f3(pj), vj = f3(__ldg(vel + j));
        if (mir) { xj = mirror3(mir, xj); vj = mirror3(mir, vj); }
        F3 r = xi - xj;
        float rn;
        F3 g = wendland_dW2(r, dot3(r, r), rn, c);
        const F3 vd = S::w(pj, c) * (vj - vi);
        G[0][0] += vd.x * g.x; G[0][1] += vd.x * g.y; G[0][2] += vd.x * g.z;
        G[1][0] += vd.y * g.x; G[1][1] += vd.y * g.y; G[1][2] += vd.y * g.z;
        G[2][0] += vd.z * g.x; G[2][1] += vd.z * g.y; G[2][2] += vd.z * g.z;
    });
    grad_v_finish<NoExtra>(c, P, i, G, pi, vi.y);
}

// ------------------------------------------------------------------ return maps
// MAT001_linear_plasticity.py:65-81
__device__ __forceinline__ float j2_return(Sym& s, float G, float sy, float H, float ep) {
    float d = 0.0f;
    if (sy > 0.0f) {
        float vm = vm_sym(s);
        float sigy = sy + H * ep;
        if (vm > sigy && (3.0f * G + H) > 0.0f) {
            d = (vm - sigy) / (3.0f * G + H);
            float sc = (sigy + H * d) / vm;
            s = {s.xx * sc, s.yy * sc, s.zz * sc, s.xy * sc, s.xz * sc, s.yz * sc};
        }
    }
    return d;
}
__device__ __forceinline__ void jc_residual(float d, float vm, float G, float A, float B, float nn,
                                            float C, float e0d, float mt, float ep, float dt,
                                            float& g, float& dg) {
    float et = ep + d;
    float ss = A, ds = 0.0f;
    if (et > 0.0f && B > 0.0f && nn > 0.0f) {
        ss += B * powf(et, nn);
        if (et > 1e-12f) ds = nn * B * powf(et, nn - 1.0f);
    }
    float rate = 1.0f;
    if (dt > 0.0f && e0d > 0.0f) rate = (d / dt) / e0d;
    float mr = 1.0f, dmr = 0.0f;
    if (rate > 1.0f && C > 0.0f) { mr = 1.0f + C * logf(rate); dmr = C / fmaxf(1e-12f, d); }
    float sy = ss * mr * mt;
    float dsy = (ds * mr + ss * dmr) * mt;
    g = vm - 3.0f * G * d - sy;
    dg = -3.0f * G - dsy;
}
// The frozen part of a Johnson-Cook return: von Mises of the trial deviator, the thermal
// softening factor at the step-start temperature, the yield stress at d = 0 and the
// upper bracket d_hi = (vm - sigma_y0) / (3 G) (MAT002_johnson_cook.py:251-300).
struct JcTrial {
    float vm, G, A, B, nn, C, e0d, mt, sy0;
    bool active;                 // material has G, A > 0
    bool yields;                 // vm > sigma_y0 > 0
};
__device__ __forceinline__ JcTrial jc_trial(const Sym& s, const Ptr& P, int k, float ep, float temp) {
    JcTrial q;
    const SphMatRow& M = P.mat[k];
    q.G = M.G; q.A = M.jc_A; q.B = M.jc_B; q.nn = M.jc_n;
    q.C = M.jc_C; q.e0d = M.jc_eps0_dot;
    const float T0 = M.jc_T0, Tm = M.jc_Tm;
    q.active = q.G > 0.0f && q.A > 0.0f;
    q.vm = vm_sym(s);
    q.mt = 1.0f;
    if (Tm > T0 && temp > T0) {
        float ts = fminf(1.0f, fmaxf(0.0f, (temp - T0) / (Tm - T0)));
        q.mt = fmaxf(0.0f, 1.0f - powf(ts, M.jc_m));
    }
    float s0 = q.A;
    if (ep > 0.0f && q.B > 0.0f && q.nn > 0.0f) s0 += q.B * powf(ep, q.nn);
    q.sy0 = s0 * q.mt;
    q.yields = q.active && q.vm > q.sy0 && q.sy0 > 0.0f;
    return q;
}
// MAT002_johnson_cook.py:277-354: bracketed Newton-bisection, at most 40 iterations.
__device__ __forceinline__ float jc_newton(const JcTrial& q, float ep, float dt, int& iters) {
    float lo = 0.0f, hi = (q.vm - q.sy0) / (3.0f * q.G);
    float dref = 0.0f;
    if (dt > 0.0f && q.e0d > 0.0f && q.C > 0.0f) dref = dt * q.e0d;
    if (dref > 0.0f && dref < hi) {
        float g, dg;
        jc_residual(dref, q.vm, q.G, q.A, q.B, q.nn, q.C, q.e0d, q.mt, ep, dt, g, dg);
        if (g > 0.0f) lo = dref; else hi = dref;
    }
    float d = lo > 0.0f ? lo : hi;
    int it = 0;
    for (; it < 40; ++it) {
        float g, dg;
        jc_residual(d, q.vm, q.G, q.A, q.B, q.nn, q.C, q.e0d, q.mt, ep, dt, g, dg);
        if (g > 0.0f) lo = d; else hi = d;
        if (fabsf(g) <= 1e-6f * q.vm || hi - lo <= 1e-6f * hi) break;
        float dn = d - g / dg;
        if (!(dn > lo && dn < hi)) dn = lo > 0.0f ? sqrtf(lo * hi) : 0.5f * hi;
        if (fabsf(dn - d) <= 1e-6f * d) { d = dn; break; }
        d = dn;
    }
    iters = it;
    return d;
}
// Radial scaling of the deviator onto the yield surface after an increment d.
__device__ __forceinline__ void jc_scale(Sym& s, const JcTrial& q, float d) {
    float syf = fmaxf(0.0f, q.vm - 3.0f * q.G * d);
    float sc = syf / q.vm;
    s = {s.xx * sc, s.yy * sc, s.zz * sc, s.xy * sc, s.xz * sc, s.yz * sc};
}
__device__ __forceinline__ float jc_return(Sym& s, const Ptr& P, int k, float ep, float temp, float dt,
                                           bool& capped, int& iters) {
    capped = false;
    iters = 0;
    const JcTrial q = jc_trial(s, P, k, ep, temp);
    if (!q.active || !q.yields) return 0.0f;
    const float d = jc_newton(q, ep, dt, iters);
    capped = iters >= 40;
    jc_scale(s, q, d);
    return d;
}
// Surrogate inputs of a yielding return (features documented in sph_mlp.cuh); eq_rate is
// the equivalent deviatoric strain rate sqrt(2/3 e':e').
__device__ __forceinline__ float4 jc_features(const JcTrial& q, float ep, float dt, float eq_rate) {
    const float d_hi = (q.vm - q.sy0) / (3.0f * q.G);
    const float r0 = q.e0d > 0.0f ? eq_rate / q.e0d : 0.0f;
    const float r1 = (q.e0d > 0.0f && dt > 0.0f) ? d_hi / (dt * q.e0d) : 0.0f;
    return make_float4(0.1f * logf(fmaxf(q.vm / q.sy0 - 1.0f, 1e-8f)), ep, 0.1f * logf(fmaxf(r0, 1.0f)),
                       0.1f * logf(fmaxf(r1, 1.0f)));
}

// ------------------------------------------------------------------ pass B
// Adds a per-thread count, summed over the block, to *dst (one atomic per block).
__device__ __forceinline__ void block_count_add(unsigned v, unsigned long long* dst) {
    __shared__ unsigned s_cnt;
    if (threadIdx.x == 0) s_cnt = 0u;
    __syncthreads();
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_cnt, v);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt && dst) atomicAdd(dst, (unsigned long long)s_cnt);
}

template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_SOLID_B) k_solid_b(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double pw = 0.0, wl = 0.0;
    bool capped_any = false;
    unsigned newton_solves = 0u, newton_iters = 0u;
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4* __restrict__ shf = as4c(P.cur.shift);
        const float* __restrict__ sdev = P.cur.sdev;
        float4 pi = pos[i], vi4 = vel[i], shi = shf[i];
        F3 xi = f3(pi);
        const float rho_i = vi4.w / pi.w, inv_rho_i = 1.0f / rho_i;
        const int ki = eos_of(P, i);
        const float dt = dt_at(c, P, ki), inv_dt = 1.0f / dt;
        const Sym s = load_s(sdev, i);
        const float4 sd1 = __ldg(reinterpret_cast<const float4*>(sdev) + 2 * i + 1);
        float ep = sd1.z;
        const float T_old = sd1.w;
        const float e_i = shi.w;
        const bool ale = S::ale_hist(c);
        const bool plastic_any = S::plastic(c);
        const F3 du_i = {shi.x * inv_dt, shi.y * inv_dt, shi.z * inv_dt};
        Sym A = {0, 0, 0, 0, 0, 0};
        float dep = 0.0f, adv = 0.0f, dif = 0.0f;
        // one mass for every particle (k_solid_a recorded the range): the sweep reads no
        // neighbour's velocity record, whose mass is all it needs
        const unsigned int m_lo = P.ac->m_min_bits;
        const bool m_uni = m_lo == P.ac->m_max_bits;
        const float m_u = __uint_as_float(m_lo);
        auto sweep = [&](auto uni) {
            constexpr bool kUni = decltype(uni)::value;
            for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
                float4 pj = __ldg(pos + j), shj = __ldg(shf + j);
                const float m_j = kUni ? m_u : __ldg(&vel[j].w);
                F3 xj = f3(pj);
                F3 du_j = {shj.x * inv_dt, shj.y * inv_dt, shj.z * inv_dt};
                float epj;
                Sym sj = load_s_ep(sdev, j, epj);
                if (mir) { xj = mirror3(mir, xj); du_j = mirror3(mir, du_j); sj = mirror_sym(mir, sj); }
                F3 r = xi - xj;
                float rn2 = dot3(r, r), rn;
                F3 g = wendland_dW2(r, rn2, rn, c);
                // rho_j only in products and sums here: the rounded quotient (2 ulp) suffices
                const float rho_j = __fdividef(m_j, pj.w);
                float wj = S::w(pj, c);
                // w_j [(rho_j du_j . gW) phi_j - (rho_i du_i . gW) phi_i - phi_i div(rho du)]
                // / rho_i (SOLID.py:1799-1862), whose rho_i du_i parts cancel:
                // w_j rho_j (du_j . gW) (phi_j - phi_i) / rho_i
                const float ka = wj * inv_rho_i * (rho_j * dot3(du_j, g));
                A.xx += ka * (sj.xx - s.xx);
                A.yy += ka * (sj.yy - s.yy);
                A.zz += ka * (sj.zz - s.zz);
                A.xy += ka * (sj.xy - s.xy);
                A.xz += ka * (sj.xz - s.xz);
                A.yz += ka * (sj.yz - s.yz);
                if (plastic_any) dep += ka * (epj - ep);
                if (S::transport_e(c)) {
                    float e_j = shj.w;
                    adv += wj * rho_j * (e_j - e_i) * dot3(du_j, g) * inv_rho_i;
                    if (S::ale_diff(c) && (S::one(c) || same_material(c, P, j, ki))) {
                        float psig = __fdividef(2.0f * (e_j - e_i) * (-dot3(r, g)), rn2 + c.eta2);
                        float rb = 0.5f * (rho_i + rho_j);
                        F3 su = du_i + du_j;
                        float sp = 0.5f * norm3(su);
                        dif += c.p.ale_diffusion * 0.5f * c.p.particle_diameter * sp * wj * psig * rb * inv_rho_i;
                    }
                }
            });
        };
        if (ale) {
            if (m_uni) sweep(std::true_type());
            else sweep(std::false_type());
        }
        // update_stress (SOLID.py:2691-3004): Jaumann rate, trace-free symmetric update
        float Lg[3][3];
        load_gradv(P, i, Lg);
        float ed[3][3], sp[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) { ed[a][b] = 0.5f * (Lg[a][b] + Lg[b][a]); sp[a][b] = 0.5f * (Lg[a][b] - Lg[b][a]); }
        float tr = ed[0][0] + ed[1][1] + ed[2][2];
        float S[3][3] = {{s.xx, s.xy, s.xz}, {s.xy, s.yy, s.yz}, {s.xz, s.yz, s.zz}};
        const SphMatRow& Mi = P.mat[ki];
        const float G2 = 2.0f * Mi.G;
        const bool spin = !c.p.objective_none;
        float Sn[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                float dev = ed[a][b] - ((a == b) ? tr / 3.0f : 0.0f);
                float ws = sp[a][0] * S[0][b] + sp[a][1] * S[1][b] + sp[a][2] * S[2][b];
                float sw = S[a][0] * sp[0][b] + S[a][1] * sp[1][b] + S[a][2] * sp[2][b];
                Sn[a][b] = spin ? G2 * dev + (ws - sw) : G2 * dev;
            }
        Sn[0][0] += A.xx; Sn[1][1] += A.yy; Sn[2][2] += A.zz;
        Sn[0][1] += A.xy; Sn[1][0] += A.xy; Sn[0][2] += A.xz; Sn[2][0] += A.xz; Sn[1][2] += A.yz; Sn[2][1] += A.yz;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) Sn[a][b] = S[a][b] + dt * Sn[a][b];
        Sym sn = {Sn[0][0], Sn[1][1], Sn[2][2], 0.5f * (Sn[0][1] + Sn[1][0]), 0.5f * (Sn[0][2] + Sn[2][0]),
                  0.5f * (Sn[1][2] + Sn[2][1])};
        float tr3 = (sn.xx + sn.yy + sn.zz) / 3.0f;
        sn.xx -= tr3; sn.yy -= tr3; sn.zz -= tr3;
        if (Mi.G <= 0.0f) sn = {0, 0, 0, 0, 0, 0};
        if (ale && plastic_any) ep = fmaxf(0.0f, ep + dt * dep);
        float dprod = 0.0f;
        if (plastic_any) {
            if (Mi.plastic_kind == 2) {
                const bool want_mlp = c.p.jc_surrogate != 0 && P.jc.count != nullptr;
                const bool want_log = P.jc.log != nullptr;
                if (want_mlp || want_log) {
                    const JcTrial q = jc_trial(sn, P, ki, ep, T_old);
                    if (q.yields) {
                        float dd = 0.0f;
#pragma unroll
                        for (int a = 0; a < 3; ++a)
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const float dv = ed[a][b] - ((a == b) ? tr / 3.0f : 0.0f);
                                dd += dv * dv;
                            }
                        const float4 f = jc_features(q, ep, dt, sqrtf((2.0f / 3.0f) * dd));
                        if (want_mlp) {
                            // deferred: k_mlp_tc proposes d, k_jc_finish checks it
                            const int slot = atomicAdd(P.jc.count, 1);
                            P.jc.idx[slot] = i;
                            P.jc.feat[slot] = f;
                        } else {
                            int it;
                            dprod = jc_newton(q, ep, dt, it);
                            capped_any = it >= 40;
                            newton_solves = 1;
                            newton_iters = (unsigned)it;
                            jc_scale(sn, q, dprod);
                            const unsigned long long row = atomicAdd(P.jc.log_count, 1ull);
                            if ((long long)row < P.jc.log_cap) {
                                const float d_hi = (q.vm - q.sy0) / (3.0f * q.G);
                                float4* out = reinterpret_cast<float4*>(P.jc.log + 8 * row);
                                out[0] = f;
                                out[1] = make_float4(dprod / d_hi, d_hi, q.vm, q.sy0);
                            }
                        }
                    }
                } else {
                    bool capped;
                    int it;
                    dprod = jc_return(sn, P, ki, ep, T_old, dt, capped, it);
                    capped_any = capped;
                    newton_solves = dprod > 0.0f ? 1u : 0u;
                    newton_iters = (unsigned)it;
                }
            } else {
                dprod = j2_return(sn, Mi.G, Mi.sy0, Mi.H, ep);
            }
            ep += dprod;
            if (dprod > 0.0f) pw = (double)(pi.w * vm_sym(sn) * dprod);
        }
        // update_internal_energy (SOLID.py:2071-2237): the previous force pass's de_int
        // plus this step's transport; the leftover with the previous acceleration.
        float4 ap = P.cur.acc ? reinterpret_cast<const float4*>(P.cur.acc)[i] : make_float4(0, 0, 0, 0);
        float de = ap.w;
        if (c.p.transport_e) de += adv + dif;
        float e_new = e_i + dt * de;
        {
            const float gx = c.p.gravity[0], gy = c.p.gravity[1], gz = c.p.gravity[2];
            F3 f = {ap.x - gx, ap.y - gy, ap.z - gz};
            wl = (double)(0.5f * vi4.w * dt * dt * (dot3(f, f) - (gx * gx + gy * gy + gz * gz)));
        }
        // update_temperature (SOLID.py:2239-2293) from the new energy and the current V
        float T_new = T_old;
        const float cv = Mi.cv;
        if (cv > 0.0f) {
            double rho = (double)vi4.w / (double)pi.w, rho0 = (double)Mi.rho0;
            double St = (double)Mi.stiff, gam = (double)Mi.gamma;
            double xx = rho / rho0, ec;
            if (fabs(gam - 1.0) < 1.0e-6) ec = (St / rho0) * (log(xx) + 1.0 / xx - 1.0);
            else ec = (St / rho0) * ((pow(xx, gam - 1.0) - 1.0) / (gam - 1.0) + 1.0 / xx - 1.0);
            if (!c.p.allow_negative_pressure && rho < rho0) ec = 0.0;
            double eth = (double)e_new - ec;
            T_new = Mi.T0 + (float)(eth / (double)cv);
        }
        P.aux[6 * i + 0] = make_float4(sn.xx, sn.yy, sn.zz, sn.xy);
        P.aux[6 * i + 1] = make_float4(sn.xz, sn.yz, ep, e_new);
        float4 a2 = P.aux[6 * i + 2];
        a2.x = T_new;
        P.aux[6 * i + 2] = a2;
    }
    if (__syncthreads_or(capped_any) && threadIdx.x == 0) atomicOr(&P.sc->err, SPH_EW_JC_NO_CONVERGE);
    block_sum_atomic(pw, &P.sc->plastic_work);
    block_sum_atomic(wl, &P.sc->leftover_work);
    if (c.any_jc && P.jc.stats) {
        block_count_add(newton_solves, P.jc.stats + 0);
        block_count_add(newton_iters, P.jc.stats + 1);
    }
}

// Completes the returns deferred to the surrogate: the prediction d = f d_hi is kept when
// the Johnson-Cook residual |g(d)| is within jc_surrogate_tol of sigma_y(d); otherwise the
// exact bracketed Newton-bisection runs, as on the plain path.
__global__ void __launch_bounds__(kBlock) k_jc_finish(Cst c, Ptr P) {
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    const int cnt = *P.jc.count;
    double pw = 0.0;
    bool capped = false;
    unsigned solved = 0u, iters = 0u, queued = 0u, accepted = 0u;
    if (qi < cnt) {
        queued = 1u;
        const int i = P.jc.idx[qi];
        const float4 a0 = P.aux[6 * i + 0];
        float4 a1 = P.aux[6 * i + 1];
        Sym sn = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y};
        float ep = a1.z;
        const int k = eos_of(P, i);
        const float T_old = P.cur.sdev[8 * i + 7];
        const float dt = dt_at(c, P, k);
        const JcTrial q = jc_trial(sn, P, k, ep, T_old);
        if (q.yields) {
            const float d_hi = (q.vm - q.sy0) / (3.0f * q.G);
            const float f = 1.0f - 0.1f * P.jc.fpred[qi];    // the network's u = 10 (1 - d / d_hi)
            float d = 0.0f;
            bool ok = false;
            if (f > 0.0f && f <= 1.0f) {              // false for NaN
                d = f * d_hi;
                float g, dg;
                jc_residual(d, q.vm, q.G, q.A, q.B, q.nn, q.C, q.e0d, q.mt, ep, dt, g, dg);
                const float sy = q.vm - 3.0f * q.G * d - g;
                ok = sy > 0.0f && fabsf(g) <= c.p.jc_surrogate_tol * sy;
            }
            if (ok) {
                accepted = 1u;
            } else {
                int it;
                d = jc_newton(q, ep, dt, it);
                capped = it >= 40;
                solved = 1u;
                iters = (unsigned)it;
            }
            jc_scale(sn, q, d);
            ep += d;
            pw = (double)(P.cur.pos[4 * i + 3] * vm_sym(sn) * d);
            P.aux[6 * i + 0] = make_float4(sn.xx, sn.yy, sn.zz, sn.xy);
            a1.x = sn.xz; a1.y = sn.yz; a1.z = ep;
            P.aux[6 * i + 1] = a1;
        }
    }
    if (__syncthreads_or(capped) && threadIdx.x == 0) atomicOr(&P.sc->err, SPH_EW_JC_NO_CONVERGE);
    block_sum_atomic(pw, &P.sc->plastic_work);
    block_count_add(solved, P.jc.stats + 0);
    block_count_add(iters, P.jc.stats + 1);
    block_count_add(queued, P.jc.stats + 2);
    block_count_add(accepted, P.jc.stats + 3);
}

// ------------------------------------------------------------------ commit + volume + EOS
__global__ void __launch_bounds__(kBlock) k_solid_commit(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        // ensembles keep their dt maxima per instance (reset in k_solid_load) and no
        // scene-wide diffusion work
        // the previous step's works, with the dt they were done over (SOLID.py:2182-2207)
        if (c.n_inst == 0) {
            const double dt_prev = (double)P.sc->dt;
            P.sc->diff_work += dt_prev * P.ac->w_diff_step;
            P.sc->hg_work += dt_prev * P.ac->hg_power;
            if (c.p.track_visc_work) P.sc->visc_work += dt_prev * P.ac->visc_power;
        }
        P.ac->w_diff_step = 0.0;
        P.ac->hg_power = 0.0;
        P.ac->visc_power = 0.0;
        P.ac->max_c_sq_bits = __float_as_uint(c.p.c_signal * c.p.c_signal);
        P.ac->max_accel_bits = __float_as_uint(1e-10f);
    }
    if (i >= c.n) return;
    const float dt = dt_at(c, P, eos_of(P, i));
    float4 a0 = P.aux[6 * i + 0], a1 = P.aux[6 * i + 1], a2 = P.aux[6 * i + 2];
    float4* sd = reinterpret_cast<float4*>(P.cur.sdev) + 2 * i;
    sd[0] = a0;
    sd[1] = make_float4(a1.x, a1.y, a1.z, a2.x);
    float4* sh = as4(P.cur.shift) + i;
    float4 s = *sh;
    s.w = a1.w;
    *sh = s;
    float4* pos = as4(P.cur.pos);
    float4 pi = pos[i];
    float V = pi.w;
    float dVdt = -V * P.div[i].x;
    if (c.p.compensated_volume) {
        float* xo = P.cur.x0 + 4 * i + 3;
        double sv = (double)V + (double)(*xo) + (double)(dt * dVdt);
        float hi = (float)sv;
        V = hi;
        *xo = (float)(sv - (double)hi);
    } else {
        V += dt * dVdt;
    }
    pi.w = V;
    pos[i] = pi;
    float m = P.cur.vel[4 * i + 3];
    const int k = eos_of(P, i);
    const float rho = m / V;
    const float p = solid_pressure(c, P, k, rho);
    P.cur.disp[4 * i + 3] = p;
    // the spare words of the symmetric velocity-gradient record carry p (and q) to the
    // neighbours' force pass, which reads that record of every neighbour for the in-loop
    // damper anyway
    P.gradv[12 * i + 9] = p;
    float q_i = 0.0f;
    if (c.p.q_l2 > 0.0f) {
        // SOLID.py:3393-3401 and :3939-3975: q = C_Q l^2 rho (tr grad v)^2 under
        // compression, and the signal speed Q + sqrt(Q^2 + c^2), Q = C_Q l |tr grad v|
        const float4* g = reinterpret_cast<const float4*>(P.gradv + 12 * i);
        const float dv = (g[0].x + g[1].x) + g[2].x;
        float q = 0.0f, ce = 0.0f;
        if (dv < 0.0f) {
            q = c.p.q_l2 * rho * dv * dv;
            const float qc = c.p.q_cl * (-dv), ci = P.mat[k].cp;
            ce = qc + sqrtf(qc * qc + ci * ci);
        }
        reinterpret_cast<float2*>(P.gradv + 12 * i + 10)[0] = make_float2(q, ce);
        q_i = q;
    }
    reinterpret_cast<float2*>(P.gsym + 2 * i + 1)[1] = make_float2(p, q_i);
    // gravity; de_int restarts for this step's force pass
    P.acc[i] = make_float4(c.p.gravity[0], c.p.gravity[1], c.p.gravity[2], 0.0f);
}

// ------------------------------------------------------------------ stress force
// kVisc: a deck with the bulk viscosity q or Monaghan's Pi_ij (SOLID.py:3386-3401,
// :3560-3570, :3727-3766); kAxi: an axisymmetric deck (its pair-radius forms and
// geometric sources).  The plain instances keep the registers of the common case.
template <bool kVisc, bool kAxi, int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_SOLID_FORCE) k_solid_force(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float amag = 0.0f, csq = 0.0f, cvisc = 0.0f;
    double hgp = 0.0, vpw = 0.0;
    int kinst = 0;
    bool on = false;
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4* __restrict__ dsp = as4c(P.cur.disp);
        const float4* __restrict__ shf = as4c(P.cur.shift);
        const float* __restrict__ sdev = P.cur.sdev;
        float4 pi = pos[i], vi4 = vel[i];
        F3 xi = f3(pi), vi = f3(vi4);
        const float p_i = dsp[i].w;
        const bool q_on = kVisc && c.p.q_l2 > 0.0f;
        const bool av_on = kVisc && (c.p.av_alpha > 0.0f || c.p.av_beta > 0.0f);
        float ptot_i = p_i, ce_q = 0.0f;
        if (q_on) {
            const float2 qc = reinterpret_cast<const float2*>(P.gradv + 12 * i + 10)[0];
            ptot_i = p_i + qc.x;
            ce_q = qc.y;
        }
        const float rho_i = vi4.w / pi.w, inv_rho_i = 1.0f / rho_i;
        const float w_i = S::w(pi, c), mw_i = S::mw(vi4.w, pi, c), inv_mw = 1.0f / mw_i;
        const int ki = eos_of(P, i);
        const float dt = dt_at(c, P, ki), inv_dt = 1.0f / dt;
        const Sym s = load_s(sdev, i);
        const bool ale = S::ale_mom(c);
        const bool hg_inloop = S::hg_inloop(c);
        const bool axc = kAxi && c.p.axi_conservative_x;
        const bool axr = kAxi && c.p.axi_conservative_r;
        const float ri = r_axi_of(pi.y, c), inv_ri = 1.0f / ri;
        SymG Si = {0, 0, 0, 0, 0, 0};
        if (hg_inloop) Si = own_gsym(P, i);
        const float hg_pre = c.p.hourglass_alpha * (P.mat[ki].rho0 * inv_rho_i) * (P.mat[ki].cp * c.inv_h)
                             / (c.p.V0 * (float)c.p.hg_W_dx0);
        const float visc = visc_at(c, P, ki);
        kinst = ki;
        on = true;
        const float eps_rho = 1e-3f * c.p.density0;
        const float csig = S::ensemble(c) ? P.irow[ki].c_signal : c.p.c_signal;
        float cl = csig * csig;
        const float c_i = kVisc ? P.mat[ki].cp : 0.0f;
        F3 a = {0, 0, 0};
        float dei = 0.0f, dhg = 0.0f, dvisc = 0.0f, mu_max = 0.0f;
        for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
            float4 pj = __ldg(pos + j), vj4 = __ldg(vel + j);
            F3 xj = f3(pj), vj = f3(vj4);
            if (mir) { xj = mirror3(mir, xj); vj = mirror3(mir, vj); }
            F3 r = xi - xj;
            float rn2 = dot3(r, r), rn;
            F3 g = wendland_dW2(r, rn2, rn, c);
            float w_j = S::w(pj, c);
            const float rj = r_axi_of(pj.y, c);
            // the pair radius over r_i, on the axial (axc) and radial (axr) pair forces
            const float ratio = (axc || axr) ? 0.5f * (ri + rj) * inv_ri : 1.0f;
            F3 vij = vi - vj;
            // the in-loop damper first: j's velocity-gradient record also carries its
            // pressure (k_solid_commit), and is dead once this term is summed
            float p_j, q_j = 0.0f;
            if (hg_inloop) {
                float qq;
                const SymG Sj = load_gsym(P, j, mir, p_j, qq);
                if (q_on) q_j = qq;
                if (rn > 1e-9f) {
                    float inv_rn = rsqrtf(rn2);
                    F3 rh = {-r.x * inv_rn, -r.y * inv_rn, -r.z * inv_rn};
                    // hg = [(v_j - v_i) - <G> (x_j - x_i)] . rhat with x_j - x_i = |r| rhat:
                    // (v_j - v_i) . rhat - |r| rhat^T <S> rhat, <S> the mean symmetric part
                    // (the antisymmetric part of <G> drops out of the quadratic form)
                    const SymG Ss = {Si.xx + Sj.xx, Si.yy + Sj.yy, Si.zz + Sj.zz, Si.xy + Sj.xy,
                                     Si.xz + Sj.xz, Si.yz + Sj.yz};
                    float hg = dot3(vj - vi, rh) - 0.5f * rn * quad_sym(Ss, rh);
                    float damp = hg_pre * w_j * wendland_W(rn, c) * hg;
                    if (S::hg_mixed(c)) damp *= hg_impedance_ratio(P, ki, j);
                    F3 ah = damp * rh;
                    if (axc) ah.x *= ratio;
                    if (axr) ah.y *= ratio;
                    a += ah;
                    dhg += -0.5f * dot3(ah, vij);
                }
            } else if (q_on) {
                const float4 r8 = __ldg(P.gsym + 2 * j + 1);
                p_j = r8.z;
                q_j = r8.w;
            } else {
                p_j = __ldg(&dsp[j].w);
            }
            Sym sj = load_s(sdev, j);
            if (mir) sj = mirror_sym(mir, sj);
            float pp = q_on ? ptot_i + (p_j + q_j) : p_i + p_j;
            Sym ss = {s.xx + sj.xx - pp, s.yy + sj.yy - pp, s.zz + sj.zz - pp, s.xy + sj.xy, s.xz + sj.xz, s.yz + sj.yz};
            float ww = w_i * w_j;
            F3 f = {ww * (ss.xx * g.x + ss.xy * g.y + ss.xz * g.z),
                    ww * (ss.xy * g.x + ss.yy * g.y + ss.yz * g.z),
                    ww * (ss.xz * g.x + ss.yz * g.y + ss.zz * g.z)};
            // axialImageRadius "signed" (and the radial form always): a mirror image's
            // radius is the coordinate it sits at
            if (axc || axr) {
                const float signed_ratio = 0.5f * (ri - rj) * inv_ri;
                if (axc) f.x *= (mir && c.p.axi_image_signed) ? signed_ratio : ratio;
                if (axr) f.y *= mir ? signed_ratio : ratio;
            }
            a += inv_mw * f;
            dei += -0.5f * dot3(f, vij) * inv_mw;
            float vxy = dot3(vij, r);
            F3 am = __fdividef(visc * w_j * vxy, rn * rn + c.eta2) * g;
            a += am;
            // the viscous work conjugates are summed once, as de_visc = -(their part of
            // de_int), and folded into de_int after the loop: one add per pair fewer
            if (S::visc(c)) dvisc += 0.5f * dot3(am, vij);
            // rho_j to within 2 ulp for the products and sums below; the dt pair test, which
            // takes the difference rho_i - rho_j, forms the exact quotient whenever the
            // rounded one is within 1% of its threshold (as the fluid's force pass)
            const float rho_j = __fdividef(vj4.w, pj.w);
            if (av_on && vxy < 0.0f) {
                // Pi_ij = (-alpha cbar mu + beta mu^2) / rhobar on an approaching pair
                const float mu = c.h * vxy / (rn * rn + c.p.av_eps * c.h * c.h);
                const float rho_bar = 0.5f * (rho_i + rho_j);
                const float c_j = c.one_material ? c_i : P.mat[eos_of(P, j)].cp;
                const float c_bar = 0.5f * (c_i + c_j);
                const float pij = (-c.p.av_alpha * c_bar * mu + c.p.av_beta * mu * mu) / rho_bar;
                F3 ap = (-S::mw(vj4.w, pj, c) * pij) * g;
                float mu_cfl = -mu;
                if (axc || axr) {
                    if (axc) ap.x *= ratio;
                    if (axr) ap.y *= ratio;
                    mu_cfl *= ratio;
                }
                a += ap;
                mu_max = fmaxf(mu_max, mu_cfl);
                dvisc += 0.5f * dot3(ap, vij);
            }
            if (ale) {
                // the ALE momentum term with its rho_i du_i parts cancelled (as the fluid's):
                // w_j rho_j (du_j . gW) (v_j - v_i) / rho_i
                float4 q = __ldg(shf + j);
                F3 du_j = {q.x * inv_dt, q.y * inv_dt, q.z * inv_dt};
                if (mir) du_j = mirror3(mir, du_j);
                a += (-(w_j * inv_rho_i) * (rho_j * dot3(du_j, g))) * vij;
            }
            if (S::dt_pairs(c) && fabsf(rho_i - rho_j) > eps_rho * (1.0f - 1e-2f) &&
                (c.p.dt_pair_mode != 2 || S::one(c) || same_material(c, P, j, ki))) {
                const float drho = fabsf(rho_i - vj4.w / pj.w);   // exact, as the reference's test
                if (drho > eps_rho) {
                    // the quotient only where it can beat the running maximum: the product
                    // rounds within 1e-6 of cl drho, so the pre-test never drops a larger one
                    const float dp = fabsf(p_i - p_j);
                    if (dp > cl * drho * (1.0f - 1e-6f)) {
                        float cij = dp / drho;
                        if (cij > cl) cl = cij;
                    }
                }
            }
        });
        if (kAxi) {
            // the geometric sources the pair sums do not generate (SOLID.py:3444-3466)
            const float inv_rho_r = 1.0f / (rho_i * ri);
            F3 ag = {axc ? 0.0f : s.xy * inv_rho_r,
                     axr ? (ptot_i - s.zz) * inv_rho_r : (s.yy - s.zz) * inv_rho_r, 0.0f};
            a += ag;
            if (axr) dei += -dot3(vi, ag);   // the hoop stress power
        }
        dei -= dvisc;
        float4 a0 = P.acc[i];
        F3 an = {a0.x + a.x, a0.y + a.y, a0.z + a.z};
        P.acc[i] = make_float4(an.x, an.y, an.z, dei);
        bool ongrid = !(isnan(pi.x) || isnan(pi.y) || isnan(pi.z));
        if (ongrid) amag = norm3(an);
        if (S::dt_pairs(c)) csq = cl;
        hgp = (double)(mw_i * dhg);
        vpw = (double)vi4.w * (double)dvisc;
        if (kVisc) {
            // SOLID.py:3977-4009: Pi_ij's signal speed where a neighbour approaches
            float ce_av = 0.0f;
            if (mu_max > 0.0f) ce_av = c_i + 1.2f * (c.p.av_alpha * c_i + c.p.av_beta * mu_max);
            cvisc = fmaxf(ce_q, ce_av);
        }
    }
    if (S::ensemble(c)) {
        inst_max_atomic(amag, kinst, on, &SphInstState::max_accel_bits, P.inst);
        inst_max_atomic(csq, kinst, on, &SphInstState::max_c_sq_bits, P.inst);
        return;
    }
    block_max_atomic(amag, &P.ac->max_accel_bits);
    block_max_atomic(csq, &P.ac->max_c_sq_bits);
    if (S::hg_inloop(c)) block_sum_atomic(hgp, &P.ac->hg_power);
    if (kVisc) block_max_atomic(cvisc, &P.ac->visc_c_bits);
    if (c.p.track_visc_work) block_sum_atomic(vpw, &P.ac->visc_power);
}

// ------------------------------------------------------------------ dt, damper cap / stage count
// sts_stage_count (SOLID.py:4510-4539): the smallest stage count whose interval covers
// rate dt -- n forward-Euler sub-steps reach 1.6 n, s RKL1 stages safety (s^2 + s) --
// or the deck's fixed count; *cap is the dt that count carries.
__device__ __forceinline__ int sts_stage_count(const Cst& c, const Ptr& P, double rate, float dt,
                                               double& cap) {
    const double want = rate * (double)dt;
    int s;
    if (!c.p.hg_sts_rkl) {
        s = c.p.hg_sts_fixed > 0 ? c.p.hg_sts_fixed : max(1, (int)ceil(want / 1.6));
        if (s > kStsMaxStages) { s = kStsMaxStages; atomicOr(&P.sc->err, SPH_EW_STS_CAP); }
        cap = s * 1.6 / rate;
    } else {
        const double safety = (double)c.p.hourglass_sts_safety;
        s = 1;
        if (c.p.hg_sts_fixed > 0) s = min(c.p.hg_sts_fixed, kStsMaxStages);
        else
            while ((double)(s * s + s) * safety < want && s < kStsMaxStages) ++s;
        cap = safety * (double)(s * s + s) / rate;
    }
    return s;
}

__global__ void k_solid_dt(Cst c, Ptr P) {
    if (c.n_inst > 0) {
        // per instance: its own CFL dt, damper cap or stage count; grips cleared
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.n_inst; k += gridDim.x * blockDim.x) {
            SphInstState& S = P.inst[k];
            const float mcs = __uint_as_float(S.max_c_sq_bits), ma = __uint_as_float(S.max_accel_bits);
            float dt = fminf(c.cfl_h / sqrtf(mcs), c.p.CFL * sqrtf(c.h / ma));
            const double rate = (double)P.irow[k].hg_rate;
            int s = 0;
            if (c.p.hourglass_alpha > 0.0f && rate > 0.0) {
                if (!c.p.hourglass_sts) {
                    dt = fminf(dt, (float)(1.6 / rate));
                } else {
                    double cap;
                    s = sts_stage_count(c, P, rate, dt, cap);
                    if ((double)dt > cap) dt = (float)cap;
                }
            } else if (c.p.hourglass_alpha > 0.0f && c.p.hourglass_sts) {
                s = 1;
            }
            S.dt = dt;
            S.sts_stages = s;
            if (s > 0) atomicMax(&P.sc->sts_stages, s);
            for (int g = 0; g < 2; ++g)
                for (int d = 0; d < 3; ++d) { S.constraint_force[g][d] = 0.0; S.constraint_disp[g][d] = 0.0; }
        }
        return;
    }
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float mcs = __uint_as_float(P.ac->max_c_sq_bits);
    float ma = __uint_as_float(P.ac->max_accel_bits);
    P.sc->max_c_sq = mcs;
    P.sc->max_accel = ma;
    float dt = fminf(c.cfl_h / sqrtf(mcs), c.p.CFL * sqrtf(c.h / ma));
    if (c.p.q_l2 > 0.0f || c.p.av_alpha > 0.0f || c.p.av_beta > 0.0f) {
        // the two viscosities' own limits (SOLID.py:3939-4009) in one: min over both of
        // CFL h / c is CFL h / (the larger c)
        const float ce = __uint_as_float(P.ac->visc_c_bits);
        P.ac->visc_c_bits = 0u;
        if (ce > 0.0f) dt = fminf(dt, c.cfl_h / ce);
    }
    const bool hg = c.p.hourglass_alpha > 0.0f;
    int s = 0;
    if (!c.p.hourglass_sts) {
        if (hg) dt = fminf(dt, (float)(1.6 / (double)c.p.hg_rate));
    } else if (hg) {
        s = 1;
        if (c.p.hg_rate > 0.0f) {
            double cap;
            s = sts_stage_count(c, P, (double)c.p.hg_rate, dt, cap);
            if ((double)dt > cap) dt = (float)cap;
        }
    }
    P.sc->dt = dt;
    P.sc->sts_stages = s;
    for (int k = 0; k < 8; ++k)
        for (int d = 0; d < 3; ++d) { P.sc->constraint_force[k][d] = 0.0; P.sc->constraint_disp[k][d] = 0.0; }
}

// ------------------------------------------------------------------ sub-cycled damper
// y lives in aux slot 0 (even stages read it) and slot 2 (odd stages read it); v_sync in
// slot 4.zw + 5.x.  The history in slots 0..2 has been committed by then.
__device__ __forceinline__ F3 y_load(const Ptr& P, int i, int buf) {
    return f3(P.aux[6 * i + (buf ? 2 : 0)]);
}
__device__ __forceinline__ void y_store(const Ptr& P, int i, int buf, F3 y) {
    P.aux[6 * i + (buf ? 2 : 0)] = make_float4(y.x, y.y, y.z, 0.0f);
}

__global__ void __launch_bounds__(kBlock) k_half_kick(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0;
    if (i < c.n) {
        const float h = 0.5f * dt_at(c, P, eos_of(P, i));
        float4* vel = as4(P.cur.vel);
        float4 v = vel[i];
        float4 a = P.acc[i];
        v.x += h * a.x; v.y += h * a.y; v.z += h * a.z;
        vel[i] = v;
        float4 b4 = P.aux[6 * i + 4];
        b4.z = v.x; b4.w = v.y;
        P.aux[6 * i + 4] = b4;
        float4 b5 = P.aux[6 * i + 5];
        b5.x = v.z;
        P.aux[6 * i + 5] = b5;
        y_store(P, i, 0, f3(v));
        if (c.p.hg_sts_rkl) y_store(P, i, 1, f3(v));   // RKL: Y_0 = Y_1 = v
        ke = (double)(0.5f * v.w * (v.x * v.x + v.y * v.y + v.z * v.z));
    }
    block_sum_atomic(ke, &P.sc->hg_work);   // + KE before the damper
}

template <int kShape>
__global__ void __launch_bounds__(kBlock) k_hg_stage(Cst c, Ptr P, int stage) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    // the stage count (an ensemble: its largest instance's) -- later stages return at once
    if (stage >= P.sc->sts_stages) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int ki = eos_of(P, i);
    const int s = c.n_inst > 0 ? P.inst[ki].sts_stages : P.sc->sts_stages;
    if (stage >= s) return;
    const int rb = stage & 1, wb = rb ^ 1;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    const float4* __restrict__ vel = as4c(P.cur.vel);
    float4 pi = pos[i];
    F3 xi = f3(pi);
    F3 yi = y_load(P, i, rb);
    const float rho_i = __ldg(&vel[i].w) / pi.w;
    const SymG Si = own_gsym(P, i);
    const bool axc = S::axi(c) && c.p.axi_conservative_x;
    const bool axr = S::axi(c) && c.p.axi_conservative_r;
    const float ri = r_axi_of(pi.y, c), inv_ri = 1.0f / ri;
    const float hg_pre = c.p.hourglass_alpha * (P.mat[ki].rho0 / rho_i) * (P.mat[ki].cp * c.inv_h)
                         / (c.p.V0 * (float)c.p.hg_W_dx0);
    F3 acc = {0, 0, 0};
    for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) {
        float4 pj = __ldg(pos + j);
        F3 xj = f3(pj);
        F3 yj = y_load(P, j, rb);
        float pj_unused, qj_unused;
        const SymG Sj = load_gsym(P, j, mir, pj_unused, qj_unused);
        if (mir) { xj = mirror3(mir, xj); yj = mirror3(mir, yj); }
        F3 r = xi - xj;
        float rn2 = dot3(r, r);
        float rn = rn2 > 0.0f ? rn2 * rsqrtf(rn2) : 0.0f;
        if (!(rn > 1e-9f)) return;
        float inv_rn = 1.0f / rn;
        F3 rh = {-r.x * inv_rn, -r.y * inv_rn, -r.z * inv_rn};
        // as the in-loop damper: (y_j - y_i) . rhat - |r| rhat^T <S> rhat
        const SymG Ss = {Si.xx + Sj.xx, Si.yy + Sj.yy, Si.zz + Sj.zz, Si.xy + Sj.xy, Si.xz + Sj.xz, Si.yz + Sj.yz};
        float hg = dot3(yj - yi, rh) - 0.5f * rn * quad_sym(Ss, rh);
        float damp = hg_pre * S::w(pj, c) * wendland_W(rn, c) * hg;
        if (S::hg_mixed(c)) damp *= hg_impedance_ratio(P, ki, j);
        F3 ah = damp * rh;
        if (axc || axr) {
            const float ratio = 0.5f * (ri + r_axi_of(pj.y, c)) * inv_ri;
            if (axc) ah.x *= ratio;
            if (axr) ah.y *= ratio;
        }
        acc += ah;
    });
    if (!c.p.hg_sts_rkl) {
        const float sub = (float)((double)dt_at(c, P, ki) / (double)s);
        y_store(P, i, wb, yi + sub * acc);
    } else {
        // RKL1 stage j (SOLID.py:4563-4575): Y_j = mu Y_(j-1) + nu Y_(j-2) + mu w1 dt M Y_(j-1),
        // the coefficients in double and then float, as the host passes them there;
        // Y_(j-2) is this particle's own entry of the buffer Y_j replaces
        const int j = stage + 1;
        double mu = 1.0, nu = 0.0;
        if (j > 1) { mu = (2.0 * j - 1.0) / j; nu = (1.0 - j) / j; }
        const double w1 = 2.0 / (double)(s * s + s);
        const float muf = (float)mu, nuf = (float)nu;
        const float mut = (float)(mu * w1 * (double)dt_at(c, P, ki));
        const F3 yo = y_load(P, i, wb);
        y_store(P, i, wb, (muf * yi + nuf * yo) + mut * acc);
    }
}

__global__ void __launch_bounds__(kBlock) k_sts_finish(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0, wl = 0.0;
    float disp = 0.0f;
    if (i < c.n) {
        const int ki = eos_of(P, i);
        const int s = c.n_inst > 0 ? P.inst[ki].sts_stages : P.sc->sts_stages;
        const float dt = dt_at(c, P, ki), h = 0.5f * dt;
        float4* vel = as4(P.cur.vel);
        float4 v = vel[i];
        F3 y = y_load(P, i, s & 1);
        v.x = y.x; v.y = y.y; v.z = y.z;
        ke = -(double)(0.5f * v.w * (v.x * v.x + v.y * v.y + v.z * v.z));   // - KE after
        float4 b4 = P.aux[6 * i + 4], b5 = P.aux[6 * i + 5];
        F3 dvv = {v.x - b4.z, v.y - b4.w, v.z - b5.x};
        float4 a = P.acc[i];
        F3 ha = {h * a.x, h * a.y, h * a.z};
        wl = (double)(v.w * dot3(dvv, ha));
        v.x += ha.x; v.y += ha.y; v.z += ha.z;
        vel[i] = v;
        float4* pos = as4(P.cur.pos);
        float4 p = pos[i];
        if (c.p.displacement_positions) {
            float4* dsp = as4(P.cur.disp);
            float4 u = dsp[i];
            float4 x0 = as4(P.cur.x0)[i];
            u.x += dt * v.x; u.y += dt * v.y; u.z += dt * v.z;
            dsp[i] = u;
            p.x = x0.x + u.x; p.y = x0.y + u.y; p.z = x0.z + u.z;
        } else {
            p.x += dt * v.x; p.y += dt * v.y; p.z += dt * v.z;
        }
        {
            const float4 po = pos[i];
            disp = norm3(F3{p.x - po.x, p.y - po.y, p.z - po.z}) * (1.0f + 1e-5f);
            if (isnan(disp)) disp = INFINITY;
        }
        pos[i] = p;
    }
    block_sum_atomic(ke, &P.sc->hg_work);
    block_sum_atomic(wl, &P.sc->leftover_work);
    block_max_atomic(disp, &P.ac->max_disp_bits);
}

__global__ void __launch_bounds__(kBlock) k_solid_advect(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float disp = 0.0f;
    if (i < c.n) {
    const float dt = dt_at(c, P, eos_of(P, i));
    float4* vel = as4(P.cur.vel);
    float4 v = vel[i];
    float4 a = P.acc[i];
    v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
    vel[i] = v;
    float4* pos = as4(P.cur.pos);
    float4 p = pos[i];
    if (c.p.displacement_positions) {
        float4* dsp = as4(P.cur.disp);
        float4 u = dsp[i];
        float4 x0 = as4(P.cur.x0)[i];
        u.x += dt * v.x; u.y += dt * v.y; u.z += dt * v.z;
        dsp[i] = u;
        p.x = x0.x + u.x; p.y = x0.y + u.y; p.z = x0.z + u.z;
    } else {
        p.x += dt * v.x; p.y += dt * v.y; p.z += dt * v.z;
    }
    {
        const float4 po = pos[i];
        disp = norm3(F3{p.x - po.x, p.y - po.y, p.z - po.z}) * (1.0f + 1e-5f);
        if (isnan(disp)) disp = INFINITY;
    }
    pos[i] = p;
    }
    block_max_atomic(disp, &P.ac->max_disp_bits);
}

// ------------------------------------------------------------------ grips
// The grip force is summed per block in shared memory (FP64) and pushed with one global
// atomic per block, grip and axis: gripped particles are contiguous in the Morton order,
// so a per-particle global atomic would serialise thousands of adds on a few addresses.
// Ensemble form: each gripped particle uses its instance's load factor and adds to its
// instance's grip (bc.y = 0 or 1), one FP64 atomic per warp and distinct grip.
__device__ __forceinline__ void constraints_ensemble(const Cst& c, const Ptr& P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int2 bc = make_int2(0, -1);
    if (i < c.n) bc = reinterpret_cast<const int2*>(P.cur.bc)[i];
    int k = 0, g = 0;
    float gdisp = 0.0f;
    double fd[3] = {0.0, 0.0, 0.0};
    bool rec[3] = {false, false, false};
    if (bc.x != 0) {
        k = eos_of(P, i);
        SphInstState& S = P.inst[k];
        const float s = S.load_s, sd = S.load_sdot;
        const float scale = c.p.axisymmetric ? (float)(2.0 * M_PI) : 1.0f;
        const float4 bd = reinterpret_cast<const float4*>(P.cur.bcdisp)[i];
        float4* pos = as4(P.cur.pos);
        float4* vel = as4(P.cur.vel);
        float4* dsp = as4(P.cur.disp);
        float4 p = pos[i], v = vel[i], u = dsp[i], a = P.acc[i];
        const float4 x0 = as4(P.cur.x0)[i];
        float* pc[3] = {&p.x, &p.y, &p.z};
        float* vc[3] = {&v.x, &v.y, &v.z};
        float* uc[3] = {&u.x, &u.y, &u.z};
        float* ac[3] = {&a.x, &a.y, &a.z};
        const float bdc[3] = {bd.x, bd.y, bd.z};
        const float x0c[3] = {x0.x, x0.y, x0.z};
        const bool record = bc.y == 0 || bc.y == 1;
        g = record ? bc.y : 0;
        const float4 po = p;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!(bc.x & (1 << d))) continue;
            if (record) {
                fd[d] = (double)(scale * v.w * *ac[d]);
                rec[d] = true;
                S.constraint_disp[g][d] = (double)(bdc[d] * s);   // one value per grip
            }
            *uc[d] = bdc[d] * s;
            *pc[d] = x0c[d] + *uc[d];
            *vc[d] = bdc[d] * sd;
            *ac[d] = 0.0f;
        }
        pos[i] = p; vel[i] = v; dsp[i] = u; P.acc[i] = a;
        gdisp = norm3(F3{p.x - po.x, p.y - po.y, p.z - po.z}) * (1.0f + 1e-5f);
        if (isnan(gdisp)) gdisp = INFINITY;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) addr_add_atomic(fd[d], &P.inst[k].constraint_force[g][d], rec[d]);
    const float wm = warp_max(gdisp);
    if ((threadIdx.x & 31) == 0 && wm > 0.0f) atomicMax(&P.ac->max_grip_disp_bits, __float_as_uint(wm));
}

__global__ void __launch_bounds__(kBlock) k_constraints(Cst c, Ptr P) {
    if (c.n_inst > 0) { constraints_ensemble(c, P); return; }
    float gdisp = 0.0f;
    __shared__ double s_force[8][3];
    __shared__ float s_disp[8][3];
    __shared__ int s_axes[8];
    if (threadIdx.x < 24) (&s_force[0][0])[threadIdx.x] = 0.0;
    if (threadIdx.x < 8) s_axes[threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int2 bc = make_int2(0, -1);
    if (i < c.n) bc = reinterpret_cast<const int2*>(P.cur.bc)[i];
    if (bc.x != 0) {
        const float s = P.sc->load_s, sd = P.sc->load_sdot;
        const float scale = c.p.axisymmetric ? (float)(2.0 * M_PI) : 1.0f;
        float4 bd = reinterpret_cast<const float4*>(P.cur.bcdisp)[i];
        float4* pos = as4(P.cur.pos);
        float4* vel = as4(P.cur.vel);
        float4* dsp = as4(P.cur.disp);
        float4 p = pos[i], v = vel[i], u = dsp[i], a = P.acc[i];
        const float4 x0 = as4(P.cur.x0)[i];
        const float m = v.w;
        float* pc[3] = {&p.x, &p.y, &p.z};
        float* vc[3] = {&v.x, &v.y, &v.z};
        float* uc[3] = {&u.x, &u.y, &u.z};
        float* ac[3] = {&a.x, &a.y, &a.z};
        const float bdc[3] = {bd.x, bd.y, bd.z};
        const float x0c[3] = {x0.x, x0.y, x0.z};
        const bool record = c.p.num_constraints > 0 && bc.y >= 0 && bc.y < 8;
        if (record) atomicOr(&s_axes[bc.y], bc.x & 7);
        const float4 po = p;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!(bc.x & (1 << d))) continue;
            if (record) {
                atomicAdd(&s_force[bc.y][d], (double)(scale * m * *ac[d]));
                s_disp[bc.y][d] = bdc[d] * s;     // one value per grip: a benign race
            }
            *uc[d] = bdc[d] * s;
            *pc[d] = x0c[d] + *uc[d];
            *vc[d] = bdc[d] * sd;
            *ac[d] = 0.0f;
        }
        pos[i] = p; vel[i] = v; dsp[i] = u; P.acc[i] = a;
        gdisp = norm3(F3{p.x - po.x, p.y - po.y, p.z - po.z}) * (1.0f + 1e-5f);
        if (isnan(gdisp)) gdisp = INFINITY;
    }
    block_max_atomic(gdisp, &P.ac->max_grip_disp_bits);
    if (threadIdx.x < 24) {
        const int k = threadIdx.x / 3, d = threadIdx.x % 3;
        if (s_axes[k] & (1 << d)) {
            atomicAdd(&P.sc->constraint_force[k][d], s_force[k][d]);
            P.sc->constraint_disp[k][d] = (double)s_disp[k][d];
        }
    }
}

__global__ void k_solid_time(Cst c, Ptr P) {
    if (c.n_inst > 0) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.n_inst; k += gridDim.x * blockDim.x)
            P.inst[k].sim_time += (double)P.inst[k].dt;
        return;
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) P.sc->sim_time += (double)P.sc->dt;
}

// ------------------------------------------------------------------ host sequencing
inline int grid_of(int n, int bs = kBlock) { return n > 0 ? (n + bs - 1) / bs : 1; }
// Launch shape of the per-instance kernels (one thread per instance, or one thread).
inline int inst_blocks(const Cst& c) { return c.n_inst > 0 ? (c.n_inst + 127) / 128 : 1; }
inline int inst_threads(const Cst& c) { return c.n_inst > 0 ? 128 : 32; }

// Launched before the rebuild of a solid step.
inline int solid_pre_step(const Cst& c, const Ptr& P, SolidScratch&, cudaStream_t st) {
    k_solid_load<<<inst_blocks(c), inst_threads(c), 0, st>>>(c, P);
    return SPH_OK;
}

template <class Mark>
inline int solid_substep_launch(const Cst& c, const Ptr& P, int n, cudaStream_t st, Mark&& mark,
                                int first_stage = 0, int last_stage = 99) {
    // the particle kernels take the handle's block size (sph_set_block); the tensor-core
    // and per-instance kernels have their own shapes
    const int bs = c.block > 0 ? c.block : kBlock;
    const int nb = grid_of(n, bs);
    auto in = [&](int s) { return s >= first_stage && s <= last_stage; };
    if (in(SPH_STAGE_LAM)) {
        SHAPED(shape_of(c), k_lam, <<<nb, bs, 0, st>>>(c, P)); mark("k_lam");
        if (c.p.kernel_correction) { SHAPED(shape_of(c), k_kc_inverse, <<<nb, bs, 0, st>>>(c, P)); mark("k_kc_inverse"); }
        SHAPED(shape_of(c), k_solid_a, <<<nb, bs, 0, st>>>(c, P)); mark("k_solid_a");
        SHAPED(shape_of(c), k_solid_b, <<<nb, bs, 0, st>>>(c, P)); mark("k_solid_b");
        if (c.p.jc_surrogate && P.jc.count) {
            const int tiles = (n + kMlpTileRows - 1) / kMlpTileRows;
            const int g = std::min(kMlpCtasPerSm * 148, std::max(tiles, 1));
            k_mlp_tc<<<g, kMlpTcThreads, 0, st>>>(P.jc.W, static_cast<const __nv_bfloat16*>(P.jc.packed),
                                                 P.jc.feat, n, P.jc.count, P.jc.fpred, &P.sc->err);
            mark("k_mlp_tc");
            k_jc_finish<<<grid_of(n), kBlock, 0, st>>>(c, P); mark("k_jc_finish");
        }
    }
    if (in(SPH_STAGE_CONTINUITY)) { k_solid_commit<<<nb, bs, 0, st>>>(c, P); mark("k_solid_commit"); }
    if (in(SPH_STAGE_FORCES)) {
        const bool visc = c.p.q_l2 > 0.0f || c.p.av_alpha > 0.0f || c.p.av_beta > 0.0f;
        if (c.p.axisymmetric) {
            if (visc) k_solid_force<true, true, 0><<<nb, bs, 0, st>>>(c, P);
            else k_solid_force<false, true, 0><<<nb, bs, 0, st>>>(c, P);
        } else if (shape_of(c) == 2) {
            if (visc) k_solid_force<true, false, 2><<<nb, bs, 0, st>>>(c, P);
            else k_solid_force<false, false, 2><<<nb, bs, 0, st>>>(c, P);
        } else if (shape_of(c) == 1) {
            if (visc) k_solid_force<true, false, 1><<<nb, bs, 0, st>>>(c, P);
            else k_solid_force<false, false, 1><<<nb, bs, 0, st>>>(c, P);
        } else if (shape_of(c) == 3) {
            if (visc) k_solid_force<true, false, 3><<<nb, bs, 0, st>>>(c, P);
            else k_solid_force<false, false, 3><<<nb, bs, 0, st>>>(c, P);
        } else {
            if (visc) k_solid_force<true, false, 0><<<nb, bs, 0, st>>>(c, P);
            else k_solid_force<false, false, 0><<<nb, bs, 0, st>>>(c, P);
        }
        mark("k_solid_force");
    }
    if (in(SPH_STAGE_DT)) { k_solid_dt<<<inst_blocks(c), inst_threads(c), 0, st>>>(c, P); mark("k_solid_dt"); }
    if (in(SPH_STAGE_ADVECT)) {
        if (c.p.hourglass_sts && c.p.hourglass_alpha > 0.0f) {
            k_half_kick<<<nb, bs, 0, st>>>(c, P); mark("k_half_kick");
            if (c.p.hg_sts_refresh) { SHAPED(shape_of(c), k_gradv, <<<nb, bs, 0, st>>>(c, P)); mark("k_gradv"); }
            for (int s = 0; s < kStsMaxStages; ++s) {
                // its plain-2D instance measured 2.7% slower than the general one on the
                // strip ensemble (5.91 against 5.75 ms per step over the stages)
                SHAPED(shape_of(c) == 3 ? 0 : shape_of(c), k_hg_stage, <<<nb, bs, 0, st>>>(c, P, s));
                mark("k_hg_stage");
            }
            k_sts_finish<<<nb, bs, 0, st>>>(c, P); mark("k_sts_finish");
        } else {
            k_solid_advect<<<nb, bs, 0, st>>>(c, P); mark("k_solid_advect");
        }
        k_constraints<<<nb, bs, 0, st>>>(c, P); mark("k_constraints");
    }
    if (in(SPH_STAGE_PST) && c.p.pst_enabled) {
        SHAPED(shape_of(c), k_pst, <<<nb, bs, 0, st>>>(c, P)); mark("k_pst");
        k_finish<<<nb, bs, 0, st>>>(c, P, last_stage >= SPH_STAGE_BOUNDARY ? 3 : 1); mark("k_finish");
    } else if (in(SPH_STAGE_BOUNDARY)) {
        k_finish<<<nb, bs, 0, st>>>(c, P, 2); mark("k_finish");
    }
    if (in(SPH_STAGE_BOUNDARY)) { k_solid_time<<<inst_blocks(c), inst_threads(c), 0, st>>>(c, P); mark("k_solid_time"); }
    return SPH_OK;
}

// HypoElasticSolver.compute_elastic_energy (SOLID.py:2296-2322): per particle of a
// material with G > 0, 0.5 K theta^2 V + 0.25 (s:s) V / G with theta = rho / rho0 - 1,
// in float32 as the reference evaluates it, summed in FP64.
__global__ void __launch_bounds__(kBlock) k_solid_elastic(Cst c, Ptr P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < c.n) {
        const int k = eos_of(P, i);
        const int rows = c.n_inst > 0 ? c.n_inst : c.p.n_materials;
        const float G = (k >= 0 && k < rows) ? P.mat[k].G : 0.0f;
        if (G > 0.0f) {
            const float K = P.mat[k].K, rho0 = P.mat[k].rho0;
            const float V = P.cur.pos[4 * i + 3];
            const float rho = P.cur.vel[4 * i + 3] / V;
            const float theta = (rho - rho0) / rho0;
            const float u_vol = 0.5f * K * theta * theta * V;
            const Sym sd = load_s(P.cur.sdev, i);
            const float ss = sd.xx * sd.xx + sd.yy * sd.yy + sd.zz * sd.zz +
                             2.0f * (sd.xy * sd.xy + sd.xz * sd.xz + sd.yz * sd.yz);
            const float u_dev = 0.25f * ss / G * V;
            e = (double)(u_vol + u_dev);
        }
    }
    block_sum_atomic(e, &P.ac->red[SPH_RED_ELASTIC]);
}

inline void solid_reduce_extra(const Cst& c, const Ptr& P, int n, cudaStream_t st) {
    k_solid_elastic<<<grid_of(n), kBlock, 0, st>>>(c, P);
}

}  // namespace sph

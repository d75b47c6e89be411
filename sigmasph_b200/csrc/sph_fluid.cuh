// sph_fluid.cuh -- the delta+-SPH step (DSPH.py DSPHSolver.substep, :1854-1883) as
// fused sm_100a kernels over the neighbour lists.
//
//   k_lam            compute_lam first pass: E, lambda, regularised L   (DSPH.py:611-681)
//   k_lamgrad_cont   compute_lam second pass + the continuity pair sum  (:683-702, :1208-1338)
//   k_eos            volume update, Tait pressure, gravity               (:1476-1521, :1642-1650)
//   k_force          pressure + Morris viscosity + ALE momentum, and the pair sound-speed
//                    and acceleration maxima of compute_adaptive_dt      (:1523-1640, :1340-1430)
//   k_dt             the two CFL limits                                  (:1416-1430)
//   k_advect         accumulate_step_work + advect                       (:1652-1763)
//   k_pst            apply_pst first pass: live-position search against the stale bins
//   k_finish         apply_pst second pass (displace) + SPHBase.step's constraints and walls
//
// Fusions relative to the reference: the grad-lambda sum and the continuity sum read the
// same start-of-step state and share one neighbour sweep; the dt pair estimate reads the
// post-EOS pressure the force pass reads and shares its sweep; the step-work reduction is
// folded into advect; the displacement of the shift is folded into the boundary pass.
#pragma once
#include <type_traits>

#include "sph_grid.cuh"

namespace sph {

__device__ __forceinline__ float4* as4(float* p) { return reinterpret_cast<float4*>(p); }
__device__ __forceinline__ const float4* as4c(const float* p) { return reinterpret_cast<const float4*>(p); }

// ------------------------------------------------------------------ compute_lam pass 1
template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_LAM) k_lam(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    float4 pi = pos[i];
    F3 xi = f3(pi);
    // E = sum V_j (x_j - x_i) (x) grad W (DSPH.py:611-681).  grad W = f r with r = x_i - x_j,
    // so each pair adds -V_j f r (x) r: a symmetric matrix, accumulated as its six entries
    float e00 = 0.f, e11 = 0.f, e22 = 0.f, e01 = 0.f, e02 = 0.f, e12 = 0.f;
    auto pair = [&](int mir, float4 pj) {
        F3 xj = f3(pj);
        if (mir) xj = mirror3(mir, xj);
        const F3 r = xi - xj;
        const float f = wendland_dW_factor(dot3(r, r), c);
        const F3 sr = (-(S::w(pj, c) * f)) * r;
        e00 += sr.x * r.x; e01 += sr.x * r.y; e11 += sr.y * r.y;
        if (!S::two_d(c)) { e02 += sr.x * r.z; e12 += sr.y * r.z; e22 += sr.z * r.z; }
    };
    for_each_neighbour<kPlain>(c, P, i, [&](int j, int mir) { pair(mir, __ldg(pos + j)); });
    const float E[3][3] = {{e00, e01, e02}, {e01, e11, e12}, {e02, e12, e22}};
    const float tol = c.p.l_eig_tol_lam;
    float L00, L11, L22, L01, L02, L12, lam;
    float4 evec = make_float4(0.f, 0.f, 0.f, 0.f);
    if (S::two_d(c)) {
        // eig_sym_2x2 (DSPH.py:35-47) on (E00, E01, E11) and spd_inverse_2x2 (spd_inverse.py:53-83)
        float a = E[0][0], b0 = E[0][1], dd = E[1][1];
        float det = sqrtf((a - dd) * (a - dd) + 4.0f * b0 * b0);
        lam = fminf(1.0f, fmaxf(0.0f, 0.5f * (a + dd - det)));
        float b = 0.5f * (E[0][1] + E[1][0]);
        float disc = sqrtf(fmaxf((a - dd) * (a - dd) + 4.0f * b * b, 0.0f));
        float e1 = 0.5f * (a + dd + disc), e2 = 0.5f * (a + dd - disc);
        float n1x = 1.0f, n1y = 0.0f;
        float scale = fabsf(a) + fabsf(dd) + 1e-30f;
        if (disc > 1e-9f * scale) {
            float v1x = b, v1y = e1 - a, v2x = e1 - dd, v2y = b;
            float l1 = sqrtf(v1x * v1x + v1y * v1y), l2 = sqrtf(v2x * v2x + v2y * v2y);
            if (l1 >= l2) { n1x = v1x / l1; n1y = v1y / l1; }
            else { n1x = v2x / l2; n1y = v2y / l2; }
        }
        float n2x = -n1y, n2y = n1x;
        float w1 = spd_weight(e1, tol), w2 = spd_weight(e2, tol);
        L00 = w1 * (n1x * n1x) + w2 * (n2x * n2x);
        L01 = w1 * (n1x * n1y) + w2 * (n2x * n2y);
        L11 = w1 * (n1y * n1y) + w2 * (n2y * n2y);
        L22 = 1.0f; L02 = 0.0f; L12 = 0.0f;
        evec = make_float4(n2x, n2y, 0.0f, 0.0f);
    } else {
        float A[3][3], ev[3], Q[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) A[a][b] = 0.5f * (E[a][b] + E[b][a]);
        sym_eig3(A, ev, Q);
        float mine = fminf(ev[0], fminf(ev[1], ev[2]));
        lam = fminf(1.0f, fmaxf(0.0f, mine));
        float w0 = spd_weight(ev[0], tol), w1 = spd_weight(ev[1], tol), w2 = spd_weight(ev[2], tol);
        L00 = w0 * (Q[0][0] * Q[0][0]) + w1 * (Q[0][1] * Q[0][1]) + w2 * (Q[0][2] * Q[0][2]);
        L11 = w0 * (Q[1][0] * Q[1][0]) + w1 * (Q[1][1] * Q[1][1]) + w2 * (Q[1][2] * Q[1][2]);
        L22 = w0 * (Q[2][0] * Q[2][0]) + w1 * (Q[2][1] * Q[2][1]) + w2 * (Q[2][2] * Q[2][2]);
        L01 = w0 * (Q[0][0] * Q[1][0]) + w1 * (Q[0][1] * Q[1][1]) + w2 * (Q[0][2] * Q[1][2]);
        L02 = w0 * (Q[0][0] * Q[2][0]) + w1 * (Q[0][1] * Q[2][1]) + w2 * (Q[0][2] * Q[2][2]);
        L12 = w0 * (Q[1][0] * Q[2][0]) + w1 * (Q[1][1] * Q[2][1]) + w2 * (Q[1][2] * Q[2][2]);
        int km = 0;
        if (ev[1] < ev[km]) km = 1;
        if (ev[2] < ev[km]) km = 2;
        evec = make_float4(Q[0][km], Q[1][km], Q[2][km], 0.0f);
    }
    P.lam[i] = lam;
    // a fluid's shift.w is free: it carries lambda to the neighbours' gradient pass, which
    // reads the shift record of every neighbour anyway (then k_eos puts p there)
    if (!c.p.is_solid) P.cur.shift[4 * i + 3] = lam;
    P.lsym[2 * i] = make_float4(L00, L11, L22, L01);
    P.lsym[2 * i + 1] = make_float4(L02, L12, 0.0f, 0.0f);
    if (c.p.pst_normal_eigvec) P.lgrad[i] = evec;
}

// ------------------------------------------------------------------ grad lambda + continuity
template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_LAMGRAD) k_lamgrad_cont(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double wdiff = 0.0;
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4* __restrict__ shf = as4c(P.cur.shift);
        const float* __restrict__ lam = P.lam;
        float4 pi = pos[i], vi4 = vel[i];
        F3 xi = f3(pi), vi = f3(vi4);
        float4 l0 = P.lsym[2 * i], l1 = P.lsym[2 * i + 1];
        const float L00 = l0.x, L11 = l0.y, L22 = l0.z, L01 = l0.w, L02 = l1.x, L12 = l1.y;
        const float lam_i = lam[i];
        const float rho_i = vi4.w / pi.w;
        const float inv_rho_i = 1.0f / rho_i;
        const float dt = P.sc->dt;
        const float inv_dt = 1.0f / dt;
        const bool pst = S::pst(c);
        const bool need_lgrad = S::lgrad(c);
        F3 lg = {0, 0, 0};
        float r0 = 0.0f, r1 = 0.0f;
        // the next neighbour's position is requested while this pair is evaluated
        for_each_neighbour_pos<kPlain>(c, P, i, pos, [&](int j, int mir, float4 pj) {
            float4 vj4 = __ldg(vel + j);
            F3 xj = f3(pj), vj = f3(vj4);
            if (mir) { xj = mirror3(mir, xj); vj = mirror3(mir, vj); }
            F3 r = xi - xj;
            float rn2 = dot3(r, r);
            float rn;
            F3 g = wendland_dW2(r, rn2, rn, c);
            float Vj = S::w(pj, c);
            const float4 sj = pst ? __ldg(shf + j) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (need_lgrad) {
                float ld = (pst ? sj.w : __ldg(lam + j)) - lam_i;
                F3 Lg = {L00 * g.x + L01 * g.y + L02 * g.z,
                         L01 * g.x + L11 * g.y + L12 * g.z,
                         L02 * g.x + L12 * g.y + L22 * g.z};
                lg += (Vj * ld) * Lg;
            }
            float rho_j = vj4.w / pj.w;   // exact: rho_j - rho_i is a small difference
            // the velocity divergence with the shift's mass flux (DSPH.py:1240-1262):
            // V_j [(rho_j du_j - rho_i du_i) . gW / rho_i + (v_i + du_i - v_j - du_j) . gW],
            // whose du_i terms cancel: V_j [(v_i - v_j) . gW + (rho_j - rho_i) / rho_i du_j . gW]
            float rr = dot3(vi - vj, g);
            if (pst) {
                F3 du_j = {sj.x * inv_dt, sj.y * inv_dt, sj.z * inv_dt};
                if (mir) du_j = mirror3(mir, du_j);
                rr += (rho_j - rho_i) * inv_rho_i * dot3(du_j, g);
            }
            r0 += Vj * rr;
            if (S::delta(c)) {
                // psi . grad W = 2 (rho_j - rho_i) (-r . grad W) / (|r|^2 + eta^2)
                float psig = __fdividef(2.0f * (rho_j - rho_i) * (-dot3(r, g)), rn2 + c.eta2);
                float rate = c.delta_coef * Vj * psig * inv_rho_i;
                r0 += rate;
                r1 += rate;
            }
        });
        if (need_lgrad) {
            if (S::two_d(c)) lg.z = 0.0f;
            P.lgrad[i] = make_float4(lg.x, lg.y, lg.z, 0.0f);
        }
        float dv = r0;
        if (S::axi(c)) dv -= vi.y / fmaxf(pi.y, c.p.axi_r_min);
        P.div[i] = make_float4(dv, r1, 0.0f, 0.0f);
        wdiff = -(double)pi.w * (double)__ldg(P.cur.disp + 4 * i + 3) * (double)r1;
    }
    block_sum_atomic(wdiff, &P.ac->w_diff_step);
}

// ------------------------------------------------------------------ volume update + EOS + gravity
__device__ __forceinline__ float tait_p(float rho, const Cst& c) {
    float p = c.p.stiffness * (powf(rho / c.p.density0, c.p.exponent) - 1.0f);
    if (!c.p.allow_negative_pressure) p = fmaxf(p, 0.0f);
    return p;
}

__global__ void __launch_bounds__(kBlock) k_eos(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float dt = P.sc->dt;
    if (i == 0) {
        // end of compute_volume_evolution: diff_work += dt * w_diff_step (DSPH.py:1495)
        P.sc->diff_work += (double)dt * P.ac->w_diff_step;
        P.ac->w_diff_step = 0.0;
        P.ac->max_c_sq_bits = __float_as_uint(c.p.c_signal * c.p.c_signal);
        P.ac->max_accel_bits = __float_as_uint(1e-10f);
    }
    if (i >= c.n) return;
    float4* pos = as4(P.cur.pos);
    float4 pi = pos[i];
    float V = pi.w;
    float dVdt = -V * P.div[i].x;
    if (c.p.compensated_volume) {
        float* xo = P.cur.x0 + 4 * i + 3;
        double s = (double)V + (double)(*xo) + (double)(dt * dVdt);
        float hi = (float)s;
        V = hi;
        *xo = (float)(s - (double)hi);
    } else {
        V += dt * dVdt;
    }
    pi.w = V;
    pos[i] = pi;
    float m = P.cur.vel[4 * i + 3];
    const float p = tait_p(m / V, c);
    P.cur.disp[4 * i + 3] = p;
    P.cur.shift[4 * i + 3] = p;   // for the neighbours' force pass (see k_lam)
    P.acc[i] = make_float4(c.p.gravity[0], c.p.gravity[1], c.p.gravity[2], 0.0f);
}

// ------------------------------------------------------------------ pressure + viscosity + dt pairs
template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_FORCE) k_force(Cst c, Ptr P) {
    using S = Shape<kShape>;
    constexpr bool kPlain = S::kPlain;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float amag = 0.0f, csq = 0.0f;
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4* __restrict__ dsp = as4c(P.cur.disp);
        const float4* __restrict__ shf = as4c(P.cur.shift);
        float4 pi = pos[i], vi4 = vel[i];
        F3 xi = f3(pi), vi = f3(vi4);
        const float p_i = dsp[i].w;
        const float rho_i = vi4.w / pi.w;
        const float w_i = S::w(pi, c);
        const float mw_i = S::mw(vi4.w, pi, c);
        const float dt = P.sc->dt;
        const bool ale = S::ale_mom(c);
        const float eps_rho = 1e-3f * c.p.density0;
        const float inv_mw_i = 1.0f / mw_i, inv_rho_i = 1.0f / rho_i, inv_dt = 1.0f / dt;
        const float inv_rho_dt = inv_rho_i * inv_dt;
        const float wi_mw = w_i * inv_mw_i;
        float cl = c.p.c_signal * c.p.c_signal;
        F3 a = {0, 0, 0};
        float dvisc = 0.0f;
        for_each_neighbour_pos<kPlain>(c, P, i, pos, [&](int j, int mir, float4 pj) {
            float4 vj4 = __ldg(vel + j);
            const float4 sj = ale ? __ldg(shf + j) : make_float4(0.f, 0.f, 0.f, 0.f);
            float p_j = ale ? sj.w : __ldg(&dsp[j].w);   // k_eos copies p to shift.w
            F3 xj = f3(pj), vj = f3(vj4);
            if (mir) { xj = mirror3(mir, xj); vj = mirror3(mir, vj); }
            F3 r = xi - xj;
            float rn;
            const float rn2 = dot3(r, r);
            F3 g = wendland_dW2(r, rn2, rn, c);
            float w_j = S::w(pj, c);
            // -w_i w_j (p_i + p_j) grad W / mw_i
            a += (-wi_mw * w_j * (p_i + p_j)) * g;
            const F3 vij = vi - vj;
            float vxy = dot3(vij, r);
            F3 fv = __fdividef(c.visc_coef * w_j * vxy, rn2 + c.eta2) * g;
            a += fv;
            dvisc += dot3(vi, fv);
            // rho_j to within 2 ulp: enough for the ALE term; the dt pair test, which takes
            // the difference rho_i - rho_j, forms the exact quotient whenever the rounded one
            // is within 1% of its threshold (2 ulp of rho_j is 2.4e-7 rho_j << 1e-2 eps_rho)
            const float rho_j = __fdividef(vj4.w, pj.w);
            if (ale) {
                // the ALE momentum term w_j [div(rho v du) - v_i div(rho du)] / rho_i
                // (DSPH.py:1630-1640), whose rho_i du_i parts cancel:
                // w_j rho_j (du_j . gW) (v_j - v_i) / rho_i; with w_j = V_j (plain decks)
                // w_j rho_j is the mass m_j, and du_j = shift_j / dt
                if (kPlain) {
                    a += (-(vj4.w * inv_rho_dt) * dot3(f3(sj), g)) * vij;
                } else {
                    F3 du_j = {sj.x * inv_dt, sj.y * inv_dt, sj.z * inv_dt};
                    if (mir) du_j = mirror3(mir, du_j);
                    a += (-(w_j * inv_rho_i) * (rho_j * dot3(du_j, g))) * vij;
                }
            }
            if (S::dt_pairs(c) && fabsf(rho_i - rho_j) > eps_rho * (1.0f - 1e-2f)) {
                float drho = fabsf(rho_i - vj4.w / pj.w);   // exact, as the reference's test
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
        float4 a0 = P.acc[i];
        F3 an = {a0.x + a.x, a0.y + a.y, a0.z + a.z};
        P.acc[i] = make_float4(an.x, an.y, an.z, c.p.track_visc_work ? dvisc : 0.0f);
        bool ongrid = !(isnan(pi.x) || isnan(pi.y) || isnan(pi.z));
        if (ongrid) amag = norm3(an);
        if (S::dt_pairs(c)) csq = cl;
    }
    block_max_atomic(amag, &P.ac->max_accel_bits);
    block_max_atomic(csq, &P.ac->max_c_sq_bits);
}

// ------------------------------------------------------------------ compute_adaptive_dt tail
__global__ void k_dt(Cst c, Ptr P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float mcs = __uint_as_float(P.ac->max_c_sq_bits);
    float ma = __uint_as_float(P.ac->max_accel_bits);
    P.sc->max_c_sq = mcs;
    P.sc->max_accel = ma;
    float cmax = sqrtf(mcs);
    float dta = c.cfl_h / cmax;
    float dtf = c.p.CFL * sqrtf(c.h / ma);
    P.sc->dt = fminf(dta, dtf);
    P.ac->max_v_bits = 0u;
}

// ------------------------------------------------------------------ step work + advect
__global__ void __launch_bounds__(kBlock) k_advect(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float dt = P.sc->dt;
    double wl = 0.0, wv = 0.0;
    float vmag = 0.0f, disp = 0.0f;
    unsigned int mlo = 0xffffffffu, mhi = 0u;
    if (i < c.n) {
        float4 a4 = P.acc[i];
        float4* vel = as4(P.cur.vel);
        float4 v4 = vel[i];
        mlo = mhi = __float_as_uint(v4.w);
        const float gx = c.p.gravity[0], gy = c.p.gravity[1], gz = c.p.gravity[2];
        float gsq = gx * gx + gy * gy + gz * gz;
        F3 f = {a4.x - gx, a4.y - gy, a4.z - gz};
        wl = (double)(0.5f * v4.w * dt * dt * (dot3(f, f) - gsq));
        if (c.p.track_visc_work) wv = (double)v4.w * (double)a4.w;
        v4.x += dt * a4.x; v4.y += dt * a4.y; v4.z += dt * a4.z;
        vel[i] = v4;
        float4* pos = as4(P.cur.pos);
        float4 p = pos[i];
        if (c.p.displacement_positions) {
            float4* dsp = as4(P.cur.disp);
            float4 u = dsp[i];
            float4 x0 = as4(P.cur.x0)[i];
            u.x += dt * v4.x; u.y += dt * v4.y; u.z += dt * v4.z;
            dsp[i] = u;
            p.x = x0.x + u.x; p.y = x0.y + u.y; p.z = x0.z + u.z;
        } else {
            p.x += dt * v4.x; p.y += dt * v4.y; p.z += dt * v4.z;
        }
        {
            // how far this particle moved, rounded up (a NaN counts as infinitely far)
            const float4 po = pos[i];
            const F3 d = {p.x - po.x, p.y - po.y, p.z - po.z};
            disp = norm3(d) * (1.0f + 1e-5f);
            if (isnan(disp)) disp = INFINITY;
        }
        pos[i] = p;
        if (c.p.pst_enabled && c.p.pst_ma_mode == 1 && !(isnan(p.x) || isnan(p.y) || isnan(p.z)))
            vmag = sqrtf(v4.x * v4.x + v4.y * v4.y + v4.z * v4.z);
    }
    __shared__ double sh[2][32];
    wl = warp_sum(wl);
    wv = warp_sum(wv);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = wl; sh[1][wid] = wv; }
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        double a = lane < nw ? sh[0][lane] : 0.0, b = lane < nw ? sh[1][lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (lane == 0) {
            atomicAdd(&P.sc->leftover_work, a);
            if (c.p.track_visc_work) atomicAdd(&P.sc->visc_work, (double)dt * b);
        }
    }
    if (c.p.pst_enabled && c.p.pst_ma_mode == 1) block_max_atomic(vmag, &P.ac->max_v_bits);
    block_max_atomic(disp, &P.ac->max_disp_bits);
    // the Sun shift weighs each neighbour by its mass: one mass for all spares that gather
    if (c.p.pst_enabled && !c.p.pst_colle) block_minmax_bits(mlo, mhi, &P.ac->m_min_bits, &P.ac->m_max_bits);
}

// ------------------------------------------------------------------ apply_pst (DSPH.py:725-1046)
// Pairs of the shift: the reference's sweep from the live positions after advect against
// the bins of this step's start (particle_system.py:1377-1411).  While the particles'
// displacement since the lists' build -- at the step's start plus this step's advect and
// grips -- is within the bound, from the candidate lists: every entry tested for
// distance at the live positions, the edge entries also for j's step-start cell (fcell,
// written by k_cells) against i's live cell.  Of the
// edge candidates, only those accepted at the step's start and the near ones need
// reading when the step moved particles less than half the near margin.  Otherwise
// (or when the candidate list overflowed) the stale-bin search.  f(j, mirror, pos_j).
template <bool kPlain, class F>
__device__ __forceinline__ void for_each_pst_neighbour(const Cst& c, const Ptr& P, int i, F3 xi, F&& f) {
    using S = Shape<kPlain ? 1 : 0>;
    if (isnan(xi.x) || isnan(xi.y) || isnan(xi.z)) return;
    const float dtot = __uint_as_float(P.ac->d_start_bits) + __uint_as_float(P.ac->max_disp_bits) +
                       __uint_as_float(P.ac->max_grip_disp_bits);
    const int lx = cell_of(xi.x, c.h), ly = cell_of(xi.y, c.h), lz = cell_of(xi.z, c.h);
    const int vc = __ldg(P.vl_cnt + i);
    if (!(dtot <= c.dlim) || vl_overflow(c, vc)) {
        stale_search(c, P, i, xi, lx, ly, lz, dtot, [&](int j, int mir, float4 pj) {
            F3 xj = f3(pj);
            if (mir) xj = mirror3(mir, xj);
            f(j, mir, pj, xj, dist2_rn(xi, xj));
        });
        return;
    }
    const float4* __restrict__ pos = as4c(P.cur.pos);
    const bool py = xi.y < c.h, pz = xi.z < c.h;
    const int d = vl_deep(vc);
    const size_t n = (size_t)c.n;
    // Near path, when this step moved no particle more than M / 2 since the filter: the
    // step's neighbour list (deep rows, then the edge entries accepted at the start) and
    // the near list.  Otherwise the deep rows and every edge candidate.
    const float step_move = __uint_as_float(P.ac->max_disp_bits) + __uint_as_float(P.ac->max_grip_disp_bits);
    const bool near = P.ac->near_m_bits != 0u && 2.0f * step_move <= __uint_as_float(P.ac->near_m_bits);
    // near path: neighbour-list rows 0 .. cnt-1, then its near rows K - nn .. K - 1; full
    // path: rows 0 .. d-1, then the candidate list's edge rows
    const int a_end = near ? __ldg(P.nbr_cnt + i) : d;
    const int b_cnt = near ? __ldg(P.nl_cnt + i) : vl_edge(vc);
    const int* __restrict__ la = P.nbr + i;
    const int* __restrict__ lb = near ? P.nbr + (size_t)(c.K - b_cnt) * n + i : P.vl + i;
    split_entries(a_end + b_cnt, [&](int k) { return k < a_end ? __ldg(la + (size_t)k * n) : __ldg(lb + (size_t)(k - a_end) * n); },
                  [&](int k, int e) {
        const int j = S::idx(e), mir = S::mir(e);
        if (mir && (((mir & 1) && !py) || ((mir & 2) && !pz))) return;
        const float4 pj = __ldg(pos + j);
        F3 xj = f3(pj);
        if (mir) xj = mirror3(mir, xj);
        const float d2 = dist2_rn(xi, xj);
        if (!(d2 < c.d2_lt)) return;
        if (k >= d) {
            // j's cell of size h at this step's start (k_cells)
            const int4 fj = __ldg(P.fcell + j);
            if (!sweep_cell_ok(mir, fj.x, fj.y, fj.z, lx, ly, lz)) return;
        }
        f(j, mir, pj, xj, d2);
    });
}

// The disorder sum's pair term from the shift pass's own test: the mirrored position xj and
// the squared separation d2 the neighbour test formed.  Arithmetic of pst_pair_term below.
// kForm 1 (Sun) and 2 (Colle) fix the deck's exponent n = 4 with W(dx0) > 0 when the pass
// is compiled, 3 is Sun's with every particle of mass m_u; kForm 0 reads the form, n and
// W(dx0) from the parameters.
constexpr int kPstAny = 0, kPstSun4 = 1, kPstColle4 = 2, kPstSun4Uni = 3;
template <bool kPlain, int kForm>
__device__ __forceinline__ F3 pst_term_d2(const Cst& c, const float4* __restrict__ vel, F3 xi, float rho_i,
                                          float inv_Wd, int j, float4 pj, F3 xj, float d2, bool m_uni,
                                          float m_u) {
    const F3 r = xi - xj;
    float Wij;
    const F3 g = wendland_W_dW2(r, d2, Wij, c);
    float f = 0.0f;
    if (kForm != kPstAny) {
        const float x = Wij * inv_Wd;
        f = c.p.pst_R * (((x * x) * x) * x);   // ipow_or_pow(x, 4)
    } else if (c.W_dx0 > 1e-10f) {
        f = c.p.pst_R * ipow_or_pow(Wij * inv_Wd, c.p.pst_n);
    }
    if (kForm == kPstColle4 || (kForm == kPstAny && c.p.pst_colle)) {
        const float Vj = Shape<kPlain ? 1 : 0>::w(pj, c);
        if (Vj > 1e-30f) return ((1.0f + f) * Vj) * g;
    } else {
        const float mj_raw = (kForm == kPstSun4Uni || m_uni) ? m_u : __ldg(&vel[j].w);
        const float mj = Shape<kPlain ? 1 : 0>::mw(mj_raw, pj, c);
        if (mj > 1e-10f) {
            // m_j / mean rho: a sum of densities, rounded quotients suffice (no cancellation)
            const float rho_j = __fdividef(mj_raw, pj.w);
            const float ra = 0.5f * (rho_i + rho_j);
            if (ra > 1e-10f) return ((1.0f + f) * __fdividef(mj, ra)) * g;
        }
    }
    return {0.0f, 0.0f, 0.0f};
}

// The disorder sum's pair term (pst_pair, DSPH.py:725-769): (1 + R (W / W(dx0))^n) grad W,
// weighted by V_j (Colle) or m_j / mean rho (Sun).
// m_uni: every particle's mass is m_u (the neighbour's is not gathered).
__device__ __forceinline__ F3 pst_pair_term(const Cst& c, const float4* __restrict__ vel, F3 xi,
                                            float rho_i, float inv_Wd, int j, int mir, float4 pj,
                                            bool m_uni = false, float m_u = 0.0f) {
    F3 xj = f3(pj);
    if (mir) xj = mirror3(mir, xj);
    F3 r = xi - xj;
    float Wij;
    F3 g = wendland_W_dW2(r, dot3(r, r), Wij, c);
    float f = 0.0f;
    if (c.W_dx0 > 1e-10f) f = c.p.pst_R * ipow_or_pow(Wij * inv_Wd, c.p.pst_n);
    if (c.p.pst_colle) {
        float Vj = w_of(pj, c);
        if (Vj > 1e-30f) return ((1.0f + f) * Vj) * g;
    } else {
        float mj_raw = m_uni ? m_u : __ldg(&vel[j].w);
        float mj = mw_of(mj_raw, pj, c);
        if (mj > 1e-10f) {
            // m_j / mean rho: a sum of densities, rounded quotients suffice (no cancellation)
            float rho_j = __fdividef(mj_raw, pj.w);
            float ra = 0.5f * (rho_i + rho_j);
            if (ra > 1e-10f) return ((1.0f + f) * __fdividef(mj, ra)) * g;
        }
    }
    return {0.0f, 0.0f, 0.0f};
}

// pst_constrain (DSPH.py:888-941): no shift, or only its tangential part (against the
// lambda gradient or the smallest eigenvector), near the free surface; the plane-strain
// z; no shift of a gripped solid particle.
__device__ __forceinline__ F3 pst_constrain(const Cst& c, const Ptr& P, int i, F3 dr) {
    float li = P.lam[i];
    bool surf = li < c.p.pst_lambda_hi;
    if (c.p.pst_surface_none) {
        if (surf) dr = {0, 0, 0};
    } else if (surf) {
        if (li < c.p.pst_lambda_lo) dr = {0, 0, 0};
        else {
            F3 ns = f3(P.lgrad[i]);
            if (c.p.two_d) ns.z = 0.0f;
            float nn = norm3(ns);
            if (nn > 1e-10f) {
                F3 nh = {ns.x / nn, ns.y / nn, ns.z / nn};
                float dd = dot3(dr, nh);
                dr = dr - dd * nh;
            }
        }
    }
    if (c.p.two_d) dr.z = 0.0f;
    if (c.p.is_solid && P.cur.bc[2 * i] != 0) dr = {0, 0, 0};
    return dr;
}

template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_PST) k_pst(Cst c, Ptr P) {
    constexpr bool kPlain = kShape >= 1;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {   // steps whose shift could not use the candidate lists
        const float dtot = __uint_as_float(P.ac->d_start_bits) + __uint_as_float(P.ac->max_disp_bits) +
                           __uint_as_float(P.ac->max_grip_disp_bits);
        if (!(dtot <= c.dlim)) P.ac->n_shift_search += 1ull;
    }
    if (i >= c.n) return;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    const float4* __restrict__ vel = as4c(P.cur.vel);
    float4 pi = pos[i];
    F3 xi = f3(pi);
    F3 sr = {0, 0, 0};
    const float m_i = __ldg(&vel[i].w);
    const float rho_i = m_i / pi.w;
    {
        const float inv_Wd = c.W_dx0 > 0.0f ? 1.0f / c.W_dx0 : 0.0f;
        // filled by this step's fluid advect (a solid's: by k_solid_a)
        const unsigned int mlo = P.ac->m_min_bits;
        const bool m_uni = !c.p.pst_colle && mlo == P.ac->m_max_bits;
        const float m_u = __uint_as_float(mlo);
        // one walk per form of the pair term, so that the loop carries no test of the form
        auto walk = [&](auto form) {
            constexpr int kForm = decltype(form)::value;
            for_each_pst_neighbour<kPlain>(c, P, i, xi, [&](int j, int, float4 pj, F3 xj, float d2) {
                sr += pst_term_d2<kPlain, kForm>(c, vel, xi, rho_i, inv_Wd, j, pj, xj, d2, m_uni, m_u);
            });
        };
        if (c.W_dx0 > 1e-10f && c.p.pst_n == 4) {
            if (c.p.pst_colle) walk(std::integral_constant<int, kPstColle4>());
            else if (m_uni) walk(std::integral_constant<int, kPstSun4Uni>());
            else walk(std::integral_constant<int, kPstSun4>());
        } else {
            walk(std::integral_constant<int, kPstAny>());
        }
    }
    float4 vi4 = vel[i];
    F3 vi = f3(vi4);
    // an ensemble instance (solid: material row = instance) has its own speed and dt
    float c0 = c.p.c0, dt = P.sc->dt;
    if (c.n_inst > 0) {
        const int k = (int)__ldg(P.cur.bcdisp + 4 * i + 3);
        c0 = P.irow[k].c0;
        dt = P.inst[k].dt;
    } else if (c.p.c0_mixed) {
        // local_c0 (DSPH.py:520-530): the particle's own material's EOS sound speed
        c0 = P.mat[(int)__ldg(P.cur.bcdisp + 4 * i + 3)].c0;
    }
    float Ma;
    if (c.p.pst_ma_mode == 2) Ma = c.p.pst_ma_fixed;
    else {
        float vref = c.p.pst_ma_mode == 1 ? __uint_as_float(P.ac->max_v_bits) : norm3(vi);
        Ma = vref / c0;
    }
    F3 dr;
    if (c.p.pst_colle) {
        float cc = c.colle_coef * c0 * Ma;
        F3 dvv = cc * sr;
        if (c.p.pst_clamp_vel) {
            float cap = c.p.pst_m_delta * norm3(vi);
            float dn = norm3(dvv);
            if (dn > cap) dvv = (cap / fmaxf(dn, 1e-30f)) * dvv;
        }
        dr = dt * dvv;
    } else {
        float cc = c.sun_coef * Ma * c.h * c.h;
        dr = cc * sr;
    }
    if (c.p.pst_clamp_disp) {
        float dn = norm3(dr);
        if (dn > c.max_shift) dr = (c.max_shift / dn) * dr;
    }
    dr = pst_constrain(c, P, i, dr);
    float4* shf = as4(P.cur.shift);
    float4 s = shf[i];
    s.x = dr.x; s.y = dr.y; s.z = dr.z;
    shf[i] = s;
}

// ------------------------------------------------------------------ initial relaxation
// relax_initial_configuration (DSPH.py:1113-1179): with the bins fresh, the drive
// g_i = pst_constrain(-h^2 S_i) from the run's own disorder sum; the residual is
// max |g_i| / dx0; the particle's step is beta g_i, capped at maxShift dx0, parked in the
// shift record until k_relax_move applies it.  Volume and mass are held.

// compute_lam's gradient pass alone (DSPH.py:591-609): grad lambda = sum V_j (lambda_j -
// lambda_i) L_i grad W, for the constraint's surface normal.
__global__ void __launch_bounds__(kBlock) k_relax_lamgrad(Cst c, Ptr P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const float4* __restrict__ pos = as4c(P.cur.pos);
    const F3 xi = f3(pos[i]);
    const float4 l0 = P.lsym[2 * i], l1 = P.lsym[2 * i + 1];
    const float L00 = l0.x, L11 = l0.y, L22 = l0.z, L01 = l0.w, L02 = l1.x, L12 = l1.y;
    const float lam_i = P.lam[i];
    F3 lg = {0, 0, 0};
    for_each_neighbour(c, P, i, [&](int j, int mir) {
        float4 pj = __ldg(pos + j);
        F3 xj = f3(pj);
        if (mir) xj = mirror3(mir, xj);
        F3 r = xi - xj;
        float rn;
        F3 g = wendland_dW2(r, dot3(r, r), rn, c);
        float ld = __ldg(P.lam + j) - lam_i;
        F3 Lg = {L00 * g.x + L01 * g.y + L02 * g.z, L01 * g.x + L11 * g.y + L12 * g.z,
                 L02 * g.x + L12 * g.y + L22 * g.z};
        lg += (w_of(pj, c) * ld) * Lg;
    });
    if (c.p.two_d) lg.z = 0.0f;
    P.lgrad[i] = make_float4(lg.x, lg.y, lg.z, 0.0f);
}

__global__ void __launch_bounds__(kBlock) k_relax(Cst c, Ptr P, float beta, float* res_each) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float res = 0.0f;
    if (i < c.n) {
        const float4* __restrict__ pos = as4c(P.cur.pos);
        const float4* __restrict__ vel = as4c(P.cur.vel);
        const float4 pi = pos[i];
        const F3 xi = f3(pi);
        const float rho_i = __ldg(&vel[i].w) / pi.w;
        const float inv_Wd = c.W_dx0 > 0.0f ? 1.0f / c.W_dx0 : 0.0f;
        F3 S = {0, 0, 0};
        for_each_neighbour(c, P, i, [&](int j, int mir) {
            S += pst_pair_term(c, vel, xi, rho_i, inv_Wd, j, mir, __ldg(pos + j));
        });
        const F3 g = pst_constrain(c, P, i, (-(c.h * c.h)) * S);
        const float gn = norm3(g);
        res = gn / c.p.particle_diameter;
        if (res_each) res_each[i] = res;
        F3 dr = beta * g;
        const float dn = norm3(dr);
        if (dn > c.max_shift) dr = (c.max_shift / dn) * dr;
        float4* shf = as4(P.cur.shift);
        float4 s = shf[i];
        s.x = dr.x; s.y = dr.y; s.z = dr.z;
        shf[i] = s;
    }
    block_max_atomic(res, &P.ac->relax_max_bits);
}

__global__ void __launch_bounds__(kBlock) k_relax_move(Cst c, Ptr P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    float4* pos = as4(P.cur.pos);
    const float4 s = as4c(P.cur.shift)[i];
    float4 p = pos[i];
    p.x += s.x; p.y += s.y; p.z += s.z;
    pos[i] = p;
}

// ------------------------------------------------------------------ displace + SPHBase.step boundary
__device__ __forceinline__ void place_component(float4& p, float4& u, const float4& x0, int k,
                                                float value, bool dpos) {
    if (k == 0) { p.x = value; if (dpos) u.x = value - x0.x; }
    else if (k == 1) { p.y = value; if (dpos) u.y = value - x0.y; }
    else { p.z = value; if (dpos) u.z = value - x0.z; }
}

__global__ void __launch_bounds__(kBlock) k_finish(Cst c, Ptr P, int mode) {
    const bool do_shift = mode & 1, do_bnd = mode & 2;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ww = 0.0;
    if (i < c.n) {
        float4* pos = as4(P.cur.pos);
        float4* vel = as4(P.cur.vel);
        float4* dsp = as4(P.cur.disp);
        float4 p = pos[i], v = vel[i], u = dsp[i];
        const float4 x0 = as4(P.cur.x0)[i];
        float4 a = P.acc[i];
        const bool dpos = c.p.displacement_positions;
        if (do_shift) {
            float4 s = as4(P.cur.shift)[i];
            if (dpos) {
                u.x += s.x; u.y += s.y; u.z += s.z;
                p.x = x0.x + u.x; p.y = x0.y + u.y; p.z = x0.z + u.z;
            } else {
                p.x += s.x; p.y += s.y; p.z += s.z;
            }
        }
        auto walls = [&](bool wx, bool wylo, bool wyhi, bool wz) {
            float4 q = p;
            float cn[3] = {0.f, 0.f, 0.f};
            const float qv[3] = {q.x, q.y, q.z};
            const bool on[3] = {wx, true, wz};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!on[k]) continue;
                bool hi_ok = k != 1 || wyhi, lo_ok = k != 1 || wylo;
                if (hi_ok && qv[k] > c.wall_hi[k]) { cn[k] += 1.0f; place_component(p, u, x0, k, c.wall_hi[k], dpos); }
                if (lo_ok && qv[k] <= c.p.padding) { cn[k] += -1.0f; place_component(p, u, x0, k, c.p.padding, dpos); }
            }
            float cl = sqrtf(cn[0] * cn[0] + cn[1] * cn[1] + cn[2] * cn[2]);
            if (cl > 1e-6f) {
                float nx = cn[0] / cl, ny = cn[1] / cl, nz = cn[2] / cl;
                float vn = v.x * nx + v.y * ny + v.z * nz;
                if (vn > 0.0f) {
                    ww += (double)(0.5f * v.w * vn * vn * c.rest_loss);
                    float k2 = c.rest_1p * vn;
                    v.x -= k2 * nx; v.y -= k2 * ny; v.z -= k2 * nz;
                }
            }
        };
        if (!do_bnd) {
        } else if (c.p.axisymmetric) {
            v.z = 0.0f; a.z = 0.0f;
            place_component(p, u, x0, 2, x0.z, dpos);
            if (p.y < 0.0f) {
                p.y = -p.y;
                if (dpos) u.y = -u.y - 2.0f * x0.y;
                v.y = -v.y;
                a.y = -a.y;
                if (c.p.is_solid) {  // M s M with M = diag(1, -1, 1): s_xy, s_yz flip
                    float4* sd = reinterpret_cast<float4*>(P.cur.sdev);
                    float4 s0 = sd[2 * i], s1 = sd[2 * i + 1];
                    s0.w = -s0.w;      // s_xy
                    s1.y = -s1.y;      // s_yz
                    sd[2 * i] = s0; sd[2 * i + 1] = s1;
                }
            }
            if (c.p.walls) walls(true, false, true, false);
        } else {
            if (c.p.sym_y && p.y < 0.0f) {
                p.y = -p.y; if (dpos) u.y = -u.y - 2.0f * x0.y;
                v.y = -v.y; a.y = -a.y;
                if (c.p.is_solid) {
                    float4* sd = reinterpret_cast<float4*>(P.cur.sdev);
                    float4 s0 = sd[2 * i], s1 = sd[2 * i + 1];
                    s0.w = -s0.w; s1.y = -s1.y;
                    sd[2 * i] = s0; sd[2 * i + 1] = s1;
                }
            }
            if (c.p.sym_z && p.z < 0.0f) {
                p.z = -p.z; if (dpos) u.z = -u.z - 2.0f * x0.z;
                v.z = -v.z; a.z = -a.z;
                if (c.p.is_solid) {  // M = diag(1, 1, -1): s_xz, s_yz flip
                    float4* sd = reinterpret_cast<float4*>(P.cur.sdev);
                    float4 s1 = sd[2 * i + 1];
                    s1.x = -s1.x; s1.y = -s1.y;
                    sd[2 * i + 1] = s1;
                }
            }
            if (c.p.walls) walls(true, true, true, !c.p.plane_strain);
            if (c.p.plane_strain) {
                v.z = 0.0f; a.z = 0.0f;
                place_component(p, u, x0, 2, x0.z, dpos);
            }
        }
        pos[i] = p; vel[i] = v; dsp[i] = u; P.acc[i] = a;
    }
    if (c.p.walls && do_bnd) block_sum_atomic(ww, &P.sc->wall_work);
}

// ------------------------------------------------------------------ FP64 reductions (sph_base.py:425-620)
__global__ void __launch_bounds__(kBlock) k_reduce(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double r[SPH_RED_COUNT];
#pragma unroll
    for (int k = 0; k < SPH_RED_COUNT; ++k) r[k] = 0.0;
    if (i < c.n)
        reduce_terms(c, as4c(P.cur.pos)[i], as4c(P.cur.vel)[i], as4c(P.cur.shift)[i].w, r);
#pragma unroll
    for (int k = 0; k < SPH_RED_COUNT; ++k) block_sum_atomic(r[k], &P.ac->red[k]);
}

}  // namespace sph

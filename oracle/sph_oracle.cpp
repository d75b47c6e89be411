// sph_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference's
// per-step hot path, used as the parity checker and as the timed CPU baseline.  See
// sph_oracle_common.hpp for its status.  Built as liboracle_sph.so by oracle/Makefile,
// loaded by tests/ and bench.py through oracle/oracle.py.  Nothing in sigmasph_b200
// links or calls it.
//
// Structure follows the reference one kernel per function, with the reference's loop
// semantics: one outer loop over particles (OpenMP here, a Taichi parallel for there),
// the serial neighbour loop of ParticleSystem.for_all_neighbors inside it, and global
// maxima/sums as reductions.  Templated on the arithmetic type: R = float follows the
// reference's float32 fields, R = double is the all-FP64 oracle build.
#include "sph_oracle_common.hpp"
#include "../include/sph_b200.h"

#include <cstdio>
#include <omp.h>

using namespace orc;

namespace {

constexpr double kPi = 3.14159265358979323846;

template <class R>
struct Sim {
    SphParams P;
    int64_t n = 0;
    // ---- persistent (sorted) fields, reference layout (particle_system.py:378-458)
    std::vector<V3<R>> x, x0, u, v, acc, pst_shift;
    std::vector<R> V, V_lo, m, pressure;
    std::vector<int32_t> pid;
    // ---- grid (particle_system.py:337-352, :378-386)
    int64_t T = 0;  // table size, a power of two >= 2N (min 131072)
    std::vector<int32_t> grid_ids, gpn, gpn_temp, grid_ids_new;
    std::vector<std::array<int32_t, 3>> cell_id;
    // ---- derived fields (DSPH.py:322-345)
    std::vector<R> lam, divergence, de_visc, div_rate1;
    std::vector<std::array<R, 6>> L_sym;
    std::vector<V3<R>> lam_grad, lam_eigvec;
    // ---- 0-d fields
    R dt = 0, max_c_sq = 0, max_accel = 0, max_v = 0;
    int32_t off_grid_num = 0;
    double off_grid_mass = 0, wall_work = 0, visc_work = 0, diff_work = 0, leftover_work = 0;
    // ---- constants folded the way the reference folds them
    R h = 0, alpha = 0, kgrad = 0, eta2 = 0, W_dx0 = 0;
    // ---- hypoelastic solid (SOLID.py); sorted unless noted
    std::vector<M3<R>> sdev;                    // deviatoric stress (symmetric)
    std::vector<R> eps_p, e_int, temperature, de_int;
    std::vector<R> q_visc, av_mu_max;           // derived (SOLID.py:1200-1204)
    std::vector<int32_t> bc_flag, bc_id, eos_id;
    std::vector<V3<R>> bc_disp;
    std::vector<M3<R>> grad_v, dsigma;          // derived
    std::vector<R> d_eps_p_rate, ale_adv, ale_diff;
    std::vector<V3<R>> hg_yb, hg_a, hg_v_sync;
    double sim_time = 0, plastic_work = 0, hg_work = 0, hg_ke_pre = 0;
    R load_s = 0, load_sdot = 0;
    double constraint_force[8][3] = {}, constraint_disp[8][3] = {};
    int sts_last = 0;

    void setup(const SphParams& p, int64_t nn) {
        P = p;
        n = nn;
        x.assign(n, {}); x0.assign(n, {}); u.assign(n, {}); v.assign(n, {});
        acc.assign(n, {}); pst_shift.assign(n, {});
        V.assign(n, 0); V_lo.assign(n, 0); m.assign(n, 0); pressure.assign(n, 0);
        pid.assign(n, 0);
        T = 131072;
        while (T < 2 * n) T <<= 1;
        grid_ids.assign(n, 0); grid_ids_new.assign(n, 0);
        gpn.assign(T + 1, 0); gpn_temp.assign(T + 1, 0);
        cell_id.assign(n, {0, 0, 0});
        lam.assign(n, 0); divergence.assign(n, 0); de_visc.assign(n, 0); div_rate1.assign(n, 0);
        L_sym.assign(n, {}); lam_grad.assign(n, {}); lam_eigvec.assign(n, {});
        // sph_base.py:42-151: alpha and 20 alpha / h are Python constants
        double hd = P.support_radius;
        double al = P.two_d ? 7.0 / (kPi * hd * hd) : 21.0 / (2.0 * kPi * hd * hd * hd);
        h = R(hd);
        alpha = R(al);
        kgrad = R(20.0 * al / hd);
        eta2 = R(0.01 * hd * hd);
        W_dx0 = W(R(P.particle_diameter));
        if (P.is_solid) {
            sdev.assign(n, M3<R>()); eps_p.assign(n, 0); e_int.assign(n, 0);
            temperature.assign(n, 0); de_int.assign(n, 0);
            q_visc.assign(n, 0); av_mu_max.assign(n, 0);
            bc_flag.assign(n, 0); bc_id.assign(n, -1); eos_id.assign(n, 0); bc_disp.assign(n, {});
            grad_v.assign(n, M3<R>()); dsigma.assign(n, M3<R>());
            d_eps_p_rate.assign(n, 0); ale_adv.assign(n, 0); ale_diff.assign(n, 0);
            hg_yb.assign(n, {}); hg_a.assign(n, {}); hg_v_sync.assign(n, {});
        }
    }

    // ------------------------------------------------------------ kernel (sph_base.py:42-92)
    R W(R r) const {
        R q = r / h;
        if (q < R(1)) {
            R t = R(1) - q;
            R t2 = t * t;
            return alpha * (t2 * t2) * (R(4) * q + R(1));
        }
        return R(0);
    }
    V3<R> dW(const V3<R>& r) const {
        R rn = norm(r);
        R q = rn / h;
        if (q < R(1) && rn > R(1e-5)) {
            R t = R(1) - q;
            R c = -(kgrad * q * (t * t * t));
            R f = c / rn;
            return f * r;
        }
        return {};
    }
    // particle_system.py:990-1004
    R w(int64_t p) const { return P.axisymmetric ? V[p] / std::max(x[p][1], R(P.axi_r_min)) : V[p]; }
    R mw(int64_t p) const { return P.axisymmetric ? m[p] / std::max(x[p][1], R(P.axi_r_min)) : m[p]; }
    R r_axi(int64_t p) const { return std::max(x[p][1], R(P.axi_r_min)); }
    static V3<R> mirror(int code, const V3<R>& a) {
        R sy = (code & 1) ? R(-1) : R(1), sz = (code & 2) ? R(-1) : R(1);
        return {a[0], sy * a[1], sz * a[2]};
    }

    // ------------------------------------------------------------ grid (particle_system.py:1220-1345)
    std::array<int32_t, 3> pos_to_index(const V3<R>& p) const {
        return {(int32_t)std::floor(p[0] / h), (int32_t)std::floor(p[1] / h), (int32_t)std::floor(p[2] / h)};
    }
    static bool on_grid(const V3<R>& p) { return !(std::isnan(p[0]) || std::isnan(p[1]) || std::isnan(p[2])); }
    int32_t hash_cell(const std::array<int32_t, 3>& c) const {
        uint32_t hh = (uint32_t)c[0] * 73856093u;
        hh ^= (uint32_t)c[1] * 19349663u;
        hh ^= (uint32_t)c[2] * 83492791u;
        return (int32_t)(hh & (uint32_t)(T - 1));
    }

    template <class F> void for_each_sorted(F&& f) {
        f(x); f(x0); f(u); f(v); f(acc); f(pst_shift); f(V); f(V_lo); f(m); f(pressure); f(pid);
        f(cell_id); f(grid_ids);
        if (P.is_solid) {
            f(sdev); f(eps_p); f(e_int); f(temperature); f(de_int); f(bc_flag); f(bc_id);
            f(eos_id); f(bc_disp);
        }
    }

    void initialize_particle_system() {
        // update_grid_id (:1300-1318)
        int32_t ogn = 0;
        double ogm = 0;
#pragma omp parallel for schedule(static) reduction(+ : ogn, ogm)
        for (int64_t i = 0; i < n; ++i) {
            int32_t g = (int32_t)T;
            auto c = pos_to_index(x[i]);
            cell_id[i] = c;
            if (on_grid(x[i])) g = hash_cell(c);
            else { ogn += 1; ogm += (double)m[i]; }
            grid_ids[i] = g;
        }
        off_grid_num = ogn;
        off_grid_mass = ogm;
        // counting_sort (:1320-1340) + PrefixSumExecutor.  Read serially, the reference's
        // sort leaves a bucket's particles in their previous order: it is a stable sort by
        // bucket, done here as a parallel LSD radix sort (stable by construction), and
        // gpn[b] is the inclusive count of particles in buckets <= b.
        std::vector<int32_t> order = stable_bucket_order();
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) grid_ids_new[order[p]] = (int32_t)p;
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) {
            const int64_t k = grid_ids[order[p]];
            const int64_t knext = (p + 1 < n) ? (int64_t)grid_ids[order[p + 1]] : T + 1;
            for (int64_t b = k; b < knext; ++b) gpn[b] = (int32_t)(p + 1);
        }
        const int64_t kfirst = n > 0 ? (int64_t)grid_ids[order[0]] : T + 1;
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < kfirst; ++b) gpn[b] = 0;
        for_each_sorted([&](auto& fld) {
            auto tmp = fld;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) tmp[grid_ids_new[i]] = fld[i];
            fld.swap(tmp);
        });
    }

    // Particle indices stably sorted by grid_ids (keys 0 .. T): LSD radix sort, 8 bits per
    // pass, each pass counting per thread over contiguous chunks.
    std::vector<int32_t> stable_bucket_order() const {
        std::vector<int32_t> a(n), b(n);
        for (int64_t i = 0; i < n; ++i) a[i] = (int32_t)i;
        const int nt = std::max(1, omp_get_max_threads());
        const int64_t chunk = (n + nt - 1) / nt;
        int passes = 0;
        while ((T >> (8 * passes)) > 0) ++passes;
        std::vector<int64_t> hist((size_t)nt * 256);
        for (int pass = 0; pass < passes; ++pass) {
            const int sh = 8 * pass;
            std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
            {
                const int t = omp_get_thread_num();
                const int64_t lo = std::min<int64_t>(n, t * chunk), hi = std::min<int64_t>(n, lo + chunk);
                int64_t* h = &hist[(size_t)t * 256];
                for (int64_t q = lo; q < hi; ++q) h[(grid_ids[a[q]] >> sh) & 255] += 1;
            }
            int64_t run = 0;
            for (int d = 0; d < 256; ++d)
                for (int t = 0; t < nt; ++t) {
                    const int64_t c = hist[(size_t)t * 256 + d];
                    hist[(size_t)t * 256 + d] = run;
                    run += c;
                }
#pragma omp parallel num_threads(nt)
            {
                const int t = omp_get_thread_num();
                const int64_t lo = std::min<int64_t>(n, t * chunk), hi = std::min<int64_t>(n, lo + chunk);
                int64_t* h = &hist[(size_t)t * 256];
                for (int64_t q = lo; q < hi; ++q) b[h[(grid_ids[a[q]] >> sh) & 255]++] = a[q];
            }
            a.swap(b);
        }
        return a;
    }

    // for_all_neighbors (particle_system.py:1348-1490).  `live` chooses the centre
    // cell from the live position (always true in the reference; both coincide before
    // advect).  task(j, mirror_code).
    template <class Task> void for_all_neighbors(int64_t i, Task&& task) const {
        if (!on_grid(x[i])) return;
        auto cc = pos_to_index(x[i]);
        for (int o0 = -1; o0 <= 1; ++o0)
            for (int o1 = -1; o1 <= 1; ++o1)
                for (int o2 = -1; o2 <= 1; ++o2) {
                    std::array<int32_t, 3> nc = {cc[0] + o0, cc[1] + o1, cc[2] + o2};
                    int32_t b = hash_cell(nc);
                    int32_t s = b == 0 ? 0 : gpn[b - 1], e = gpn[b];
                    for (int32_t j = s; j < e; ++j) {
                        if (cell_id[j] != nc) continue;
                        if (j != i && norm(x[i] - x[j]) < h) task((int64_t)j, 0);
                    }
                }
        bool my = P.axisymmetric || P.sym_y, mz = P.sym_z;
        if (my && x[i][1] < h) {
            V3<R> xm = mirror(1, x[i]);
            for (int o0 = -1; o0 <= 1; ++o0)
                for (int o1 = -1; o1 <= 1; ++o1) {
                    std::array<int32_t, 3> nc = {cc[0] + o0, 0, cc[2] + o1};
                    int32_t b = hash_cell(nc);
                    int32_t s = b == 0 ? 0 : gpn[b - 1], e = gpn[b];
                    for (int32_t j = s; j < e; ++j) {
                        if (cell_id[j] != nc) continue;
                        if (norm(xm - x[j]) < h) task((int64_t)j, 1);
                    }
                }
        }
        if (mz && x[i][2] < h) {
            V3<R> xm = mirror(2, x[i]);
            for (int o0 = -1; o0 <= 1; ++o0)
                for (int o1 = -1; o1 <= 1; ++o1) {
                    std::array<int32_t, 3> nc = {cc[0] + o0, cc[1] + o1, 0};
                    int32_t b = hash_cell(nc);
                    int32_t s = b == 0 ? 0 : gpn[b - 1], e = gpn[b];
                    for (int32_t j = s; j < e; ++j) {
                        if (cell_id[j] != nc) continue;
                        if (norm(xm - x[j]) < h) task((int64_t)j, 2);
                    }
                }
        }
        if (my && mz && x[i][1] < h && x[i][2] < h) {
            V3<R> xm = mirror(3, x[i]);
            for (int o0 = -1; o0 <= 1; ++o0) {
                std::array<int32_t, 3> nc = {cc[0] + o0, 0, 0};
                int32_t b = hash_cell(nc);
                int32_t s = b == 0 ? 0 : gpn[b - 1], e = gpn[b];
                for (int32_t j = s; j < e; ++j) {
                    if (cell_id[j] != nc) continue;
                    if (norm(xm - x[j]) < h) task((int64_t)j, 3);
                }
            }
        }
    }

    V3<R> xj_of(int64_t j, int mir) const { return mir ? mirror(mir, x[j]) : x[j]; }
    V3<R> vj_of(int64_t j, int mir) const { return mir ? mirror(mir, v[j]) : v[j]; }

    // ------------------------------------------------------------ compute_lam (DSPH.py:611-702)
    void compute_lam() {
        const R tol = R(P.l_eig_tol_lam);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            M3<R> E;
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir);
                V3<R> d = xj - x[i];
                V3<R> g = dW(x[i] - xj);
                R Vj = w(j);
                int nd = P.two_d ? 2 : 3;
                for (int a = 0; a < nd; ++a)
                    for (int b = 0; b < nd; ++b) E[a][b] += Vj * (d[a] * g[b]);
            });
            std::array<R, 6> Ls{};
            if (P.two_d) {
                // eig_sym_2x2 (DSPH.py:35-47) on (E00, E01, E11)
                R a = E[0][0], b = E[0][1], dd = E[1][1];
                R det = std::sqrt((a - dd) * (a - dd) + R(4) * b * b);
                R ev2 = R(0.5) * (a + dd - det);
                lam[i] = std::min(R(1), std::max(R(0), ev2));
                R L2[2][2];
                spd_inverse_2x2(E[0][0], E[0][1], E[1][0], E[1][1], tol, L2);
                Ls = {L2[0][0], L2[1][1], R(1), L2[0][1], R(0), R(0)};
                if (P.pst_normal_eigvec) {
                    R nv[2];
                    min_eig_vec_2x2(E[0][0], E[0][1], E[1][0], E[1][1], nv);
                    lam_eigvec[i] = {nv[0], nv[1], R(0)};
                }
            } else {
                R mine, mv[3];
                M3<R> L = spd_inverse_3x3(E, tol, &mine, mv);
                lam[i] = std::min(R(1), std::max(R(0), mine));
                Ls = {L[0][0], L[1][1], L[2][2], L[0][1], L[0][2], L[1][2]};
                if (P.pst_normal_eigvec) lam_eigvec[i] = {mv[0], mv[1], mv[2]};
            }
            L_sym[i] = Ls;
        }
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            const auto& s = L_sym[i];
            R L[3][3] = {{s[0], s[3], s[4]}, {s[3], s[1], s[5]}, {s[4], s[5], s[2]}};
            V3<R> lg;
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> g = dW(x[i] - xj_of(j, mir));
                R Vj = w(j);
                R ld = lam[j] - lam[i];
                V3<R> Lg = {L[0][0] * g[0] + L[0][1] * g[1] + L[0][2] * g[2],
                            L[1][0] * g[0] + L[1][1] * g[1] + L[1][2] * g[2],
                            L[2][0] * g[0] + L[2][1] * g[1] + L[2][2] * g[2]};
                lg += (Vj * ld) * Lg;
            });
            if (P.two_d) lg[2] = 0;
            lam_grad[i] = lg;
        }
    }

    // ------------------------------------------------------------ continuity (DSPH.py:1208-1338, 1432-1495)
    void compute_volume_evolution() {
        const R dtl = dt;
        double w_diff_step = 0;
        const R coef = R(P.delta_sph) * h * R(P.c0);
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : w_diff_step)
        for (int64_t i = 0; i < n; ++i) {
            R r0 = 0, r1 = 0;
            const R rho_i = m[i] / V[i];
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir), vj = vj_of(j, mir);
                V3<R> r = x[i] - xj;
                V3<R> g = dW(r);
                R rho_j = m[j] / V[j];
                V3<R> vi = v[i];
                if (P.pst_enabled) {
                    V3<R> du_i = {pst_shift[i][0] / dtl, pst_shift[i][1] / dtl, pst_shift[i][2] / dtl};
                    V3<R> du_j = {pst_shift[j][0] / dtl, pst_shift[j][1] / dtl, pst_shift[j][2] / dtl};
                    if (mir) du_j = mirror(mir, du_j);
                    vi += du_i;
                    vj += du_j;
                    r0 += w(j) * dot(rho_j * du_j - rho_i * du_i, g) / rho_i;
                }
                V3<R> vd = vi - vj;
                r0 += w(j) * dot(vd, g);
                // the solid's pair_delta (SOLID.py:4103-4114) on same-material pairs, or on
                // every pair under Diffusion.pairs "all" (DSPH.py:1271-1282), sized on
                // pair_c0 (DSPH.py:483-511)
                R cpair = coef;
                bool diffuse = P.delta_sph > 0.0f;
                if (P.is_solid) {
                    R di = R(P.mat_delta[eos_id[i]]), dj = R(P.mat_delta[eos_id[j]]);
                    R den = di + dj;
                    R dl = den > R(1e-12) ? R(2) * di * dj / den : R(0);
                    diffuse = (P.delta_pairs_all || eos_id[i] == eos_id[j]) && dl > R(0);
                    const R c0p = P.c0_mixed ? R(0.5) * (R(P.mat_c0[eos_id[i]]) + R(P.mat_c0[eos_id[j]]))
                                             : R(P.c0);
                    cpair = dl * h * c0p;
                }
                if (diffuse) {
                    R rn2 = dot(r, r);
                    R a2 = R(2) * (rho_j - rho_i);
                    R den = rn2 + eta2;
                    V3<R> psi = {a2 * (-r[0]) / den, a2 * (-r[1]) / den, a2 * (-r[2]) / den};
                    R diffusion = cpair * w(j) * dot(psi, g);
                    R rate = diffusion / rho_i;
                    r0 += rate;
                    r1 += rate;
                }
            });
            R dv = r0;
            if (P.axisymmetric) dv -= v[i][1] / r_axi(i);
            divergence[i] = dv;
            div_rate1[i] = r1;
            w_diff_step += -(double)V[i] * (double)pressure[i] * (double)r1;
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            R dVdt = -V[i] * divergence[i];
            if (P.compensated_volume) {
                double s = (double)V[i] + (double)V_lo[i] + (double)(R)(dtl * dVdt);
                R hi = (R)s;
                V[i] = hi;
                V_lo[i] = (R)(s - (double)hi);
            } else {
                V[i] += dtl * dVdt;
            }
        }
        diff_work += (double)dtl * w_diff_step;
    }

    R pressure_from_density(R rho) const {
        R p = R(P.stiffness) * (std::pow(rho / R(P.density0), R(P.exponent)) - R(1));
        if (!P.allow_negative_pressure) p = std::max(p, R(0));
        return p;
    }

    // ------------------------------------------------------------ forces (DSPH.py:1497-1650)
    void compute_forces() {
        // compute_non_pressure_forces
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            acc[i] = {R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
            pressure[i] = pressure_from_density(m[i] / V[i]);
            de_visc[i] = 0;
        }
        const R dtl = dt;
        const R visc_coef = R(10.0 * (double)P.viscosity);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> dv;
            R dvisc = 0;
            const R rho_i = m[i] / V[i];
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir), vj = vj_of(j, mir);
                V3<R> r = x[i] - xj;
                V3<R> g = dW(r);
                R fp = -w(i) * w(j) * (pressure[i] + pressure[j]);
                V3<R> f_p = fp * g;
                dv += {f_p[0] / mw(i), f_p[1] / mw(i), f_p[2] / mw(i)};
                R vxy = dot(v[i] - vj, r);
                R rn = norm(r);
                R rn2 = rn * rn;
                V3<R> f_v = (visc_coef * w(j) * vxy / (rn2 + eta2)) * g;
                dv += f_v;
                if (P.track_visc_work) dvisc += dot(v[i], f_v);
                if (P.pst_enabled && P.pst_ale_momentum) {
                    V3<R> du_i = {pst_shift[i][0] / dtl, pst_shift[i][1] / dtl, pst_shift[i][2] / dtl};
                    V3<R> du_j = {pst_shift[j][0] / dtl, pst_shift[j][1] / dtl, pst_shift[j][2] / dtl};
                    if (mir) du_j = mirror(mir, du_j);
                    R rho_j = m[j] / V[j];
                    V3<R> a = (rho_j * dot(du_j, g)) * vj - (rho_i * dot(du_i, g)) * v[i];
                    R b = dot(rho_j * du_j - rho_i * du_i, g);
                    V3<R> t = a - b * v[i];
                    R c = w(j);
                    dv += {c * t[0] / rho_i, c * t[1] / rho_i, c * t[2] / rho_i};
                }
            });
            acc[i] += dv;
            de_visc[i] = dvisc;
        }
    }

    // ------------------------------------------------------------ dt (DSPH.py:1340-1430)
    void compute_adaptive_dt() {
        R cs2 = R(P.c_signal) * R(P.c_signal);
        R mcs = cs2, ma = R(1e-10);
        const R eps = R(1e-3) * R(P.density0);
#pragma omp parallel for schedule(dynamic, 256) reduction(max : mcs, ma)
        for (int64_t i = 0; i < n; ++i) {
            if (on_grid(x[i])) ma = std::max(ma, norm(acc[i]));
            if (P.dt_pair_mode != 0) {
                R c = cs2;
                const R rho_i = m[i] / V[i];
                for_all_neighbors(i, [&](int64_t j, int) {
                    if (P.is_solid && P.dt_pair_mode == 2 && eos_id[i] != eos_id[j]) return;
                    R dp = std::fabs(pressure[i] - pressure[j]);
                    R rho_j = m[j] / V[j];
                    R drho = std::fabs(rho_i - rho_j);
                    if (drho > eps) {
                        R cij = dp / drho;
                        if (cij > c) c = cij;
                    }
                });
                mcs = std::max(mcs, c);
            }
        }
        max_c_sq = mcs;
        max_accel = ma;
        R cmax = std::sqrt(max_c_sq);
        R dta = R((double)P.CFL * (double)P.support_radius) / cmax;
        R dtf = R(P.CFL) * std::sqrt(h / max_accel);
        dt = std::min(dta, dtf);
    }

    // ------------------------------------------------------------ step work + advect (DSPH.py:1652-1763)
    void advect_and_work() {
        const R dtl = dt;
        V3<R> g = {R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
        R gsq = dot(g, g);
        double wv = 0, wl = 0;
#pragma omp parallel for schedule(static) reduction(+ : wv, wl)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> f = acc[i] - g;
            wl += (double)(R(0.5) * m[i] * dtl * dtl * (dot(f, f) - gsq));
            if (P.track_visc_work) wv += (double)m[i] * (double)de_visc[i];
            v[i] += dtl * acc[i];
            displace(i, dtl * v[i]);
        }
        visc_work += (double)dtl * wv;
        leftover_work += wl;
    }
    void displace(int64_t p, const V3<R>& d) {
        if (P.displacement_positions) { u[p] += d; x[p] = x0[p] + u[p]; }
        else x[p] += d;
    }
    void place_component(int64_t p, int k, R value) {
        x[p][k] = value;
        if (P.displacement_positions) u[p][k] = value - x0[p][k];
    }
    void reflect_component(int64_t p, int k) {
        x[p][k] = -x[p][k];
        if (P.displacement_positions) u[p][k] = -u[p][k] - R(2) * x0[p][k];
    }

    // ------------------------------------------------------------ PST (DSPH.py:712-1049)
    V3<R> pst_pair(int64_t i, int64_t j, int mir) const {
        V3<R> xj = xj_of(j, mir);
        V3<R> r = x[i] - xj;
        R rn = norm(r);
        V3<R> g = dW(r);
        R Wij = W(rn);
        R f = 0;
        if (W_dx0 > R(1e-10)) f = R(P.pst_R) * std::pow(Wij / W_dx0, R(P.pst_n));
        if (P.pst_colle) {
            R Vj = w(j);
            if (Vj > R(1e-30)) return ((R(1) + f) * Vj) * g;
        } else {
            R mj = mw(j);
            if (mj > R(1e-10)) {
                R rho_i = m[i] / V[i], rho_j = m[j] / V[j];
                R ra = R(0.5) * (rho_i + rho_j);
                if (ra > R(1e-10)) return ((R(1) + f) * (mj / ra)) * g;
            }
        }
        return {};
    }
    V3<R> pst_constrain(int64_t i, V3<R> dr) const {
        R li = lam[i];
        bool surf = li < R(P.pst_lambda_hi);
        if (P.pst_surface_none) {
            if (surf) dr = {};
        } else if (surf) {
            if (li < R(P.pst_lambda_lo)) dr = {};
            else {
                V3<R> ns = P.pst_normal_eigvec ? lam_eigvec[i] : lam_grad[i];
                if (P.two_d) ns[2] = 0;
                R nn = norm(ns);
                if (nn > R(1e-10)) {
                    V3<R> nh = {ns[0] / nn, ns[1] / nn, ns[2] / nn};
                    dr = dr - dot(dr, nh) * nh;
                }
            }
        }
        if (P.two_d) dr[2] = 0;
        if (P.is_solid && bc_flag[i] != 0) dr = {};
        return dr;
    }
    void apply_pst() {
        if (P.pst_ma_mode == 1) {
            R mv = 0;
#pragma omp parallel for schedule(static) reduction(max : mv)
            for (int64_t i = 0; i < n; ++i) if (on_grid(x[i])) mv = std::max(mv, norm(v[i]));
            max_v = mv;
        }
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> s;
            for_all_neighbors(i, [&](int64_t j, int mir) { s += pst_pair(i, j, mir); });
            // local_c0 (DSPH.py:520-530): the particle's own material's speed when the
            // materials' EOS speeds differ
            const R c0l = (P.is_solid && P.c0_mixed) ? R(P.mat_c0[eos_id[i]]) : R(P.c0);
            R Ma;
            if (P.pst_ma_mode == 2) Ma = R(P.pst_ma_fixed);
            else {
                R vref = P.pst_ma_mode == 1 ? max_v : norm(v[i]);
                Ma = vref / c0l;
            }
            V3<R> dr;
            if (P.pst_colle) {
                R c = R(-2.0 * (double)P.support_radius) * c0l * Ma;
                V3<R> dvv = c * s;
                if (P.pst_clamp_vel) {
                    R cap = R(P.pst_m_delta) * norm(v[i]);
                    R dn = norm(dvv);
                    if (dn > cap) dvv = (cap / std::max(dn, R(1e-30))) * dvv;
                }
                dr = dt * dvv;
            } else {
                R c = R(-(double)P.CFL) * Ma * h * h;
                dr = c * s;
            }
            if (P.pst_clamp_disp) {
                R ms = R((double)P.pst_max_shift * (double)P.particle_diameter);
                R dn = norm(dr);
                if (dn > ms) dr = (ms / dn) * dr;
            }
            pst_shift[i] = pst_constrain(i, dr);
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) displace(i, pst_shift[i]);
    }

    // ------------------------------------------------------------ boundary (sph_base.py:160-655)
    // the wall work of one collision (added by the caller)
    double simulate_collisions(int64_t i, const V3<R>& nv) {
        R vn = dot(v[i], nv);
        if (vn > R(0)) {
            R c = R(P.wall_restitution);
            v[i] -= (R(1.0 + (double)c) * vn) * nv;
            return (double)(R(0.5) * m[i] * vn * vn * R(1.0 - (double)P.wall_restitution * P.wall_restitution));
        }
        return 0.0;
    }
    void enforce_walls(int faces) {  // faces: bit0 x, bit1 y-low, bit2 y-high, bit3 z
        double ww = 0;
#pragma omp parallel for schedule(static) reduction(+ : ww)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> pos = x[i];
            V3<R> cn;
            for (int k = 0; k < 3; ++k) {
                if (k == 2 && !(faces & 8)) continue;
                R hi = R((double)P.domain_size[k] - (double)P.padding), lo = R(P.padding);
                bool do_hi = k != 1 || (faces & 4);
                bool do_lo = k != 1 || (faces & 2);
                if (do_hi && pos[k] > hi) { cn[k] += R(1); place_component(i, k, hi); }
                if (do_lo && pos[k] <= lo) { cn[k] += R(-1); place_component(i, k, lo); }
            }
            R cl = norm(cn);
            if (cl > R(1e-6)) ww += simulate_collisions(i, {cn[0] / cl, cn[1] / cl, cn[2] / cl});
        }
        wall_work += ww;
    }
    void boundary() {
        if (P.axisymmetric) {
            for (int64_t i = 0; i < n; ++i) {
                v[i][2] = 0; acc[i][2] = 0;
                place_component(i, 2, x0[i][2]);
                if (x[i][1] < R(0)) {
                    reflect_component(i, 1);
                    v[i][1] = -v[i][1];
                    acc[i][1] = -acc[i][1];
                    if (P.is_solid) sdev[i] = mirror_mat(1, sdev[i]);
                }
            }
            if (P.walls) enforce_walls(1 | 4);
        } else {
            if (P.sym_y || P.sym_z) {
                for (int64_t i = 0; i < n; ++i) {
                    if (P.sym_y && x[i][1] < R(0)) {
                        reflect_component(i, 1); v[i][1] = -v[i][1]; acc[i][1] = -acc[i][1];
                        if (P.is_solid) sdev[i] = mirror_mat(1, sdev[i]);
                    }
                    if (P.sym_z && x[i][2] < R(0)) {
                        reflect_component(i, 2); v[i][2] = -v[i][2]; acc[i][2] = -acc[i][2];
                        if (P.is_solid) sdev[i] = mirror_mat(2, sdev[i]);
                    }
                }
            }
            if (P.walls) enforce_walls(P.plane_strain ? (1 | 2 | 4) : (1 | 2 | 4 | 8));
            if (P.plane_strain) {
                for (int64_t i = 0; i < n; ++i) {
                    v[i][2] = 0; acc[i][2] = 0;
                    place_component(i, 2, x0[i][2]);
                }
            }
        }
    }

    // ============================================================ hypoelastic solid (SOLID.py)
    static M3<R> mirror_mat(int code, const M3<R>& T) {
        R s[3] = {R(1), (code & 1) ? R(-1) : R(1), (code & 2) ? R(-1) : R(1)};
        M3<R> o;
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) o[a][b] = s[a] * T[a][b] * s[b];
        return o;
    }
    R matc_G(int64_t p) const { return R(P.mat_G[eos_id[p]]); }
    // _hg_impedance_ratio (SOLID.py:4184-4239): 2 Z_j / (Z_i + Z_j), Z = rho0 c_p
    R hg_impedance_ratio(int64_t i, int64_t j) const {
        const R zi = R(P.mat_rho0[eos_id[i]]) * R(P.mat_cp[eos_id[i]]);
        const R zj = R(P.mat_rho0[eos_id[j]]) * R(P.mat_cp[eos_id[j]]);
        const R den = zi + zj;
        return den > R(0) ? R(2) * zj / den : R(1);
    }
    R r_of(int64_t p) const { return std::max(x[p][1], R(P.axi_r_min)); }

    // SOLID.py:5001-5017
    void update_load_factor() {
        double T = P.ramp_time;
        if (T <= 0.0) { load_s = R(1); load_sdot = R(0); return; }
        double uu = std::min(1.0, std::max(0.0, sim_time / T));
        load_s = R(uu * uu * (3.0 - 2.0 * uu));
        load_sdot = R(6.0 * uu * (1.0 - uu) / T);
    }

    // SOLID.py:1721-1794
    void compute_velocity_gradient() {
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            M3<R> G;
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir), vj = vj_of(j, mir);
                V3<R> g = dW(x[i] - xj);
                V3<R> dv = vj - v[i];
                R wj = w(j);
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) G[a][b] += wj * (dv[a] * g[b]);
            });
            if (P.kernel_correction) {
                M3<R> E;
                for_all_neighbors(i, [&](int64_t j, int mir) {
                    V3<R> xj = xj_of(j, mir);
                    V3<R> d = xj - x[i];
                    V3<R> g = dW(x[i] - xj);
                    R Vj = w(j);
                    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) E[a][b] += Vj * (d[a] * g[b]);
                });
                M3<R> L;
                if (P.two_d) {
                    R L2[2][2];
                    spd_inverse_2x2(E[0][0], E[0][1], E[1][0], E[1][1], R(P.l_eig_tol), L2);
                    L[0][0] = L2[0][0]; L[0][1] = L2[0][1]; L[1][0] = L2[1][0]; L[1][1] = L2[1][1];
                    L[2][2] = R(1);
                } else {
                    L = spd_inverse_3x3(E, R(P.l_eig_tol));
                }
                M3<R> GL;
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
                    R s = 0;
                    for (int k = 0; k < 3; ++k) s += G[a][k] * L[k][b];
                    GL[a][b] = s;
                }
                G = GL;
            }
            if (P.two_d) for (int d = 0; d < 3; ++d) { G[2][d] = 0; G[d][2] = 0; }
            if (P.axisymmetric) G[2][2] = v[i][1] / r_axi(i);
            grad_v[i] = G;
        }
    }

    // MAT001_linear_plasticity.py:65-81
    static R vm_of(const M3<R>& s) {
        R t = 0;
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) t += s[a][b] * s[a][b];
        return std::sqrt(R(1.5) * t);
    }
    static R j2_return(M3<R>& s, R G, R sy, R H, R ep) {
        R d = 0;
        if (sy > R(0)) {
            R vm = vm_of(s);
            R sigy = sy + H * ep;
            if (vm > sigy && (R(3) * G + H) > R(0)) {
                d = (vm - sigy) / (R(3) * G + H);
                R sc = (sigy + H * d) / vm;
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s[a][b] = s[a][b] * sc;
            }
        }
        return d;
    }
    // MAT002_johnson_cook.py:251-354 (bracketed Newton-bisection)
    static void jc_residual(R d, R vm, R G, R A, R B, R nn, R C, R e0d, R mt, R ep, R dt, R& g, R& dg) {
        R et = ep + d;
        R ss = A, ds = 0;
        if (et > R(0) && B > R(0) && nn > R(0)) {
            ss += B * std::pow(et, nn);
            if (et > R(1e-12)) ds = nn * B * std::pow(et, nn - R(1));
        }
        R rate = 1;
        if (dt > R(0) && e0d > R(0)) rate = (d / dt) / e0d;
        R mr = 1, dmr = 0;
        if (rate > R(1) && C > R(0)) { mr = R(1) + C * std::log(rate); dmr = C / std::max(R(1e-12), d); }
        R sy = ss * mr * mt;
        R dsy = (ds * mr + ss * dmr) * mt;
        g = vm - R(3) * G * d - sy;
        dg = -R(3) * G - dsy;
    }
    R jc_return(M3<R>& s, int k, R ep, R temp, R dt, int* iters = nullptr) const {
        return jc_return_of(s, R(P.mat_G[k]), R(P.jc_A[k]), R(P.jc_B[k]), R(P.jc_n[k]),
                            R(P.jc_C[k]), R(P.jc_eps0_dot[k]), R(P.jc_T0[k]), R(P.jc_Tm[k]),
                            R(P.jc_m[k]), ep, temp, dt, iters);
    }
    static R jc_return_of(M3<R>& s, R G, R A, R B, R nn, R C, R e0d, R T0, R Tm, R mexp,
                          R ep, R temp, R dt, int* iters = nullptr) {
        R d = 0;
        if (!(G > R(0) && A > R(0))) return 0;
        R vm = vm_of(s);
        R mt = 1;
        if (Tm > T0 && temp > T0) {
            R ts = std::min(R(1), std::max(R(0), (temp - T0) / (Tm - T0)));
            mt = std::max(R(0), R(1) - std::pow(ts, mexp));
        }
        R s0 = A;
        if (ep > R(0) && B > R(0) && nn > R(0)) s0 += B * std::pow(ep, nn);
        R sy0 = s0 * mt;
        if (!(vm > sy0 && sy0 > R(0))) return 0;
        R lo = 0, hi = (vm - sy0) / (R(3) * G);
        R dref = 0;
        if (dt > R(0) && e0d > R(0) && C > R(0)) dref = dt * e0d;
        if (dref > R(0) && dref < hi) {
            R g, dg;
            jc_residual(dref, vm, G, A, B, nn, C, e0d, mt, ep, dt, g, dg);
            if (g > R(0)) lo = dref; else hi = dref;
        }
        d = hi;
        if (lo > R(0)) d = lo;
        int it = 0;
        for (; it < 40; ++it) {
            R g, dg;
            jc_residual(d, vm, G, A, B, nn, C, e0d, mt, ep, dt, g, dg);
            if (g > R(0)) lo = d; else hi = d;
            if (std::fabs(g) <= R(1e-6) * vm || hi - lo <= R(1e-6) * hi) break;
            R dn = d - g / dg;
            if (!(dn > lo && dn < hi)) dn = lo > R(0) ? std::sqrt(lo * hi) : R(0.5) * hi;
            if (std::fabs(dn - d) <= R(1e-6) * d) { d = dn; break; }
            d = dn;
        }
        if (iters) *iters = it;
        R syf = std::max(R(0), vm - R(3) * G * d);
        R sc = syf / vm;
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s[a][b] = s[a][b] * sc;
        return d;
    }

    // SOLID.py:2691-3004 with the ALE tasks :1799-1862
    void update_stress() {
        const R dtl = dt;
        const bool ale = P.ale_history != 0;
        const bool plastic_any = [&] {
            for (int k = 0; k < P.n_materials; ++k) if (P.plastic_sy0[k] > 0.0f) return true;
            return false;
        }();
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            const M3<R>& Lv = grad_v[i];
            M3<R> ed, sp;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
                ed[a][b] = R(0.5) * (Lv[a][b] + Lv[b][a]);
                sp[a][b] = R(0.5) * (Lv[a][b] - Lv[b][a]);
            }
            R tr = ed[0][0] + ed[1][1] + ed[2][2];
            const M3<R>& s = sdev[i];
            R G2 = R(2) * matc_G(i);
            M3<R> sd;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
                R dev = ed[a][b] - ((a == b) ? tr / R(3) : R(0));
                R ws = 0, sw = 0;
                for (int k = 0; k < 3; ++k) { ws += sp[a][k] * s[k][b]; sw += s[a][k] * sp[k][b]; }
                // SOLID.py:2721-2722: the spin terms only under the Jaumann rate
                sd[a][b] = P.objective_none ? G2 * dev : G2 * dev + (ws - sw);
            }
            R dep = 0;
            if (ale) {
                M3<R> A;
                const V3<R> du_i = {pst_shift[i][0] / dtl, pst_shift[i][1] / dtl, pst_shift[i][2] / dtl};
                const R rho_i = m[i] / V[i];
                for_all_neighbors(i, [&](int64_t j, int mir) {
                    V3<R> xj = xj_of(j, mir);
                    V3<R> du_j = {pst_shift[j][0] / dtl, pst_shift[j][1] / dtl, pst_shift[j][2] / dtl};
                    M3<R> sj = sdev[j];
                    if (mir) { du_j = mirror(mir, du_j); sj = mirror_mat(mir, sj); }
                    V3<R> g = dW(x[i] - xj);
                    R rho_j = m[j] / V[j];
                    R a_j = rho_j * dot(du_j, g), a_i = rho_i * dot(du_i, g);
                    R div = dot(rho_j * du_j - rho_i * du_i, g);
                    R wj = w(j);
                    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
                        R flux = a_j * sj[a][b] - a_i * s[a][b];
                        A[a][b] += wj * (flux - s[a][b] * div) / rho_i;
                    }
                    if (plastic_any) {
                        R flux = a_j * eps_p[j] - a_i * eps_p[i];
                        dep += wj * (flux - eps_p[i] * div) / rho_i;
                    }
                });
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) sd[a][b] += A[a][b];
            }
            dsigma[i] = sd;
            d_eps_p_rate[i] = dep;
        }
        double pw = 0;
#pragma omp parallel for schedule(static) reduction(+ : pw)
        for (int64_t i = 0; i < n; ++i) {
            M3<R> sn;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) sn[a][b] = sdev[i][a][b] + dtl * dsigma[i][a][b];
            M3<R> ss;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) ss[a][b] = R(0.5) * (sn[a][b] + sn[b][a]);
            R tr3 = (ss[0][0] + ss[1][1] + ss[2][2]) / R(3);
            for (int a = 0; a < 3; ++a) ss[a][a] -= tr3;
            if (matc_G(i) <= R(0)) ss = M3<R>();
            if (ale && plastic_any) eps_p[i] = std::max(R(0), eps_p[i] + dtl * d_eps_p_rate[i]);
            R dprod = 0;
            if (plastic_any) {
                int k = eos_id[i];
                if (P.plastic_kind[k] == 2) dprod = jc_return(ss, k, eps_p[i], temperature[i], dtl);
                else dprod = j2_return(ss, matc_G(i), R(P.plastic_sy0[k]), R(P.plastic_H[k]), eps_p[i]);
                eps_p[i] += dprod;
                if (dprod > R(0)) pw += (double)(V[i] * vm_of(ss) * dprod);
            }
            sdev[i] = ss;
        }
        plastic_work += pw;
    }

    // SOLID.py:1949-2069 (ALE advection and upwind diffusion of e)
    void compute_ale_e_rates() {
        const R dtl = dt;
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            R adv = 0, dif = 0;
            const V3<R> du_i = {pst_shift[i][0] / dtl, pst_shift[i][1] / dtl, pst_shift[i][2] / dtl};
            const R rho_i = m[i] / V[i];
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir);
                V3<R> du_j = {pst_shift[j][0] / dtl, pst_shift[j][1] / dtl, pst_shift[j][2] / dtl};
                if (mir) du_j = mirror(mir, du_j);
                V3<R> g = dW(x[i] - xj);
                R rho_j = m[j] / V[j];
                adv += w(j) * rho_j * (e_int[j] - e_int[i]) * dot(du_j, g) / rho_i;
                if (P.ale_diffusion > 0.0f && eos_id[i] == eos_id[j]) {
                    V3<R> r = x[i] - xj;
                    R sc = R(2) * (e_int[j] - e_int[i]);
                    R den = dot(r, r) + eta2;
                    V3<R> psi = {sc * (-r[0]) / den, sc * (-r[1]) / den, sc * (-r[2]) / den};
                    R rb = R(0.5) * (rho_i + rho_j);
                    R sp = R(0.5) * norm(du_i + du_j);
                    dif += R(P.ale_diffusion) * R(0.5) * R(P.particle_diameter) * sp * w(j) * dot(psi, g) * rb / rho_i;
                }
            });
            ale_adv[i] = adv;
            ale_diff[i] = dif;
        }
    }

    // SOLID.py:2071-2237 (state part) and :2239-2293
    void update_internal_energy() {
        const R dtl = dt;
        V3<R> g = {R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
        R gsq = dot(g, g);
        double wl = 0;
        for (int64_t i = 0; i < n; ++i) {
            R de = de_int[i];
            if (P.transport_e) de += ale_adv[i] + ale_diff[i];
            e_int[i] += dtl * de;
            V3<R> f = acc[i] - g;
            wl += (double)(R(0.5) * m[i] * dtl * dtl * (dot(f, f) - gsq));
        }
        leftover_work += wl;
        // SOLID.py:2182-2207: the explicit damper's and the viscosities' work of the
        // previous step's force pass, banked with the dt it was done over
        hg_work += (double)dtl * hg_step_power;
        hg_step_power = 0;
        if (P.track_visc_work) visc_work += (double)dtl * visc_step_power;
        visc_step_power = 0;
    }
    void update_temperature() {
        for (int64_t i = 0; i < n; ++i) {
            int k = eos_id[i];
            R cv = R(P.mat_cv[k]);
            if (!(cv > R(0))) continue;
            double rho = (double)m[i] / (double)V[i], rho0 = (double)(R)P.mat_rho0[k];
            double S = (double)(R)P.mat_stiff[k], gam = (double)(R)P.mat_gamma[k];
            double xx = rho / rho0, ec;
            if (std::fabs(gam - 1.0) < 1.0e-6) ec = (S / rho0) * (std::log(xx) + 1.0 / xx - 1.0);
            else ec = (S / rho0) * ((std::pow(xx, gam - 1.0) - 1.0) / (gam - 1.0) + 1.0 / xx - 1.0);
            if (!P.allow_negative_pressure && rho < rho0) ec = 0.0;
            double eth = (double)e_int[i] - ec - 0.0;
            temperature[i] = R(P.mat_T0[k]) + (R)(eth / (double)cv);
        }
    }

    R solid_pressure(int64_t i, R rho) const {
        int k = eos_id[i];
        R rho0 = R(P.mat_rho0[k]), S = R(P.mat_stiff[k]), gam = R(P.mat_gamma[k]);
        bool all_one = true;
        for (int q = 0; q < P.n_materials; ++q) if (P.mat_gamma[q] != 1.0f) all_one = false;
        R p = all_one ? S * (rho / rho0 - R(1)) : S * (std::pow(rho / rho0, gam) - R(1));
        if (!P.allow_negative_pressure) p = std::max(p, R(0));
        return p;
    }

    // SOLID.py:3204-3852
    void compute_stress_accelerations() {
        const bool q_on = P.q_l2 > 0.0f;
        const bool av_on = P.av_alpha > 0.0f || P.av_beta > 0.0f;
        for (int64_t i = 0; i < n; ++i) {
            acc[i] = {R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
            const R rho = m[i] / V[i];
            pressure[i] = solid_pressure(i, rho);
            de_int[i] = 0;
            // SOLID.py:3393-3401: q from the trace of this step's grad v, compression only
            q_visc[i] = 0;
            if (q_on) {
                R dvv = grad_v[i][0][0] + grad_v[i][1][1] + grad_v[i][2][2];
                if (dvv < R(0)) q_visc[i] = R(P.q_l2) * rho * dvv * dvv;
            }
        }
        const R dtl = dt;
        const R visc = R(10.0 * (double)P.viscosity);
        const bool hg_inloop = P.hourglass_alpha > 0.0f && !P.hourglass_sts;
        const bool ale = P.pst_enabled && P.pst_ale_momentum;
        double hgw = 0, vw = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : hgw, vw)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> dv;
            R dei = 0, dhg = 0, dvisc = 0, mu_max = 0;
            const R rho_i = m[i] / V[i];
            const R mwi = mw(i), wi = w(i);
            const R ptot_i = pressure[i] + q_visc[i];
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir), vj = vj_of(j, mir);
                M3<R> sj = sdev[j];
                if (mir) sj = mirror_mat(mir, sj);
                V3<R> r = x[i] - xj;
                V3<R> g = dW(r);
                V3<R> f;
                for (int a = 0; a < 3; ++a) {
                    R t = 0;
                    for (int b = 0; b < 3; ++b) {
                        R sig = (sdev[i][a][b] + sj[a][b]) - ((a == b) ? (ptot_i + (pressure[j] + q_visc[j])) : R(0));
                        t += sig * g[b];
                    }
                    f[a] = wi * w(j) * t;
                }
                const bool axc = P.axisymmetric && P.axi_conservative_x;
                const bool axr = P.axisymmetric && P.axi_conservative_r;
                if (axc) {
                    // SOLID.py:3598-3609: a mirror image at its signed radius under "signed"
                    const R rs = (mir && P.axi_image_signed) ? r_of(i) - r_of(j) : r_of(i) + r_of(j);
                    f[0] = f[0] * (R(0.5) * rs / r_of(i));
                }
                if (axr) {
                    // SOLID.py:3609-3614: the radial form, an image always at its signed radius
                    const R rs = mir ? r_of(i) - r_of(j) : r_of(i) + r_of(j);
                    f[1] = f[1] * (R(0.5) * rs / r_of(i));
                }
                const R pratio = (axc || axr) ? R(0.5) * (r_of(i) + r_of(j)) / r_of(i) : R(1);
                dv += {f[0] / mwi, f[1] / mwi, f[2] / mwi};
                V3<R> vij = v[i] - vj;
                dei += -R(0.5) * dot(f, vij) / mwi;
                R vxy = dot(vij, r);
                R rn = norm(r);
                V3<R> am = (visc * w(j) * vxy / (rn * rn + eta2)) * g;
                dv += am;
                if (P.viscosity > 0.0f) {
                    R wm = -R(0.5) * dot(am, vij);
                    dei += wm;
                    dvisc += -wm;
                }
                // SOLID.py:3727-3766: Monaghan's Pi_ij on approaching pairs
                if (av_on && vxy < R(0)) {
                    const R hav = h;
                    R mu = hav * vxy / (rn * rn + R(P.av_eps) * hav * hav);
                    R rho_j = m[j] / V[j];
                    R rho_bar = R(0.5) * (rho_i + rho_j);
                    R c_bar = R(0.5) * (R(P.mat_cp[eos_id[i]]) + R(P.mat_cp[eos_id[j]]));
                    R pij = (-R(P.av_alpha) * c_bar * mu + R(P.av_beta) * mu * mu) / rho_bar;
                    V3<R> ap = (-mw(j) * pij) * g;
                    R mu_cfl = -mu;
                    if (axc) ap[0] = ap[0] * pratio;
                    if (axr) ap[1] = ap[1] * pratio;
                    if (axc || axr) mu_cfl = mu_cfl * pratio;
                    dv += ap;
                    mu_max = std::max(mu_max, mu_cfl);
                    R wp = -R(0.5) * dot(ap, vij);
                    dei += wp;
                    dvisc += -wp;
                }
                if (hg_inloop && rn > R(1e-9)) {
                    V3<R> rh = {-r[0] / rn, -r[1] / rn, -r[2] / rn};
                    M3<R> gvj = grad_v[j];
                    if (mir) gvj = mirror_mat(mir, gvj);
                    V3<R> dvh;
                    for (int a = 0; a < 3; ++a) {
                        R t = 0;
                        for (int b = 0; b < 3; ++b) t += R(0.5) * (grad_v[i][a][b] + gvj[a][b]) * (-r[b]);
                        dvh[a] = (vj[a] - v[i][a]) - t;
                    }
                    R hg = dot(dvh, rh);
                    R Wij = W(rn);
                    int k = eos_id[i];
                    R damp = R(P.hourglass_alpha) * (R(P.mat_rho0[k]) / rho_i) * (R(P.mat_cp[k]) / h)
                             * (w(j) / R(P.V0)) * (Wij / R(P.hg_W_dx0)) * hg;
                    if (P.hg_mixed_impedance) damp = damp * hg_impedance_ratio(i, j);
                    V3<R> ah = damp * rh;
                    if (axc) ah[0] = ah[0] * pratio;
                    if (axr) ah[1] = ah[1] * pratio;
                    dv += ah;
                    dhg += -R(0.5) * dot(ah, vij);
                }
                if (ale) {
                    V3<R> du_i = {pst_shift[i][0] / dtl, pst_shift[i][1] / dtl, pst_shift[i][2] / dtl};
                    V3<R> du_j = {pst_shift[j][0] / dtl, pst_shift[j][1] / dtl, pst_shift[j][2] / dtl};
                    if (mir) du_j = mirror(mir, du_j);
                    R rho_j = m[j] / V[j];
                    V3<R> a = (rho_j * dot(du_j, g)) * vj - (rho_i * dot(du_i, g)) * v[i];
                    R b = dot(rho_j * du_j - rho_i * du_i, g);
                    V3<R> t = a - b * v[i];
                    R c = w(j);
                    dv += {c * t[0] / rho_i, c * t[1] / rho_i, c * t[2] / rho_i};
                }
            });
            if (P.axisymmetric) {
                // SOLID.py:3444-3466: the sources the pair sums do not generate
                R inv = R(1) / (rho_i * r_axi(i));
                V3<R> ag = {P.axi_conservative_x ? R(0) : sdev[i][0][1] * inv,
                            P.axi_conservative_r ? (ptot_i - sdev[i][2][2]) * inv
                                                 : (sdev[i][1][1] - sdev[i][2][2]) * inv,
                            R(0)};
                dv += ag;
                if (P.axi_conservative_r) dei += -dot(v[i], ag);
            }
            acc[i] += dv;
            de_int[i] = dei;
            av_mu_max[i] = mu_max;
            hgw += (double)(mwi * dhg);
            vw += (double)m[i] * (double)dvisc;
        }
        hg_step_power = hgw;
        visc_step_power = vw;
    }
    double hg_step_power = 0, visc_step_power = 0;

    // SOLID.py:3939-4009: the two viscosities' own CFL limits, after the acoustic one
    void clamp_dt_viscosities() {
        const R cfl_h = R((double)P.CFL * (double)P.support_radius);
        if (P.q_l2 > 0.0f) {
            R cmax = 0;
            for (int64_t i = 0; i < n; ++i) {
                R dvv = grad_v[i][0][0] + grad_v[i][1][1] + grad_v[i][2][2];
                if (dvv < R(0)) {
                    R qc = R(P.q_cl) * (-dvv);
                    R ci = R(P.mat_cp[eos_id[i]]);
                    cmax = std::max(cmax, qc + std::sqrt(qc * qc + ci * ci));
                }
            }
            if (cmax > R(0)) dt = std::min(dt, cfl_h / cmax);
        }
        if (P.av_alpha > 0.0f || P.av_beta > 0.0f) {
            R cmax = 0;
            for (int64_t i = 0; i < n; ++i) {
                R mu = av_mu_max[i];
                if (mu > R(0)) {
                    R ci = R(P.mat_cp[eos_id[i]]);
                    cmax = std::max(cmax, ci + R(1.2) * (R(P.av_alpha) * ci + R(P.av_beta) * mu));
                }
            }
            if (cmax > R(0)) dt = std::min(dt, cfl_h / cmax);
        }
    }

    // SOLID.py:4241-4309 (the damper operator on the sub-stepped velocity y)
    void compute_hg_accel() {
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> a;
            const R rho_i = m[i] / V[i];
            for_all_neighbors(i, [&](int64_t j, int mir) {
                V3<R> xj = xj_of(j, mir);
                V3<R> yj = hg_yb[j];
                M3<R> gvj = grad_v[j];
                if (mir) { yj = mirror(mir, yj); gvj = mirror_mat(mir, gvj); }
                V3<R> r = x[i] - xj;
                R rn = norm(r);
                if (!(rn > R(1e-9))) return;
                V3<R> rh = {-r[0] / rn, -r[1] / rn, -r[2] / rn};
                V3<R> dvh;
                for (int q = 0; q < 3; ++q) {
                    R t = 0;
                    for (int b = 0; b < 3; ++b) t += R(0.5) * (grad_v[i][q][b] + gvj[q][b]) * (-r[b]);
                    dvh[q] = (yj[q] - hg_yb[i][q]) - t;
                }
                R hg = dot(dvh, rh);
                R Wij = W(rn);
                int k = eos_id[i];
                R damp = R(P.hourglass_alpha) * (R(P.mat_rho0[k]) / rho_i) * (R(P.mat_cp[k]) / h)
                         * (w(j) / R(P.V0)) * (Wij / R(P.hg_W_dx0)) * hg;
                if (P.hg_mixed_impedance) damp = damp * hg_impedance_ratio(i, j);
                V3<R> ah = damp * rh;
                if (P.axisymmetric && (P.axi_conservative_x || P.axi_conservative_r)) {
                    const R ratio = R(0.5) * (r_of(i) + r_of(j)) / r_of(i);
                    if (P.axi_conservative_x) ah[0] = ah[0] * ratio;
                    if (P.axi_conservative_r) ah[1] = ah[1] * ratio;
                }
                a += ah;
            });
            hg_a[i] = a;
        }
    }
    double kinetic() const {
        double ke = 0;
        for (int64_t i = 0; i < n; ++i) ke += (double)(R(0.5) * m[i] * dot(v[i], v[i]));
        return ke;
    }

    // SOLID.py:5019-5055
    void apply_constraints() {
        for (int k = 0; k < 8; ++k) for (int d = 0; d < 3; ++d) { constraint_force[k][d] = 0; constraint_disp[k][d] = 0; }
        const R s = load_s, sd = load_sdot;
        const R scale = P.axisymmetric ? R(2.0 * kPi) : R(1);
        for (int64_t i = 0; i < n; ++i) {
            int fl = bc_flag[i];
            if (!fl) continue;
            int cid = bc_id[i];
            for (int d = 0; d < 3; ++d) {
                if (!(fl & (1 << d))) continue;
                if (P.num_constraints > 0 && cid >= 0) {
                    constraint_force[cid][d] += (double)(scale * m[i] * acc[i][d]);
                    constraint_disp[cid][d] = (double)(bc_disp[i][d] * s);
                }
                u[i][d] = bc_disp[i][d] * s;
                x[i][d] = x0[i][d] + u[i][d];
                v[i][d] = bc_disp[i][d] * sd;
                acc[i][d] = 0;
            }
        }
    }

    // The step in the stage grouping of the GPU (SPH_STAGE_*), for stage-by-stage checks.
    void stage_solid(int s) {
        switch (s) {
            case SPH_STAGE_SORT: update_load_factor(); initialize_particle_system(); break;
            case SPH_STAGE_LAM: {
                compute_lam();
                compute_velocity_gradient();
                update_stress();
                if (P.transport_e) compute_ale_e_rates();
                update_internal_energy();
                bool thermal = false;
                for (int k = 0; k < P.n_materials; ++k) if (P.mat_cv[k] > 0.0f) thermal = true;
                if (thermal) update_temperature();
                break;
            }
            case SPH_STAGE_CONTINUITY: compute_volume_evolution(); break;
            case SPH_STAGE_FORCES: compute_stress_accelerations(); break;
            case SPH_STAGE_DT: solid_dt(); break;
            case SPH_STAGE_ADVECT: solid_advect(); apply_constraints(); break;
            case SPH_STAGE_PST: if (P.pst_enabled) apply_pst(); break;
            case SPH_STAGE_BOUNDARY: boundary(); sim_time += (double)dt; break;
            default: break;
        }
    }
    void solid_dt() {
        compute_adaptive_dt();
        clamp_dt_viscosities();
        const bool hg = P.hourglass_alpha > 0.0f;
        sts_last = 0;
        if (!P.hourglass_sts) {
            if (hg) dt = std::min(dt, R(1.6 / (double)P.hg_rate));
        } else if (hg) {
            // sts_stage_count (SOLID.py:4510-4539)
            int s = 1;
            if (P.hg_rate > 0.0f) {
                double want = (double)P.hg_rate * (double)dt, cap;
                if (!P.hg_sts_rkl) {
                    s = P.hg_sts_fixed > 0 ? P.hg_sts_fixed : std::max(1, (int)std::ceil(want / 1.6));
                    s = std::min(s, 32);
                    cap = s * 1.6 / (double)P.hg_rate;
                } else {
                    const double safety = (double)P.hourglass_sts_safety;
                    if (P.hg_sts_fixed > 0) s = P.hg_sts_fixed;
                    else
                        while ((double)(s * s + s) * safety < want && s < 32) ++s;
                    cap = safety * (double)(s * s + s) / (double)P.hg_rate;
                }
                if ((double)dt > cap) dt = R(cap);
            }
            sts_last = s;
        }
    }
    void step_solid() {
        for (int s = SPH_STAGE_SORT; s <= SPH_STAGE_BOUNDARY; ++s) stage_solid(s);
    }
    void solid_advect() {
        const bool hg = P.hourglass_alpha > 0.0f;
        if (P.hourglass_sts && hg) {
            const int s = sts_last;
            for (int64_t i = 0; i < n; ++i) { v[i] += (R(0.5) * dt) * acc[i]; hg_v_sync[i] = v[i]; }
            if (P.hg_sts_refresh) compute_velocity_gradient();
            hg_ke_pre = kinetic();
            for (int64_t i = 0; i < n; ++i) hg_yb[i] = v[i];
            if (!P.hg_sts_rkl) {
                R sub = R((double)dt / s);
                for (int st = 0; st < s; ++st) {
                    compute_hg_accel();
                    for (int64_t i = 0; i < n; ++i) hg_yb[i] = hg_yb[i] + sub * hg_a[i];
                }
            } else {
                // hourglass_sts, 'rkl' (SOLID.py:4541-4576): Y_j = mu Y_(j-1) + nu Y_(j-2)
                // + mu w1 dt M Y_(j-1), Y_0 = Y_1 = v, coefficients in double, then float
                std::vector<V3<R>> ya(hg_yb);
                const double w1 = 2.0 / (double)(s * s + s);
                for (int j = 1; j <= s; ++j) {
                    double mu = 1.0, nu = 0.0;
                    if (j > 1) { mu = (2.0 * j - 1.0) / j; nu = (1.0 - j) / j; }
                    const R muf = R(mu), nuf = R(nu), mut = R(mu * w1 * (double)dt);
                    compute_hg_accel();
                    for (int64_t i = 0; i < n; ++i) {
                        V3<R> y = (muf * hg_yb[i] + nuf * ya[i]) + mut * hg_a[i];
                        ya[i] = hg_yb[i];
                        hg_yb[i] = y;
                    }
                }
            }
            for (int64_t i = 0; i < n; ++i) v[i] = hg_yb[i];
            hg_work += hg_ke_pre - kinetic();
            R hh = R(0.5) * dt;
            double wsum = 0;
            for (int64_t i = 0; i < n; ++i) {
                V3<R> dvv = v[i] - hg_v_sync[i];
                wsum += (double)(m[i] * dot(dvv, hh * acc[i]));
                v[i] += hh * acc[i];
            }
            leftover_work += wsum;
            for (int64_t i = 0; i < n; ++i) displace(i, dt * v[i]);
        } else {
            for (int64_t i = 0; i < n; ++i) { v[i] += dt * acc[i]; displace(i, dt * v[i]); }
        }
    }

    // ------------------------------------------------------------ step (sph_base.py:622-655, DSPH.py:1854-1883)
    void substep() {
        compute_lam();
        compute_volume_evolution();
        compute_forces();
        compute_adaptive_dt();
        advect_and_work();
        if (P.pst_enabled) apply_pst();
    }
    void step() {
        if (P.is_solid) { step_solid(); return; }
        initialize_particle_system();
        substep();
        boundary();
    }
    void stage(int s) {
        if (P.is_solid) { stage_solid(s); return; }
        switch (s) {
            case SPH_STAGE_SORT: initialize_particle_system(); break;
            case SPH_STAGE_LAM: compute_lam(); break;
            case SPH_STAGE_CONTINUITY: compute_volume_evolution(); break;
            case SPH_STAGE_FORCES: compute_forces(); break;
            case SPH_STAGE_DT: compute_adaptive_dt(); break;
            case SPH_STAGE_ADVECT: advect_and_work(); break;
            case SPH_STAGE_PST: if (P.pst_enabled) apply_pst(); break;
            case SPH_STAGE_BOUNDARY: boundary(); break;
            default: break;
        }
    }

    int64_t pairs(int32_t* pi, int32_t* pj, int32_t* mr, int64_t cap) const {
        int64_t k = 0;
        for (int64_t i = 0; i < n; ++i)
            for_all_neighbors(i, [&](int64_t j, int mir) {
                if (k < cap) { pi[k] = (int32_t)i; pj[k] = (int32_t)j; mr[k] = mir; }
                ++k;
            });
        return k;
    }
};

// Interface state: every array crosses as float64 (exact for float32 inputs).
struct OracleState {
    const double* x; const double* x0; const double* u; const double* v; const double* acc;
    const double* V; const double* V_lo; const double* m; const double* pressure;
    const double* pst_shift; const int32_t* pid;
    // solid (may be NULL for a fluid)
    const double* sdev; const double* eps_p; const double* e_int; const double* temperature;
    const double* de_int; const int32_t* bc_flag; const int32_t* bc_id; const double* bc_disp;
    const int32_t* eos_id;
};
struct OracleOut {
    double* x; double* x0; double* u; double* v; double* acc;
    double* V; double* V_lo; double* m; double* pressure; double* pst_shift; int32_t* pid;
    double* lam; double* L_sym; double* lam_grad; double* divergence; double* de_visc;
    double* sdev; double* eps_p; double* e_int; double* temperature; double* de_int;
    int32_t* bc_flag; double* grad_v;
};

struct Handle {
    int fp64;
    Sim<float> f;
    Sim<double> d;
};

template <class R> void put(Sim<R>& s, const OracleState* st) {
    for (int64_t i = 0; i < s.n; ++i) {
        for (int k = 0; k < 3; ++k) {
            s.x[i][k] = (R)st->x[3 * i + k];
            s.x0[i][k] = (R)st->x0[3 * i + k];
            s.u[i][k] = (R)st->u[3 * i + k];
            s.v[i][k] = (R)st->v[3 * i + k];
            s.acc[i][k] = st->acc ? (R)st->acc[3 * i + k] : R(0);
            s.pst_shift[i][k] = (R)st->pst_shift[3 * i + k];
        }
        s.V[i] = (R)st->V[i]; s.V_lo[i] = (R)st->V_lo[i]; s.m[i] = (R)st->m[i];
        s.pressure[i] = (R)st->pressure[i]; s.pid[i] = st->pid[i];
        if (s.P.is_solid && st->sdev) {
            const double* q = st->sdev + 6 * i;
            M3<R> S;
            S[0][0] = (R)q[0]; S[1][1] = (R)q[1]; S[2][2] = (R)q[2];
            S[0][1] = S[1][0] = (R)q[3]; S[0][2] = S[2][0] = (R)q[4]; S[1][2] = S[2][1] = (R)q[5];
            s.sdev[i] = S;
            s.eps_p[i] = (R)st->eps_p[i];
            s.e_int[i] = (R)st->e_int[i];
            s.temperature[i] = (R)st->temperature[i];
            s.de_int[i] = st->de_int ? (R)st->de_int[i] : R(0);
            s.bc_flag[i] = st->bc_flag[i];
            s.bc_id[i] = st->bc_id[i];
            s.eos_id[i] = st->eos_id[i];
            for (int k = 0; k < 3; ++k) s.bc_disp[i][k] = (R)st->bc_disp[3 * i + k];
        }
    }
}
template <class R> void get(const Sim<R>& s, OracleOut* o) {
    for (int64_t i = 0; i < s.n; ++i) {
        for (int k = 0; k < 3; ++k) {
            if (o->x) o->x[3 * i + k] = s.x[i][k];
            if (o->x0) o->x0[3 * i + k] = s.x0[i][k];
            if (o->u) o->u[3 * i + k] = s.u[i][k];
            if (o->v) o->v[3 * i + k] = s.v[i][k];
            if (o->acc) o->acc[3 * i + k] = s.acc[i][k];
            if (o->pst_shift) o->pst_shift[3 * i + k] = s.pst_shift[i][k];
            if (o->lam_grad) o->lam_grad[3 * i + k] = s.lam_grad[i][k];
        }
        if (o->V) o->V[i] = s.V[i];
        if (o->V_lo) o->V_lo[i] = s.V_lo[i];
        if (o->m) o->m[i] = s.m[i];
        if (o->pressure) o->pressure[i] = s.pressure[i];
        if (o->pid) o->pid[i] = s.pid[i];
        if (o->lam) o->lam[i] = s.lam[i];
        if (o->divergence) o->divergence[i] = s.divergence[i];
        if (o->de_visc) o->de_visc[i] = s.de_visc[i];
        if (o->L_sym) for (int k = 0; k < 6; ++k) o->L_sym[6 * i + k] = s.L_sym[i][k];
        if (s.P.is_solid) {
            const M3<R>& S = s.sdev[i];
            if (o->sdev) {
                double* q = o->sdev + 6 * i;
                q[0] = S[0][0]; q[1] = S[1][1]; q[2] = S[2][2]; q[3] = S[0][1]; q[4] = S[0][2]; q[5] = S[1][2];
            }
            if (o->eps_p) o->eps_p[i] = s.eps_p[i];
            if (o->e_int) o->e_int[i] = s.e_int[i];
            if (o->temperature) o->temperature[i] = s.temperature[i];
            if (o->de_int) o->de_int[i] = s.de_int[i];
            if (o->bc_flag) o->bc_flag[i] = s.bc_flag[i];
            if (o->grad_v) for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) o->grad_v[9 * i + 3 * a + b] = s.grad_v[i][a][b];
        }
    }
}

}  // namespace

extern "C" {

void* orc_create(const SphParams* p, int64_t n, int fp64) {
    auto* h = new Handle();
    h->fp64 = fp64;
    if (fp64) h->d.setup(*p, n); else h->f.setup(*p, n);
    return h;
}
void orc_destroy(void* hp) { delete (Handle*)hp; }
void orc_set_threads(int nt) { if (nt > 0) omp_set_num_threads(nt); }
int orc_max_threads(void) { return omp_get_max_threads(); }
void orc_set_state(void* hp, const OracleState* st) {
    auto* h = (Handle*)hp;
    if (h->fp64) put(h->d, st); else put(h->f, st);
}
void orc_get_state(void* hp, OracleOut* o) {
    auto* h = (Handle*)hp;
    if (h->fp64) get(h->d, o); else get(h->f, o);
}
void orc_set_dt(void* hp, double dt) {
    auto* h = (Handle*)hp;
    if (h->fp64) h->d.dt = dt; else h->f.dt = (float)dt;
}
// scalars: dt, max_c_sq, max_accel, max_v, off_grid_num, off_grid_mass, wall, visc, diff, leftover
void orc_get_scalars(void* hp, double* out) {
    auto* h = (Handle*)hp;
    auto fill = [&](auto& s) {
        out[0] = s.dt; out[1] = s.max_c_sq; out[2] = s.max_accel; out[3] = s.max_v;
        out[4] = s.off_grid_num; out[5] = s.off_grid_mass; out[6] = s.wall_work;
        out[7] = s.visc_work; out[8] = s.diff_work; out[9] = s.leftover_work;
        out[10] = s.sim_time; out[11] = s.plastic_work; out[12] = s.hg_work;
        out[13] = s.load_s; out[14] = s.load_sdot; out[15] = s.sts_last;
        for (int k = 0; k < 8; ++k)
            for (int d = 0; d < 3; ++d) {
                out[16 + 3 * k + d] = s.constraint_force[k][d];
                out[40 + 3 * k + d] = s.constraint_disp[k][d];
            }
    };
    if (h->fp64) fill(h->d); else fill(h->f);
}
void orc_step(void* hp, int nsteps) {
    auto* h = (Handle*)hp;
    for (int k = 0; k < nsteps; ++k) { if (h->fp64) h->d.step(); else h->f.step(); }
}
void orc_stage(void* hp, int s) {
    auto* h = (Handle*)hp;
    if (h->fp64) h->d.stage(s); else h->f.stage(s);
}
int64_t orc_pairs(void* hp, int32_t* pi, int32_t* pj, int32_t* mr, int64_t cap) {
    auto* h = (Handle*)hp;
    return h->fp64 ? h->d.pairs(pi, pj, mr, cap) : h->f.pairs(pi, pj, mr, cap);
}
// Restated 3x3 eigensolver and regularised inverse, exposed for the eigen tests.
void orc_sym_eig3(const double* A, double* ev, double* Q) {
    M3<double> M, QQ;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = A[3 * i + j];
    sym_eig3(M, ev, QQ);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[3 * i + j] = QQ[i][j];
}
void orc_sym_eig3_f32(const float* A, float* ev, float* Q) {
    M3<float> M, QQ;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = A[3 * i + j];
    sym_eig3(M, ev, QQ);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[3 * i + j] = QQ[i][j];
}
// Return maps on one deviator (row-major 3x3), for the known-answer tests.
double orc_j2_return(const double* s_in, double G, double sy, double H, double ep, double* s_out) {
    M3<double> s;
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s[a][b] = s_in[3 * a + b];
    double d = Sim<double>::j2_return(s, G, sy, H, ep);
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s_out[3 * a + b] = s[a][b];
    return d;
}
double orc_jc_return(const double* s_in, const double* k11, double ep, double temp, double dt,
                     double* s_out, int* iters) {
    // k11 = {G, A, B, n, C, eps0_dot, T0, Tm, m}
    M3<double> s;
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s[a][b] = s_in[3 * a + b];
    double d = Sim<double>::jc_return_of(s, k11[0], k11[1], k11[2], k11[3], k11[4], k11[5],
                                         k11[6], k11[7], k11[8], ep, temp, dt, iters);
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s_out[3 * a + b] = s[a][b];
    return d;
}
void orc_spd_inverse3(const double* E, double tol, double* L) {
    M3<double> M;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = E[3 * i + j];
    M3<double> R = spd_inverse_3x3(M, tol);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) L[3 * i + j] = R[i][j];
}
}

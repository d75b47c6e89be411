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
    }

    void initialize_particle_system() {
        // update_grid_id (:1300-1318)
        std::fill(gpn.begin(), gpn.end(), 0);
        off_grid_num = 0;
        off_grid_mass = 0;
        for (int64_t i = 0; i < n; ++i) {
            int32_t g = (int32_t)T;
            auto c = pos_to_index(x[i]);
            cell_id[i] = c;
            if (on_grid(x[i])) g = hash_cell(c);
            else { off_grid_num += 1; off_grid_mass += (double)m[i]; }
            grid_ids[i] = g;
            gpn[g] += 1;
        }
        gpn_temp = gpn;
        // PrefixSumExecutor (inclusive)
        for (int64_t b = 1; b <= T; ++b) gpn[b] += gpn[b - 1];
        // counting_sort (:1320-1340), executed serially so the order is reproducible
        for (int64_t i = 0; i < n; ++i) {
            int64_t I = n - 1 - i;
            int32_t g = grid_ids[I];
            int32_t base = (g - 1 >= 0) ? gpn[g - 1] : 0;
            gpn_temp[g] -= 1;
            grid_ids_new[I] = gpn_temp[g] + base;
        }
        for_each_sorted([&](auto& fld) {
            auto tmp = fld;
            for (int64_t i = 0; i < n; ++i) tmp[grid_ids_new[i]] = fld[i];
            fld.swap(tmp);
        });
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
                if (P.delta_sph > 0.0f) {
                    R rn2 = dot(r, r);
                    R a2 = R(2) * (rho_j - rho_i);
                    R den = rn2 + eta2;
                    V3<R> psi = {a2 * (-r[0]) / den, a2 * (-r[1]) / den, a2 * (-r[2]) / den};
                    R diffusion = coef * w(j) * dot(psi, g);
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
        for (int64_t i = 0; i < n; ++i) acc[i] = {R(P.gravity[0]), R(P.gravity[1]), R(P.gravity[2])};
        for (int64_t i = 0; i < n; ++i) {
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
        for (int64_t i = 0; i < n; ++i) {
            V3<R> f = acc[i] - g;
            wl += (double)(R(0.5) * m[i] * dtl * dtl * (dot(f, f) - gsq));
            if (P.track_visc_work) wv += (double)m[i] * (double)de_visc[i];
        }
        visc_work += (double)dtl * wv;
        leftover_work += wl;
        for (int64_t i = 0; i < n; ++i) {
            v[i] += dtl * acc[i];
            displace(i, dtl * v[i]);
        }
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
        return dr;
    }
    void apply_pst() {
        if (P.pst_ma_mode == 1) {
            R mv = 0;
            for (int64_t i = 0; i < n; ++i) if (on_grid(x[i])) mv = std::max(mv, norm(v[i]));
            max_v = mv;
        }
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i) {
            V3<R> s;
            for_all_neighbors(i, [&](int64_t j, int mir) { s += pst_pair(i, j, mir); });
            R Ma;
            if (P.pst_ma_mode == 2) Ma = R(P.pst_ma_fixed);
            else {
                R vref = P.pst_ma_mode == 1 ? max_v : norm(v[i]);
                Ma = vref / R(P.c0);
            }
            V3<R> dr;
            if (P.pst_colle) {
                R c = R(-2.0 * (double)P.support_radius) * R(P.c0) * Ma;
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
        for (int64_t i = 0; i < n; ++i) displace(i, pst_shift[i]);
    }

    // ------------------------------------------------------------ boundary (sph_base.py:160-655)
    void simulate_collisions(int64_t i, const V3<R>& nv) {
        R vn = dot(v[i], nv);
        if (vn > R(0)) {
            R c = R(P.wall_restitution);
            wall_work += (double)(R(0.5) * m[i] * vn * vn * R(1.0 - (double)P.wall_restitution * P.wall_restitution));
            v[i] -= (R(1.0 + (double)c) * vn) * nv;
        }
    }
    void enforce_walls(int faces) {  // faces: bit0 x, bit1 y-low, bit2 y-high, bit3 z
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
            if (cl > R(1e-6)) simulate_collisions(i, {cn[0] / cl, cn[1] / cl, cn[2] / cl});
        }
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
                }
            }
            if (P.walls) enforce_walls(1 | 4);
        } else {
            if (P.sym_y || P.sym_z) {
                for (int64_t i = 0; i < n; ++i) {
                    if (P.sym_y && x[i][1] < R(0)) { reflect_component(i, 1); v[i][1] = -v[i][1]; acc[i][1] = -acc[i][1]; }
                    if (P.sym_z && x[i][2] < R(0)) { reflect_component(i, 2); v[i][2] = -v[i][2]; acc[i][2] = -acc[i][2]; }
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
        initialize_particle_system();
        substep();
        boundary();
    }
    void stage(int s) {
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
};
struct OracleOut {
    double* x; double* x0; double* u; double* v; double* acc;
    double* V; double* V_lo; double* m; double* pressure; double* pst_shift; int32_t* pid;
    double* lam; double* L_sym; double* lam_grad; double* divergence; double* de_visc;
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
void orc_spd_inverse3(const double* E, double tol, double* L) {
    M3<double> M;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = E[3 * i + j];
    M3<double> R = spd_inverse_3x3(M, tol);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) L[3 * i + j] = R[i][j];
}
}

// sph_host.cuh -- host-side derivation of the kernel constants (Cst) from SphParams,
// shared by the handle-based entry points and the handle-free one.
#pragma once
#include <cmath>

#include "sph_device.cuh"

namespace sph {

// Smallest float t with sqrtf(t) >= h, so |r| < h  <=>  |r|^2 < t for the rounded |r|^2
// (sqrt rounded to nearest is monotone, so the set {d2 : sqrt(d2) < h} is an interval).
inline float d2_threshold(float h) {
    float t = (float)((double)h * (double)h);
    for (int k = 0; k < 64 && std::sqrt(std::nextafter(t, 0.0f)) >= h; ++k) t = std::nextafter(t, 0.0f);
    for (int k = 0; k < 64 && std::sqrt(t) < h; ++k) t = std::nextafter(t, INFINITY);
    return t;
}

// Constants the reference folds into its kernels at compile time (sph_base.py:42-151,
// DSPH.py, SOLID.py), computed in double and rounded once, as Python folds them.
inline void fill_constants_from(const SphParams& p, int64_t n, Cst& c) {
    c.p = p;
    c.n = (int)n;
    c.n_inst = 0;
    c.any_plastic = 0;
    c.all_gamma_one = 1;
    c.any_jc = 0;
    c.one_material = p.n_materials <= 1;
    c.block = kBlock;
    // skin of the candidate lists: a tenth of the support.  The squared cut is rounded up
    // so that it holds every pair a float32 distance test could place within h + skin;
    // the bound keeps 2 dlim a thousandth of the skin short of it, far beyond the
    // rounding of the displacement, distance and coarse-cell computations.
    {
        const double hs = p.support_radius;
        c.skin = (float)(0.1 * hs);
        c.hc = (float)(1.1 * hs);
        c.dlim = (float)(0.05 * hs * (1.0 - 1e-3));
        c.d2_skin = (float)((1.1 * hs) * (1.1 * hs) * (1.0 + 1e-5));
        c.d2_deep = (float)((0.9 * hs) * (0.9 * hs) * (1.0 - 1e-5));
    }
    double hd = p.support_radius;
    double al = p.two_d ? 7.0 / (M_PI * hd * hd) : 21.0 / (2.0 * M_PI * hd * hd * hd);
    c.h = (float)hd;
    c.inv_h = (float)(1.0 / hd);
    c.alpha = (float)al;
    c.kgrad = (float)(20.0 * al / hd);
    c.eta2 = (float)(0.01 * hd * hd);
    {
        float r = p.particle_diameter, q = r / c.h;
        float W = 0.0f;
        if (q < 1.0f) { float t = 1.0f - q; float t2 = t * t; W = c.alpha * (t2 * t2) * (4.0f * q + 1.0f); }
        c.W_dx0 = W;
    }
    c.d2_lt = d2_threshold(c.h);
    c.visc_coef = (float)(10.0 * (double)p.viscosity);
    c.delta_coef = p.delta_sph * c.h * p.c0;
    c.cfl_h = (float)((double)p.CFL * (double)p.support_radius);
    for (int k = 0; k < 3; ++k) c.wall_hi[k] = (float)((double)p.domain_size[k] - (double)p.padding);
    c.rest_1p = (float)(1.0 + (double)p.wall_restitution);
    c.rest_loss = (float)(1.0 - (double)p.wall_restitution * (double)p.wall_restitution);
    c.max_shift = (float)((double)p.pst_max_shift * (double)p.particle_diameter);
    c.colle_coef = (float)(-2.0 * (double)p.support_radius);
    c.sun_coef = -p.CFL;
    c.mirror_y = (p.axisymmetric || p.sym_y) ? 1 : 0;
    c.mirror_z = p.sym_z ? 1 : 0;
}

}  // namespace sph

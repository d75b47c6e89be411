"""Solid-solver constants of SphParams (SOLID.py HypoElasticSolver.__init__,
SOLID.py:138-1452): per-material tables in declaration order, the hourglass damper's
rate and lattice kernel sum, the dt pair mode, the grip ramp."""
from __future__ import annotations

import math

import numpy as np

from .materials import PLASTIC_JOHNSON_COOK


def wendland_scalar(r, h, two_d):
    """W(r) in float64 (SOLID.py:1705-1716)."""
    alpha = 7.0 / (math.pi * h * h) if two_d else 21.0 / (2.0 * math.pi * h ** 3)
    q = r / h
    return alpha * (1.0 - q) ** 4 * (4.0 * q + 1.0) if q < 1.0 else 0.0


def reference_kernel_sum(dx0, h, two_d):
    """S = sum_j W(|r_j|) / W(dx0) over the lattice around a particle (SOLID.py:1632-1657):
    6.64 at 3 dx0 in a single layer, 15.41 in 3D."""
    reach = int(math.ceil(h / dx0))
    w_ref = wendland_scalar(dx0, h, two_d)
    if w_ref <= 0.0:
        return 1.0
    total = 0.0
    span = range(-reach, reach + 1)
    cells = ([(i, j, 0) for i in span for j in span] if two_d else
             [(i, j, k) for i in span for j in span for k in span])
    for c in cells:
        r = dx0 * math.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2)
        if r > 0.0:
            total += wendland_scalar(r, h, two_d)
    return total / w_ref


def fill_solid_params(ps, p):
    cfg = ps.cfg
    g = cfg.get_cfg
    mats = sorted(cfg.get_materials().values(), key=lambda m: m.index)
    if not 1 <= len(mats) <= 4:
        raise ValueError("the solid path takes 1 to 4 materials")
    p.n_materials = len(mats)
    for k, m in enumerate(mats):
        p.mat_rho0[k] = m.rho0
        p.mat_K[k] = m.K
        p.mat_G[k] = m.G
        p.mat_cp[k] = m.c_p
        p.mat_c0[k] = m.c_eos
        p.mat_delta[k] = m.delta
        p.mat_cv[k] = m.specific_heat
        p.mat_stiff[k] = m.stiffness
        p.mat_gamma[k] = m.exponent
        p.plastic_kind[k] = int(m.plastic_kind)
        p.plastic_sy0[k] = m.sigma_y0
        p.plastic_H[k] = m.hardening
        p.mat_T0[k] = m.jc["T0"] if m.plastic_kind == PLASTIC_JOHNSON_COOK else 293.0
        if m.jc is not None:
            p.jc_A[k], p.jc_B[k], p.jc_n[k] = m.jc["A"], m.jc["B"], m.jc["n"]
            p.jc_C[k], p.jc_eps0_dot[k] = m.jc["C"], m.jc["eps0_dot"]
            p.jc_T0[k], p.jc_Tm[k] = m.jc["T0"], m.jc["Tm"]
            p.jc_m[k], p.jc_chi[k] = m.jc["m"], m.jc["chi"]
    c_p = max(m.c_p for m in mats)
    p.c_signal = c_p
    # SOLID.py:222-245: do the materials differ in acoustic impedance rho0 c_p (the
    # damper's pair force) or in EOS sound speed (the delta-SPH and Colle coefficients)?
    # Compared as the reference compares them, on the resolved double-precision values.
    p.hg_mixed_impedance = int(len({m.rho0 * m.c_p for m in mats}) > 1)
    p.c0_mixed = int(len({m.c_eos for m in mats}) > 1)
    p.delta_pairs_all = int(str(g("DELTA_PAIRS") or "samematerial").lower() != "samematerial")
    mode = str(g("DT_PAIR_SOUND_SPEED") or "samematerial").lower()
    p.dt_pair_mode = {"off": 0, "all": 1, "samematerial": 2}[mode]
    p.kernel_correction = int(bool(g("KERNEL_CORRECTION")))
    tol = g("L_EIG_TOL")
    p.l_eig_tol = 0.1 if tol is None else float(tol)
    # Domain.conservativeAxialMomentum (default on) and axialImageRadius (SOLID.py:262-315)
    cx = g("AXI_CONSERVATIVE_X")
    p.axi_conservative_x = int(bool(ps.axisymmetric) and (True if cx is None else bool(cx)))
    p.axi_conservative_r = int(bool(ps.axisymmetric) and bool(g("AXI_CONSERVATIVE_R")))
    p.axi_image_signed = int(bool(p.axi_conservative_x)
                             and str(g("AXI_IMAGE_RADIUS") or "ring").lower() == "signed")
    dx0 = ps.particle_diameter
    h = ps.support_radius
    p.hourglass_alpha = float(g("HOURGLASS_ALPHA") or 0.0)
    p.hourglass_sts = int(bool(g("HOURGLASS_STS")))
    p.hourglass_sts_cap = 32
    sf = g("HOURGLASS_STS_SAFETY")
    p.hourglass_sts_safety = 0.8 if sf is None else float(sf)
    p.objective_none = int(str(g("OBJECTIVE_RATE") or "jaumann").lower() == "none")
    p.hg_sts_rkl = int(str(g("HOURGLASS_STS_MODE") or "subcycle").lower() == "rkl")
    p.hg_sts_fixed = int(g("HOURGLASS_STS_STAGES") or 0)
    rg = g("HOURGLASS_STS_REFRESH")
    p.hg_sts_refresh = int(True if rg is None else bool(rg))
    p.hg_S = reference_kernel_sum(dx0, h, ps.two_d)
    p.hg_W_dx0 = wendland_scalar(dx0, h, ps.two_d)
    ratio_max = (1.0 + h / (2.0 * ps.axi_r_min)
                 if (p.axi_conservative_x or p.axi_conservative_r) else 1.0)
    p.hg_rate = (p.hourglass_alpha * c_p / ps.h_min * reference_kernel_sum(dx0, h, ps.two_d)
                 * ratio_max) if p.hourglass_alpha > 0.0 else 0.0
    hist = g("PST_ALE_HISTORY")
    p.ale_history = int((True if hist is None else bool(hist)) and bool(g("PST_ENABLED")))
    p.transport_e = p.ale_history
    d = g("PST_ALE_DIFFUSION")
    p.ale_diffusion = 1.0 if d is None else float(d)
    p.num_constraints = len(cfg.get_constraints())
    if p.num_constraints > 8:
        raise ValueError("at most 8 constraints")
    p.ramp_time = float(g("rampTime") or 0.0)
    p.jc_surrogate = 0
    p.jc_surrogate_tol = 1e-3
    # the in-loop viscosities (SOLID.py:667-716): q = C_Q l^2 rho (div v)^2 under
    # compression, added to the pressure of the stress pair; Monaghan's Pi_ij on
    # approaching pairs; C_Q l^2 and C_Q l folded in double as the reference folds them
    q_bulk = float(g("BULK_VISCOSITY_Q") or 0.0)
    q_len = str(g("BULK_VISCOSITY_LENGTH") or "dx0").lower()
    q_length = float(dx0 if q_len == "dx0" else h)
    p.q_l2 = q_bulk * q_length ** 2
    p.q_cl = q_bulk * q_length
    p.av_alpha = float(g("MONAGHAN_ALPHA") or 0.0)
    p.av_beta = float(g("MONAGHAN_BETA") or 0.0)
    eps = g("MONAGHAN_EPS")
    p.av_eps = 0.01 if eps is None else float(eps)
    av_on = p.av_alpha > 0.0 or p.av_beta > 0.0
    # the solid's viscous work: Morris and Monaghan, not q (SOLID.py:1255-1264)
    track = g("TRACK_VISCOUS_WORK")
    p.track_visc_work = int((True if track is None else bool(track))
                            and (float(g("viscosity")) > 0.0 or av_on))

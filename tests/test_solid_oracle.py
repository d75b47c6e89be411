"""The solid half of the CPU oracle against the reference's known answers (no GPU):
the J2 and Johnson-Cook return maps against the reference's own float64 mirrors
(tests/golden/make_golden.py), the hourglass lattice constant, and conservation
properties of the oracle's solid step."""
import json
import os

import numpy as np
import pytest

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import scene_path
from sigmasph_b200.solid_params import reference_kernel_sum
from sigmasph_b200.solver import build_params
from oracle.oracle import Oracle, state_from_sets, j2_return, jc_return

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_host.json")))


def vm(s):
    s = np.asarray(s)
    return float(np.sqrt(1.5 * np.sum(s * s)))


@pytest.mark.parametrize("k", range(len(GOLD["plasticity"]["j2"])))
def test_j2_return_matches_reference(k):
    """MAT001_linear_plasticity.py:65-81 (j2_radial_return_py)."""
    e = GOLD["plasticity"]["j2"][k]
    s_new, d = j2_return(e["s"], e["G"], e["sy0"], e["H"], e["eps_p"])
    s_ref, d_ref = np.array(e["out"][0]), e["out"][1]
    assert d == pytest.approx(d_ref, rel=1e-12, abs=1e-15)
    assert np.abs(s_new - s_ref).max() <= 1e-12 * np.abs(s_ref).max()
    if d > 0:   # consistency: the returned state sits on the hardened yield surface
        assert vm(s_new) == pytest.approx(e["sy0"] + e["H"] * (e["eps_p"] + d), rel=1e-12)


@pytest.mark.parametrize("k", range(len(GOLD["plasticity"]["jc"])))
def test_jc_return_matches_reference(k):
    """MAT002_johnson_cook.py:172-250 (jc_radial_return_py): bracketed Newton-bisection,
    40 iterations at most, T* frozen at the step start."""
    e = GOLD["plasticity"]["jc"][k]
    (s, G, rho0, A, B, n, C, e0d, T0, Tm, m, Cp, chi, ep, temp, dt) = e["args"]
    s_new, d, it = jc_return(s, G, A, B, n, C, e0d, T0, Tm, m, ep, temp, dt)
    s_ref, d_ref = np.array(e["out"][0]), e["out"][1]
    assert it < 40
    assert d == pytest.approx(d_ref, rel=1e-12, abs=1e-15)
    assert np.abs(s_new - s_ref).max() <= 1e-12 * max(np.abs(s_ref).max(), 1e-30)


def test_jc_return_is_elastic_below_yield():
    s = np.diag([0.1, -0.05, -0.05])
    s_new, d, _ = jc_return(s, 76.92, 0.31, 1.0, 0.65, 0.02, 1.0, 293.0, 1720.0, 1.0, 0.0, 293.0, 1e-5)
    assert d == 0.0 and np.array_equal(s_new, s)


@pytest.mark.parametrize("two_d,expect", [(True, 6.639), (False, 15.413)])
def test_hourglass_lattice_sum(two_d, expect):
    """SOLID.py:1632-1657: S = sum_j W(|r_j|) / W(dx0) at support 3 dx0 (6.6 in plane
    strain, SOLID.py:763); scale-free in dx0."""
    assert reference_kernel_sum(0.1, 0.3, two_d) == pytest.approx(expect, abs=1e-3)
    assert reference_kernel_sum(2.0, 6.0, two_d) == pytest.approx(expect, abs=1e-3)


def test_dogbone_params():
    ps = ParticleSystem(SimConfig(scene_path("tensile_axi_dogbone_dx0.1.json")), device="cpu")
    p = build_params(ps)
    assert p.is_solid and p.axisymmetric and p.hourglass_sts
    assert p.hg_S == pytest.approx(6.639, abs=2e-3)
    assert p.num_constraints == 2
    # the signal speed is the dilatational speed of stainless steel (E 193 GPa, nu 0.3)
    E, nu, rho = 193.0, 0.3, 7.9e-6
    K, G = E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu))
    assert p.c_signal == pytest.approx(np.sqrt((K + 4 * G / 3) / rho), rel=1e-6)


def free_block(dx=0.5):
    """A free 3D elastic-plastic block (no grips, no gravity) with a random velocity
    field: the pair forces are antisymmetric, so linear momentum is conserved."""
    return {
        "Domain": {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "boundary": "open"},
        "Time": {"CFL": 0.3},
        "Solver": {"type": "hypoElastic", "viscosity": 0.02, "allowNegativePressure": True},
        "Materials": [{"name": "steel", "density0": 7.9e-6, "eos": {"type": "linear"},
                       "strength": {"type": "hypoElastic", "youngsModulus": 200.0,
                                    "poissonRatio": 0.3,
                                    "plasticity": {"model": "linear", "yieldStress": 0.03,
                                                   "hardeningModulus": 1.0}}}],
        "Load": {"gravitation": [0.0, 0.0, 0.0]},
        "Diffusion": {"delta": 0.1},
        "Shifting": {"enabled": False},
        "Hourglass": {"alpha": 4.0},
        "SolidBlocks": [{"objectId": 0, "start": [0.0, 0.0, 0.0], "end": [6.0, 6.0, 6.0],
                         "material": "steel", "density": 7.9e-6}],
    }


def test_free_block_conserves_momentum():
    ps = ParticleSystem(SimConfig(free_block()), device="cpu")
    rng = np.random.default_rng(3)
    n = ps.particle_max_num
    ps.v.from_numpy(rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32))
    p = build_params(ps)
    o = Oracle(p, n, fp64=True)
    st = state_from_sets(ps.state_numpy())
    o.set_state(st, p.CFL * p.support_radius / p.c_signal)
    m = st["m"].astype(np.float64)
    P0 = (m[:, None] * st["v"].astype(np.float64)).sum(0)
    o.stage(abi.STAGE_SORT)
    o.step(20)
    r = o.get_state()
    P1 = (r["m"][:, None] * r["v"]).sum(0)
    gross = (r["m"][:, None] * np.abs(r["v"])).sum(0)
    assert np.abs(P1 - P0).max() <= 1e-10 * gross.max()
    assert r["eps_p"].max() > 0.0       # the random field yields somewhere


ALUMINIUM = {"name": "aluminium", "density0": 2.7e-6, "eos": {"type": "linear"},
             "strength": {"type": "hypoElastic", "youngsModulus": 70.0, "poissonRatio": 0.33,
                          "plasticity": {"model": "linear", "yieldStress": 0.02,
                                         "hardeningModulus": 0.5}}}


def two_material_block(dx=0.5, pairs="samematerial"):
    """The free block as two materials, steel below y = 3 and aluminium above: their EOS
    sound speeds and their acoustic impedances rho0 c_p differ."""
    sc = free_block(dx)
    sc["Materials"].append(ALUMINIUM)
    sc["Diffusion"]["pairs"] = pairs
    sc["SolidBlocks"] = [
        {"objectId": 0, "start": [0.0, 0.0, 0.0], "end": [6.0, 2.9, 6.0], "material": "steel",
         "density": 7.9e-6},
        {"objectId": 1, "start": [0.0, 3.0, 0.0], "end": [6.0, 6.0, 6.0], "material": "aluminium",
         "density": 2.7e-6}]
    return sc


def test_two_materials_set_the_mixed_flags():
    """SOLID.py:222-245: c0_mixed when the EOS speeds differ, hg_mixed_impedance when
    rho0 c_p differ; Diffusion.pairs "all" lets the diffusion cross the interface."""
    p1 = build_params(ParticleSystem(SimConfig(free_block()), device="cpu"))
    assert (p1.c0_mixed, p1.hg_mixed_impedance, p1.delta_pairs_all) == (0, 0, 0)
    ps = ParticleSystem(SimConfig(two_material_block(pairs="all")), device="cpu")
    p2 = build_params(ps)
    assert (p2.n_materials, p2.c0_mixed, p2.hg_mixed_impedance, p2.delta_pairs_all) == (2, 1, 1, 1)
    assert sorted(set(np.rint(ps.state_numpy()["bcdisp"][:, 3]).astype(int))) == [0, 1]
    from sigmasph_b200.config import SceneError
    sc = two_material_block()
    sc["Diffusion"]["pairs"] = "some"
    with pytest.raises(SceneError):
        SimConfig(sc)


@pytest.mark.parametrize("ratio", [True, False], ids=["impedance_ratio", "own_impedance"])
def test_two_material_damper_conserves_momentum(ratio):
    """_hg_impedance_ratio (SOLID.py:4184-4239): the in-loop damper's pair force carries
    rho0 c_p; with the pair's harmonic mean (2 Z_j / (Z_i + Z_j) on particle i's own) it is
    antisymmetric across the steel/aluminium interface and the free two-material block
    conserves momentum to round-off; with each particle's own impedance it does not.  The
    Morris viscosity is off: its pair term m_i w_j (...) is antisymmetric only between
    particles of one density, so across the interface it moves momentum by construction
    in the reference too."""
    sc = two_material_block()
    sc["Solver"]["viscosity"] = 0.0
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    rng = np.random.default_rng(4)
    n = ps.particle_max_num
    ps.v.from_numpy(rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32))
    p = build_params(ps)
    p.hg_mixed_impedance = int(ratio)
    o = Oracle(p, n, fp64=True)
    st = state_from_sets(ps.state_numpy())
    o.set_state(st, p.CFL * p.support_radius / p.c_signal)
    m = st["m"].astype(np.float64)
    P0 = (m[:, None] * st["v"].astype(np.float64)).sum(0)
    o.stage(abi.STAGE_SORT)
    o.step(10)
    r = o.get_state()
    P1 = (r["m"][:, None] * r["v"]).sum(0)
    gross = (r["m"][:, None] * np.abs(r["v"])).sum(0)
    drift = np.abs(P1 - P0).max() / gross.max()
    if ratio:
        assert drift <= 1e-10, drift
    else:
        assert drift > 1e-6, drift


def test_mlp_oracle_gradient_matches_finite_differences():
    """The float64 surrogate-MLP oracle (the checker of the GPU training kernels):
    analytic gradient against central differences."""
    from oracle import mlp
    rng = np.random.default_rng(5)
    w = rng.normal(0.0, 0.3, mlp.N_PARAMS)
    X = rng.uniform(0.0, 1.0, (7, 4))
    T = rng.uniform(0.5, 1.0, 7)
    _, g = mlp.loss_and_grad(w, X, T)
    idx = rng.choice(mlp.N_PARAMS, 40, replace=False)
    for q in idx:
        e = np.zeros_like(w)
        e[q] = 1e-6
        fd = (mlp.loss_and_grad(w + e, X, T)[0] - mlp.loss_and_grad(w - e, X, T)[0]) / 2e-6
        assert fd == pytest.approx(g[q], rel=1e-5, abs=1e-9)


def _viscous(sc, q=1.5, alpha=1.0, beta=2.0):
    sc["Solver"]["bulkViscosity"] = {"quadratic": q}
    sc["Solver"]["artificialViscosity"] = {"alpha": alpha, "beta": beta}
    return sc


def _forces(sc, v_of_x, fp64=True):
    """The oracle's force stage on a free block with velocities v_of_x(x)."""
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    x = ps.x.to_numpy().astype(np.float64)
    ps.v.from_numpy(v_of_x(x).astype(np.float32))
    p = build_params(ps)
    o = Oracle(p, ps.particle_max_num, fp64=fp64)
    o.set_state(state_from_sets(ps.state_numpy()), p.CFL * p.support_radius / p.c_signal)
    for s in range(abi.STAGE_FORCES + 1):
        o.stage(s)
    return o, o.get_state()


def test_viscosities_conserve_momentum():
    """q enters the stress pair and Pi_ij is pair-symmetric against an antisymmetric
    grad W (SOLID.py:3560-3570, :3727-3766): a free block keeps its momentum."""
    ps = ParticleSystem(SimConfig(_viscous(free_block())), device="cpu")
    rng = np.random.default_rng(5)
    n = ps.particle_max_num
    ps.v.from_numpy(rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32))
    p = build_params(ps)
    assert p.q_l2 > 0 and p.av_alpha == 1.0 and p.track_visc_work == 1
    o = Oracle(p, n, fp64=True)
    st = state_from_sets(ps.state_numpy())
    o.set_state(st, p.CFL * p.support_radius / p.c_signal)
    m = st["m"].astype(np.float64)
    P0 = (m[:, None] * st["v"].astype(np.float64)).sum(0)
    o.stage(abi.STAGE_SORT)
    o.step(20)
    r = o.get_state()
    P1 = (r["m"][:, None] * r["v"]).sum(0)
    gross = (r["m"][:, None] * np.abs(r["v"])).sum(0)
    assert np.abs(P1 - P0).max() <= 1e-10 * gross.max()
    assert o.scalars()["visc_work"] < 0.0     # dissipation is booked negative


def test_viscous_work_conjugate_balances_the_power():
    """de_int carries the work conjugate of every pair force (stress with q, Morris,
    Pi_ij), so in 3D sum_i m_i (de_i + a_i . v_i) = 0 with no damper, gravity or ALE."""
    sc = _viscous(free_block())
    sc["Hourglass"] = {"alpha": 0.0}
    rng = np.random.default_rng(6)
    _, r = _forces(sc, lambda x: rng.uniform(-2.0, 2.0, x.shape))
    m = r["m"]
    pw = m * (r["acc"] * r["v"]).sum(1)
    assert np.abs((m * r["de_int"] + pw).sum()) <= 1e-10 * np.abs(pw).sum()


def test_viscosities_act_only_under_compression():
    """Under a uniform expansion every pair separates and div v > 0: q and Pi_ij vanish
    and the accelerations are the plain deck's.  Under the same compression both act."""
    base = free_block()
    base["Hourglass"] = {"alpha": 0.0}
    c = np.array([3.0, 3.0, 3.0])
    for sign, same in ((1.0, True), (-1.0, False)):
        _, r0 = _forces(base, lambda x: sign * 0.5 * (x - c))
        _, r1 = _forces(_viscous(json.loads(json.dumps(base))), lambda x: sign * 0.5 * (x - c))
        d = np.abs(r1["acc"] - r0["acc"]).max()
        if same:
            assert d == 0.0
        else:
            assert d > 1e-3 * np.abs(r0["acc"]).max()


@pytest.mark.parametrize("mode", ["subcycle", "rkl"])
def test_sts_carries_a_rigid_translation(mode):
    """The sub-cycled damper annihilates only what the linear velocity field does not
    explain; under RKL1 each stage's mu + nu = 1 carries the null space through
    (SOLID.py:4493-4502).  A free block translating rigidly keeps its velocity through
    several steps of s > 1 stages."""
    sc = free_block()
    sc["Hourglass"] = {"alpha": 4.0, "superTimeStepping": {"mode": mode}}
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    n = ps.particle_max_num
    v0 = np.array([1.0, 0.5, -0.3], np.float32)
    ps.v.from_numpy(np.tile(v0, (n, 1)))
    p = build_params(ps)
    assert p.hg_sts_rkl == (mode == "rkl")
    o = Oracle(p, n, fp64=False)
    o.set_state(state_from_sets(ps.state_numpy()), p.CFL * p.support_radius / p.c_signal)
    o.stage(abi.STAGE_SORT)
    o.step(5)
    assert o.scalars()["sts_stages"] > 1
    r = o.get_state()
    assert np.abs(r["v"] - v0).max() <= 1e-5 * np.abs(v0).max()


def test_objective_rate_none_drops_the_spin():
    """Under a rigid rotation the strain rate vanishes in the interior, so there the
    Jaumann rate turns the stress with the body while objectiveRate "none" leaves it
    (SOLID.py:2721-2722)."""
    out = {}
    for rate in ("jaumann", "none"):
        sc = free_block()
        sc["Solver"]["objectiveRate"] = rate
        sc["Hourglass"] = {"alpha": 0.0}
        ps = ParticleSystem(SimConfig(sc), device="cpu")
        x = ps.x.to_numpy().astype(np.float64)
        c = x.mean(0)
        w = np.array([0.0, 0.0, 2.0])
        ps.v.from_numpy(np.cross(w, x - c).astype(np.float32))
        s = np.zeros((ps.particle_max_num, 3, 3), np.float32)
        s[:, 0, 0], s[:, 1, 1] = 0.01, -0.01          # deviatoric, below yield
        ps.sigma_dev.from_numpy(s)
        p = build_params(ps)
        assert p.objective_none == (rate == "none")
        o = Oracle(p, ps.particle_max_num, fp64=True)
        o.set_state(state_from_sets(ps.state_numpy()), 1e-4)
        for st in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY):
            o.stage(st)
        r = o.get_state()
        inner = np.all(np.abs(r["x"] - c) < 1.5, axis=1)
        out[rate] = np.abs(r["sdev"][inner][:, 3]).max()   # s_xy: the rotated shear
    assert out["jaumann"] > 1e-6 and out["none"] <= 1e-3 * out["jaumann"], out


def _axi_power_imbalance(radial):
    """sum_i m_i (de_i + a_i . v_i) / sum_i |m_i a_i . v_i| of the axisymmetric dogbone's
    force stage (no damper, viscosity, shift or grips), with the conservative axial form
    and the conservative radial form on or off."""
    from sigmasph_b200.config import strip_json_comments
    with open(scene_path("tensile_axi_dogbone_dx0.1.json")) as f:
        sc = json.loads(strip_json_comments(f.read()))
    sc["Domain"].update({"conservativeAxialMomentum": True, "conservativeRadialForce": radial})
    sc["Hourglass"] = {"alpha": 0.0}
    sc["Solver"]["viscosity"] = 0.0
    sc["Shifting"] = {"enabled": False}
    sc.pop("Constraints", None)
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    rng = np.random.default_rng(3)
    n = ps.particle_max_num
    v = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    v[:, 2] = 0.0
    ps.v.from_numpy(v)
    s = rng.normal(0.0, 0.05, (n, 3, 3))
    s = 0.5 * (s + s.transpose(0, 2, 1))
    s -= (np.trace(s, axis1=1, axis2=2) / 3.0)[:, None, None] * np.eye(3)
    s[:, 0, 2] = s[:, 2, 0] = s[:, 1, 2] = s[:, 2, 1] = 0.0
    ps.sigma_dev.from_numpy(s.astype(np.float32))
    p = build_params(ps)
    assert p.axi_conservative_r == int(radial)
    o = Oracle(p, n, fp64=True)
    o.set_state(state_from_sets(ps.state_numpy()), 1e-5)
    for st in range(abi.STAGE_FORCES + 1):
        o.stage(st)
    r = o.get_state()
    pw = r["m"] * (r["acc"] * r["v"]).sum(1)
    return abs((r["m"] * r["de_int"] + pw).sum()) / np.abs(pw).sum()


def test_conservative_radial_form_closes_the_ring_power():
    """Domain.conservativeRadialForce carries the pair radius in the radial pair forces and
    banks the hoop power -v . a_geom in de_int (SOLID.py:3444-3466, :3609-3614), so the
    pair work telescopes in the ring measure m: the power imbalance of the force stage
    falls by two orders of magnitude (what is left is the axis images, which are not
    reciprocal pairs)."""
    plain, radial = _axi_power_imbalance(False), _axi_power_imbalance(True)
    assert plain > 1e-3 and radial < 0.02 * plain, (plain, radial)


# ------------------------------------------------------------------ analytic identities
def _bar_after_forces(sc, v_of=None, s_of=None):
    """The FP64 oracle's state after the sort, lambda / stress and force stages of one step
    on the deck, with the velocity and deviatoric stress set from functions of position."""
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    st = state_from_sets(ps.state_numpy())
    x = st["x"].astype(np.float64)
    if v_of is not None:
        st["v"] = v_of(x)
    if s_of is not None:
        st["sdev"] = s_of(x)
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-7)
    for s in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY, abi.STAGE_FORCES):
        o.stage(s)
    g = o.get_state()
    order = np.argsort(g["pid"])
    return {k: (v[order] if hasattr(v, "shape") and v.shape and v.shape[0] == len(order) else v)
            for k, v in g.items()}


def test_hourglass_damper_does_not_resist_a_linear_deformation():
    """The in-loop damper's pair term [(v_j - v_i) - <G> (x_j - x_i)] . rhat (SOLID.py:
    3768-3816) measures the departure from the linear field the velocity gradient G
    predicts ("dv_ij vanishes for any affine motion").  With the kernel-corrected G exact for v = A x, the term vanishes on every
    pair, so switching the damper on changes no acceleration (to 1e-10 of its scale)."""
    from tests.test_solid_gpu import bar3d_kc_deck
    A = np.random.default_rng(5).normal(size=(3, 3)) * 1e-3
    out = {}
    for alpha in (4.0, 0.0):
        sc = bar3d_kc_deck()
        sc["Hourglass"] = dict(sc.get("Hourglass", {}), alpha=alpha)
        out[alpha] = _bar_after_forces(sc, v_of=lambda x: x @ A.T)
    scale = np.abs(out[0.0]["acc"]).max()
    assert scale > 0.0
    assert np.abs(out[4.0]["acc"] - out[0.0]["acc"]).max() <= 1e-10 * scale


def test_stress_acceleration_of_a_linear_stress_field():
    """A deviatoric stress linear in position (s_xx = -s_yy = c x, s_xy = b y; the density
    at rho0, so p = 0; at rest, so no damper, viscosity or rate): the symmetric stress
    force sum_j w_i w_j (s_i + s_j) . grad W / mw_i (SOLID.py:3545-3700) is
    lambda div(s) / rho = lambda (b + c, 0, 0) / rho where the kernel's moment is lambda I
    (the bar's interior, lambda at its plateau: to 5e-3, the moment's anisotropy there)."""
    from tests.test_solid_gpu import bar3d_deck
    b, c = 2e-3, 1e-3

    def s_of(x):
        s = np.zeros((len(x), 6))
        s[:, 0], s[:, 1], s[:, 3] = c * x[:, 0], -c * x[:, 0], b * x[:, 1]
        return s
    sc = bar3d_deck()
    sc["Solver"]["viscosity"] = 0.0
    g = _bar_after_forces(sc, s_of=s_of)
    inn = g["lam"] >= 0.9999
    assert inn.sum() > 5000
    want = g["lam"][:, None] * np.array([b + c, 0.0, 0.0])[None, :] / (g["m"] / g["V"])[:, None]
    assert np.abs(g["acc"][inn] - want[inn]).max() <= 5e-3 * np.abs(want[inn]).max()


def test_jaumann_update_only_rotates_under_a_rigid_spin():
    """Objectivity of the Jaumann rate s_dot = 2 G dev(D) + W s - s W (SOLID.py:2691-2760):
    under a rigid spin v = W x the strain rate D vanishes (the kernel-corrected gradient is
    exact), so a uniform stress below yield is only rotated, s + dt (W s - s W), with no
    plastic strain (to float64 rounding of the stress, 1e-12 of |s|: 1e-8 of the 4e-5
    rotation)."""
    from tests.test_solid_gpu import bar3d_kc_deck
    sc = bar3d_kc_deck()
    sc["Solver"]["viscosity"] = 0.0
    ps = ParticleSystem(SimConfig(sc), device="cpu")
    st = state_from_sets(ps.state_numpy())
    x = st["x"].astype(np.float64)
    w = np.array([0.3, -0.2, 0.5]) * 10.0
    W = np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])
    st["v"] = x @ W.T
    s0 = np.array([[0.05, 0.02, -0.01], [0.02, -0.03, 0.015], [-0.01, 0.015, -0.02]])
    six = lambda m: np.array([m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2]])
    st["sdev"] = np.tile(six(s0), (len(x), 1))
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=True)
    o.set_state(st, 1e-4)
    o.stage(abi.STAGE_SORT)
    o.stage(abi.STAGE_LAM)
    g = o.get_state()
    dt = o.scalars()["dt"]
    S = s0 + dt * (W @ s0 - s0 @ W)
    S -= np.trace(S) / 3.0 * np.eye(3)
    change = np.abs(six(S) - six(s0)).max()
    err = np.abs(g["sdev"] - six(S)[None]).max()
    assert change > 1e-5
    assert err <= 1e-12 * np.abs(s0).max() and err <= 1e-8 * change
    assert g["eps_p"].max() == 0.0

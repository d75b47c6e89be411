"""GPU parity of the hypoelastic tensile-solid step against the CPU oracle, through the
C-ABI.  Tolerances as for the fluid (tests/test_fluid_gpu.py): stage fields within 5e-5
of the float32 oracle (the Johnson-Cook return map is an iterative solve and the stress
update cancels in its trace-free part), within 2e-4 of the float64 oracle; after several
steps the GPU stays as close to float64 as the float32 oracle is (4x + floor)."""
import numpy as np
import pytest

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import scene_path
from sigmasph_b200.solver import build_params
from oracle.oracle import Oracle, state_from_sets
from tests.helpers import pair_set, perturb, check_shift_pairs, check_pp

pytestmark = pytest.mark.gpu


def perturb_solid(ps, seed=11, s_amp=0.25, ep_max=0.05):
    """A plastic state: random deviators near yield, plastic strain, heat."""
    rng = np.random.default_rng(seed)
    n = ps.particle_max_num
    perturb(ps, seed=seed, dv=0.5, drho=2e-4, dshift=2e-3)
    s = rng.normal(0.0, s_amp, (n, 3, 3))
    s = 0.5 * (s + np.transpose(s, (0, 2, 1)))
    s -= (np.trace(s, axis1=1, axis2=2) / 3.0)[:, None, None] * np.eye(3)[None]
    if ps.two_d:
        s[:, 0, 2] = s[:, 2, 0] = s[:, 1, 2] = s[:, 2, 1] = 0.0
    ps.sigma_dev.from_numpy(s.astype(np.float32))
    ps.eps_plastic.from_numpy(rng.uniform(0.0, ep_max, n).astype(np.float32))
    ps.e_int.from_numpy(rng.uniform(0.0, 5.0, n).astype(np.float32))
    ps.temperature.from_numpy(rng.uniform(293.0, 400.0, n).astype(np.float32))


def solid_gpu_fields(ps):
    st = ps.state_numpy()
    d = {k: t.detach().cpu().numpy().copy() for k, t in ps.derived().items()}
    o = np.argsort(st["pid"])
    out = {"x": st["pos"][o, :3], "V": st["pos"][o, 3], "v": st["vel"][o, :3],
           "pressure": st["disp"][o, 3], "u": st["disp"][o, :3], "pst_shift": st["shift"][o, :3],
           "e_int": st["shift"][o, 3], "sdev": st["sdev"][o, :6], "eps_p": st["sdev"][o, 6],
           "temperature": st["sdev"][o, 7], "acc": st["acc"][o, :3], "de_int": st["acc"][o, 3],
           "lam": d["lam"][o, 0], "divergence": d["div"][o, 0],
           "grad_v": d["gradv"][o][:, :9]}
    return {k: np.asarray(v, dtype=np.float64) for k, v in out.items()}


def solid_oracle_fields(orc):
    r = orc.get_state()
    o = np.argsort(r["pid"])
    return {k: (v[o] if hasattr(v, "shape") and v.shape and v.shape[0] == len(o) else v)
            for k, v in r.items()}


def errs(g, r, keys):
    out = {}
    for k in keys:
        a, b = np.asarray(g[k], dtype=np.float64), np.asarray(r[k], dtype=np.float64)
        sc = np.abs(b).max()
        out[k] = float(np.abs(a - b).max() / sc) if sc > 0 else float(np.abs(a - b).max())
    return out


def make_solid(scene, perturbed=True):
    cfg = SimConfig(scene)
    ps = ParticleSystem(cfg, device="cuda")
    if perturbed:
        perturb_solid(ps)
    solver = ps.build_solver()
    st0 = state_from_sets(ps.state_numpy())
    p = build_params(ps)
    o64 = Oracle(p, ps.particle_max_num, fp64=True)
    o32 = Oracle(p, ps.particle_max_num, fp64=False)
    for o in (o64, o32):
        o.set_state(st0, solver.dt[None])
    return ps, solver, o64, o32


def axi_deck():
    return scene_path("tensile_axi_dogbone_dx0.1.json")


def bar3d_deck(dx=0.4):
    """A small 3D round bar (the revolved parallel-gauge profile), J2 linear hardening,
    in-loop hourglass damper, grips on both heads."""
    return {
        "Domain": {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "boundary": "open"},
        "Time": {"CFL": 0.3},
        "Solver": {"type": "hypoElastic", "viscosity": 0.02, "allowNegativePressure": True},
        "Materials": [{"name": "steel", "density0": 7.9e-6, "eos": {"type": "linear"},
                       "strength": {"type": "hypoElastic", "youngsModulus": 200.0,
                                    "poissonRatio": 0.3,
                                    "plasticity": {"model": "linear", "yieldStress": 0.3,
                                                   "hardeningModulus": 1.0}}}],
        "Load": {"gravitation": [0.0, 0.0, 0.0], "rampTime": 0.05},
        "Diffusion": {"delta": 0.1},
        "Shifting": {"enabled": True, "mode": "colle", "maMode": "fixed", "maFixed": 0.05},
        "Hourglass": {"alpha": 4.0},
        "SolidBlocks": [{"objectId": 0, "start": [-5.0, -12.0, -5.0], "end": [5.0, 12.0, 5.0],
                         "translation": [0, 0, 0], "scale": [1, 1, 1], "velocity": [0, 0, 0],
                         "density": 7.9e-6, "color": [1, 1, 1], "material": "steel",
                         "shape": {"type": "gaugedogbone3d", "tabWidth": 10.0, "tabHeight": 5.0,
                                   "gaugeWidth": 6.0, "radius": 3.0, "gaugeLength": 6.0}}],
        "Constraints": [
            {"name": "low", "region": [[-6, -12.5, -6], [6, -9.0, 6]], "components": "xyz",
             "displacement": [0.0, -0.5, 0.0]},
            {"name": "high", "region": [[-6, 9.0, -6], [6, 12.5, 6]], "components": "xyz",
             "displacement": [0.0, 0.5, 0.0]}],
    }


def strip_ps_deck(dx=0.1):
    """A plane-strain strip (a single particle layer) with Johnson-Cook hardening."""
    sc = bar3d_deck()
    sc["Domain"] = {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "planeStrain": True,
                    "boundary": "open"}
    sc["Materials"][0]["strength"]["plasticity"] = {"model": "johnson_cook", "A": 0.31, "B": 1.0,
                                                    "n": 0.65, "C": 0.02, "eps0_dot": 1.0}
    sc["Hourglass"] = {"alpha": 4.0, "superTimeStepping": {"mode": "subcycle"}}
    sc["SolidBlocks"][0].pop("shape")
    sc["SolidBlocks"][0]["start"] = [0.0, 0.0, 0.0]
    sc["SolidBlocks"][0]["end"] = [3.0, 6.0, 0.5 * dx]
    sc["Constraints"] = [
        {"name": "low", "region": [[-1, -1, -1], [4, 0.55, 1]], "components": "xy",
         "displacement": [0.0, -0.3, 0.0]},
        {"name": "high", "region": [[-1, 5.4, -1], [4, 7, 1]], "components": "xy",
         "displacement": [0.0, 0.3, 0.0]}]
    return sc


def bar3d_visc_deck():
    """The bar with both in-loop viscosities: the VNR bulk viscosity (l = dx0) and
    Monaghan's pair viscosity, beside the Morris term and the in-loop damper."""
    sc = bar3d_deck()
    sc["Solver"]["bulkViscosity"] = {"quadratic": 1.5}
    sc["Solver"]["artificialViscosity"] = {"alpha": 1.0, "beta": 2.0}
    return sc


def axi_visc_deck():
    """The axisymmetric dogbone (conservative axial form, sub-cycled damper) with q on the
    kernel support (l = h) and Monaghan's viscosity."""
    import json
    from sigmasph_b200.config import strip_json_comments
    with open(axi_deck()) as f:
        sc = json.loads(strip_json_comments(f.read()))
    sc["Solver"]["bulkViscosity"] = {"quadratic": 0.5, "lengthScale": "h"}
    sc["Solver"]["artificialViscosity"] = {"alpha": 0.5, "beta": 1.0, "epsilon": 0.02}
    return sc


def bar3d_no_spin_deck():
    """The bar with Solver.objectiveRate "none": the stress rate without its spin terms."""
    sc = bar3d_deck()
    sc["Solver"]["objectiveRate"] = "none"
    return sc


def _axi_json():
    import json
    from sigmasph_b200.config import strip_json_comments
    with open(axi_deck()) as f:
        return json.loads(strip_json_comments(f.read()))


def axi_signed_deck():
    """Domain.axialImageRadius "signed": the axial stress pair reads a mirror image's
    radius as the coordinate it sits at (SOLID.py:3598-3609)."""
    sc = _axi_json()
    sc["Domain"]["axialImageRadius"] = "signed"
    return sc


def axi_plain_axial_deck():
    """Domain.conservativeAxialMomentum false: no pair-radius rescaling of the axial
    forces, and the damper's rate without the axis ratio."""
    sc = _axi_json()
    sc["Domain"]["conservativeAxialMomentum"] = False
    return sc


def axi_radial_deck():
    """Domain.conservativeRadialForce with Monaghan's viscosity and q: the pair radius in
    every radial pair force (stress with an image's signed radius, Pi_ij, the damper) and
    the source (p + q - s_tt) / (rho r) with its hoop power (SOLID.py:3444-3466)."""
    sc = axi_visc_deck()
    sc["Domain"]["conservativeRadialForce"] = True
    return sc


def axi_rkl_deck():
    """The axisymmetric dogbone with its sub-cycled damper as s-stage RKL1
    (Hourglass.superTimeStepping.mode "rkl", SOLID.py:4510-4576)."""
    import json
    from sigmasph_b200.config import strip_json_comments
    with open(axi_deck()) as f:
        sc = json.loads(strip_json_comments(f.read()))
    sc["Hourglass"]["superTimeStepping"]["mode"] = "rkl"
    return sc


def bar3d_kc_deck():
    """The bar with Solver.kernelCorrection: grad v through the regularised inverse of E
    (SOLID.py:1757-1771, spd_inverse.py:45-101), which departs from the identity at the
    bar's free surface, where the float64 inverse is taken."""
    sc = bar3d_deck()
    sc["Solver"]["kernelCorrection"] = True
    return sc


def axi_kc_deck():
    """The axisymmetric dogbone with Solver.kernelCorrection (the 2x2 inverse)."""
    sc = _axi_json()
    sc["Solver"]["kernelCorrection"] = True
    return sc


def two_material_bar_deck(pairs="samematerial"):
    """A square bar of two materials, steel below y = 0 and aluminium above, J2 both, with
    the in-loop damper, Colle shifting at a fixed Mach number and delta-SPH: the EOS sound
    speeds and the acoustic impedances differ, so pair_c0, local_c0 and the damper's
    impedance ratio are all live (SOLID.py:222-245, :4184-4239, DSPH.py:483-530)."""
    sc = bar3d_deck()
    sc["Materials"].append({"name": "aluminium", "density0": 2.7e-6, "eos": {"type": "linear"},
                            "strength": {"type": "hypoElastic", "youngsModulus": 70.0,
                                         "poissonRatio": 0.33,
                                         "plasticity": {"model": "linear", "yieldStress": 0.1,
                                                        "hardeningModulus": 0.5}}})
    sc["Diffusion"]["pairs"] = pairs
    blk = dict(sc["SolidBlocks"][0])
    blk.pop("shape")
    sc["SolidBlocks"] = [dict(blk, start=[-2.0, -12.0, -2.0], end=[2.0, -0.2, 2.0]),
                         dict(blk, objectId=1, material="aluminium", density=2.7e-6,
                              start=[-2.0, 0.0, -2.0], end=[2.0, 12.0, 2.0])]
    return sc


def two_material_bar_all_deck():
    """The two-material bar with Diffusion.pairs "all": the diffusion crosses the
    interface with the harmonic mean of the two deltas."""
    return two_material_bar_deck("all")


# The GPU writes the return-mapped stress, plastic strain and energy to scratch in the
# LAM stage and commits them with the volume update, so they are compared after it.
STAGE_FIELDS = {
    abi.STAGE_LAM: ["lam", "grad_v"],
    abi.STAGE_CONTINUITY: ["V", "sdev", "eps_p", "e_int", "temperature"],
    abi.STAGE_FORCES: ["acc", "de_int", "pressure"],
    abi.STAGE_ADVECT: ["v", "x", "u"],
    abi.STAGE_PST: ["pst_shift", "x"],
    abi.STAGE_BOUNDARY: ["x", "v", "sdev"],
}
# The linear EOS K (m / (V rho0) - 1) cancels: with |rho / rho0 - 1| ~ 2e-4 (these decks'
# density perturbation) one float32 ulp of V (6e-8) is ~3e-4 of max |p|.
TOL32 = {"de_int": 2e-4, "pressure": 1e-3, "grad_v": 1e-4}
TOL64 = {"de_int": 1e-3, "pressure": 2e-3, "acc": 5e-4, "grad_v": 2e-4}


@pytest.mark.parametrize("deck", [axi_deck, bar3d_deck, strip_ps_deck, bar3d_visc_deck, axi_visc_deck,
                                  axi_rkl_deck, bar3d_no_spin_deck, axi_signed_deck, axi_plain_axial_deck,
                                  axi_radial_deck, bar3d_kc_deck, axi_kc_deck, two_material_bar_deck,
                                  two_material_bar_all_deck],
                         ids=["axi_dogbone_jc_sts", "bar3d_j2_inloop", "plane_strain_jc",
                              "bar3d_q_monaghan", "axi_q_monaghan", "axi_rkl", "bar3d_no_spin",
                              "axi_signed_image", "axi_plain_axial", "axi_radial",
                              "bar3d_kernel_correction", "axi_kernel_correction",
                              "two_materials", "two_materials_pairs_all"])
def test_solid_stages_match_oracle(cuda, deck):
    ps, solver, o64, o32 = make_solid(deck())
    p = solver.params
    if deck in (two_material_bar_deck, two_material_bar_all_deck):
        assert p.n_materials == 2 and p.c0_mixed and p.hg_mixed_impedance
    for s in range(8):
        solver.run_stage(s)
        o64.stage(s)
        o32.stage(s)
        if s == abi.STAGE_LAM and p.kernel_correction and not p.two_d:
            # the free surface is in the deck: there the inverse is taken in float64
            assert (ps.lam.to_numpy() < 0.75).any()
        if s == abi.STAGE_SORT:
            gi, gj, gm = solver.pairs(0)
            oi, oj, om = o32.pairs()
            A = pair_set(gi, gj, gm, ps.pid.to_numpy())
            B = pair_set(oi, oj, om, o32.get_state()["pid"])
            assert A == B
        if s not in STAGE_FIELDS:
            continue
        g = solid_gpu_fields(ps)
        r32, r64 = solid_oracle_fields(o32), solid_oracle_fields(o64)
        e32 = errs(g, r32, STAGE_FIELDS[s])
        e64 = errs(g, r64, STAGE_FIELDS[s])
        for k, e in e32.items():
            assert e <= TOL32.get(k, 5e-5), (s, k, e, e32)
        for k, e in e64.items():
            assert e <= TOL64.get(k, 2e-4), (s, k, e, e64)
        check_pp(g, r32, r64, STAGE_FIELDS[s])
    sg = solver._scalars()
    s32 = o32.scalars()
    assert sg.sts_stages == int(s32["sts_stages"])
    assert abs(sg.dt - s32["dt"]) <= 1e-6 * s32["dt"]
    assert abs(sg.sim_time - s32["sim_time"]) <= 1e-6 * s32["sim_time"]
    nc = solver.num_constraints
    fg = np.array([[sg.constraint_force[k][d] for d in range(3)] for k in range(nc)])
    fo = s32["constraint_force"][:nc]
    assert np.abs(fg - fo).max() <= 1e-4 * np.abs(fo).max()
    assert abs(sg.plastic_work - s32["plastic_work"]) <= 1e-4 * abs(s32["plastic_work"]) + 1e-12


@pytest.mark.parametrize("deck", [bar3d_deck, strip_ps_deck], ids=["bar3d", "plane_strain"])
def test_solid_shift_pairs_from_lists(cuda, deck):
    """A solid lattice starts on the cell boundaries, so small moves change many
    particles' cells: the shift's list path must still give the stale-bin pair set, for
    host-made moves under a given bound and after the real step's advect and grips."""
    ps, solver, _, _ = make_solid(deck())
    solver.initialize()
    crossed = check_shift_pairs(ps, solver, seed=9, reach=0.045)
    assert crossed[1:].sum() > 0.05 * crossed.sum()
    ps, solver, _, _ = make_solid(deck())
    for s in range(abi.STAGE_ADVECT + 1):
        solver.run_stage(s)
    pid = ps.pid.to_numpy()
    A = pair_set(*solver.shift_pairs(), pid)
    B = pair_set(*solver.pairs(1), pid)
    assert A == B


@pytest.mark.parametrize("deck", [bar3d_deck, strip_ps_deck], ids=["bar3d", "plane_strain"])
def test_solid_lists_between_builds_match_oracle(cuda, deck):
    """Steps that filter the candidate lists instead of building them give the
    reference's neighbour pairs (the oracle sorts the same state afresh)."""
    ps, solver, _, _ = make_solid(deck())
    solver.initialize()
    solver.list_stats(reset=True)
    solver.step_many(6)
    stats = solver.list_stats()
    solver.run_stage(abi.STAGE_SORT)
    assert solver.list_stats()["builds"] == stats["builds"] < stats["steps"] == 6, stats
    orc = Oracle(build_params(ps), ps.particle_max_num, fp64=False)
    orc.set_state(state_from_sets(ps.state_numpy()), solver.dt[None])
    orc.stage(abi.STAGE_SORT)
    B = pair_set(*orc.pairs(), orc.get_state()["pid"])
    A = pair_set(*solver.pairs(0), ps.pid.to_numpy())
    assert A == B


@pytest.mark.parametrize("deck", [axi_deck, bar3d_deck, bar3d_visc_deck, axi_rkl_deck],
                         ids=["axi_dogbone", "bar3d", "bar3d_q_monaghan", "axi_rkl"])
def test_solid_multistep_tracks_fp64(cuda, deck):
    ps, solver, o64, o32 = make_solid(deck())
    for o in (o64, o32):
        o.stage(abi.STAGE_SORT)
    solver.initialize()
    # the oracle's first stage also advanced its load factor; the GPU's step does that
    nsteps = 10
    solver.step_many(nsteps)
    o64.step(nsteps)
    o32.step(nsteps)
    g, r64, r32 = solid_gpu_fields(ps), solid_oracle_fields(o64), solid_oracle_fields(o32)
    keys = ["x", "v", "V", "sdev", "eps_p", "e_int", "pressure"]
    eg = errs(g, r64, keys)
    eo = errs(r32, r64, keys)
    for k in keys:
        assert eg[k] <= 4.0 * eo[k] + 2e-6, (k, eg[k], eo[k])
    check_pp(g, r32, r64, keys, slack=1e-5)
    sg = solver._scalars()
    s64 = o64.scalars()
    fg = np.array([[sg.constraint_force[k][d] for d in range(3)] for k in range(solver.num_constraints)])
    fo = s64["constraint_force"][:solver.num_constraints]
    assert np.abs(fg - fo).max() <= 1e-3 * np.abs(fo).max() + 1e-9
    assert solver.error_word() & ~(abi.EW_HASHED_GRID) == 0


@pytest.mark.parametrize("deck", [bar3d_deck, bar3d_visc_deck], ids=["bar3d", "bar3d_q_monaghan"])
def test_solid_work_channels(cuda, deck):
    """The explicit damper's and the viscosities' work (SOLID.py:2182-2207): each step's
    force-pass power banked at the next step's start with the dt it was done over, so
    after N steps the totals hold N - 1 steps, as the float32 oracle's; the viscosity
    limits of the time step are the oracle's (dt within 1e-6)."""
    ps, solver, o64, o32 = make_solid(deck())
    o32.stage(abi.STAGE_SORT)
    solver.initialize()
    nsteps = 6
    solver.step_many(nsteps)
    o32.step(nsteps)
    sg, s32 = solver._scalars(), o32.scalars()
    assert abs(sg.dt - s32["dt"]) <= 1e-5 * s32["dt"]
    for k in ("visc_work", "hg_work"):
        want, got = s32[k], getattr(sg, k)
        assert want != 0.0, k
        assert abs(got - want) <= 2e-3 * abs(want), (k, got, want)
    b = solver.energy_budget()
    assert b["visc"] == sg.visc_work and b["hg"] == sg.hg_work
    assert b["total"] == pytest.approx(b["ke"] + b["ie"] + b["hg"] + b["pe"] - b["leftover"])


def test_grip_force_and_time_bookkeeping(cuda):
    """Unperturbed dogbone: after a few hundred steps the two grips pull equal and
    opposite forces, the load factor follows the smoothstep ramp of the device clock,
    and the hourglass sub-step count is the reference's (20 at this deck's CFL)."""
    cfg = SimConfig(axi_deck())
    ps = ParticleSystem(cfg, device="cuda")
    sv = ps.build_solver()
    sv.initialize()
    sv.step_many(300)
    sg = sv._scalars()
    # the load factor of the last step is taken at that step's start time
    u = min(1.0, (sg.sim_time - sg.dt) / 0.9)
    assert abs(sv.load_s[None] - u * u * (3 - 2 * u)) <= 1e-6
    assert sg.sts_stages == 20
    d = sv.get_constraint_data()
    F0, F1 = d[0]["force"][0], d[1]["force"][0]
    assert F0 > 0 and F1 < 0 and abs(F0 + F1) <= 0.05 * abs(F0)
    assert d[1]["displacement"][0] == pytest.approx(10.0 * sv.load_s[None], rel=1e-5)


def test_constraint_data_through_the_abi(cuda):
    """sph_constraints (get_constraint_data, SOLID.py:5198-5225): each grip's FP64 force and
    displacement after a step equal the float32 oracle's apply_constraints sums; more grips
    than the scene has, and a fluid handle, are refused."""
    ps, solver, _, o32 = make_solid(bar3d_deck())
    for s in range(8):
        solver.run_stage(s)
        o32.stage(s)
    d = solver.get_constraint_data()
    s32 = o32.scalars()
    assert [e["name"] for e in d] == ["low", "high"]
    F = np.array([e["force"] for e in d])
    U = np.array([e["displacement"] for e in d])
    Fo, Uo = s32["constraint_force"][:2], s32["constraint_disp"][:2]
    assert np.abs(F).max() > 0.0
    assert np.abs(F - Fo).max() <= 1e-4 * np.abs(Fo).max()
    assert np.allclose(U, Uo, rtol=1e-6, atol=0.0)
    buf = np.zeros(3 * 8)
    assert solver.L.sph_constraints(solver.h, buf.ctypes.data, None, 3, None) == -1
    from sigmasph_b200.scenes import dambreak3d, dx_for_particles
    fps = ParticleSystem(SimConfig(dambreak3d(dx=dx_for_particles(2000))), device="cuda")
    fsv = fps.build_solver()
    assert fsv.L.sph_constraints(fsv.h, buf.ctypes.data, None, 0, None) == -1


def test_solid_reductions_match_numpy(cuda):
    """HypoElasticSolver energy reductions (SOLID.py:2296-2322, sph_base.py:451-507) on a
    perturbed plastic state against float64 numpy sums of the same fields."""
    ps = ParticleSystem(SimConfig(bar3d_deck()), device="cuda")
    perturb_solid(ps)
    sv = ps.build_solver()
    st = ps.state_numpy()
    V = st["pos"][:, 3].astype(np.float64)
    m = st["vel"][:, 3].astype(np.float64)
    v = st["vel"][:, :3].astype(np.float64)
    s = st["sdev"][:, :6].astype(np.float64)
    p = build_params(ps)
    K, G, rho0 = float(p.mat_K[0]), float(p.mat_G[0]), float(p.mat_rho0[0])
    theta = (m / V - rho0) / rho0
    ss = (s[:, :3] ** 2).sum(1) + 2.0 * (s[:, 3:] ** 2).sum(1)
    elastic = (0.5 * K * theta ** 2 * V + 0.25 * ss / G * V).sum()
    ke = (0.5 * m * (v ** 2).sum(1)).sum()
    ie = (m * st["shift"][:, 3].astype(np.float64)).sum()
    assert sv.compute_elastic_energy() == pytest.approx(elastic, rel=1e-5)
    assert sv.compute_kinetic_energy() == pytest.approx(ke, rel=1e-5)
    assert sv.compute_internal_energy() == pytest.approx(ie, rel=1e-5)
    assert sv.compute_total_mass() == pytest.approx(m.sum(), rel=1e-6)
    P = sv.compute_momentum()
    assert np.abs(P - (m[:, None] * v).sum(0)).max() <= 1e-5 * (m[:, None] * np.abs(v)).sum()


def test_kernel_corrected_gradient_is_exact_on_the_gpu(cuda):
    """v = A x on the kernel-corrected bar: the CUDA path's grad v (float32 pair sums, the
    FP64 regularised inverse) is A at every particle, the free surface included, to float32
    rounding amplified by the inverse where lambda falls to ~0.2 (bound 1e-3 of |A|)."""
    ps = ParticleSystem(SimConfig(bar3d_kc_deck()), device="cuda")
    A = np.random.default_rng(5).normal(size=(3, 3)) * 1e-3
    ps.v.from_numpy((ps.x.to_numpy().astype(np.float64) @ A.T).astype(np.float32))
    solver = ps.build_solver()
    solver.run_stage(abi.STAGE_SORT)
    solver.run_stage(abi.STAGE_LAM)
    g = solid_gpu_fields(ps)
    assert g["lam"].min() < 0.3
    G = g["grad_v"].reshape(-1, 3, 3)
    assert np.abs(G - A[None]).max() <= 1e-3 * np.abs(A).max()


def _gpu_bar_forces(sc, v=None, s=None):
    ps = ParticleSystem(SimConfig(sc), device="cuda")
    if v is not None:
        ps.v.from_numpy(v(ps.x.to_numpy().astype(np.float64)).astype(np.float32))
    if s is not None:
        sd = np.zeros((ps.particle_max_num, 3, 3))
        s6 = s(ps.x.to_numpy().astype(np.float64))
        sd[:, 0, 0], sd[:, 1, 1], sd[:, 2, 2] = s6[:, 0], s6[:, 1], s6[:, 2]
        sd[:, 0, 1] = sd[:, 1, 0] = s6[:, 3]
        sd[:, 0, 2] = sd[:, 2, 0] = s6[:, 4]
        sd[:, 1, 2] = sd[:, 2, 1] = s6[:, 5]
        ps.sigma_dev.from_numpy(sd.astype(np.float32))
    solver = ps.build_solver()
    for st in (abi.STAGE_SORT, abi.STAGE_LAM, abi.STAGE_CONTINUITY, abi.STAGE_FORCES):
        solver.run_stage(st)
    assert solver.error_word() & ~abi.EW_HASHED_GRID == 0
    g = solid_gpu_fields(ps)
    st = ps.state_numpy()
    g["m"] = st["vel"][np.argsort(st["pid"]), 3].astype(np.float64)
    return g


def test_damper_leaves_an_affine_motion_alone_on_the_gpu(cuda):
    """The CUDA path's in-loop damper under the kernel-corrected gradient: for v = A x it
    changes the accelerations by less than 5% of what it does to the same field with a
    non-affine part of 1e-3 of its size added (float32 sums leave ~1e-6 of A in the
    corrected gradient, against the 1e-3 the damper is there to remove)."""
    A = np.random.default_rng(5).normal(size=(3, 3)) * 1e-3
    rng = np.random.default_rng(9)

    def affine(x):
        return x @ A.T

    def perturbed(x):
        v = x @ A.T
        return v + 1e-3 * np.abs(v).max() * rng.standard_normal(v.shape)
    acc = {}
    for name, vf in (("affine", affine), ("perturbed", perturbed)):
        for alpha in (4.0, 0.0):
            sc = bar3d_kc_deck()
            sc["Hourglass"] = dict(sc.get("Hourglass", {}), alpha=alpha)
            rng = np.random.default_rng(9)
            acc[name, alpha] = _gpu_bar_forces(sc, v=vf)["acc"]
    response = np.abs(acc["perturbed", 4.0] - acc["perturbed", 0.0]).max()
    assert response > 0.0
    assert np.abs(acc["affine", 4.0] - acc["affine", 0.0]).max() <= 0.05 * response


def test_linear_stress_field_on_the_gpu(cuda):
    """The CUDA path's stress force for s_xx = -s_yy = c x, s_xy = b y at rest and at rho0:
    lambda (b + c, 0, 0) / rho where lambda is at its plateau (bound 1e-2: the moment's
    anisotropy, 5e-3, and float32 sums)."""
    b, c = 2e-3, 1e-3

    def s_of(x):
        s = np.zeros((len(x), 6))
        s[:, 0], s[:, 1], s[:, 3] = c * x[:, 0], -c * x[:, 0], b * x[:, 1]
        return s
    sc = bar3d_deck()
    sc["Solver"]["viscosity"] = 0.0
    g = _gpu_bar_forces(sc, s=s_of)
    inn = g["lam"] >= 0.9999
    assert inn.sum() > 5000
    want = g["lam"][:, None] * np.array([b + c, 0.0, 0.0])[None, :] / (g["m"] / g["V"])[:, None]
    assert np.abs(g["acc"][inn] - want[inn]).max() <= 1e-2 * np.abs(want[inn]).max()

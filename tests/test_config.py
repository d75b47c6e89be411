"""Host-side set-up against golden values produced by the reference's own host code
(tests/golden/make_golden.py): resolved scene parameters, material constants, and the
particle lattice (count and exact float32 positions)."""
import hashlib
import json
import os

import numpy as np
import pytest

from sigmasph_b200.config import SimConfig, SceneError
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import scene_path

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_host.json")))
DECKS = {"tensile_axi_dogbone_dx0.1": scene_path("tensile_axi_dogbone_dx0.1.json"),
         "dambreak3d_1M": scene_path("dambreak3d_1M.json")}


def _same(a, b):
    if isinstance(b, float) or isinstance(a, float):
        return a is not None and b is not None and abs(float(a) - float(b)) <= 1e-12 * max(1.0, abs(float(b)))
    if isinstance(b, list):
        return len(a) == len(b) and all(_same(x, y) for x, y in zip(a, b))
    if isinstance(b, str) and isinstance(a, str):
        return a.lower() == b.lower()
    return a == b


@pytest.mark.parametrize("deck", sorted(DECKS))
def test_resolved_parameters_match_reference(deck):
    cfg = SimConfig(DECKS[deck])
    gold = GOLD["decks"][deck]["config"]
    bad = {k: (cfg.get_cfg(k), v) for k, v in gold.items() if not _same(cfg.get_cfg(k), v)}
    assert not bad, bad


@pytest.mark.parametrize("deck", sorted(DECKS))
def test_material_constants_match_reference(deck):
    cfg = SimConfig(DECKS[deck])
    gold = GOLD["decks"][deck]["materials"]
    for name, g in gold.items():
        m = cfg.get_materials()[name]
        for key, attr in (("rho0", "rho0"), ("K", "K"), ("G", "G"), ("c_p", "c_p"),
                          ("c_eos", "c_eos"), ("sigma_y0", "sigma_y0"),
                          ("hardening", "hardening"), ("plastic_kind", "plastic_kind"),
                          ("specific_heat", "specific_heat"), ("delta", "delta")):
            assert _same(getattr(m, attr), g[key]), (name, key, getattr(m, attr), g[key])


@pytest.mark.parametrize("deck", sorted(DECKS))
def test_lattice_is_the_reference_lattice(deck):
    ps = ParticleSystem(SimConfig(DECKS[deck]), device="cpu")
    g = GOLD["decks"][deck]
    assert ps.particle_max_num == g["particles"]
    x = np.ascontiguousarray(ps.x.to_numpy().astype(np.float32))
    assert hashlib.sha256(x.tobytes()).hexdigest() == g["positions_sha256"]


def test_axisymmetric_mass_and_volume():
    ps = ParticleSystem(SimConfig(DECKS["tensile_axi_dogbone_dx0.1"]), device="cpu")
    x = ps.x.to_numpy()
    m = ps.m.to_numpy()
    V = ps.V.to_numpy()
    rmin = np.float32(0.5 * ps.particle_diameter)
    vol = (np.float32(ps.V0) * np.maximum(x[:, 1], rmin)).astype(np.float32)
    assert np.array_equal(m, (vol * np.float32(7.9e-6)).astype(np.float32))
    assert np.array_equal(V, (m / np.float32(7.9e-6)).astype(np.float32))
    assert ps.bc_flag.to_numpy().max() == 3
    assert set(np.unique(ps.bc_id.to_numpy())) == {-1, 0, 1}


def test_unknown_and_unimplemented_keys_are_rejected():
    sc = json.loads(json.dumps(GOLD["decks"]["dambreak3d_1M"]["config"]))
    from sigmasph_b200.scenes import dambreak3d
    bad = dambreak3d(dx=0.05)
    bad["Solver"]["notAKey"] = 1
    with pytest.raises(SceneError):
        SimConfig(bad)
    bad = dambreak3d(dx=0.05)
    bad["Erosion"] = {"mode": "erode"}
    with pytest.raises(SceneError):
        SimConfig(bad)
    bad = dambreak3d(dx=0.05)
    bad["Shifting"]["mode"] = "other"
    with pytest.raises(SceneError):
        SimConfig(bad)


def test_comments_are_stripped():
    from sigmasph_b200.config import strip_json_comments
    assert json.loads(strip_json_comments('{"a": "x#y", # c\n "b": 2 // d\n}')) == {"a": "x#y", "b": 2}


def test_relaxation_switches():
    """Shifting.initialRelaxation / initialRelaxationTolerance and the relaxation dump's
    Output switches resolve to the reference's names and defaults (params.py:1038-1052,
    :1245-1263)."""
    from sigmasph_b200.scenes import dambreak3d
    sc = dambreak3d(dx=0.05)
    cfg = SimConfig(sc)
    assert (cfg.get_cfg("PST_RELAX_STEPS"), cfg.get_cfg("PST_RELAX_TOL")) == (0, 0.03)
    assert (cfg.get_cfg("exportRelaxationNetcdf"), cfg.get_cfg("exportRelaxationInterval")) == (False, 1)
    sc["Shifting"].update({"initialRelaxation": 40, "initialRelaxationTolerance": 0.01})
    sc["Output"] = {"relaxationNetcdf": True, "relaxationInterval": 5, "netcdf": True}
    cfg = SimConfig(sc)
    assert (cfg.get_cfg("PST_RELAX_STEPS"), cfg.get_cfg("PST_RELAX_TOL")) == (40, 0.01)
    assert (cfg.get_cfg("exportRelaxationNetcdf"), cfg.get_cfg("exportRelaxationInterval")) == (True, 5)


def test_sts_modes():
    """Hourglass.superTimeStepping: 'subcycle' and 'rkl' (params.py:1170-1191); a fixed
    count above the device's 32 stages is refused."""
    from sigmasph_b200.solver import build_params
    from sigmasph_b200.config import strip_json_comments
    with open(DECKS["tensile_axi_dogbone_dx0.1"]) as f:
        base = json.loads(strip_json_comments(f.read()))
    for mode, rkl in (("subcycle", 0), ("rkl", 1)):
        sc = json.loads(json.dumps(base))
        sc["Hourglass"]["superTimeStepping"] = {"mode": mode, "safety": 0.7}
        ps = ParticleSystem(SimConfig(sc), device="cpu")
        p = build_params(ps)
        assert p.hourglass_sts == 1 and p.hg_sts_rkl == rkl
        assert p.hourglass_sts_safety == pytest.approx(0.7)
    sc = json.loads(json.dumps(base))
    sc["Hourglass"]["superTimeStepping"] = {"mode": "rkl", "stages": 40}
    with pytest.raises(SceneError, match="above 32"):
        SimConfig(sc)


def test_axisymmetric_forms():
    """Domain.conservativeAxialMomentum / conservativeRadialForce / axialImageRadius
    select the axisymmetric pair forms (params.py:302-355)."""
    from sigmasph_b200.solver import build_params
    from sigmasph_b200.config import strip_json_comments
    with open(DECKS["tensile_axi_dogbone_dx0.1"]) as f:
        base = json.loads(strip_json_comments(f.read()))
    ps = ParticleSystem(SimConfig(base), device="cpu")
    p0 = build_params(ps)
    assert (p0.axi_conservative_x, p0.axi_image_signed) == (1, 0)
    sc = json.loads(json.dumps(base))
    sc["Domain"].update({"conservativeAxialMomentum": False, "axialImageRadius": "signed"})
    p1 = build_params(ParticleSystem(SimConfig(sc), device="cpu"))
    assert (p1.axi_conservative_x, p1.axi_image_signed) == (0, 0)
    assert p1.hg_rate < p0.hg_rate                 # no axis ratio in the damper's rate
    assert p0.axi_conservative_r == 0
    sc = json.loads(json.dumps(base))
    sc["Domain"].update({"conservativeAxialMomentum": False, "conservativeRadialForce": True})
    p2 = build_params(ParticleSystem(SimConfig(sc), device="cpu"))
    assert (p2.axi_conservative_x, p2.axi_conservative_r) == (0, 1)
    assert p2.hg_rate == p0.hg_rate                # the axis ratio is back with either form

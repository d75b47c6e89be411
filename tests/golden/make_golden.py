"""Generates tests/golden/reference_host.json from the reference's own host-side code.

Runs only where the reference source is present (it imports config_builder, materials,
geometry and the material models' float64 `_py` mirrors from it, with a stand-in
`taichi` module that turns the decorators into no-ops; no Taichi kernel runs).  The
fixture it writes is committed and is all the tests read.

    python tests/golden/make_golden.py /path/to/reference
    SIGMASPH_REFERENCE=/path/to/reference python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIGMASPH_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py /path/to/sigmaSPH (or set SIGMASPH_REFERENCE)")
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

STUB = '''
def func(f=None, **k): return f if f is not None else (lambda g: g)
def kernel(f=None, **k): return f if f is not None else (lambda g: g)
def data_oriented(c): return c
class _Any:
    def __getattr__(self, n): return _Any()
    def __call__(self, *a, **k): return _Any()
    def __getitem__(self, k): return _Any()
    def __setitem__(self, k, v): pass
f32 = float; f64 = float; i32 = int; u32 = int; float32 = float; float64 = float; int32 = int
def template(): return None
def static(x): return x
types = _Any(); math = _Any(); algorithms = _Any(); Vector = _Any(); Matrix = _Any(); field = _Any()
def __getattr__(n): return _Any()
'''

KEYS = ["particleRadius", "supportRadiusFactor", "axisymmetric", "planeStrain", "CFL",
        "viscosity", "allowNegativePressure", "DISPLACEMENT_POSITIONS", "COMPENSATED_VOLUME",
        "DOMAIN_BOUNDARY", "DOMAIN_RESTITUTION", "c0", "density0", "exponent", "DELTA_SPH",
        "DELTA_PAIRS", "PST_ENABLED", "PST_MODE", "PST_MA_MODE", "PST_MA_FIXED", "PST_R",
        "PST_N", "PST_MAX_SHIFT", "PST_LAMBDA_LO", "PST_LAMBDA_HI", "PST_CLAMP",
        "PST_M_DELTA", "PST_NORMAL", "PST_SURFACE_SHIFT", "PST_ALE_MOMENTUM",
        "PST_ALE_HISTORY", "L_EIG_TOL_LAM", "L_EIG_TOL", "KERNEL_CORRECTION",
        "TRACK_VISCOUS_WORK", "HOURGLASS_ALPHA", "HOURGLASS_STS_MODE",
        "HOURGLASS_STS_STAGES", "HOURGLASS_STS_REFRESH", "HOURGLASS_STS_SAFETY",
        "rampTime", "gravitation", "DT_PAIR_SOUND_SPEED", "AXI_R_MIN", "timeStepSize"]


def main():
    tmp = tempfile.mkdtemp()
    os.makedirs(os.path.join(tmp, "taichi"))
    with open(os.path.join(tmp, "taichi", "__init__.py"), "w") as f:
        f.write(STUB)
    sys.path[:0] = [tmp, REF]
    from config_builder import SimConfig
    from geometry import lattice_points, region_from_spec
    from material_models.EOS001_tait import tait_pressure_py, tait_specific_energy_py
    from material_models.EOS000_linear import linear_pressure_py
    from material_models.MAT001_linear_plasticity import j2_radial_return_py
    from material_models import MAT002_johnson_cook as jc

    decks = {
        "tensile_axi_dogbone_dx0.1": os.path.join(REF, "data", "scenes",
                                                  "tensile_axi_dogbone_nofail_dx0.1.json"),
        "dambreak3d_1M": os.path.join(REPO, "sigmasph_b200", "scenes", "dambreak3d_1M.json"),
    }
    out = {"decks": {}, "eos": {}, "plasticity": {}}
    for name, path in decks.items():
        c = SimConfig(path, verbose=False)
        d = {"config": {k: c.get_cfg(k) for k in KEYS}, "materials": {}}
        for mname, m in c.get_materials().items():
            d["materials"][mname] = {"rho0": m.rho0, "K": m.K, "G": m.G, "c_p": m.c_p,
                                     "c_eos": m.c_eos, "sigma_y0": m.sigma_y0,
                                     "hardening": m.hardening, "plastic_kind": int(m.plastic_kind),
                                     "specific_heat": m.specific_heat, "delta": m.delta}
        blocks = c.get_fluid_blocks() + c.get_solid_blocks()
        dxp = 2.0 * float(c.get_cfg("particleRadius"))
        pos = []
        for b in blocks:
            lower = np.array(b["start"]) + np.array(b["translation"])
            size = (np.array(b["end"]) - np.array(b["start"])) * np.array(b["scale"])
            pts = lattice_points(lower, size, dxp, 3)
            region = region_from_spec(b.get("shape"), pts.astype(np.float64).mean(axis=0))
            if region is not None:
                pts = pts[region.contains(pts)]
            pos.append(pts)
        pos = np.concatenate(pos).astype(np.float32)
        d["particles"] = int(len(pos))
        d["positions_sha256"] = hashlib.sha256(np.ascontiguousarray(pos).tobytes()).hexdigest()
        d["first_positions"] = pos[:4].tolist()
        out["decks"][name] = d

    rng = np.random.default_rng(20260101)
    rho = (1000.0 * (1.0 + rng.uniform(-0.05, 0.05, 16))).tolist()
    out["eos"]["tait"] = [{"rho": r, "rho0": 1000.0, "S": 1.682e5, "gamma": 7.0,
                           "p": tait_pressure_py(r, 1000.0, 1.682e5, 7.0),
                           "e": tait_specific_energy_py(r, 1000.0, 1.682e5, 7.0)} for r in rho]
    out["eos"]["linear"] = [{"rho": 7.9e-6 * (1 + d), "rho0": 7.9e-6, "K": 160.83,
                             "p": linear_pressure_py(7.9e-6 * (1 + d), 7.9e-6, 160.83)}
                            for d in rng.uniform(-0.01, 0.01, 8).tolist()]
    j2 = []
    for _ in range(24):
        s = rng.normal(0.0, 0.4, (3, 3))
        s = 0.5 * (s + s.T)
        s -= np.trace(s) / 3.0 * np.eye(3)
        ep = float(rng.uniform(0.0, 0.3))
        res = j2_radial_return_py(s.tolist(), 76.92, 0.3, 1.0, ep)
        j2.append({"s": s.tolist(), "eps_p": ep, "sy0": 0.3, "H": 1.0, "G": 76.92,
                   "out": [np.asarray(r).tolist() if hasattr(r, "__len__") else float(r) for r in res]})
    out["plasticity"]["j2"] = j2
    jcs = []
    for _ in range(24):
        s = rng.normal(0.0, 0.6, (3, 3))
        s = 0.5 * (s + s.T)
        s -= np.trace(s) / 3.0 * np.eye(3)
        ep = float(rng.uniform(0.0, 0.5))
        dt = float(10 ** rng.uniform(-6, -4))
        temp = float(rng.uniform(293.0, 600.0))
        # (s_trial, G, rho0, A, B, n, C, eps0_dot, T0, Tm, m, Cp, chi, eps_p, temp, dt)
        args = [s.tolist(), 76.92, 7.9e-6, 0.31, 1.0, 0.65, 0.02, 1.0, 293.0, 1720.0, 1.0,
                500.0, 0.9, ep, temp, dt]
        res = jc.jc_radial_return_py(*args)
        jcs.append({"args": args,
                    "out": [np.asarray(r).tolist() if hasattr(r, "__len__") else float(r) for r in res]})
    out["plasticity"]["jc"] = jcs
    path = os.path.join(HERE, "reference_host.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()

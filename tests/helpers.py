"""Shared test helpers: build a scene on the GPU and the matching oracle run."""
import numpy as np

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.solver import build_params
from oracle.oracle import Oracle, state_from_sets


def by_pid(a, pid):
    order = np.argsort(pid)
    return a[order]


def perturb(ps, seed=20260101, dv=0.05, drho=0.003, dshift=2e-3):
    """Seeded random velocity, density and previous-shift fields, so every term of the
    step (viscosity, diffusion, pressure, ALE transport) is active from the first step."""
    rng = np.random.default_rng(seed)
    n = ps.particle_max_num
    v = ps.v.to_numpy() + rng.uniform(-dv, dv, (n, 3)).astype(np.float32)
    if ps.two_d:
        v[:, 2] = 0.0
    ps.v.from_numpy(v)
    V = ps.V.to_numpy() * (1.0 + rng.uniform(-drho, drho, n)).astype(np.float32)
    ps.V.from_numpy(V.astype(np.float32))
    sh = (rng.uniform(-1.0, 1.0, (n, 3)) * dshift * ps.particle_diameter).astype(np.float32)
    if ps.two_d:
        sh[:, 2] = 0.0
    ps.pst_shift.from_numpy(sh)


def make_pair(scene, fp64=True, device="cuda", perturbed=True, oracles=None):
    """(ps, solver, oracle) at the same initial state, both before the first sort."""
    cfg = SimConfig(scene)
    ps = ParticleSystem(cfg, device=device)
    if perturbed:
        perturb(ps)
    solver = ps.build_solver()
    st0 = state_from_sets(ps.state_numpy())
    p = build_params(ps)
    orc = Oracle(p, ps.particle_max_num, fp64=fp64)
    orc.set_state(st0, solver.dt[None])
    return ps, solver, orc


def pair_set(pi, pj, pm, pid):
    """Pairs as a set of (pid_i, pid_j, mirror)."""
    return set(zip(pid[pi].tolist(), pid[pj].tolist(), pm.tolist()))


def rel_err(a, b, floor):
    return np.abs(a - b).max() / max(np.abs(b).max(), floor)


def gpu_fields(ps):
    """Reference-layout dict of the GPU state, rows ordered by pid."""
    s = ps.state_numpy()
    d = {k: t.detach().cpu().numpy().copy() for k, t in ps.derived().items()}
    pid = s["pid"]
    o = np.argsort(pid)
    out = {"x": s["pos"][o, :3], "V": s["pos"][o, 3], "v": s["vel"][o, :3], "m": s["vel"][o, 3],
           "x0": s["x0"][o, :3], "V_lo": s["x0"][o, 3], "u": s["disp"][o, :3],
           "pressure": s["disp"][o, 3], "pst_shift": s["shift"][o, :3],
           "acc": d["acc"][o, :3], "de_visc": d["acc"][o, 3], "lam": d["lam"][o, 0],
           "L_sym": d["lsym"][o, :6], "lam_grad": d["lgrad"][o, :3],
           "divergence": d["div"][o, 0]}
    return {k: np.asarray(v, dtype=np.float64) for k, v in out.items()}


def oracle_fields(orc):
    r = orc.get_state()
    o = np.argsort(r["pid"])
    return {k: (v[o] if hasattr(v, "shape") and v.shape and v.shape[0] == len(o) else v)
            for k, v in r.items()}


def field_errors(g, r, keys):
    """max |g - r| / max |r| per field."""
    out = {}
    for k in keys:
        a, b = np.asarray(g[k], dtype=np.float64), np.asarray(r[k], dtype=np.float64)
        scale = np.abs(b).max()
        out[k] = float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a - b).max())
    return out

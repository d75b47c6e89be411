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


def make_pair(scene, fp64=True, device="cuda", perturbed=True, oracles=None, mass_jitter=0.0):
    """(ps, solver, oracle) at the same initial state, both before the first sort;
    mass_jitter > 0 gives every particle its own mass (m (1 + U(-j, j)))."""
    cfg = SimConfig(scene)
    ps = ParticleSystem(cfg, device=device)
    if perturbed:
        perturb(ps)
    if mass_jitter > 0.0:
        m = ps.m.to_numpy().astype(np.float64)
        m *= 1.0 + np.random.default_rng(17).uniform(-mass_jitter, mass_jitter, m.shape)
        ps.m.from_numpy(m.astype(np.float32))
    solver = ps.build_solver()
    st0 = state_from_sets(ps.state_numpy())
    p = build_params(ps)
    orc = Oracle(p, ps.particle_max_num, fp64=fp64)
    orc.set_state(st0, solver.dt[None])
    return ps, solver, orc


def pair_set(pi, pj, pm, pid):
    """Pairs as a set of (pid_i, pid_j, mirror)."""
    return set(zip(pid[pi].tolist(), pid[pj].tolist(), pm.tolist()))


def check_shift_pairs(ps, solver, seed, reach):
    """After the sort, moves every particle by at most reach * h (random direction and
    length), then checks that the pairs the shift pass takes from the sort's lists equal,
    as a set, the live search against the stale bins (particle_system.py:1377-1411).
    Returns how many particles changed cells along 0, 1, 2 and 3 axes."""
    h = float(ps.support_radius)
    x = ps.x.to_numpy()
    rng = np.random.default_rng(seed)
    d = rng.normal(size=x.shape)
    if ps.two_d:
        d[:, 2] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d *= rng.uniform(0.0, reach * h, (len(x), 1))
    # half of the particles that can reach a cell corner (3 axes) or edge (2 axes) within
    # the bound step just past it, so multi-axis cell changes are always covered
    ax = 2 if ps.two_d else 3
    xd = x[:, :ax].astype(np.float64)
    o = np.round(xd / h) * h - xd
    o += np.where(o < 0, -1e-3, 1e-3) * h + np.where(o == 0, -2e-3, 0.0) * h
    order = np.argsort(np.abs(o), axis=1)
    for k in (ax, 2):
        t = np.zeros_like(o)
        rows = np.arange(len(x))[:, None]
        t[rows, order[:, :k]] = o[rows, order[:, :k]]
        ok = (np.linalg.norm(t, axis=1) < reach * h) & (rng.uniform(size=len(x)) < 0.5)
        d[ok] = 0.0
        d[ok, :ax] = t[ok]
    x1 = (x + d).astype(np.float32)
    moved = np.linalg.norm(x1.astype(np.float64) - x.astype(np.float64), axis=1).max()
    ps.x.from_numpy(x1)
    pid = ps.pid.to_numpy()
    A = solver.shift_pairs(float(moved) * (1.0 + 1e-5))
    B = solver.pairs(1)
    SA, SB = pair_set(*A, pid), pair_set(*B, pid)
    assert len(SA) == len(A[0]), "duplicate pairs in the shift's enumeration"
    assert SA == SB, (len(SA - SB), len(SB - SA))
    axes = (np.floor(x1.astype(np.float64) / h) != np.floor(x.astype(np.float64) / h)).sum(axis=1)
    return np.bincount(axes, minlength=4)


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


# Per-particle relative error: |g_i - r_i| / max(|r_i|, PP_FLOOR * max |r|).  Values above
# 1% of the field's largest are compared relative to themselves, so a particle whose
# value is small but wrong shows, which the field-wide max |g - r| / max |r| hides.
PP_FLOOR = 1e-2


def pp_errors(g, r, keys, floor=PP_FLOOR):
    """max over particles (and components) of the per-particle relative error, per field."""
    out = {}
    for k in keys:
        a, b = np.asarray(g[k], dtype=np.float64), np.asarray(r[k], dtype=np.float64)
        scale = np.abs(b).max()
        den = np.maximum(np.abs(b), floor * scale)
        d = np.abs(a - b)
        out[k] = float((d / np.where(den > 0, den, 1.0)).max()) if scale > 0 else float(d.max())
    return out


def check_pp(g, r32, r64, keys, factor=4.0, slack=1e-5):
    """Every particle of the GPU field is as close to the float64 oracle, relative to its
    own value (floor PP_FLOOR of the largest), as the float32 oracle's worst particle is:
    max_i e_i(GPU, FP64) <= factor * max_i e_i(FP32, FP64) + slack.  Both sides carry
    float32 rounding in a different order, so a factor of a few covers the summation-order
    noise; a wrong particle anywhere above 1% of the field's largest fails it."""
    eg = pp_errors(g, r64, keys)
    eo = pp_errors(r32, r64, keys)
    for k in keys:
        assert eg[k] <= factor * eo[k] + slack, (k, eg[k], eo[k])
    return eg, eo


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


def gpu_state(ps):
    s = ps.state_numpy()
    d = {k: v.detach().cpu().numpy().copy() for k, v in ps.derived().items()}
    return s, d


def make_pair(scene, fp64=True, device="cuda"):
    """(ps, solver, oracle) at the same initial state, both after the first sort."""
    cfg = SimConfig(scene)
    ps = ParticleSystem(cfg, device=device)
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

"""Stage-by-stage parity at the benchmarked sizes.

The small-deck tests (test_fluid_gpu.py, test_solid_gpu.py) cover every branch; these run
one step of the workloads bench.py times, each stage against the float32 and float64
oracles with the small decks' tolerances and the per-particle check:
  * the 3D dam break at 1,000,188 particles (dx = 4.762 mm), perturbed so that every term
    of the step is live;
  * the 3D round bar at dx = 0.16 mm (about 0.84M particles: the bench's 2.38M at
    dx = 0.113 mm takes the oracle tens of seconds per step), J2, in-loop damper.
The neighbour pair sets are compared as sorted 64-bit keys (pid_i, pid_j, mirror), all
80M (dam break) pairs bit for bit.  Field tolerances: the small decks' bounds, or three
times the float32 oracle's own distance to the float64 oracle where that is larger (the
field-wide maximum over a million particles reaches further into the tails of the
float32 rounding than over eight thousand).
"""
import os

import numpy as np
import pytest

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import dambreak3d, tensile_bar3d
from sigmasph_b200.solver import build_params
from oracle.oracle import Oracle, state_from_sets
from tests.helpers import (perturb, gpu_fields, oracle_fields, field_errors, check_pp)
from tests.test_fluid_gpu import STAGE_FIELDS, LOOSE32, LOOSE64
from tests import test_solid_gpu as tsg

pytestmark = pytest.mark.gpu


def pair_keys(pi, pj, pm, pid):
    """Sorted int64 keys pid_i << 33 | pid_j << 2 | mirror (pid < 2^29)."""
    pid = np.asarray(pid, dtype=np.int64)
    k = (pid[pi] << 33) | (pid[pj] << 2) | np.asarray(pm, dtype=np.int64)
    k.sort()
    return k


def _oracles(ps, solver):
    Oracle.threads(os.cpu_count())
    p = build_params(ps)
    st0 = state_from_sets(ps.state_numpy())
    out = []
    for fp64 in (False, True):
        o = Oracle(p, ps.particle_max_num, fp64=fp64)
        o.set_state(st0, solver.dt[None])
        out.append(o)
    return out


def _same_pairs(ps, solver, o32):
    gk = pair_keys(*solver.pairs(0), ps.pid.to_numpy())
    ok = pair_keys(*o32.pairs(), o32.get_state()["pid"])
    assert gk.size == ok.size, (gk.size, ok.size)
    assert np.array_equal(gk, ok)
    assert np.all(np.diff(gk) > 0), "duplicate pairs on the GPU"
    return gk.size


def test_dambreak_1m_stage_parity(cuda):
    ps = ParticleSystem(SimConfig(dambreak3d()), device="cuda")
    assert ps.particle_max_num == 1000188
    perturb(ps)
    solver = ps.build_solver()
    o32, o64 = _oracles(ps, solver)
    for s in range(8):
        solver.run_stage(s)
        o32.stage(s)
        o64.stage(s)
        if s == abi.STAGE_SORT:
            npairs = _same_pairs(ps, solver, o32)
            assert npairs > 70_000_000
        if s not in STAGE_FIELDS:
            continue
        g, r32, r64 = gpu_fields(ps), oracle_fields(o32), oracle_fields(o64)
        keys = STAGE_FIELDS[s]
        e32, e64 = field_errors(g, r32, keys), field_errors(g, r64, keys)
        eo = field_errors(r32, r64, keys)
        for k, e in e32.items():
            assert e <= max(LOOSE32.get(k, 2e-5), 3.0 * eo[k]), (s, k, e, eo[k])
        for k, e in e64.items():
            assert e <= max(LOOSE64.get(k, 1e-4), 3.0 * eo[k]), (s, k, e, eo[k])
        check_pp(g, r32, r64, keys)
        if s == abi.STAGE_ADVECT:
            assert abs(solver.dt[None] - o32.scalars()["dt"]) <= 1e-6 * o32.scalars()["dt"]
    assert solver.error_word() & ~abi.EW_HASHED_GRID == 0


def test_bar3d_stage_parity_at_scale(cuda):
    ps = ParticleSystem(SimConfig(tensile_bar3d(dx=0.16)), device="cuda")
    assert ps.particle_max_num > 800_000
    tsg.perturb_solid(ps)
    solver = ps.build_solver()
    o32, o64 = _oracles(ps, solver)
    for s in range(8):
        solver.run_stage(s)
        o32.stage(s)
        o64.stage(s)
        if s == abi.STAGE_SORT:
            _same_pairs(ps, solver, o32)
        if s not in tsg.STAGE_FIELDS:
            continue
        g = tsg.solid_gpu_fields(ps)
        r32, r64 = tsg.solid_oracle_fields(o32), tsg.solid_oracle_fields(o64)
        keys = tsg.STAGE_FIELDS[s]
        e32, e64 = tsg.errs(g, r32, keys), tsg.errs(g, r64, keys)
        eo = tsg.errs(r32, r64, keys)
        for k, e in e32.items():
            assert e <= max(tsg.TOL32.get(k, 5e-5), 3.0 * eo[k]), (s, k, e, eo[k])
        for k, e in e64.items():
            assert e <= max(tsg.TOL64.get(k, 2e-4), 3.0 * eo[k]), (s, k, e, eo[k])
        check_pp(g, r32, r64, keys)
    sg, s32 = solver._scalars(), o32.scalars()
    assert abs(sg.dt - s32["dt"]) <= 1e-6 * s32["dt"]
    fg = np.array([[sg.constraint_force[k][d] for d in range(3)] for k in range(2)])
    assert np.abs(fg - s32["constraint_force"][:2]).max() <= 1e-4 * np.abs(s32["constraint_force"][:2]).max()
    assert solver.error_word() & ~abi.EW_HASHED_GRID == 0

"""GPU parity of the delta+-SPH step against the CPU oracle (through the C-ABI)."""
import numpy as np
import pytest

from sigmasph_b200 import abi
from sigmasph_b200.scenes import dambreak3d, dx_for_particles
from tests.helpers import make_pair, pair_set, by_pid, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(cuda):
    return dambreak3d(dx=dx_for_particles(8000))


def test_pair_set_bit_exact(small):
    ps, solver, orc = make_pair(small, fp64=False)
    solver.initialize()
    orc.stage(abi.STAGE_SORT)
    gi, gj, gm = solver.pairs(0)
    pid_g = ps.pid.to_numpy()
    oi, oj, om = orc.pairs()
    pid_o = orc.get_state()["pid"]
    sg = pair_set(gi, gj, gm, pid_g)
    so = pair_set(oi, oj, om, pid_o)
    assert len(gi) == len(sg)
    assert sg == so
    assert solver.error_word() & abi.EW_NBR_OVERFLOW == 0


def test_one_step_matches_fp64_oracle(small):
    ps, solver, orc = make_pair(small, fp64=True)
    solver.initialize()
    orc.stage(abi.STAGE_SORT)
    solver.step()
    orc.step(1)
    g = ps.state_numpy()
    r = orc.get_state()
    pid = g["pid"]
    xg = by_pid(g["pos"][:, :3].astype(np.float64), pid)
    xr = by_pid(r["x"], r["pid"])
    vg = by_pid(g["vel"][:, :3].astype(np.float64), pid)
    vr = by_pid(r["v"], r["pid"])
    assert np.abs(xg - xr).max() < 1e-5 * ps.particle_diameter
    assert rel_err(vg, vr, 1e-9) < 1e-5
    assert abs(solver.dt[None] - orc.scalars()["dt"]) <= 1e-6 * orc.scalars()["dt"]

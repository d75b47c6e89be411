"""Ensembles of plane-strain strips in one packed handle (sigmasph_b200.ensemble): each
strip, re-expressed in units of its own spacing and run alongside strips of other
spacings and materials, reproduces the same strip run alone as an ordinary scene --
clock, time step, grip force and fields within 1e-3 of the single run after 150 steps
(float32 rounding of the rescaled quantities differs, nothing else); the block size
changes no field; the bucketed, autotuned, graph-captured ensemble runs."""
import numpy as np
import pytest
import torch

from sigmasph_b200.config import SimConfig
from sigmasph_b200.ensemble import Ensemble, StripSpec, strip_deck, strip_specs
from sigmasph_b200.particle_system import ParticleSystem

pytestmark = pytest.mark.gpu


def small_specs():
    return [StripSpec(2.4, 12.0, 0.2, 0.31, 1.0, 0.65, speed=50.0),
            StripSpec(3.0, 10.0, 0.125, 0.25, 0.8, 0.4, speed=50.0),
            StripSpec(2.0, 9.0, 0.1, 0.45, 1.3, 0.55, speed=50.0)]


def _fields(ps, sel, scale):
    st = ps.state_numpy()
    pid = st["pid"]
    rows = np.nonzero(sel[pid])[0]
    o = rows[np.argsort(pid[rows])]
    return {"x": st["pos"][o, :3].astype(np.float64) * scale,
            "v": st["vel"][o, :3].astype(np.float64) * scale,
            "sdev": st["sdev"][o, :6].astype(np.float64),
            "eps_p": st["sdev"][o, 6].astype(np.float64),
            "p": st["disp"][o, 3].astype(np.float64)}


def test_packed_strips_match_single_runs(cuda):
    specs = small_specs()
    ens = Ensemble(specs, buckets=1)
    b = ens.buckets[0]
    steps = 150
    b.solver.step_many(steps)
    states = b.state()
    inst = b.inst
    for k0, s in enumerate(specs):
        _, k = ens.locate(k0)              # the bucket orders its strips by size
        ps = ParticleSystem(SimConfig(strip_deck(s)), device="cuda")
        sv = ps.build_solver()
        sv.initialize()
        sv.step_many(steps)
        sc = sv._scalars()
        st = states[k]
        assert st["sim_time"] == pytest.approx(sc.sim_time, rel=1e-5)
        assert st["dt"] == pytest.approx(sc.dt, rel=1e-5)
        assert st["sts_stages"] == sc.sts_stages
        fs = np.array([[sc.constraint_force[g][d] for d in range(3)] for g in range(2)])
        assert np.abs(st["force"] - fs).max() <= 1e-3 * np.abs(fs).max() + 1e-12
        single = _fields(ps, np.ones(ps.particle_max_num, dtype=bool), 1.0)
        packed = _fields(b.ps, inst == k, s.dx)
        for key in ("v", "sdev", "eps_p", "p"):
            sc_ = max(np.abs(single[key]).max(), 1e-30)
            assert np.abs(packed[key] - single[key]).max() <= 1e-3 * sc_, (k, key)
        # positions: the same lattice, shifted to the strip's tile in the packing (the
        # tile origin is a whole number of spacings, read off the first particle's x0)
        x0p = b.ps.x_0.to_numpy()[np.nonzero(inst[b.ps.pid.to_numpy()] == k)[0]]
        origin = np.floor(x0p.min(axis=0) + 0.5) * s.dx
        assert np.abs(packed["x"] - origin - single["x"]).max() <= 1e-3 * s.dx, k
        assert single["eps_p"].max() > 0.0       # the strips have yielded


def test_block_size_changes_no_field(cuda):
    out = []
    for threads in (128, 256):
        ens = Ensemble(small_specs(), buckets=1)
        ens.buckets[0].set_block(threads)
        ens.buckets[0].solver.step_many(20)
        torch.cuda.synchronize()
        out.append(ens.buckets[0].ps.state_numpy())
    for key in ("pos", "vel", "sdev"):
        assert np.array_equal(out[0][key], out[1][key]), key


def test_bucketed_autotuned_graph_ensemble(cuda):
    specs = strip_specs(count=12, seed=5, target=60000, n_min=2000, n_max=8000)
    ens = Ensemble(specs, buckets=2)
    choice = ens.autotune(candidates=(64, 128, 256), steps=2)
    assert len(choice) == 2 and all(c["block"] in (64, 128, 256) for c in choice)
    ens.capture()
    for _ in range(5):
        ens.step2()
    torch.cuda.synchronize()
    for k in range(len(specs)):
        st = ens.state(k)
        assert np.isfinite(st["force"]).all()
        assert st["sim_time"] > 0.0 and st["dt"] > 0.0
    # every strip advanced by its own dt: 2 x (2 autotune warm-up + 2 timed) x 3 sizes + 2 + 10 steps
    t = np.array([ens.state(k)["sim_time"] / ens.state(k)["dt"] for k in range(len(specs))])
    assert np.all(t > 10)

"""Ensembles of independent plane-strain tensile strips run as packed batches.

No counterpart in the reference, which runs one scene per process
(run_simulation.py:649-708).  Every strip is resolved as an ordinary scene (the deck of
`strip_deck`, through the same SimConfig / build_params as a single run) and then
re-expressed in units of its own particle spacing dx: lengths / dx, velocities and
sound speeds (the delta-SPH and shift speed c0 among them) / dx, density * dx^2,
kinematic viscosity and specific heat / dx^2; stresses, times, rates, the time step and
the dimensionless coefficients are unchanged.  The SPH
equations are invariant under that scaling, so strips of different dx share one support
radius (3) and one cell grid, and a bucket of strips runs as ONE solid handle: one set of
kernel launches over all of its particles, each particle's material row being its
strip's, with per-strip time step, clock, load ramp, damper stage count and grips on the
device (sph_ensemble_set).  The strips are tiled with gaps wider than two supports, so
no pair crosses between strips.

By default all strips share one handle (buckets=1): one set of ~60 kernel launches per
step over all ~6M particles, 16.0 ms per ensemble step for the 256 strips against 16.5 ms
as four size buckets.  Strips can also be grouped into size buckets (one handle each);
`autotune` picks each bucket's threads per block by timing; `capture` records two steps
of every bucket into one CUDA graph, so `step2()` advances the whole ensemble two steps
with one graph launch.  The
cell size is the support radius in every bucket: it is the stale-bin window of the
reference's shift search (particle_system.py:1377-1411), which the pair set must keep.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import abi
from .config import SimConfig
from .particle_system import ParticleSystem
from .solver import build_params

GAP = 10.0          # normalised units between strips (> 2 x support radius 3)


@dataclass
class StripSpec:
    width: float          # mm (x)
    length: float         # mm (y, pull axis)
    dx: float             # mm
    A: float              # GPa
    B: float              # GPa
    n: float
    speed: float = 1.0    # grip speed, m/s = mm/ms
    disp: float = 1.0     # mm per grip

    @property
    def nx(self):
        return max(1, int(round(self.width / self.dx)))

    @property
    def ny(self):
        return max(1, int(round(self.length / self.dx)))

    @property
    def particles(self):
        return self.nx * self.ny


def strip_specs(count=256, seed=20260101, n_min=2000, n_max=60000, target=6_000_000):
    """Widths U(2, 8) mm, lengths U(20, 60) mm, dx U(0.05, 0.2) mm; Johnson-Cook A U(0.2, 0.5),
    B U(0.5, 1.5) GPa, n U(0.3, 0.7).  The spacings are then rescaled together (within
    0.05-0.2 mm) toward `target` particles in all, each strip kept within n_min..n_max."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        w, L, dx = rng.uniform(2.0, 8.0), rng.uniform(20.0, 60.0), rng.uniform(0.05, 0.2)
        s = StripSpec(w, L, dx, rng.uniform(0.2, 0.5), rng.uniform(0.5, 1.5), rng.uniform(0.3, 0.7))
        if n_min <= s.particles <= n_max:
            out.append(s)
    if target:
        for _ in range(20):
            scale = math.sqrt(sum(s.particles for s in out) / float(target))
            if abs(scale - 1.0) < 1e-3:
                break
            for s in out:
                lo = math.sqrt(s.width * s.length / n_max)     # spacing giving n_max
                hi = math.sqrt(s.width * s.length / n_min)
                s.dx = min(max(s.dx * scale, 0.05, lo * 1.001), 0.2, hi * 0.999)
    return out


def shard(specs, world, rank):
    """The strips `rank` steps when `world` GPUs share one ensemble: largest first, each to
    the rank holding the fewest particles so far (ties to the lower rank), so the ranks'
    particle counts differ by at most one strip.  Deterministic; returned in spec order."""
    load = [0] * int(world)
    owner = [0] * len(specs)
    for k in sorted(range(len(specs)), key=lambda k: (-specs[k].particles, k)):
        r = min(range(int(world)), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += specs[k].particles
    return [k for k in range(len(specs)) if owner[k] == rank]


STATE_COLUMNS = ("sim_time", "dt", "load_s", "sts_stages", "force_x0", "force_y0", "force_z0",
                 "force_x1", "force_y1", "force_z1", "disp_x0", "disp_y0", "disp_z0",
                 "disp_x1", "disp_y1", "disp_z1")


def state_row(st):
    """One strip's state (Ensemble.state) as a float64 row in STATE_COLUMNS order."""
    return np.concatenate([[st["sim_time"], st["dt"], st["load_s"], st["sts_stages"]],
                           np.asarray(st["force"], np.float64).ravel(),
                           np.asarray(st["disp"], np.float64).ravel()]).astype(np.float64)


def strip_deck(s: StripSpec):
    """One strip as an ordinary plane-strain scene in physical units (mm, GPa, ms): steel
    (rho 7.9e-6, E 200, nu 0.3, linear EOS), Johnson-Cook (C 0, no thermal softening),
    sub-cycled hourglass damper, Colle shifting at a fixed Mach 0.05, delta 0.1,
    viscosity 0.02; grips = the outer 10% of the length, pulled apart by `disp` each over
    a smoothstep ramp of disp / speed."""
    dx = s.dx
    Lx, Ly = (s.nx - 0.5) * dx, (s.ny - 0.5) * dx
    g = 0.1 * (s.ny - 1) * dx
    return {
        "Domain": {"particleRadius": 0.5 * dx, "supportRadiusFactor": 6.0, "planeStrain": True,
                   "boundary": "open"},
        "Time": {"CFL": 0.3},
        "Solver": {"type": "hypoElastic", "viscosity": 0.02, "allowNegativePressure": True},
        "Materials": [{"name": "steel", "density0": 7.9e-6, "eos": {"type": "linear"},
                       "strength": {"type": "hypoElastic", "youngsModulus": 200.0, "poissonRatio": 0.3,
                                    "plasticity": {"model": "johnson_cook", "A": s.A, "B": s.B, "n": s.n,
                                                   "C": 0.0, "eps0_dot": 1.0, "T0": 293.0, "Tm": 0.0}}}],
        "Load": {"gravitation": [0.0, 0.0, 0.0], "rampTime": s.disp / s.speed},
        "Diffusion": {"delta": 0.1},
        "Shifting": {"enabled": True, "mode": "colle", "maMode": "fixed", "maFixed": 0.05},
        "Hourglass": {"alpha": 4.0, "superTimeStepping": {"mode": "subcycle"}},
        "SolidBlocks": [{"objectId": 0, "start": [0.0, 0.0, 0.0], "end": [Lx, Ly, 0.5 * dx],
                         "material": "steel", "density": 7.9e-6}],
        "Constraints": [
            {"name": "low", "region": [[-1.0, -1.0, -1.0], [Lx + 1.0, g + 1e-6 * dx, 1.0]],
             "components": "xy", "displacement": [0.0, -s.disp, 0.0]},
            {"name": "high", "region": [[-1.0, Ly - g - 1e-6 * dx, -1.0], [Lx + 1.0, Ly + 1.0, 1.0]],
             "components": "xy", "displacement": [0.0, s.disp, 0.0]}],
    }


def normalised_rows(s: StripSpec):
    """(SphMatRow, SphInstRow, dt0, mass per particle) of a strip in units of its dx,
    from the strip's own resolved scene parameters."""
    ps = ParticleSystem(SimConfig(strip_deck(s)), device="cpu")
    p = build_params(ps)
    dx = s.dx
    m = abi.SphMatRow()
    m.rho0 = p.mat_rho0[0] * dx * dx
    m.K, m.G = p.mat_K[0], p.mat_G[0]
    m.cp, m.c0 = p.mat_cp[0] / dx, p.mat_c0[0] / dx
    m.delta = p.mat_delta[0]
    m.plastic_kind, m.sy0, m.H = p.plastic_kind[0], p.plastic_sy0[0], p.plastic_H[0]
    m.jc_A, m.jc_B, m.jc_n, m.jc_C = p.jc_A[0], p.jc_B[0], p.jc_n[0], p.jc_C[0]
    m.jc_eps0_dot, m.jc_T0, m.jc_Tm, m.jc_m, m.jc_chi = (p.jc_eps0_dot[0], p.jc_T0[0], p.jc_Tm[0],
                                                        p.jc_m[0], p.jc_chi[0])
    m.cv = p.mat_cv[0] / (dx * dx)
    m.stiff, m.gamma, m.T0 = p.mat_stiff[0], p.mat_gamma[0], p.mat_T0[0]
    r = abi.SphInstRow()
    r.c_signal = p.c_signal / dx
    r.hg_rate = p.hg_rate
    r.ramp_time = p.ramp_time
    r.c0 = p.c0 / dx
    r.visc_coef = 10.0 * p.viscosity / (dx * dx)
    dt0 = p.CFL * p.support_radius / p.c_signal
    mass = float(ps.m.to_numpy()[0])
    return m, r, dt0, mass, p


class _Bucket:
    """One packed handle over a group of strips."""

    def __init__(self, specs, device="cuda"):
        self.specs = list(specs)
        self.device = torch.device(device)
        # tile the strips in rows of roughly square overall extent, in normalised units
        total_w = sum(s.nx + GAP for s in self.specs)
        row_w = max(max(s.nx for s in self.specs) + GAP, math.sqrt(total_w * max(s.ny for s in self.specs)))
        blocks, origins, x, y, row_h = [], [], 0.0, 0.0, 0.0
        for k, s in enumerate(self.specs):
            if x > 0.0 and x + s.nx > row_w:
                x, y, row_h = 0.0, y + row_h + GAP, 0.0
            origins.append((x, y))
            blocks.append({"objectId": k, "start": [x, y, 0.0], "end": [x + s.nx - 0.5, y + s.ny - 0.5, 0.5],
                           "material": "strip", "density": 1.0})
            x += s.nx + GAP
            row_h = max(row_h, s.ny)
        rows = [normalised_rows(s) for s in self.specs]
        template = strip_deck(self.specs[0])
        template["Domain"] = {"particleRadius": 0.5, "supportRadiusFactor": 6.0, "planeStrain": True,
                              "boundary": "open"}
        mat = template["Materials"][0]
        mat["name"], mat["density0"] = "strip", 1.0
        template["SolidBlocks"] = blocks
        template.pop("Constraints")
        self.ps = ParticleSystem(SimConfig(template), device=device)
        ps = self.ps
        n = ps.particle_max_num
        assert n == sum(s.particles for s in self.specs), "lattice does not match the strip specs"
        obj = ps.object_id.to_numpy()              # creation order: strip index per particle
        x0 = ps.x.to_numpy()
        inst = obj.astype(np.int32)
        mass = np.array([r[3] for r in rows], dtype=np.float32)[inst]
        bc = np.zeros((n, 2), dtype=np.int32)
        bcd = np.zeros((n, 4), dtype=np.float32)
        bcd[:, 3] = inst.astype(np.float32)
        for k, s in enumerate(self.specs):
            sel = inst == k
            yl = x0[sel, 1] - origins[k][1]
            g = 0.1 * (s.ny - 1)
            low, high = yl <= g + 1e-6, yl >= (s.ny - 1) - g - 1e-6
            b = np.zeros((sel.sum(), 2), dtype=np.int32)
            b[:, 1] = -1
            b[low, 0], b[low, 1] = 3, 0
            b[high, 0], b[high, 1] = 3, 1
            bc[sel] = b
            d = np.zeros((sel.sum(), 4), dtype=np.float32)
            d[low, 1] = -s.disp / s.dx
            d[high, 1] = s.disp / s.dx
            d[:, 3] = k
            bcd[sel] = d
        s0 = ps.buffer_sets()[0]
        s0["vel"][:, 3].copy_(torch.from_numpy(mass))
        s0["bc"].copy_(torch.from_numpy(bc))
        s0["bcdisp"].copy_(torch.from_numpy(bcd))
        self.inst = inst
        self.solver = ps.build_solver()
        L = self.solver.L
        nI = len(self.specs)
        self._mats = (abi.SphMatRow * nI)(*[r[0] for r in rows])
        self._irows = (abi.SphInstRow * nI)(*[r[1] for r in rows])
        self._dt0 = (C.c_float * nI)(*[r[2] for r in rows])
        abi.check(L.sph_ensemble_set(self.solver.h, self._mats, self._irows, nI, self._dt0,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream)), "sph_ensemble_set")
        self.block = 256

    @property
    def particles(self):
        return self.ps.particle_max_num

    def set_block(self, threads):
        abi.check(self.solver.L.sph_set_block(self.solver.h, int(threads)), "sph_set_block")
        self.block = int(threads)

    def state(self):
        nI = len(self.specs)
        out = (abi.SphInstState * nI)()
        abi.check(self.solver.L.sph_ensemble_state(self.solver.h, out, nI,
                                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)),
                  "sph_ensemble_state")
        res = []
        for k, s in enumerate(self.specs):
            st = out[k]
            # forces per unit thickness scale back by dx, displacements by dx
            res.append({"sim_time": st.sim_time, "dt": st.dt, "load_s": st.load_s,
                        "sts_stages": st.sts_stages,
                        "force": np.array([[st.constraint_force[g][d] * s.dx for d in range(3)] for g in range(2)]),
                        "disp": np.array([[st.constraint_disp[g][d] * s.dx for d in range(3)] for g in range(2)])})
        return res


class Ensemble:
    """Strips grouped into size buckets, each a packed handle."""

    def __init__(self, specs, buckets=1, device="cuda"):
        self.specs = list(specs)
        order = sorted(range(len(self.specs)), key=lambda k: self.specs[k].particles)
        groups = [g for g in np.array_split(np.array(order), max(1, min(buckets, len(order)))) if len(g)]
        self.buckets = [_Bucket([self.specs[k] for k in g], device=device) for g in groups]
        self.index = [(b, j) for b, g in enumerate(groups) for j in range(len(g))]
        self._where = {int(k): (b, j) for b, g in enumerate(groups) for j, k in enumerate(g)}
        self.graph = None
        for b in self.buckets:
            b.solver.initialize()

    @property
    def particles(self):
        return sum(b.particles for b in self.buckets)

    def autotune(self, candidates=(64, 128, 192, 256), steps=6):
        """Times `steps` steps of each bucket at each block size and keeps the fastest."""
        choice = []
        for b in self.buckets:
            best, best_ms = None, None
            for t in candidates:
                b.set_block(t)
                b.solver.step_many(2)              # warm-up, graph rebuilt for this shape
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                b.solver.step_many(steps)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / steps
                if best_ms is None or ms < best_ms:
                    best, best_ms = t, ms
            b.set_block(best)
            choice.append({"particles": b.particles, "strips": len(b.specs), "block": best,
                           "ms_per_step": best_ms})
        self.graph = None
        return choice

    def capture(self):
        """One CUDA graph with two steps of every bucket."""
        for b in self.buckets:                     # warm the per-handle state outside capture
            b.solver.step_many(2)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for b in self.buckets:
                b.solver.step()
                b.solver.step()
        self.graph = g
        return g

    def step2(self):
        """Two steps of every strip: one graph launch."""
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def locate(self, k):
        """(bucket, instance within the bucket) of strip k; buckets hold strips by size."""
        return self._where[k]

    def state(self, k):
        b, j = self._where[k]
        return self.buckets[b].state()[j]

    def state_rows(self):
        """Every strip's state as float64 rows (STATE_COLUMNS), in spec order; one read
        per bucket."""
        per = [b.state() for b in self.buckets]
        return np.stack([state_row(per[b][j]) for b, j in (self._where[k] for k in range(len(self.specs)))])

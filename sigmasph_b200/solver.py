"""The solvers' Python API (DSPH.py DSPHSolver, SOLID.py HypoElasticSolver, sph_base.py
SPHBase) over libsph_b200.

`solver.step()` is one asynchronous launch sequence on the current torch stream (one
CUDA graph per pair of steps when `step_many` is used); nothing is computed on the host.
The 0-d fields of the reference (`dt[None]`, `load_s[None]`, ...) read the device
scalars back, which synchronises, exactly like a Taichi `[None]` read.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import abi
from .particle_system import ScalarRef


def _stream_ptr():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def build_params(ps) -> abi.SphParams:
    """Flatten the resolved scene into SphParams (DSPH.py:64-450, SOLID.py:138-1452)."""
    cfg = ps.cfg
    g = lambda k: cfg.get_cfg(k)
    p = abi.SphParams()
    p.struct_size = C.sizeof(abi.SphParams)
    p.is_solid = int(ps.is_solid)
    p.two_d = int(ps.two_d)
    p.axisymmetric = int(ps.axisymmetric)
    p.plane_strain = int(ps.plane_strain)
    p.sym_y, p.sym_z = int(ps.sym_y), int(ps.sym_z)
    p.walls = int(ps.walls)
    p.displacement_positions = int(ps.displacement_positions)
    p.compensated_volume = int(ps.compensated_volume)
    p.support_radius = ps.support_radius
    p.particle_diameter = ps.particle_diameter
    p.V0 = ps.V0
    p.axi_r_min = ps.axi_r_min
    for k in range(3):
        p.domain_size[k] = float(ps.domain_size[k])
        p.gravity[k] = float((g("gravitation") or [0, 0, 0])[k])
    p.padding = ps.padding
    p.wall_restitution = ps.wall_restitution
    c0 = float(g("c0"))
    rho0 = float(g("density0"))
    gam = float(g("exponent") or 1.0)
    p.density0, p.c0, p.exponent = rho0, c0, gam
    p.stiffness = c0 * c0 * rho0 / gam
    p.viscosity = float(g("viscosity"))
    p.CFL = float(g("CFL"))
    p.delta_sph = float(g("DELTA_SPH") or 0.0)
    p.allow_negative_pressure = int(bool(g("allowNegativePressure")))
    track = g("TRACK_VISCOUS_WORK")
    p.track_visc_work = int((True if track is None else bool(track)) and p.viscosity > 0.0
                            and not ps.is_solid)
    tl = g("L_EIG_TOL_LAM")
    p.l_eig_tol_lam = 0.02 if tl is None else float(tl)
    p.c_signal = c0
    p.dt_pair_mode = 1
    p.pst_enabled = int(bool(g("PST_ENABLED")))
    mode = str(g("PST_MODE") or "sun").lower()
    p.pst_colle = int(mode == "colle")
    ma = str(g("PST_MA_MODE") or "local").lower()
    p.pst_ma_mode = {"local": 0, "global": 1, "fixed": 2}[ma]
    clamp = str(g("PST_CLAMP")).lower()
    p.pst_clamp_disp = int(clamp in ("displacement", "both"))
    p.pst_clamp_vel = int(clamp in ("velocity", "both"))
    p.pst_surface_none = int(str(g("PST_SURFACE_SHIFT") or "tangential").lower() == "none")
    p.pst_normal_eigvec = int(str(g("PST_NORMAL") or "gradlam").lower() == "eigvec")
    am = g("PST_ALE_MOMENTUM")
    p.pst_ale_momentum = int(True if am is None else bool(am))
    p.pst_R = float(g("PST_R"))
    p.pst_n = int(g("PST_N"))
    p.pst_max_shift = float(g("PST_MAX_SHIFT"))
    p.pst_ma_fixed = float(g("PST_MA_FIXED"))
    p.pst_m_delta = float(g("PST_M_DELTA"))
    p.pst_lambda_lo = float(g("PST_LAMBDA_LO"))
    p.pst_lambda_hi = float(g("PST_LAMBDA_HI"))
    if ps.is_solid:
        from .solid_params import fill_solid_params
        fill_solid_params(ps, p)
    return p


class ResidualField:
    """relax_res (DSPH.py:1097-1100): each particle's relaxation residual |g| / dx0 from
    the latest pass, in the current storage order, one float per particle slot."""

    def __init__(self, n, device):
        self.t = torch.zeros(n, dtype=torch.float32, device=device)

    def data_ptr(self):
        return self.t.data_ptr()

    def to_numpy(self):
        return self.t.cpu().numpy()


class _SolverBase:
    """SPHBase + the shared half of DSPHSolver (sph_base.py, DSPH.py)."""

    def __init__(self, ps):
        if ps.device.type != "cuda":
            raise RuntimeError("sigmasph_b200 solvers run on a CUDA device only (no CPU "
                               "fallback); construct the ParticleSystem with device='cuda'")
        self.ps = ps
        self.L = abi.lib()
        self.params = build_params(ps)
        self.h = C.c_void_p()
        abi.check(self.L.sph_create(C.byref(self.params), ps.particle_max_num, C.byref(self.h)),
                  "sph_create")
        self._bind()
        ps._parity_fn = lambda: self.L.sph_parity(self.h)
        ps._solver = self
        cfg = ps.cfg
        self.CFL = float(cfg.get_cfg("CFL"))
        self.c0 = float(cfg.get_cfg("c0"))
        self.density_0 = float(cfg.get_cfg("density0"))
        self.exponent = float(cfg.get_cfg("exponent") or 1.0)
        self.stiffness = self.c0 ** 2 * self.density_0 / self.exponent
        self.viscosity = float(cfg.get_cfg("viscosity"))
        self.g = np.array(cfg.get_cfg("gravitation"), dtype=np.float64)
        self.dt = ScalarRef(self._get_dt, self._set_dt)
        user_dt = cfg.get_cfg("timeStepSize")
        if user_dt is not None:
            self._set_dt(float(user_dt))
        self.dt_max = float(self._get_dt())
        self.lam = ps.lam
        self.relax_frame_hook = None
        self.relax_res = None
        from .particle_system import Field
        self.lam_grad = Field(ps, "lgrad", slice(0, 3))
        self.L_sym = Field(ps, "lsym", slice(0, 6))

    def _bind(self):
        ps = self.ps
        b = abi.SphBuffers()
        for k, s in enumerate(ps.buffer_sets()):
            fs = b.set[k]
            for key in ("pos", "vel", "x0", "disp", "shift", "pid", "sdev", "bc", "bcdisp", "acc"):
                t = s.get(key)
                setattr(fs, key, t.data_ptr() if t is not None else None)
        d = ps.derived()
        for key in ("acc", "lam", "lsym", "lgrad", "div", "gradv", "aux"):
            t = d.get(key)
            setattr(b, key, t.data_ptr() if t is not None else None)
        self._buffers = b
        abi.check(self.L.sph_bind(self.h, C.byref(b), ps.particle_max_num), "sph_bind")

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                self.L.sph_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    # ------------------------------------------------------------------ scalars
    def _scalars(self) -> abi.SphScalars:
        s = abi.SphScalars()
        abi.check(self.L.sph_get_scalars(self.h, C.byref(s), _stream_ptr()), "sph_get_scalars")
        return s

    def _get_dt(self):
        v = C.c_float()
        abi.check(self.L.sph_get_dt(self.h, C.byref(v), _stream_ptr()), "sph_get_dt")
        return float(v.value)

    def _set_dt(self, value):
        abi.check(self.L.sph_set_dt(self.h, C.c_float(float(value)), _stream_ptr()), "sph_set_dt")

    def error_word(self):
        return int(self._scalars().err)

    def clear_error(self):
        abi.check(self.L.sph_clear_error(self.h, _stream_ptr()))

    # ------------------------------------------------------------------ stepping
    def _initialize_grid(self):
        abi.check(self.L.sph_initialize(self.h, _stream_ptr()), "sph_initialize")

    def initialize(self):
        """SPHBase.initialize (sph_base.py:154): the first neighbour build; then, with the
        shift on and Shifting.initialRelaxation > 0, the initial relaxation
        (DSPH.py:1060-1063)."""
        self._initialize_grid()
        self.relax_report = None
        steps = int(self.ps.cfg.get_cfg("PST_RELAX_STEPS") or 0)
        if steps > 0 and bool(self.ps.cfg.get_cfg("PST_ENABLED")):
            tol = self.ps.cfg.get_cfg("PST_RELAX_TOL")
            self.relax_report = self.relax_initial_configuration(steps, 0.03 if tol is None else float(tol))

    def relax_initial_configuration(self, steps, tol, beta=0.05):
        """relax_initial_configuration (DSPH.py:1113-1179): before t = 0, move the frozen
        body by the run's own shift drive -- disorder sum, free-surface treatment, gripped
        particles held -- until the residual max h^2 |S| / dx0 falls below `tol` or for
        `steps` passes, each particle keeping its volume and mass; the relaxed positions
        become x_0, the displacement and the stored shift are cleared.  Returns {passes,
        residual_first, residual_last, converged, moved_max, moved_mean} (moves in units of
        the spacing).

        relax_frame_hook (DSPH.py:217-221), when set, is called as hook(k, residual, final)
        with the body at the positions of pass k (k = 0 the laid positions) and lam and
        relax_res (each particle's |g| / dx0, storage order) computed there: before every
        move, and once more at the relaxed positions with final=True."""
        ps = self.ps
        pid0 = ps.pid.to_numpy()
        x_start = ps.x.to_numpy()[np.argsort(pid0)].astype(np.float64)
        res = C.c_float()
        hook = self.relax_frame_hook
        each = None
        if hook is not None:
            self.relax_res = ResidualField(ps.particle_max_num, ps.device)
            each = self.relax_res.data_ptr()

        def one_pass():
            abi.check(self.L.sph_relax_pass(self.h, float(beta), C.byref(res), each,
                                            _stream_ptr()), "sph_relax_pass")
            return float(res.value)

        first = last = 0.0
        k = 0
        for k in range(1, int(steps) + 1):
            last = one_pass()
            if hook is not None:
                hook(k - 1, last, False)
            abi.check(self.L.sph_relax_move(self.h, _stream_ptr()), "sph_relax_move")
            if k == 1:
                first = last
            if last < tol:
                break
        if hook is not None:
            hook(k, one_pass(), True)
        ps.pst_shift.fill(0.0)
        self._initialize_grid()
        x = ps.x.to_numpy()
        moved = np.linalg.norm(x[np.argsort(ps.pid.to_numpy())].astype(np.float64) - x_start,
                               axis=1) / ps.particle_diameter
        ps.x_0.copy_from(ps.x)
        ps.u.fill(0.0)
        return {"passes": k, "residual_first": first, "residual_last": last,
                "converged": bool(last < tol), "moved_max": float(moved.max()),
                "moved_mean": float(moved.mean())}

    def step(self):
        """SPHBase.step (sph_base.py:622-655): one asynchronous step."""
        abi.check(self.L.sph_step(self.h, 1, _stream_ptr()), "sph_step")

    def step_many(self, nsteps):
        """nsteps steps with dt kept on the device; pairs of steps replay one CUDA graph."""
        abi.check(self.L.sph_step(self.h, int(nsteps), _stream_ptr()), "sph_step")

    def profile(self, on=True):
        """Per-kernel CUDA-event timing of eager launches (step(), run_stage())."""
        abi.check(self.L.sph_profile_enable(self.h, int(bool(on))))

    def profile_read(self):
        """{kernel: (total_ms, launches)} since the last read."""
        cap = 64
        names = C.create_string_buffer(4096)
        ms = (C.c_double * cap)()
        cnt = (C.c_int * cap)()
        m = C.c_int()
        abi.check(self.L.sph_profile_read(self.h, names, 4096, ms, cnt, cap, C.byref(m)))
        keys = names.value.decode().split("\n")
        return {keys[k]: (ms[k], cnt[k]) for k in range(m.value)}

    def run_stage(self, stage):
        abi.check(self.L.sph_run_stage(self.h, int(stage), _stream_ptr()), "sph_run_stage")

    def pairs(self, mode=0):
        """(i, j, mirror) neighbour triples of the current bins, current-order indices."""
        cnt = C.c_int64()
        abi.check(self.L.sph_pairs(self.h, mode, None, None, None, 0, C.byref(cnt), _stream_ptr()))
        n = cnt.value
        pi = np.zeros(n, dtype=np.int32)
        pj = np.zeros(n, dtype=np.int32)
        pm = np.zeros(n, dtype=np.int32)
        if n:
            abi.check(self.L.sph_pairs(self.h, mode, pi.ctypes.data, pj.ctypes.data, pm.ctypes.data,
                                       n, C.byref(cnt), _stream_ptr()))
        return pi, pj, pm

    def shift_pairs(self, disp_bound=-1.0):
        """(i, j, mirror) triples the shift pass evaluates at the current positions;
        disp_bound >= 0 is the caller's bound on every particle's move since the sort."""
        cnt = C.c_int64()
        f = self.L.sph_shift_pairs
        abi.check(f(self.h, disp_bound, None, None, None, 0, C.byref(cnt), _stream_ptr()))
        n = cnt.value
        pi = np.zeros(n, dtype=np.int32)
        pj = np.zeros(n, dtype=np.int32)
        pm = np.zeros(n, dtype=np.int32)
        if n:
            abi.check(f(self.h, disp_bound, pi.ctypes.data, pj.ctypes.data, pm.ctypes.data, n,
                        C.byref(cnt), _stream_ptr()))
        return pi, pj, pm

    def list_stats(self, reset=False):
        """Candidate-list statistics: steps, steps that built the lists, shift passes that
        searched the coarse table."""
        out = (C.c_uint64 * 3)()
        abi.check(self.L.sph_list_stats(self.h, out, int(bool(reset)), _stream_ptr()), "sph_list_stats")
        return {"steps": out[0], "builds": out[1], "shift_searches": out[2]}

    # ------------------------------------------------------------------ reductions
    def _reduce(self):
        out = (C.c_double * abi.RED_COUNT)()
        abi.check(self.L.sph_reduce(self.h, out, _stream_ptr()), "sph_reduce")
        return list(out)

    def compute_total_mass(self):
        return self._reduce()[abi.RED_MASS]

    def compute_kinetic_energy(self):
        return self._reduce()[abi.RED_KE]

    def compute_kinetic_energy_off_grid(self):
        return self._reduce()[abi.RED_KE_OFFGRID]

    def compute_potential_energy(self):
        return self._reduce()[abi.RED_PE]

    def compute_internal_energy(self):
        return self._reduce()[abi.RED_IE]

    def compute_momentum(self):
        r = self._reduce()
        return np.array([r[abi.RED_PX], r[abi.RED_PY], r[abi.RED_PZ]], dtype=np.float64)

    def compute_gross_momentum(self):
        return float(self._reduce()[abi.RED_GROSS_P])

    def compute_wall_energy(self):
        return float(self._scalars().wall_work)

    def compute_leftover_energy(self):
        return float(self._scalars().leftover_work)

    def compute_viscous_energy(self):
        return float(self._scalars().visc_work)

    def compute_diffusion_work(self):
        return float(self._scalars().diff_work)

    def compute_integrated_gap(self):
        return self.compute_diffusion_work()


class DSPHSolver(_SolverBase):
    """delta+-SPH fluid solver (DSPH.py:50-1883)."""

    def compute_elastic_energy(self):
        return self._reduce()[abi.RED_SE]

    def compute_hourglass_energy(self):
        return 0.0

    def energy_budget(self):
        """DSPH.py:1800-1852."""
        r = self._reduce()
        s = self._scalars()
        ke, se, pe = r[abi.RED_KE], r[abi.RED_SE], r[abi.RED_PE]
        lw = float(s.leftover_work)
        wd = float(s.diff_work)
        return {"ke": ke, "se": se, "pe": pe, "ie": 0.0, "hg": 0.0,
                "wall": float(s.wall_work), "visc": float(s.visc_work),
                "leftover": lw, "leftover_raw": lw, "comp": se, "comp_complete": True,
                "e_neg": 0.0, "pw": 0.0, "wd": wd, "gap_integrated": wd,
                "total": ke + se + pe}


class HypoElasticSolver(_SolverBase):
    """Hypoelastic tensile-solid solver (SOLID.py:136-5231)."""

    def __init__(self, ps):
        super().__init__(ps)
        self.load_s = ScalarRef(lambda: float(self._scalars().load_s))
        self.load_sdot = ScalarRef(lambda: float(self._scalars().load_sdot))
        self.constraints_list = list(ps.cfg.get_constraints())
        self.num_constraints = len(self.constraints_list)

    @property
    def sim_time(self):
        return float(self._scalars().sim_time)

    def compute_elastic_energy(self):
        return self._reduce()[abi.RED_ELASTIC]

    def compute_hourglass_energy(self):
        return float(self._scalars().hg_work)

    def compute_plastic_work(self):
        return float(self._scalars().plastic_work)

    def get_constraint_data(self):
        """SOLID.py:5198-5225: each grip's FP64 force and displacement of the last step
        (sph_constraints)."""
        k = self.num_constraints
        if k == 0:
            return []
        force = np.zeros((k, 3), dtype=np.float64)
        disp = np.zeros((k, 3), dtype=np.float64)
        abi.check(self.L.sph_constraints(self.h, force.ctypes.data, disp.ctypes.data, k, _stream_ptr()),
                  "sph_constraints")
        out = []
        for g in range(k):
            name = self.constraints_list[g].get("name", f"constraint_{g}")
            out.append({"index": g, "name": name, "displacement": disp[g].copy(),
                        "force": force[g].copy()})
        return out

    # ------------------------------------------------------------------ JC surrogate
    def enable_jc_surrogate(self, surrogate, tol=1e-3):
        """Johnson-Cook returns proposed by `surrogate` (a JCSurrogate) on the tensor
        cores and kept where |g| / sigma_y <= tol; the exact Newton elsewhere."""
        self._jc_surrogate = surrogate          # keeps its parameters alive
        abi.check(self.L.sph_jc_surrogate(self.h, C.c_void_p(surrogate.W.data_ptr()), C.c_float(tol),
                                          1, _stream_ptr()), "sph_jc_surrogate")

    def disable_jc_surrogate(self):
        abi.check(self.L.sph_jc_surrogate(self.h, None, C.c_float(1.0), 0, _stream_ptr()),
                  "sph_jc_surrogate")

    def attach_jc_log(self, rows, count):
        """Log every exact Johnson-Cook return into rows [cap][8] (float32 CUDA tensor),
        counting into count (one int64 CUDA tensor); None detaches."""
        self._jc_log = (rows, count)
        if rows is None:
            abi.check(self.L.sph_jc_log(self.h, None, 0, None), "sph_jc_log")
            return
        abi.check(self.L.sph_jc_log(self.h, C.c_void_p(rows.data_ptr()), rows.shape[0],
                                    C.c_void_p(count.data_ptr())), "sph_jc_log")

    def jc_stats(self, reset=False):
        """{newton_solves, newton_iterations, proposals, accepted} since the last reset."""
        out = (C.c_uint64 * 4)()
        abi.check(self.L.sph_jc_stats(self.h, out, int(bool(reset)), _stream_ptr()), "sph_jc_stats")
        return dict(zip(("newton_solves", "newton_iterations", "proposals", "accepted"), list(out)))

    def energy_budget(self):
        r = self._reduce()
        s = self._scalars()
        ke, ie, el = r[abi.RED_KE], r[abi.RED_IE], r[abi.RED_ELASTIC]
        pe, hg, lw = r[abi.RED_PE], float(s.hg_work), float(s.leftover_work)
        return {"ke": ke, "ie": ie, "se": el, "pe": pe, "hg": hg,
                "wall": float(s.wall_work), "visc": float(s.visc_work), "leftover": lw,
                "leftover_raw": lw, "pw": float(s.plastic_work), "wd": float(s.diff_work),
                "total": ke + ie + hg + pe - lw}

"""ParticleSystem: the reference's particle store (particle_system.py:23-1849) with its
field API, over PyTorch tensors laid out for the sm_100a kernels.

Every persistent per-particle field lives in buffer set A; set B is the scratch of the
reorder (a neighbour-list build gathers A into B in the new Morton cell order and copies
it back), and the library reports which set is current.  The attributes below always read
and write the current set, so a caller sees exactly the reference's fields:

    ps.x, ps.V         set.pos   [n, 4]  (x, y, z, V)
    ps.v, ps.m         set.vel   [n, 4]  (vx, vy, vz, m)
    ps.x_0, ps.V_lo    set.x0    [n, 4]
    ps.u, ps.pressure  set.disp  [n, 4]
    ps.pst_shift, ps.e_int   set.shift [n, 4]  (fluid: w is the kernels' scratch)
    ps.sigma_dev, ps.eps_plastic, ps.temperature   set.sdev [n, 8] (solid)
    ps.bc_flag, ps.bc_id     set.bc     [n, 2] int32 (solid)
    ps.bc_disp, ps.eos_id    set.bcdisp [n, 4] (solid)

Constant per-particle tags (object_id, material, color) are kept once, in creation
order, and looked up through the persistent particle id `pid` that travels with the
sort; they are never copied by it.
"""
from __future__ import annotations

import numpy as np
import torch

from .config import SimConfig, SceneError
from .geometry import lattice_points, region_from_spec


class ScalarRef:
    """A 0-d field: ``f[None]`` reads, ``f[None] = v`` writes (Taichi's scalar API)."""

    def __init__(self, get, set_=None):
        self._get = get
        self._set = set_

    def __getitem__(self, key):
        return self._get()

    def __setitem__(self, key, value):
        if self._set is None:
            raise AttributeError("read-only scalar")
        self._set(value)


class Field:
    """A per-particle field with the Taichi field methods the reference's callers use
    (to_numpy / from_numpy / fill / shape).  `view()` returns the torch view of the
    current buffer set."""

    def __init__(self, ps, set_key, cols, kind="vec", dtype=np.float32, n_comp=None,
                 by_pid=None):
        self.ps = ps
        self.set_key = set_key      # name of the tensor in a buffer set, or a derived tensor
        self.cols = cols            # slice of columns (or an int)
        self.kind = kind            # "vec", "scalar", "symmat", "int_from_float", "pid_table"
        self.dtype = dtype
        self.by_pid = by_pid        # for constant tags: the creation-order array

    @property
    def shape(self):
        n = self.ps.particle_max_num
        if self.kind == "vec":
            return (n, self.cols.stop - self.cols.start)
        if self.kind == "symmat":
            return (n, 3, 3)
        if self.kind == "pid_table" and self.by_pid.ndim > 1:
            return (n,) + self.by_pid.shape[1:]
        return (n,)

    def view(self):
        t = self.ps._tensor(self.set_key)
        return t if self.cols is None else t[:, self.cols]

    def to_numpy(self):
        if self.kind == "pid_table":
            pid = self.ps.pid.to_numpy()
            return self.by_pid[pid]
        a = self.view().detach().cpu().numpy()
        if self.kind == "symmat":
            out = np.empty((a.shape[0], 3, 3), dtype=np.float32)
            out[:, 0, 0], out[:, 1, 1], out[:, 2, 2] = a[:, 0], a[:, 1], a[:, 2]
            out[:, 0, 1] = out[:, 1, 0] = a[:, 3]
            out[:, 0, 2] = out[:, 2, 0] = a[:, 4]
            out[:, 1, 2] = out[:, 2, 1] = a[:, 5]
            return out
        if self.kind == "int_from_float":
            return np.rint(a).astype(np.int32)
        return a.copy()

    def from_numpy(self, arr):
        if self.kind == "pid_table":
            raise AttributeError("constant per-particle tag: set at creation")
        arr = np.asarray(arr)
        if self.kind == "symmat":
            a = np.stack([arr[:, 0, 0], arr[:, 1, 1], arr[:, 2, 2],
                          0.5 * (arr[:, 0, 1] + arr[:, 1, 0]),
                          0.5 * (arr[:, 0, 2] + arr[:, 2, 0]),
                          0.5 * (arr[:, 1, 2] + arr[:, 2, 1])], axis=1)
            arr = a
        v = self.view()
        src = torch.as_tensor(np.ascontiguousarray(arr), device=v.device).to(v.dtype)
        v.copy_(src.reshape(v.shape))
        self.ps._invalidate()

    def fill(self, value):
        self.view().fill_(value)
        self.ps._invalidate()

    def copy_from(self, other):
        self.view().copy_(other.view())
        self.ps._invalidate()


SET_KEYS = ("pos", "vel", "x0", "disp", "shift", "pid", "sdev", "bc", "bcdisp")


class ParticleSystem:
    """The particle store and its field API (particle_system.py:25-475, 956-1146)."""

    def __init__(self, config: SimConfig, GGUI=False, device=None):
        if GGUI:
            raise SceneError("the GGUI window is not available: sigmasph_b200 runs headless")
        self.cfg = config
        self.GGUI = False
        self.device = torch.device(device if device is not None else
                                   ("cuda" if torch.cuda.is_available() else "cpu"))
        c = config
        ds = c.get_cfg("domainStart")
        de = c.get_cfg("domainEnd")
        self.domain_start = np.array(ds if ds is not None else [0.0, 0.0, 0.0])
        self.domain_end = np.array(de if de is not None else [1.0, 1.0, 1.0])
        self.domain_size = self.domain_end - self.domain_start
        self.plane_strain = bool(c.get_cfg("planeStrain") or False)
        self.axisymmetric = bool(c.get_cfg("axisymmetric") or False)
        if self.axisymmetric and self.plane_strain:
            raise SceneError("planeStrain and axisymmetric cannot both be on")
        self.two_d = self.plane_strain or self.axisymmetric
        self.dim = 3
        sym = str(c.get_cfg("symmetryPlanes") or "").strip().lower()
        self.sym_y = "y" in sym
        self.sym_z = "z" in sym
        if sym and self.two_d:
            raise SceneError("Domain.symmetryPlanes needs a full 3D domain")
        self.mirror_y = self.axisymmetric or self.sym_y
        self.mirror_z = self.sym_z
        dp = c.get_cfg("DISPLACEMENT_POSITIONS")
        self.displacement_positions = True if dp is None else bool(dp)
        cv = c.get_cfg("COMPENSATED_VOLUME")
        self.compensated_volume = True if cv is None else bool(cv)
        self.simulation_method = c.get_cfg("simulationMethod")
        self.is_solid = self.simulation_method == "hypoElastic"
        self.walls = str(c.get_cfg("DOMAIN_BOUNDARY") or "open").lower() == "reflect"
        cf = c.get_cfg("DOMAIN_RESTITUTION")
        self.wall_restitution = 0.5 if cf is None else float(cf)
        if not 0.0 <= self.wall_restitution <= 1.0:
            raise ValueError("Domain.restitution must lie in [0, 1]")
        self.material_fluid, self.material_solid = 1, 2
        self.particle_radius = float(c.get_cfg("particleRadius"))
        self.particle_diameter = 2 * self.particle_radius
        srf = c.get_cfg("supportRadiusFactor")
        self.support_radius_factor = 4.0 if srf is None else float(srf)
        self.support_radius = self.particle_radius * self.support_radius_factor
        self.variable_h = False
        self.h_max = self.h_min = self.support_radius
        self.dt_length = self.support_radius
        self.V0 = self.particle_diameter ** 2 if self.two_d else self.particle_diameter ** 3
        rmin = c.get_cfg("AXI_R_MIN")
        self.axi_r_min = (0.5 if rmin is None else float(rmin)) * self.particle_diameter
        self.grid_size = self.support_radius
        self.padding = self.grid_size

        # ---------------------------------------------------------------- particles
        blocks = ([(b, self.material_fluid) for b in c.get_fluid_blocks()] +
                  [(b, self.material_solid) for b in c.get_solid_blocks()])
        xs, vs, rhos, mats, cols, objs, eos_ids = [], [], [], [], [], [], []
        mat_index = {name: m.index for name, m in c.get_materials().items()}
        self.object_collection = {}
        pfile = c.get_cfg("ParticlesFile")
        if pfile:
            self._particles_from_file(pfile, blocks, mat_index, xs, vs, rhos, mats, cols, objs, eos_ids)
            blocks = []
        for blk, mtag in blocks:
            for key in ("rotVelocity", "divVelocity"):
                if blk.get(key) is not None:
                    raise SceneError(f"block {key} initial conditions are not implemented by "
                                     "sigmasph_b200")
            lower = np.array(blk["start"], dtype=float) + np.array(blk["translation"], dtype=float)
            size = (np.array(blk["end"], dtype=float) - np.array(blk["start"], dtype=float)) * \
                np.array(blk["scale"], dtype=float)
            pts = lattice_points(lower, size, self.particle_diameter, self.dim)
            region = region_from_spec(blk.get("shape"), pts.astype(np.float64).mean(axis=0))
            if region is not None:
                pts = pts[region.contains(pts)]
            if len(pts) == 0:
                raise SceneError(f"block {blk['objectId']} is empty")
            blk["particleNum"] = len(pts)
            self.object_collection[blk["objectId"]] = blk
            n_b = len(pts)
            xs.append(pts.astype(np.float32))
            vs.append(np.tile(np.asarray(blk["velocity"], dtype=np.float32), (n_b, 1)))
            rhos.append(np.full(n_b, blk.get("density", 1000.0), dtype=np.float32))
            mats.append(np.full(n_b, mtag, dtype=np.int32))
            cols.append(np.tile(np.asarray(blk["color"], dtype=np.int32), (n_b, 1)))
            objs.append(np.full(n_b, int(blk["objectId"]), dtype=np.int32))
            eos_ids.append(np.full(n_b, mat_index.get(blk.get("material"), 0), dtype=np.int32))
        if not xs:
            raise SceneError("the scene lays no particles")
        x = np.concatenate(xs)
        n = len(x)
        self.fluid_particle_num = n
        self.particle_max_num = n
        self._particle_num = n
        self.particle_num = ScalarRef(lambda: self._particle_num)
        self._object_id = np.concatenate(objs)
        self._material = np.concatenate(mats)
        self._color = np.concatenate(cols)
        self._eos_id = np.concatenate(eos_ids)
        v = np.concatenate(vs)
        rho = np.concatenate(rhos)

        if self.two_d:
            if abs(float(x[:, 2].min()) - float(x[:, 2].max())) > 1.0e-8:
                raise SceneError("a single-layer (plane strain / axisymmetric) deck must lay one "
                                 "z layer")
        if self.axisymmetric:
            if float(x[:, 1].min()) < 0.0:
                raise SceneError("axisymmetric: every particle must have y >= 0")
            if abs(float(x[:, 2].min())) > 1.0e-8:
                raise SceneError("axisymmetric: every particle must sit at z = 0")
        for axis, on, name in ((1, self.sym_y, "y"), (2, self.sym_z, "z")):
            if on and float(x[:, axis].min()) < 0.0:
                raise SceneError(f"symmetryPlanes '{name}': every particle must have {name} >= 0")

        # add_particle (particle_system.py:1128-1146): m = rho V0 (r V0 in axisymmetry),
        # V = m / rho, all in float32
        V0 = np.float32(self.V0)
        vol = np.full(n, V0, dtype=np.float32)
        if self.axisymmetric:
            vol = (V0 * np.maximum(x[:, 1], np.float32(self.axi_r_min))).astype(np.float32)
        m = (vol * rho).astype(np.float32)
        V = (m / rho).astype(np.float32)

        # ---------------------------------------------------------------- buffers
        dev = self.device
        f32, i32 = torch.float32, torch.int32

        def z(*shape, dtype=f32):
            return torch.zeros(*shape, dtype=dtype, device=dev)

        self._sets = []
        for _ in range(2):
            s = {"pos": z(n, 4), "vel": z(n, 4), "x0": z(n, 4), "disp": z(n, 4),
                 "shift": z(n, 4), "pid": z(n, dtype=i32)}
            if self.is_solid:
                s["sdev"] = z(n, 8)
                s["bc"] = z(n, 2, dtype=i32)
                s["bcdisp"] = z(n, 4)
                s["acc"] = z(n, 4)     # acceleration + de_int, carried across the sort
            self._sets.append(s)
        self._derived = {"acc": z(n, 4), "lam": z(n, 1), "lsym": z(n, 8), "lgrad": z(n, 4),
                         "div": z(n, 4)}
        if self.is_solid:
            self._derived["gradv"] = z(n, 12)
            self._derived["aux"] = z(n, 24)
            # the solid's acceleration is persistent: it lives in the buffer sets
            del self._derived["acc"]
        s0 = self._sets[0]
        pos = np.zeros((n, 4), dtype=np.float32)
        pos[:, :3] = x
        pos[:, 3] = V
        vel = np.zeros((n, 4), dtype=np.float32)
        vel[:, :3] = v
        vel[:, 3] = m
        x0 = np.zeros((n, 4), dtype=np.float32)
        x0[:, :3] = x
        s0["pos"].copy_(torch.from_numpy(pos))
        s0["vel"].copy_(torch.from_numpy(vel))
        s0["x0"].copy_(torch.from_numpy(x0))
        s0["pid"].copy_(torch.arange(n, dtype=i32))
        if self.is_solid:
            bcd = np.zeros((n, 4), dtype=np.float32)
            bcd[:, 3] = self._eos_id.astype(np.float32)
            # reference temperature per material (materials.py:429-435); e_int starts at 0
            mats = sorted(config.get_materials().values(), key=lambda mm: mm.index)
            t0 = np.array([mm.jc["T0"] if mm.jc is not None else 293.0 for mm in mats],
                          dtype=np.float32)
            s0["sdev"][:, 7].copy_(torch.from_numpy(t0[self._eos_id]))
            s0["bcdisp"].copy_(torch.from_numpy(bcd))
        self._parity_fn = lambda: 0
        self._on_write = None

        # ---------------------------------------------------------------- field API
        sl = slice
        self.x = Field(self, "pos", sl(0, 3))
        self.V = Field(self, "pos", 3, "scalar")
        self.v = Field(self, "vel", sl(0, 3))
        self.m = Field(self, "vel", 3, "scalar")
        self.x_0 = Field(self, "x0", sl(0, 3))
        self.V_lo = Field(self, "x0", 3, "scalar")
        self.u = Field(self, "disp", sl(0, 3))
        self.pressure = Field(self, "disp", 3, "scalar")
        self.pst_shift = Field(self, "shift", sl(0, 3))
        self.pid = Field(self, "pid", None, "scalar", np.int32)
        self.acceleration = Field(self, "acc", sl(0, 3))
        self.lam = Field(self, "lam", 0, "scalar")
        self.divergence = Field(self, "div", 0, "scalar")
        self.object_id = Field(self, "pid", None, "pid_table", by_pid=self._object_id)
        self.material = Field(self, "pid", None, "pid_table", by_pid=self._material)
        self.color = Field(self, "pid", None, "pid_table", by_pid=self._color)
        if self.is_solid:
            self.e_int = Field(self, "shift", 3, "scalar")
            self.sigma_dev = Field(self, "sdev", sl(0, 6), "symmat")
            self.eps_plastic = Field(self, "sdev", 6, "scalar")
            self.temperature = Field(self, "sdev", 7, "scalar")
            self.bc_flag = Field(self, "bc", 0, "scalar", np.int32)
            self.bc_id = Field(self, "bc", 1, "scalar", np.int32)
            self.bc_disp = Field(self, "bcdisp", sl(0, 3))
            self.eos_id = Field(self, "bcdisp", 3, "int_from_float")
            self._apply_constraint_regions()
        self.off_grid_num = ScalarRef(lambda: self._scalar("off_grid_num"))
        self.off_grid_mass = ScalarRef(lambda: self._scalar("off_grid_mass"))
        self._solver = None

    # ------------------------------------------------------------------ internals
    def _particles_from_file(self, path, blocks, mat_index, xs, vs, rhos, mats, cols, objs, eos_ids):
        """_load_particles_from_file (particle_system.py:728-854): the file's particles,
        grouped by object id in ascending order; an object's material type, colour and
        material row come from the block of that objectId, an object without one is laid
        as solid with a grey of its id."""
        from .particles_file import read_particles_file, ParticlesFileError
        try:
            data = read_particles_file(path, self.two_d)
        except ParticlesFileError as e:
            raise SceneError(str(e))
        if data["size"] is not None and not np.allclose(data["size"], self.V0, rtol=1e-5, atol=0.0):
            raise SceneError(f"ParticlesFile '{path}' gives particles their own sizes: the variable "
                             f"smoothing length that needs is not implemented by sigmasph_b200")
        by_id = {int(b["objectId"]): (b, m) for b, m in blocks}
        oid = data["object_id"]
        for obj in sorted(np.unique(oid).tolist()):
            mask = oid == obj
            n_b = int(mask.sum())
            blk, mtag = by_id.get(obj, (None, self.material_solid))
            color = blk["color"] if blk is not None else [100 + obj * 50] * 3
            entry = {"objectId": obj, "particleNum": n_b}
            if blk is not None and blk.get("material") is not None:
                entry["material"] = blk["material"]
            self.object_collection[obj] = entry
            xs.append(data["position"][mask])
            vs.append(data["velocity"][mask])
            rhos.append(data["density"][mask])
            mats.append(np.full(n_b, mtag, dtype=np.int32))
            cols.append(np.tile(np.asarray(color, dtype=np.int32), (n_b, 1)))
            objs.append(np.full(n_b, obj, dtype=np.int32))
            eos_ids.append(np.full(n_b, mat_index.get(entry.get("material"), 0), dtype=np.int32))

    def _tensor(self, key):
        if key in self._derived:
            return self._derived[key]
        return self._sets[self._parity_fn()][key]

    def _invalidate(self):
        if self._on_write is not None:
            self._on_write()

    def _scalar(self, name):
        if self._solver is None:
            return 0
        return getattr(self._solver._scalars(), name)

    def buffer_sets(self):
        return self._sets

    def derived(self):
        return self._derived

    def _apply_constraint_regions(self):
        """particle_system.py:875-911: tag the particles inside each constraint box."""
        constraints = self.cfg.get_constraints()
        n = self.particle_max_num
        flag = np.zeros(n, dtype=np.int32)
        disp = np.zeros((n, 3), dtype=np.float32)
        cid = np.full(n, -1, dtype=np.int32)
        if constraints:
            xn = self.x.to_numpy()
            for k, con in enumerate(constraints):
                lo = np.array(con["region"][0], dtype=np.float64)
                hi = np.array(con["region"][1], dtype=np.float64)
                sel = np.all((xn >= lo) & (xn <= hi), axis=1)
                bits = 0
                for i, axis in enumerate("xyz"):
                    if axis in con.get("components", "xyz"):
                        bits |= 1 << i
                flag[sel] |= bits
                disp[sel] = np.array(con.get("displacement", [0.0] * 3), dtype=np.float32)
                cid[sel] = k
            if not flag.any():
                raise SceneError("Constraints were given but no particle falls inside any region")
        s0 = self._sets[0]
        s0["bc"][:, 0].copy_(torch.from_numpy(flag))
        s0["bc"][:, 1].copy_(torch.from_numpy(cid))
        s0["bcdisp"][:, :3].copy_(torch.from_numpy(disp))

    # ------------------------------------------------------------------ API
    def build_solver(self):
        """particle_system.py:958-966."""
        from .solver import DSPHSolver, HypoElasticSolver
        method = self.cfg.get_cfg("simulationMethod")
        if method == "deltaPlusSPH":
            return DSPHSolver(self)
        if method == "hypoElastic":
            return HypoElasticSolver(self)
        raise ValueError(f"simulationMethod must be 'deltaPlusSPH' or 'hypoElastic', got {method!r}")

    def initialize_particle_system(self):
        if self._solver is None:
            raise RuntimeError("build_solver() first: the neighbour build runs in libsph_b200")
        self._solver._initialize_grid()

    def resync_displacement(self):
        """u = x - x_0 after a write of x from outside the solver."""
        self.u.view().copy_(self.x.view() - self.x_0.view())

    def state_numpy(self):
        """Every persistent field of the current set, as numpy arrays keyed by set name."""
        p = self._parity_fn()
        return {k: t.detach().cpu().numpy().copy() for k, t in self._sets[p].items()}

    def dump(self, obj_id=None):
        """particle_system.py:1669-1755."""
        oid = self.object_id.to_numpy()
        mask = (oid >= 0).nonzero() if obj_id is None else (oid == obj_id).nonzero()
        pres = self.pressure.to_numpy()[mask]
        out = {"position": self.x.to_numpy()[mask], "velocity": self.v.to_numpy()[mask],
               "divergence": self.divergence.to_numpy()[mask], "lam": self.lam.to_numpy()[mask],
               "pressure": pres, "object_id": oid[mask],
               "density": self.m.to_numpy()[mask] / self.V.to_numpy()[mask]}
        if self.is_solid:
            s = self.sigma_dev.to_numpy()[mask]
            sig = -pres[:, None, None] * np.eye(3)[None] + s
            for (a, b), nm in {(0, 0): "xx", (1, 1): "yy", (2, 2): "zz", (0, 1): "xy",
                               (0, 2): "xz", (1, 2): "yz"}.items():
                out["sigma_" + nm] = sig[:, a, b]
            out["von_mises"] = np.sqrt(1.5 * np.einsum("kij,kij->k", s, s))
            out["eps_plastic"] = self.eps_plastic.to_numpy()[mask]
            out["eroded"] = np.zeros(len(pres), dtype=np.int32)
            out["e_int"] = self.e_int.to_numpy()[mask]
            out["temperature"] = self.temperature.to_numpy()[mask]
        return out

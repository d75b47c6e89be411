"""Trajectory output in the AMBER NetCDF convention (the reference's netcdf_writer.py:101-225),
for OVITO and other AMBER-aware readers, without the netCDF4 package.

The reference writes through netCDF4 in the classic 64-bit-offset container; netCDF4 is
not available here, so this module writes that container itself.  The classic format
(the "CDF-2" variant: magic "CDF\\x02", 8-byte variable offsets) is a short, published
layout: a header of dimensions, global attributes and variables, then the fixed-size
variables, then one record per frame holding every record variable's slab in order, all
big-endian and padded to 4 bytes.  A frame is appended by writing its record at the end
and then the header's record count, so a run killed at any point leaves a readable file
of every frame written so far.

What is written follows the reference, because the variable names are what OVITO maps
(`coordinates` and `velocities` become its Position and Velocity properties, every other
(frame, atom) variable a custom property of the same name): the AMBER label variables,
`time`, `coordinates`, `velocities`, `cell_lengths`, `cell_angles`, `id`, then the
per-particle fields of ParticleSystem.dump() -- always object_id, density, pressure, lam;
for a solid sigma_xx, sigma_yy, sigma_zz, sigma_xy, von_mises, eps_plastic, eroded, and in
3D sigma_xz, sigma_yz; then those optional fields the first dump carries; then the
caller's extra fields.  object_id and eroded are int32, the rest float32.
"""
from __future__ import annotations

import os
import struct

import numpy as np

_NC_CHAR, _NC_INT, _NC_FLOAT, _NC_DOUBLE = 2, 4, 5, 6
_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 0x0A, 0x0B, 0x0C
_SIZE = {_NC_CHAR: 1, _NC_INT: 4, _NC_FLOAT: 4, _NC_DOUBLE: 8}
_BE = {_NC_CHAR: "S1", _NC_INT: ">i4", _NC_FLOAT: ">f4", _NC_DOUBLE: ">f8"}

FIELDS_ALWAYS = [("object_id", "object_id"), ("density", "density"), ("pressure", "pressure"),
                 ("lam", "lam")]
FIELDS_SOLID = [("sigma_xx", "sigma_xx"), ("sigma_yy", "sigma_yy"), ("sigma_zz", "sigma_zz"),
                ("sigma_xy", "sigma_xy"), ("von_mises", "von_mises"),
                ("eps_plastic", "eps_plastic"), ("eroded", "eroded")]
FIELDS_SOLID_3D = [("sigma_xz", "sigma_xz"), ("sigma_yz", "sigma_yz")]
FIELDS_OPTIONAL = [("e_int", "e_int"), ("temperature", "temperature"), ("burn_f", "burn_f"),
                   ("damage", "damage"), ("porosity", "porosity"), ("ale_e_work", "ale_e_work"),
                   ("damage_t", "damage_t"), ("flaw_eps_min", "flaw_eps_min"),
                   ("jc_omega", "jc_omega"), ("h", "h")]
INTEGER_FIELDS = {"object_id", "eroded"}


def _pad(n):
    return (4 - n % 4) % 4


def _name(s):
    b = s.encode("ascii")
    return struct.pack(">i", len(b)) + b + b"\0" * _pad(len(b))


def _attrs(attrs):
    """Attribute list: text attributes as NC_CHAR."""
    if not attrs:
        return struct.pack(">ii", 0, 0)
    out = struct.pack(">ii", _NC_ATTRIBUTE, len(attrs))
    for k, v in attrs.items():
        b = str(v).encode("ascii")
        out += _name(k) + struct.pack(">ii", _NC_CHAR, len(b)) + b + b"\0" * _pad(len(b))
    return out


class _Var:
    def __init__(self, name, nc_type, dims, attrs=None, data=None):
        self.name, self.nc_type, self.dims = name, nc_type, dims
        self.attrs = attrs or {}
        self.data = data
        self.begin = 0
        self.vsize = 0


class NetCDFTrajectoryWriter:
    """One growing .nc file for the whole run, a frame at a time (the reference's class of
    the same name: created at the first write(), whose dump fixes the particle count and
    the field list)."""

    def __init__(self, path, domain_size, is_solid, two_d=False, extra_fields=()):
        self.path = path
        self.domain_size = np.asarray(domain_size, dtype=np.float64)
        self.fields = list(FIELDS_ALWAYS)
        if is_solid:
            self.fields += list(FIELDS_SOLID)
            if not two_d:
                self.fields += list(FIELDS_SOLID_3D)
        self.fields += list(extra_fields)
        self._f = None
        self._n = 0
        self.frames_written = 0

    # ------------------------------------------------------------------ layout
    def _create(self, n, keys=()):
        self.fields += [(k, nm) for k, nm in FIELDS_OPTIONAL if k in keys]
        self._n = n
        dims = [("frame", 0), ("atom", n), ("spatial", 3), ("cell_spatial", 3),
                ("cell_angular", 3), ("label", 5)]
        did = {nm: k for k, (nm, _) in enumerate(dims)}
        fixed = [
            _Var("spatial", _NC_CHAR, ["spatial"], data=np.frombuffer(b"xyz", "S1")),
            _Var("cell_spatial", _NC_CHAR, ["cell_spatial"], data=np.frombuffer(b"abc", "S1")),
            _Var("cell_angular", _NC_CHAR, ["cell_angular", "label"],
                 data=np.frombuffer(b"alphabeta gamma", "S1")),
        ]
        rec = [
            _Var("time", _NC_FLOAT, ["frame"], {"units": "picosecond"}),
            _Var("coordinates", _NC_FLOAT, ["frame", "atom", "spatial"], {"units": "angstrom"}),
            _Var("velocities", _NC_FLOAT, ["frame", "atom", "spatial"],
                 {"units": "angstrom/picosecond"}),
            _Var("cell_lengths", _NC_DOUBLE, ["frame", "cell_spatial"], {"units": "angstrom"}),
            _Var("cell_angles", _NC_DOUBLE, ["frame", "cell_angular"], {"units": "degree"}),
            _Var("id", _NC_INT, ["frame", "atom"]),
        ]
        for _key, nm in self.fields:
            rec.append(_Var(nm, _NC_INT if nm in INTEGER_FIELDS else _NC_FLOAT, ["frame", "atom"]))
        size = dict(dims)
        for v in fixed + rec:
            count = 1
            for d in v.dims:
                if d != "frame":
                    count *= size[d]
            raw = count * _SIZE[v.nc_type]
            v.vsize = raw + _pad(raw)
        gatts = {"Conventions": "AMBER", "ConventionVersion": "1.0", "program": "sigmasph_b200",
                 "programVersion": "0.1"}

        def header(begins):
            out = b"CDF\x02" + struct.pack(">i", 0)
            out += struct.pack(">ii", _NC_DIMENSION, len(dims))
            for nm, ln in dims:
                out += _name(nm) + struct.pack(">i", ln)
            out += _attrs(gatts)
            allv = fixed + rec
            out += struct.pack(">ii", _NC_VARIABLE, len(allv))
            for v, b in zip(allv, begins):
                out += _name(v.name) + struct.pack(">i", len(v.dims))
                out += b"".join(struct.pack(">i", did[d]) for d in v.dims)
                out += _attrs(v.attrs) + struct.pack(">ii", v.nc_type, v.vsize) + struct.pack(">q", b)
            return out

        allv = fixed + rec
        off = len(header([0] * len(allv)))
        for v in fixed:
            v.begin = off
            off += v.vsize
        self._rec_begin = off
        for v in rec:
            v.begin = off
            off += v.vsize
        self._rec_size = off - self._rec_begin
        self._fixed, self._rec = fixed, rec
        self._f = open(self.path, "wb+")
        self._f.write(header([v.begin for v in allv]))
        for v in fixed:
            raw = v.data.tobytes()
            self._f.write(raw + b"\0" * (v.vsize - len(raw)))
        self._f.flush()

    # ------------------------------------------------------------------ frames
    def write(self, obj_data, sim_time):
        """Append one frame; `obj_data` is what ParticleSystem.dump() returned."""
        pos = np.asarray(obj_data["position"])
        if self._f is None:
            self._create(pos.shape[0], obj_data.keys())
        elif pos.shape[0] != self._n:
            raise RuntimeError(f"particle count changed from {self._n} to {pos.shape[0]}; the NetCDF "
                               f"atom dimension is fixed when the file is created")
        n = self._n
        values = {"time": np.array([sim_time], np.float64),
                  "coordinates": pos, "velocities": np.asarray(obj_data["velocity"]),
                  "cell_lengths": self.domain_size, "cell_angles": np.array([90.0, 90.0, 90.0]),
                  "id": np.arange(n)}
        for key, nm in self.fields:
            values[nm] = np.asarray(obj_data[key])
        chunks = []
        for v in self._rec:
            raw = np.ascontiguousarray(values[v.name], dtype=_BE[v.nc_type]).tobytes()
            if len(raw) + _pad(len(raw)) != v.vsize:
                raise ValueError(f"{v.name}: {len(raw)} bytes for a {v.vsize}-byte slab")
            chunks.append(raw + b"\0" * (v.vsize - len(raw)))
        k = self.frames_written
        self._f.seek(self._rec_begin + k * self._rec_size)
        self._f.write(b"".join(chunks))
        self._f.seek(4)
        self._f.write(struct.pack(">i", k + 1))
        self._f.flush()
        os.fsync(self._f.fileno())
        self.frames_written += 1

    def close(self):
        if self._f is not None:
            self._f.close()
            self._f = None


def attach_relaxation_writer(ps, solver, path, interval=1):
    """Output.relaxationNetcdf (run_simulation.py:686-713, params.py:1245-1263): a second
    trajectory of the initial relaxation's passes.  Installs the solver's relax_frame_hook;
    frame k holds the body after k passes with lam and `relax_residual` (each particle's
    h^2 |S| / dx0) computed there, `time` is the pass number, every `interval`-th pass and
    the last are written, and rows follow the laid positions (x_0 until the relaxation
    ends) so a row is the same particle in every frame.  Call before solver.initialize();
    close the returned writer afterwards."""
    writer = NetCDFTrajectoryWriter(path, ps.domain_size, ps.is_solid, ps.two_d,
                                    extra_fields=[("relax_residual", "relax_residual")])
    interval = max(1, int(interval or 1))

    def relax_frame(k, residual, final):
        if k % interval and not final:
            return
        obj = ps.dump()
        mask = (ps.object_id.to_numpy() >= 0).nonzero()
        obj["relax_residual"] = solver.relax_res.to_numpy()[mask]
        order = np.lexsort(ps.x_0.to_numpy()[mask].T[::-1])
        n = len(order)
        obj = {key: (a[order] if isinstance(a, np.ndarray) and a.shape[:1] == (n,) else a)
               for key, a in obj.items()}
        writer.write(obj, k)

    solver.relax_frame_hook = relax_frame
    return writer

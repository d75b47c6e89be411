"""ParticlesFile reader: particle initial conditions from a preprocessed NetCDF file
(the reference's particle_system.py:666-854).

The file holds `position` (n, 3), `velocity` (n, 3), `density` (n) and `object_id` (n);
it may also hold each particle's size, `area` for a single-layer deck or `volume` in 3D.
The reference reads it through netCDF4; that package is not available here, so the file
is read with scipy's reader of the classic container (CDF-1 and the 64-bit-offset CDF-2).
A NetCDF-4 (HDF5) file is refused with a note on converting it (`nccopy -k 64-bit-offset`).

Per-particle sizes switch the reference to a variable smoothing length, which is outside
this package: a file whose sizes all equal the deck's lattice cell (V0) is accepted as
the uniform case, any other is refused.
"""
from __future__ import annotations

import os

import numpy as np


class ParticlesFileError(ValueError):
    pass


def read_particles_file(path, two_d):
    """{position, velocity, density, object_id, size (None when the file has none)} in
    file order, as float32 / int32 numpy arrays (size float64)."""
    if not os.path.exists(path):
        raise ParticlesFileError(f"ParticlesFile '{path}' does not exist")
    with open(path, "rb") as fh:
        magic = fh.read(4)
    if magic[:3] != b"CDF":
        raise ParticlesFileError(
            f"ParticlesFile '{path}' is not a classic NetCDF file (a NetCDF-4/HDF5 file needs "
            f"converting, e.g. `nccopy -k 64-bit-offset in.nc out.nc`)")
    from scipy.io import netcdf_file
    with netcdf_file(path, "r", mmap=False) as ds:
        v = ds.variables
        for need in ("position", "velocity", "density", "object_id"):
            if need not in v:
                raise ParticlesFileError(f"ParticlesFile '{path}' has no `{need}` variable")
        pos = np.array(v["position"][:], dtype=np.float32)
        vel = np.array(v["velocity"][:], dtype=np.float32)
        rho = np.array(v["density"][:], dtype=np.float32)
        oid = np.array(v["object_id"][:], dtype=np.int64)
        name, other = ("area", "volume") if two_d else ("volume", "area")
        size = None
        if name in v:
            size = np.array(v[name][:], dtype=np.float64)
        elif other in v:
            raise ParticlesFileError(
                f"ParticlesFile '{path}' carries `{other}`, but a "
                f"{'single-layer' if two_d else '3D'} deck needs `{name}` to give each particle "
                f"its size")
    n = len(pos)
    if pos.shape != (n, 3) or vel.shape != (n, 3) or rho.shape != (n,) or oid.shape != (n,):
        raise ParticlesFileError(f"ParticlesFile '{path}': position/velocity must be (n, 3) and "
                                 f"density/object_id (n,)")
    if size is not None:
        if size.shape != (n,) or not np.all(np.isfinite(size)) or size.min() <= 0.0:
            raise ParticlesFileError(f"ParticlesFile '{path}': every `{name}` must be positive "
                                     f"and finite")
    if not (np.all(np.isfinite(pos)) and np.all(np.isfinite(vel)) and np.all(rho > 0)):
        raise ParticlesFileError(f"ParticlesFile '{path}': positions and velocities must be "
                                 f"finite and densities positive")
    return {"position": pos, "velocity": vel, "density": rho, "object_id": oid.astype(np.int32),
            "size": size}

"""ParticlesFile decks (the reference's particle_system.py:666-854) on CPU: a file written
from a lattice deck lays exactly that deck's particles; objects take their block's
material; the refusals (variable sizes, NetCDF-4, missing variables) are explicit."""
import copy
import os
import tempfile

import numpy as np
import pytest
from scipy.io import netcdf_file

from sigmasph_b200.config import SceneError, SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import dambreak3d, dx_for_particles


def _write(path, pos, vel, rho, oid, size=None, size_name="volume"):
    with netcdf_file(path, "w", version=2) as f:
        f.createDimension("particle", len(pos))
        f.createDimension("spatial", 3)
        for name, arr, dims, t in (("position", pos, ("particle", "spatial"), "f"),
                                   ("velocity", vel, ("particle", "spatial"), "f"),
                                   ("density", rho, ("particle",), "f"),
                                   ("object_id", oid, ("particle",), "i")):
            v = f.createVariable(name, t, dims)
            v[:] = arr
        if size is not None:
            f.createVariable(size_name, "d", ("particle",))[:] = size


def _file_deck(scene, path):
    sc = copy.deepcopy(scene)
    sc["ParticlesFile"] = path
    for b in sc["FluidBlocks"]:
        for k in ("start", "end"):
            b.pop(k, None)
    return sc


def test_file_deck_lays_the_lattice_decks_particles():
    scene = dambreak3d(dx=dx_for_particles(2000))
    ref = ParticleSystem(SimConfig(scene), device="cpu")
    x = ref.x.to_numpy()
    rng = np.random.default_rng(4)
    v = rng.normal(0.0, 0.1, x.shape).astype(np.float32)
    rho = (ref.m.to_numpy() / ref.V.to_numpy()).astype(np.float32)
    oid = ref.object_id.to_numpy()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "particles.nc")
        _write(path, x, v, rho, oid)
        ps = ParticleSystem(SimConfig(_file_deck(scene, path)), device="cpu")
    assert ps.particle_max_num == ref.particle_max_num
    assert np.array_equal(ps.x.to_numpy(), x)
    assert np.array_equal(ps.v.to_numpy(), v)
    assert np.array_equal(ps.V.to_numpy(), ref.V.to_numpy())
    assert np.array_equal(ps.m.to_numpy(), ref.m.to_numpy())
    assert np.array_equal(ps.object_id.to_numpy(), oid)
    assert np.array_equal(ps.material.to_numpy(), ref.material.to_numpy())
    blk = scene["FluidBlocks"][0]
    assert ps.object_collection[int(blk["objectId"])]["particleNum"] == len(x)


def test_objects_without_a_block_are_grey_solids_and_sizes_must_be_uniform():
    scene = dambreak3d(dx=dx_for_particles(500))
    ref = ParticleSystem(SimConfig(scene), device="cpu")
    x = ref.x.to_numpy()
    n = len(x)
    oid = np.where(np.arange(n) % 2 == 0, int(scene["FluidBlocks"][0]["objectId"]), 7).astype(np.int32)
    v = np.zeros_like(x)
    rho = np.full(n, 1000.0, np.float32)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "p.nc")
        _write(path, x, v, rho, oid, size=np.full(n, ref.V0))
        ps = ParticleSystem(SimConfig(_file_deck(scene, path)), device="cpu")
        mat = ps.material.to_numpy()
        got = ps.object_id.to_numpy()
        assert np.all(mat[got == 7] == ps.material_solid)
        assert np.all(ps.color.to_numpy()[got == 7] == 100 + 7 * 50)
        _write(path, x, v, rho, oid, size=np.linspace(0.5, 1.5, n) * ref.V0)
        with pytest.raises(SceneError, match="own sizes"):
            ParticleSystem(SimConfig(_file_deck(scene, path)), device="cpu")
        _write(path, x, v, rho, oid, size=np.full(n, ref.V0), size_name="area")
        with pytest.raises(SceneError, match="needs `volume`"):
            ParticleSystem(SimConfig(_file_deck(scene, path)), device="cpu")


def test_unreadable_files_are_refused():
    scene = dambreak3d(dx=dx_for_particles(500))
    with tempfile.TemporaryDirectory() as d:
        h5 = os.path.join(d, "p4.nc")
        with open(h5, "wb") as f:
            f.write(b"\x89HDF\r\n\x1a\n" + bytes(64))
        with pytest.raises(SceneError, match="not a classic NetCDF"):
            ParticleSystem(SimConfig(_file_deck(scene, h5)), device="cpu")
        part = os.path.join(d, "partial.nc")
        with netcdf_file(part, "w", version=2) as f:
            f.createDimension("particle", 3)
            f.createVariable("density", "f", ("particle",))[:] = 1.0
        with pytest.raises(SceneError, match="no `position`"):
            ParticleSystem(SimConfig(_file_deck(scene, part)), device="cpu")
        with pytest.raises(SceneError, match="does not exist"):
            ParticleSystem(SimConfig(_file_deck(scene, os.path.join(d, "none.nc"))), device="cpu")

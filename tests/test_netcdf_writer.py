"""The AMBER NetCDF trajectory writer (the reference's netcdf_writer.py:101-225) against an
independent reader of the classic container (scipy.io.netcdf_file), on CPU."""
import os
import tempfile

import numpy as np
import pytest
from scipy.io import netcdf_file

from sigmasph_b200.netcdf_writer import NetCDFTrajectoryWriter


def _dump(n, rng, solid=False):
    d = {"position": rng.normal(size=(n, 3)).astype(np.float32),
         "velocity": rng.normal(size=(n, 3)).astype(np.float32),
         "object_id": rng.integers(0, 3, n).astype(np.int32),
         "density": rng.uniform(900, 1100, n).astype(np.float32),
         "pressure": rng.normal(size=n).astype(np.float32),
         "lam": rng.uniform(0, 1, n).astype(np.float32),
         "divergence": rng.normal(size=n).astype(np.float32)}
    if solid:
        for k in ("sigma_xx", "sigma_yy", "sigma_zz", "sigma_xy", "sigma_xz", "sigma_yz",
                  "von_mises", "eps_plastic", "e_int", "temperature"):
            d[k] = rng.normal(size=n).astype(np.float32)
        d["eroded"] = np.zeros(n, np.int32)
    return d


@pytest.mark.parametrize("solid,two_d", [(False, False), (True, False), (True, True)],
                         ids=["fluid", "solid3d", "solid2d"])
def test_frames_read_back(solid, two_d):
    rng = np.random.default_rng(1)
    n = 137                          # odd: every slab needs padding
    frames = [_dump(n, rng, solid) for _ in range(3)]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "traj.nc")
        w = NetCDFTrajectoryWriter(path, [1.6, 1.0, 0.6], solid, two_d=two_d)
        for k, fr in enumerate(frames):
            w.write(fr, 0.25 * k)
        w.close()
        with netcdf_file(path, "r", mmap=False) as f:
            assert f.version_byte == 2
            assert f.Conventions == b"AMBER"
            assert f.dimensions["atom"] == n and f.dimensions["frame"] is None
            v = f.variables
            assert v["coordinates"].shape == (3, n, 3) and v["coordinates"].units == b"angstrom"
            assert b"".join(v["cell_angular"][:].ravel()) == b"alphabeta gamma"
            for k, fr in enumerate(frames):
                assert v["time"][k] == pytest.approx(0.25 * k)
                assert np.array_equal(v["coordinates"][k], fr["position"])
                assert np.array_equal(v["velocities"][k], fr["velocity"])
                assert np.array_equal(v["object_id"][k], fr["object_id"])
                assert v["object_id"].typecode() == "i"
                assert np.array_equal(v["pressure"][k], fr["pressure"])
                assert np.array_equal(v["id"][k], np.arange(n))
                assert np.allclose(v["cell_lengths"][k], [1.6, 1.0, 0.6])
            names = set(v.keys())
            assert ("sigma_xx" in names) == solid and ("e_int" in names) == solid
            assert ("sigma_xz" in names) == (solid and not two_d)
            assert "divergence" not in names


def test_readable_before_close_and_fixed_atom_count():
    rng = np.random.default_rng(2)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "traj.nc")
        w = NetCDFTrajectoryWriter(path, [1, 1, 1], False)
        w.write(_dump(10, rng), 0.0)
        w.write(_dump(10, rng), 1.0)
        with netcdf_file(path, "r", mmap=False) as f:   # a run killed here
            assert f.variables["time"].shape == (2,)
        with pytest.raises(RuntimeError):
            w.write(_dump(11, rng), 2.0)
        w.close()

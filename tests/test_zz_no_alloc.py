"""The handle-free, allocation-free reduction entry point (sph_reduce_noalloc).

It exists for callers that cannot allocate GPU memory -- a host inside another
framework's fixed device pool, code that may not allocate during CUDA graph capture, or
an FFI caller holding only raw device pointers -- so it must produce what the handle's
sph_reduce produces from the caller's buffers alone.  This file is collected last so a
failure here cannot hide any other test's result.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import dambreak3d, dx_for_particles
from tests.helpers import perturb

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 4194304      # SPH_NOALLOC_MAX_PARTICLES in include/sph_b200.h
SPH_ERR_SCRATCH_CAP = -8


def _entry():
    f = abi.lib().sph_reduce_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.SphParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                  C.c_void_p, C.c_void_p]
    return f


def test_noalloc_reduction_matches_handle_reduction(cuda):
    cfg = SimConfig(dambreak3d(dx=dx_for_particles(20000)))
    ps = ParticleSystem(cfg, device="cuda")
    perturb(ps, dv=0.3)
    sv = ps.build_solver()
    sv.initialize()
    sv.step_many(3)
    ref = np.array(sv._reduce(), dtype=np.float64)
    f = _entry()
    n = ps.particle_max_num
    cur = ps.buffer_sets()[abi.lib().sph_parity(sv.h)]
    out = torch.empty(abi.RED_COUNT, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    results = []
    for _ in range(2):                       # two calls in a row share the static scratch
        out.fill_(float("nan"))
        rc = f(C.byref(sv.params), cur["pos"].data_ptr(), cur["vel"].data_ptr(),
               cur["shift"].data_ptr(), n, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        scale = np.abs(ref).max()
        assert np.all(np.abs(got - ref) <= 1e-10 * np.abs(ref) + 1e-13 * scale), (got, ref)
        results.append(got)
    assert np.array_equal(results[0], results[1])
    # beyond the fixed scratch: refused with a clear status, nothing launched
    rc = f(C.byref(sv.params), cur["pos"].data_ptr(), cur["vel"].data_ptr(),
           cur["shift"].data_ptr(), MAX_PARTICLES + 1, out.data_ptr(), stream)
    assert rc == SPH_ERR_SCRATCH_CAP

"""The handle-free, allocation-free reduction entry point (sph_reduce_noalloc).

It exists for callers that cannot allocate GPU memory -- a host inside another
framework's fixed device pool, code that may not allocate during CUDA graph capture, or
an FFI caller holding only raw device pointers -- so it must produce what the handle's
sph_reduce produces from the caller's buffers alone.  It serves fluids; a solid's
parameters are refused, because the solid's elastic energy needs the stress and material
rows that this call is not given.  This file is collected last so a failure here cannot
hide any other test's result.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from sigmasph_b200 import abi
from sigmasph_b200.config import SimConfig
from sigmasph_b200.particle_system import ParticleSystem
from sigmasph_b200.scenes import dambreak3d, dx_for_particles
from sigmasph_b200.solver import build_params
from tests.helpers import perturb

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 4194304      # SPH_NOALLOC_MAX_PARTICLES in include/sph_b200.h
SPH_ERR_UNSUPPORTED = -4
SPH_ERR_SCRATCH_CAP = -8


def _entry():
    f = abi.lib().sph_reduce_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.SphParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                  C.c_void_p, C.c_void_p]
    return f


def _stepped_fluid():
    cfg = SimConfig(dambreak3d(dx=dx_for_particles(20000)))
    ps = ParticleSystem(cfg, device="cuda")
    perturb(ps, dv=0.3)
    sv = ps.build_solver()
    sv.initialize()
    sv.step_many(3)
    return ps, sv


def _close(got, ref):
    scale = np.abs(ref).max()
    return np.all(np.abs(got - ref) <= 1e-10 * np.abs(ref) + 1e-13 * scale)


def test_noalloc_reduction_matches_handle_reduction(cuda):
    ps, sv = _stepped_fluid()
    ref = np.array(sv._reduce(), dtype=np.float64)
    f = _entry()
    n = ps.particle_max_num
    cur = ps.buffer_sets()[abi.lib().sph_parity(sv.h)]
    out = torch.empty(abi.RED_COUNT, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    results = []
    # two calls in a row share the static scratch; a fluid may pass no shift array
    for shift in (cur["shift"].data_ptr(), None):
        out.fill_(float("nan"))
        rc = f(C.byref(sv.params), cur["pos"].data_ptr(), cur["vel"].data_ptr(), shift, n,
               out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert _close(got, ref), (got, ref)
        results.append(got)
    assert np.array_equal(results[0], results[1])
    # no particles: every sum is zero
    out.fill_(float("nan"))
    assert f(C.byref(sv.params), None, None, None, 0, out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.zeros(abi.RED_COUNT))
    # beyond the fixed scratch: refused with a clear status, nothing launched
    rc = f(C.byref(sv.params), cur["pos"].data_ptr(), cur["vel"].data_ptr(),
           cur["shift"].data_ptr(), MAX_PARTICLES + 1, out.data_ptr(), stream)
    assert rc == SPH_ERR_SCRATCH_CAP


def test_noalloc_refuses_a_solid(cuda):
    """A solid's reductions include its elastic energy, which needs each particle's stress
    and material row: the call refuses the solid's parameters and writes nothing."""
    from tests.test_solid_gpu import bar3d_deck
    ps = ParticleSystem(SimConfig(bar3d_deck(dx=0.8)), device="cuda")
    p = build_params(ps)
    assert p.is_solid
    cur = ps.buffer_sets()[0]
    out = torch.full((abi.RED_COUNT,), float("nan"), dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _entry()(C.byref(p), cur["pos"].data_ptr(), cur["vel"].data_ptr(), cur["shift"].data_ptr(),
                  ps.particle_max_num, out.data_ptr(), stream)
    assert rc == SPH_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert np.isnan(out.cpu().numpy()).all()

"""sigmasph_b200 -- a B200-native (sm_100a) per-step particle hot path for the sigmaSPH
delta+-SPH fluid and hypoelastic tensile-solid solvers.

The public API mirrors the reference's: a scene file is read by `SimConfig`, particles
are laid by `ParticleSystem`, `ps.build_solver()` returns a `DSPHSolver` or a
`HypoElasticSolver`, and `solver.step()` advances one step on the GPU through the C-ABI
of libsph_b200.so (include/sph_b200.h).
"""
from .config import SimConfig, SceneError
from .materials import Material, MaterialError

__all__ = ["SimConfig", "SceneError", "Material", "MaterialError", "ParticleSystem"]


def __getattr__(name):
    # torch is imported lazily so the host-side modules stay importable without it
    if name == "ParticleSystem":
        from .particle_system import ParticleSystem
        return ParticleSystem
    raise AttributeError(name)

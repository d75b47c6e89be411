// sph_solid.cuh -- hypoelastic tensile-solid step (SOLID.py HypoElasticSolver).
#pragma once
#include "sph_fluid.cuh"

namespace sph {

struct SolidScratch {
    int unused = 0;
};

inline void solid_fill_constants(Cst&) {}
inline int solid_alloc(SolidScratch&, const SphParams&, int64_t) { return SPH_ERR_UNSUPPORTED; }
inline void solid_free(SolidScratch&) {}
inline int solid_pre_step(const Cst&, const Ptr&, SolidScratch&, cudaStream_t) { return SPH_ERR_UNSUPPORTED; }
inline int solid_substep_and_boundary(const Cst&, const Ptr&, SolidScratch&, int, cudaStream_t) {
    return SPH_ERR_UNSUPPORTED;
}
template <class Rebuild>
inline int solid_run_stage(const Cst&, const Ptr&, SolidScratch&, int, int, cudaStream_t, Rebuild&&) {
    return SPH_ERR_UNSUPPORTED;
}
inline void solid_reduce_extra(const Cst&, const Ptr&, int, cudaStream_t) {}

}  // namespace sph

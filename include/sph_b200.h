/*
 * sph_b200.h -- C-ABI of libsph_b200.so, the B200 (sm_100a) per-step particle hot path
 * of the sigmaSPH delta+-SPH fluid and hypoelastic tensile-solid solvers.
 *
 * The reference has no FFI: its hot path sits behind the solver object's Python API
 * (ParticleSystem fields, solver.initialize(), solver.step(), solver.dt[None], the
 * energy/momentum reductions and get_constraint_data()).  Each entry point below
 * replaces one of those calls; the reference method it stands in for is cited beside it
 * by file:line within the sigmaSPH source tree.  The Python package sigmasph_b200 binds
 * these with ctypes and keeps the reference's attribute names.
 *
 * Conventions
 *  - Plain C types only.  Device pointers are passed as raw pointers; `stream` is a
 *    cudaStream_t passed as void* (NULL = the legacy default stream).
 *  - Every function returns an int status: 0 = SPH_OK, < 0 = error (sph_strerror()).
 *    No exception crosses the boundary.
 *  - The caller owns every per-particle buffer (PyTorch tensors in the Python host
 *    layer).  The library allocates only scratch: sort keys, permutation, cell table,
 *    neighbour lists, device scalars.
 *  - The persistent particle state lives in buffer set A; set B is the reorder's
 *    scratch.  A build of the neighbour candidates gathers the state into B in the new
 *    order and copies it back to A.  sph_parity() says which set is current (always A,
 *    0, since the copy back; kept so that a host need not assume it).
 */
#ifndef SPH_B200_H
#define SPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH_ABI_VERSION 4

/* ---------------------------------------------------------------- status codes */
#define SPH_OK                 0
#define SPH_ERR_ARG           -1   /* bad argument (null pointer, n > n_max, ...)          */
#define SPH_ERR_CUDA          -2   /* a CUDA runtime call failed                           */
#define SPH_ERR_NOMEM         -3   /* scratch allocation failed                            */
#define SPH_ERR_UNSUPPORTED   -4   /* option the library does not implement                */
#define SPH_ERR_NOT_BOUND     -5   /* sph_bind() has not been called                       */
#define SPH_ERR_NEIGHBOUR_CAP -6   /* reserved: neighbour-list overflow is handled in-kernel */
#define SPH_ERR_TIMEOUT       -7   /* a bounded device wait ran out                        */
#define SPH_ERR_SCRATCH_CAP   -8   /* request exceeds the fixed static scratch capacity    */

/* Device error-word bits (SphScalars.err).  Set by kernels, never by a trap. */
#define SPH_EW_NBR_OVERFLOW   0x1  /* a particle had more neighbours within h than its
                                      list holds (twice the lattice count within 1.1 h);
                                      the extra pairs went to the overflow pool          */
#define SPH_EW_HASHED_GRID    0x2  /* the occupied cell box did not fit the dense Morton
                                      table; the step ran on the hashed fallback table   */
#define SPH_EW_JC_NO_CONVERGE 0x4  /* a Johnson-Cook return map hit its iteration cap     */
#define SPH_EW_STS_CAP        0x8  /* the hourglass sub-cycle count hit its cap          */
#define SPH_EW_MLP_TIMEOUT    0x10 /* a tensor-core surrogate pass gave up waiting for its
                                      MMAs; its returns fell back to the exact Newton      */
#define SPH_EW_CAND_OVERFLOW  0x20 /* a particle had more candidates within h + skin than
                                      its candidate list holds; its pairs came from a
                                      direct search of the coarse cell table              */
#define SPH_EW_NBR_DROPPED    0x40 /* the overflow pool (as many entries as the lists of
                                      all particles) ran out: pairs were dropped and the
                                      step is not exact                                    */

/* ------------------------------------------------------------------ parameters */
/* Flattened, resolved scene configuration.  Field meanings follow the reference's
 * registry (params.py) and the solver constructors (DSPH.py:64-450, SOLID.py:138-1452).
 * Appended-to only; struct_size guards the layout. */
typedef struct SphParams {
    int32_t struct_size;          /* sizeof(SphParams), checked by sph_create           */
    int32_t is_solid;             /* simulationMethod == hypoElastic                    */
    /* --- domain (particle_system.py:25-350) --- */
    int32_t two_d;                /* plane_strain || axisymmetric                       */
    int32_t axisymmetric;
    int32_t plane_strain;
    int32_t sym_y, sym_z;         /* Cartesian symmetry planes (mirror sweeps)          */
    int32_t walls;                /* Domain.boundary == reflect                          */
    int32_t displacement_positions;
    int32_t compensated_volume;
    float   support_radius;       /* h: kernel support == grid cell size                */
    float   particle_diameter;    /* dx0                                                */
    float   V0;                   /* dx0^2 (single layer) or dx0^3                      */
    float   axi_r_min;            /* floor on r in axisymmetry                          */
    float   domain_size[3];
    float   padding;              /* wall offset == grid size                           */
    float   wall_restitution;
    /* --- fluid solver (DSPH.py) --- */
    float   density0;
    float   c0;
    float   exponent;
    float   stiffness;            /* c0^2 rho0 / exponent                               */
    float   viscosity;
    float   CFL;
    float   delta_sph;
    float   gravity[3];
    int32_t allow_negative_pressure;
    int32_t track_visc_work;
    float   l_eig_tol_lam;        /* regularised-inverse tolerance for L (0.02)         */
    float   c_signal;             /* CFL floor speed: c0 (fluid) or c_p (solid)         */
    int32_t dt_pair_mode;         /* 0 off, 1 all pairs, 2 same-material pairs          */
    /* --- particle shifting (DSPH.py:190-330, 943-1049) --- */
    int32_t pst_enabled;
    int32_t pst_colle;            /* 0 = Sun, 1 = Colle                                 */
    int32_t pst_ma_mode;          /* 0 local, 1 global, 2 fixed                         */
    int32_t pst_clamp_disp;
    int32_t pst_clamp_vel;
    int32_t pst_surface_none;
    int32_t pst_normal_eigvec;
    int32_t pst_ale_momentum;
    float   pst_R;
    int32_t pst_n;
    float   pst_max_shift;
    float   pst_ma_fixed;
    float   pst_m_delta;
    float   pst_lambda_lo;
    float   pst_lambda_hi;
    /* --- hypoelastic solid (SOLID.py); ignored unless is_solid --- */
    int32_t n_materials;          /* rows used in the material tables below (<= 4)      */
    float   mat_rho0[4];
    float   mat_K[4];
    float   mat_G[4];
    float   mat_cp[4];            /* dilatational speed sqrt((K + 4G/3)/rho0)           */
    float   mat_c0[4];            /* EOS sound speed sqrt(K/rho0)                       */
    float   mat_delta[4];         /* per-material delta-SPH coefficient                 */
    int32_t plastic_kind[4];      /* 0 none, 1 linear (J2), 2 Johnson-Cook              */
    float   plastic_sy0[4];
    float   plastic_H[4];
    float   jc_A[4], jc_B[4], jc_n[4], jc_C[4], jc_eps0_dot[4];
    float   jc_T0[4], jc_Tm[4], jc_m[4], jc_chi[4];
    float   mat_cv[4];            /* specific heat (0: temperature stays at T0)         */
    float   mat_stiff[4];         /* EOS stiffness: K (linear) or c0^2 rho0 / gamma     */
    float   mat_gamma[4];         /* EOS exponent (1 for linear)                        */
    float   mat_T0[4];            /* reference temperature                              */
    int32_t axi_conservative_x;   /* axisymmetric conservative axial momentum form      */
    float   hg_rate;              /* alpha c_p / h_min * S * axis ratio (1/time)        */
    int32_t kernel_correction;    /* grad v through the regularised inverse of E        */
    float   l_eig_tol;            /* tolerance of that inverse (0.1)                    */
    float   hourglass_alpha;
    int32_t hourglass_sts;        /* 0 in-loop damper + dt clamp, 1 sub-cycled          */
    int32_t hourglass_sts_cap;    /* max sub-cycle stages                               */
    float   hourglass_sts_safety; /* RKL: the fraction of s^2+s dt may use (0.8)     */
    float   hg_S;                 /* lattice kernel sum of the damper (SOLID.py:1632)   */
    float   hg_W_dx0;             /* W(dx0)                                            */
    int32_t hg_sts_refresh;       /* recompute grad v after the half kick               */
    int32_t ale_history;          /* ALE transport of s, eps_p                          */
    int32_t transport_e;          /* ALE transport of e_int                             */
    float   ale_diffusion;        /* xi of the upwind ALE diffusion (1.0)               */
    int32_t num_constraints;      /* grips (<= 8)                                       */
    float   ramp_time;
    int32_t jc_surrogate;         /* 1: MLP return map with Newton fallback             */
    float   jc_surrogate_tol;     /* |f_yield| / sigma_y acceptance (1e-3)              */
    int32_t hg_sts_fixed;         /* > 0: that many damper sub-steps, else automatic    */
    /* --- the solid's in-loop viscosities (SOLID.py:640-716) --- */
    float   q_l2;                 /* VNR bulk viscosity C_Q l^2 (0: off)                */
    float   q_cl;                 /* C_Q l, for the viscosity's own CFL limit           */
    float   av_alpha;             /* Monaghan pair viscosity alpha (0 with beta: off)   */
    float   av_beta;
    float   av_eps;               /* mu_ij regulariser epsilon (0.01)                   */
    int32_t hg_sts_rkl;           /* sub-cycled damper as s-stage RKL1 (else forward
                                     Euler sub-steps), SOLID.py:4510-4576              */
    int32_t objective_none;       /* Solver.objectiveRate "none": no spin terms in the
                                     stress rate (SOLID.py:368, :2721-2722)            */
    int32_t axi_image_signed;     /* conservative axial stress pair: a mirror image's
                                     radius is its signed coordinate (SOLID.py:3598-3609)*/
    int32_t axi_conservative_r;   /* axisymmetric conservative radial form: the pair
                                     radius in every radial pair force, the source
                                     (p + q - s_tt) / (rho r)  (SOLID.py:3444-3466)    */
    /* --- several solid materials (SOLID.py:222-245) --- */
    int32_t delta_pairs_all;      /* Diffusion.pairs "all": the delta-SPH diffusion also on
                                     pairs of two materials, with the harmonic mean of the
                                     two deltas (DSPH.py:1271-1282, SOLID.py:4102-4114)  */
    int32_t c0_mixed;             /* the materials' EOS sound speeds differ: pair terms take
                                     the mean of the two (pair_c0), the shift particle i's
                                     own (local_c0)         (DSPH.py:483-530, SOLID.py:244) */
    int32_t hg_mixed_impedance;   /* the materials' rho0 c_p differ: the damper's pair force
                                     carries 2 Z_j / (Z_i + Z_j)  (SOLID.py:228-229,
                                     :4184-4239)                                        */
} SphParams;

/* ------------------------------------------------------------------ buffers */
/* One set of the persistent (sorted) per-particle state.  Row-major [n][k] float32
 * unless noted.  Vector fields carry a fourth float so every record is one 16-byte
 * load; the fourth slot holds a scalar field of the reference (named below). */
typedef struct SphFieldSet {
    float*   pos;      /* [n][4] x, y, z, V         (ps.x, ps.V)                         */
    float*   vel;      /* [n][4] vx, vy, vz, m      (ps.v, ps.m)                         */
    float*   x0;       /* [n][4] x0, y0, z0, V_lo   (ps.x_0, ps.V_lo)                    */
    float*   disp;     /* [n][4] ux, uy, uz, p      (ps.u, ps.pressure)                  */
    float*   shift;    /* [n][4] dr_x, dr_y, dr_z, e_int (ps.pst_shift, ps.e_int)        */
    int32_t* pid;      /* [n] persistent particle id (index at creation)                 */
    /* solid only (may be NULL for a fluid run) */
    float*   sdev;     /* [n][8] s_xx, s_yy, s_zz, s_xy, s_xz, s_yz, eps_p, T            */
    int32_t* bc;       /* [n][2] bc_flag, bc_id                                         */
    float*   bcdisp;   /* [n][4] bc_disp xyz, eos_id (as float)                         */
    float*   acc;      /* [n][4] acceleration, de_int: carried across the sort, since the
                          next step's energy update reads them (SOLID.py:2071-2237)      */
} SphFieldSet;

/* Per-step derived fields (one copy, overwritten every step before they are read). */
typedef struct SphBuffers {
    SphFieldSet set[2];
    float* acc;        /* [n][4] ax, ay, az, de_visc (de_int on the solid path)          */
    float* lam;        /* [n]                                                            */
    float* lsym;       /* [n][8] L_00, L_11, L_22, L_01, L_02, L_12, -, -                */
    float* lgrad;      /* [n][4] grad lambda (or the min eigenvector under eigvec)       */
    float* div;        /* [n][4] divergence, diffusion rate, -, -                        */
    float* gradv;      /* [n][12] grad v (row-major 3x3) + 3 spare (solid)               */
    float* aux;        /* [n][24] solid per-step scratch: updated s, eps_p, e, T; the
                          kernel-correction inverse; the damper's velocity buffers        */
} SphBuffers;

/* Device scalars copied back by sph_get_scalars (the reference's 0-d fields). */
typedef struct SphScalars {
    float   dt;               /* solver.dt[None]                                         */
    float   max_c_sq;         /* solver.max_c_sq[None]                                   */
    float   max_accel;        /* solver.max_accel[None]                                  */
    float   max_v;            /* solver.max_v[None]                                      */
    int32_t off_grid_num;     /* ps.off_grid_num[None]                                   */
    int32_t err;              /* SPH_EW_* bits accumulated since the last reset           */
    int32_t sts_stages;       /* last hourglass sub-cycle count (ensembles: the largest)  */
    int32_t pad0;
    double  off_grid_mass;    /* ps.off_grid_mass[None]                                  */
    double  wall_work;        /* SPHBase.wall_work                                       */
    double  visc_work;        /* DSPHSolver.visc_work                                    */
    double  diff_work;        /* DSPHSolver.diff_work                                    */
    double  leftover_work;    /* DSPHSolver.leftover_work                                */
    double  plastic_work;     /* HypoElasticSolver plastic work                          */
    double  hg_work;          /* HypoElasticSolver hourglass work                        */
    double  sim_time;         /* HypoElasticSolver.sim_time                              */
    float   load_s, load_sdot;/* HypoElasticSolver.load_s / load_sdot                    */
    double  constraint_force[8][3];
    double  constraint_disp[8][3];
} SphScalars;

/* ---- Solid material rows and ensemble instances (no counterpart in the reference,
 * which runs one scene per process: run_simulation.py:649-708).  A solid handle keeps
 * its material rows in device memory (built from SphParams for an ordinary scene).  An
 * ensemble packs many independent scenes into one handle: instance k's particles carry
 * material row k, each instance has its own time step, clock, load ramp, damper stage
 * count and two grips, and the instances are placed far enough apart that no pair
 * crosses between them. */
typedef struct SphMatRow {
    float   rho0, K, G, cp, c0, delta;   /* as SphParams mat_*                              */
    int32_t plastic_kind;                /* 0 none, 1 J2, 2 Johnson-Cook                    */
    float   sy0, H;                      /* J2 / JC: yield stress at zero plastic strain, H */
    float   jc_A, jc_B, jc_n, jc_C, jc_eps0_dot, jc_T0, jc_Tm, jc_m, jc_chi;
    float   cv, stiff, gamma, T0;        /* specific heat, EOS stiffness / exponent, T ref   */
} SphMatRow;

typedef struct SphInstRow {              /* constants of one ensemble instance               */
    float   c_signal;                    /* CFL floor speed                                  */
    float   hg_rate;                     /* hourglass damper rate (sub-cycle count)          */
    float   ramp_time;                   /* load ramp                                        */
    float   c0;                          /* speed c0 of delta-SPH and the Colle shift        */
    float   visc_coef;                   /* Morris viscosity coefficient 10 nu               */
    float   reserved[3];
} SphInstRow;

typedef struct SphInstState {            /* per-instance device state (sph_ensemble_state)  */
    double  sim_time;
    float   dt, load_s, load_sdot;
    int32_t sts_stages;
    uint32_t max_c_sq_bits, max_accel_bits;  /* internal: the step's dt maxima           */
    double  constraint_force[2][3];      /* grips 0 and 1 (FP64, x 2 pi if axisymmetric)    */
    double  constraint_disp[2][3];
} SphInstState;

/* Reduction indices of sph_reduce(). */
enum {
    SPH_RED_KE = 0, SPH_RED_KE_OFFGRID, SPH_RED_PE, SPH_RED_SE, SPH_RED_IE,
    SPH_RED_MASS, SPH_RED_PX, SPH_RED_PY, SPH_RED_PZ, SPH_RED_GROSS_P,
    SPH_RED_ELASTIC, SPH_RED_COUNT
};

typedef struct SphHandle SphHandle;

/* Library identity and layout checks. */
int         sph_abi_version(void);
size_t      sph_params_size(void);
size_t      sph_scalars_size(void);
const char* sph_strerror(int status);
/* Writes "name=offset;..." for every SphParams field into buf (for the host layer's
 * layout check).  Returns the number of bytes needed. */
int         sph_params_layout(char* buf, int cap);

/* Set-up: ParticleSystem.__init__ + build_solver (particle_system.py:25-475, :958-966,
 * DSPH.py:64-450, SOLID.py:138-1452).  Allocates scratch for n_max particles. */
int  sph_create(const SphParams* p, int64_t n_max, SphHandle** out);
void sph_destroy(SphHandle* h);
/* Attach the caller's buffers; n = particle_num[None] (particle_system.py:269). */
int  sph_bind(SphHandle* h, const SphBuffers* b, int64_t n);
/* Which SphFieldSet holds the current state (0 or 1). */
int  sph_parity(const SphHandle* h);
/* Upload per-material constraint/material tables after a change on the host. */
int  sph_set_params(SphHandle* h, const SphParams* p);

/* ParticleSystem.initialize_particle_system (particle_system.py:1342-1345): rebuild the
 * cell table, reorder every persistent field, rebuild the neighbour lists. */
int  sph_initialize(SphHandle* h, void* stream);
/* SPHBase.step (sph_base.py:622-655) / HypoElasticSolver.step (SOLID.py:5227-5231),
 * nsteps times, asynchronously on `stream`; dt stays on the device.  Replays CUDA graphs
 * of two steps and of one step, captured at the first call (eager launches while the
 * per-kernel profile is on). */
int  sph_step(SphHandle* h, int nsteps, void* stream);
/* One named stage of the step, for stage-by-stage parity tests (SPH_STAGE_*). */
int  sph_run_stage(SphHandle* h, int stage, void* stream);
/* solver.dt[None] read/write (DSPH.py:124-131, run_simulation.py:1190-1211). */
int  sph_set_dt(SphHandle* h, float dt, void* stream);
/* solver.dt[None] read: 4 bytes device -> page-locked host (synchronises `stream`). */
int  sph_get_dt(SphHandle* h, float* dt, void* stream);
/* Copies the device scalars (synchronises `stream`). */
int  sph_get_scalars(SphHandle* h, SphScalars* out, void* stream);
/* HypoElasticSolver.get_constraint_data (SOLID.py:5198-5225): the FP64 force and the
 * displacement of grips 0 .. k-1 of the last step into force[k][3] and disp[k][3] (host
 * arrays; either may be NULL).  The force is summed over the grip's particles in FP64
 * (x 2 pi in axisymmetry), as apply_constraints does (SOLID.py:5026-5055).  k must not
 * exceed the scene's constraint count; a fluid handle or an ensemble returns
 * SPH_ERR_ARG (an ensemble's grips are per instance: sph_ensemble_state).  Synchronises. */
int  sph_constraints(SphHandle* h, double* force, double* disp, int k, void* stream);
int  sph_clear_error(SphHandle* h, void* stream);
/* FP64 reductions: compute_kinetic_energy / _off_grid / potential / elastic /
 * internal / total_mass (sph_base.py:425-557, DSPH.py:1670-1712) and compute_momentum /
 * compute_gross_momentum (sph_base.py:560-620), into out[SPH_RED_COUNT]. */
int  sph_reduce(SphHandle* h, double* out, void* stream);
/* Neighbour pairs (for_all_neighbors, particle_system.py:1348-1490): mode 0 = this
 * step's list (the sweep against the bins of the step's start); mode 1 = a fresh search
 * from the current positions against those bins (the PST sweep, DSPH.py:771-886).  Writes
 * up to cap (i, j, mirror) triples as current-order indices and the total into *count. */
int  sph_pairs(SphHandle* h, int mode, int32_t* pi, int32_t* pj, int32_t* mir,
               int64_t cap, int64_t* count, void* stream);
/* The pairs the shift pass evaluates at the current positions (the PST sweep,
 * DSPH.py:771-886): the candidate lists of the last build re-tested at the current
 * positions, or the coarse-table search when the displacement bound does not hold.
 * disp_bound >= 0 stands for the largest distance a particle moved since the lists were
 * built (the caller vouches for it); < 0 uses what the step recorded.  As a set, equal to
 * sph_pairs mode 1 whenever the bound holds.  Output as sph_pairs. */
int  sph_shift_pairs(SphHandle* h, float disp_bound, int32_t* pi, int32_t* pj, int32_t* mir,
                     int64_t cap, int64_t* count, void* stream);
/* One pass of the initial relaxation against the shift (relax_initial_configuration,
 * DSPH.py:1113-1179): the neighbour lists at the current positions, lambda and its
 * gradient, then each particle's drive g = pst_constrain(-h^2 S) from the run's own
 * disorder sum; *residual = max |g| / dx0; the step beta g, capped at maxShift dx0, is
 * left in the shift record.  residual_each: NULL, or a device array of n floats that
 * receives each particle's |g| / dx0 in the current storage order (the reference's
 * relax_res, DSPH.py:1100).  Synchronises. */
int  sph_relax_pass(SphHandle* h, float beta, float* residual, float* residual_each,
                    void* stream);
/* Moves every particle by the step the last sph_relax_pass left in its shift record. */
int  sph_relax_move(SphHandle* h, void* stream);
/* Candidate-list statistics since creation or the last reset: out[0] steps, out[1] steps
 * that built the candidate lists, out[2] shift passes that searched the coarse table
 * instead of reading the lists.  reset != 0 zeroes them after reading. */
int  sph_list_stats(SphHandle* h, uint64_t* out, int reset, void* stream);

/* Per-kernel timing with CUDA events recorded on the launching stream around every
 * kernel of eagerly launched steps (sph_step while profiling, sph_run_stage).  Off by
 * default; graph replays are not instrumented. */
int  sph_profile_enable(SphHandle* h, int on);
/* Synchronises, then writes up to cap entries: '\n'-separated kernel names into names,
 * total milliseconds into ms and launch counts into launches; *count = entries.  Resets
 * the accumulators. */
int  sph_profile_read(SphHandle* h, char* names, int names_cap, double* ms, int* launches,
                      int cap, int* count);

/* Measured FP32 fused multiply-add throughput of the current device (TFLOP/s, 2 FLOP per
 * FMA) from a microbenchmark kernel: eight independent FMA chains per thread, eight
 * 256-thread blocks per SM.  The denominator of the FP32-issue bound bench.py reports
 * beside the HBM roofline.  Synchronises; allocates a 4 kB result buffer. */
int  sph_fma_peak(double* tflops, void* stream);

/* The FP64 reductions of sph_reduce for a FLUID, without a handle and without
 * allocating: no counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host running inside another framework's fixed device-memory pool, code that may not
 * allocate while a CUDA graph is being captured, FFI callers that hold only raw device
 * pointers).  The caller passes the current buffer set's pos, vel and shift arrays
 * ([n][4] float32, 16-byte aligned; shift may be NULL) and `out`, a device array of
 * SPH_RED_COUNT doubles it owns; the result is written there asynchronously on `stream`.
 * A solid's parameters (is_solid) return SPH_ERR_UNSUPPORTED and write nothing: its
 * elastic energy needs every particle's stress and material row, which this call is not
 * given (use sph_reduce on the solid's handle).  n = 0 writes zeros.
 * The scratch is a fixed array compiled into the library (1.44 MB on each GPU that loads
 * it, held until the process exits), which caps n at SPH_NOALLOC_MAX_PARTICLES: larger n
 * returns SPH_ERR_SCRATCH_CAP and launches nothing.  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress) with the device current; make it
 * before any stream capture.  The address is kept for the life of the process: a
 * cudaDeviceReset between calls is not supported.  All calls share the array, so calls
 * whose GPU work overlaps (other streams, other host threads) race: serialise them.  The
 * sum is deterministic (per-block partials added in a fixed order). */
#define SPH_NOALLOC_MAX_PARTICLES 4194304
int  sph_reduce_noalloc(const SphParams* p, const float* pos, const float* vel,
                        const float* shift, int64_t n, double* out, void* stream);

/* ---- Johnson-Cook return-map surrogate (no counterpart in the reference; its return
 * map is the Newton-bisection of MAT002_johnson_cook.py:251-354, called from
 * SOLID.py:2889-2913).  A 4 -> 64 -> 64 -> 64 -> 1 SiLU MLP of sph_mlp_param_count()
 * float32 parameters (W1[64][4], b1, W2[64][64], b2, W3[64][64], b3, W4[64], b4) maps the
 * features of a yielding return, f0 = ln(max(vm/sigma_y0 - 1, 1e-8))/10, f1 = eps_p,
 * f2 = ln(max(eps_dot_eq/eps0_dot, 1))/10, f3 = ln(max(d_hi/(dt eps0_dot), 1))/10, to
 * u = 10 (1 - d/d_hi), with d_hi = (vm - sigma_y0)/(3G).  Every pointer is device memory; X rows are
 * float4 (16-byte aligned), Y and T one float per row.  Calls are asynchronous on stream. */
int     sph_mlp_param_count(void);
int64_t sph_mlp_packed_bytes(void);
/* Float32 forward on CUDA cores (the training reference). */
int  sph_mlp_forward(const float* W, const float* X, int64_t n, float* Y, void* stream);
/* Mean-squared-error gradient over n rows into G[param_count] (overwritten) and the loss
 * into *loss (one double, overwritten). */
int  sph_mlp_grad(const float* W, const float* X, const float* T, int64_t n, float* G,
                  double* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected; step counts from 1). */
int  sph_mlp_adam(float* W, const float* G, float* M, float* V, int64_t step, float lr,
                  void* stream);
/* BF16 copy of W2 and W3 in the tensor cores' operand layout (sph_mlp_packed_bytes(),
 * 16-byte aligned). */
int  sph_mlp_pack(const float* W, void* packed, void* stream);
/* BF16 tensor-core (tcgen05) inference with FP32 accumulation; *err gets
 * SPH_EW_MLP_TIMEOUT if a bounded wait gave up. */
int  sph_mlp_infer_tc(const float* W, const void* packed, const float* X, int64_t n, float* Y,
                      int* err, void* stream);
/* Enables (enable = 1, W = the parameters, tol = the |g|/sigma_y acceptance) or disables
 * the surrogate in a solid handle's Johnson-Cook returns: yielding returns are queued,
 * the network proposes d, and the exact Newton runs wherever the residual exceeds tol. */
int  sph_jc_surrogate(SphHandle* h, const float* W, float tol, int enable, void* stream);
/* Attaches (rows != NULL) or detaches a sample log: every exact Johnson-Cook return of the
 * plain path appends {f0, f1, f2, f3, d/d_hi, d_hi, vm, sigma_y0} to rows[capacity][8];
 * *count (device, zeroed by the caller) counts every return, logged or not. */
int  sph_jc_log(SphHandle* h, float* rows, int64_t capacity, unsigned long long* count);
/* Counters since the last reset: {Newton solves, Newton iterations, surrogate proposals,
 * proposals accepted}; reset != 0 zeroes them after the read (synchronises stream). */
int  sph_jc_stats(SphHandle* h, uint64_t* out, int reset, void* stream);

/* Turns a solid handle into an ensemble of n_inst instances (1 <= n_inst <= 1024):
 * mat[k] and inst[k] are instance k's material row and constants (host arrays, copied),
 * every particle's material id (bcdisp.w) must be its instance, constraint ids (bc.y)
 * 0 or 1 within the instance; dt0[k] (host) is the first step of instance k.  n_inst = 0
 * returns the handle to single-scene mode.  A handle with the bulk or the Monaghan
 * viscosity on returns SPH_ERR_UNSUPPORTED (the instances' steps carry no viscosity
 * limits). */
int  sph_ensemble_set(SphHandle* h, const SphMatRow* mat, const SphInstRow* inst, int n_inst,
                      const float* dt0, void* stream);
/* Copies the per-instance state into out[n_inst] (host; synchronises stream). */
int  sph_ensemble_state(SphHandle* h, SphInstState* out, int n_inst, void* stream);
/* Threads per block of the particle kernels (a multiple of 32, 64..256; 0 = 256). */
int  sph_set_block(SphHandle* h, int threads);

/* Stage ids for sph_run_stage. */
enum {
    SPH_STAGE_SORT = 0,        /* initialize_particle_system                           */
    SPH_STAGE_LAM = 1,         /* DSPHSolver.compute_lam, both passes                  */
    SPH_STAGE_CONTINUITY = 2,  /* compute_volume_evolution                             */
    SPH_STAGE_FORCES = 3,      /* non-pressure + pressure accelerations (+ dt pair max) */
    SPH_STAGE_DT = 4,          /* compute_adaptive_dt                                  */
    SPH_STAGE_ADVECT = 5,      /* accumulate_step_work + advect                        */
    SPH_STAGE_PST = 6,         /* apply_pst                                            */
    SPH_STAGE_BOUNDARY = 7,    /* constraints / walls at the end of SPHBase.step       */
    SPH_STAGE_COUNT_FLUID = 8
};

#ifdef __cplusplus
}
#endif
#endif /* SPH_B200_H */

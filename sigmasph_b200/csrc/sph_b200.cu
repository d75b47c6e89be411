// sph_b200.cu -- libsph_b200.so: the C-ABI of include/sph_b200.h over the sm_100a
// kernels of sph_grid.cuh / sph_fluid.cuh / sph_solid.cuh.  One translation unit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <string>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "sph_fluid.cuh"
#include "sph_host.cuh"
#include "sph_solid.cuh"

using namespace sph;

struct SphHandle {
    SphParams p;
    Cst c;
    int64_t n_max = 0;
    int64_t n = 0;
    int parity = 0;
    bool bound = false;
    SphBuffers buf;
    int device = 0;
    // scratch
    int4* cell = nullptr;
    int* key = nullptr;
    int* rank = nullptr;
    int* perm = nullptr;
    int* hist = nullptr;
    int* start = nullptr;
    int* bsum = nullptr;
    int* bbox = nullptr;
    GridLayout* layout = nullptr;
    int* nbr = nullptr;
    int* nbr_cnt = nullptr;
    int* vl = nullptr;
    int* vl_cnt = nullptr;
    int* nl_cnt = nullptr;
    int* ovf = nullptr;
    int* ovf_off = nullptr;
    int4* fcell = nullptr;
    float4* xb = nullptr;
    bool force_pending = true;      // the next step builds the candidate lists
    DevScalars* sc = nullptr;
    DevAccum* ac = nullptr;
    SphScalars* pinned = nullptr;   // page-locked staging of the scalar copies
    SolidScratch solid;
    // CUDA graph of two consecutive steps
    cudaGraphExec_t graph2 = nullptr;
    cudaGraphExec_t graph1 = nullptr;   // one step (sph_step with an odd count)
    cudaStream_t cap_stream = nullptr;
    // per-kernel event profile of eager launches
    bool prof_on = false;
    bool capturing = false;
    std::vector<std::pair<const char*, cudaEvent_t>> prof_marks;
    std::vector<cudaEvent_t> prof_pool;
    size_t prof_used = 0;
};

namespace {

// Records an event after a launch when profiling an eager launch sequence; the kernel's
// time is the interval since the previous mark.
void prof_mark(SphHandle* h, const char* name, cudaStream_t st) {
    if (!h->prof_on || h->capturing) return;
    if (h->prof_used == h->prof_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        h->prof_pool.push_back(e);
    }
    cudaEvent_t e = h->prof_pool[h->prof_used++];
    cudaEventRecord(e, st);
    h->prof_marks.emplace_back(name, e);
}
#define LAUNCH(name, ...)            \
    do {                             \
        __VA_ARGS__;                 \
        prof_mark(h, name, st);      \
    } while (0)

#define CK(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            fprintf(stderr, "libsph_b200: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
            return SPH_ERR_CUDA;                                                     \
        }                                                                            \
    } while (0)

inline int blocks_for(int64_t n) { return (int)((n + kBlock - 1) / kBlock) > 0 ? (int)((n + kBlock - 1) / kBlock) : 1; }
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

void fill_constants(SphHandle* h) {
    fill_constants_from(h->p, h->n, h->c);
    solid_fill_constants(h->c);
}

Ptr make_ptr(SphHandle* h) {
    Ptr P;
    P.cur = h->buf.set[h->parity];
    P.nxt = h->buf.set[1 - h->parity];
    // the solid's acceleration (and de_int) is persistent, carried in the field sets
    P.acc = reinterpret_cast<float4*>(h->p.is_solid ? P.cur.acc : h->buf.acc);
    P.lam = h->buf.lam;
    P.lsym = reinterpret_cast<float4*>(h->buf.lsym);
    P.lgrad = reinterpret_cast<float4*>(h->buf.lgrad);
    P.div = reinterpret_cast<float4*>(h->buf.div);
    P.gradv = h->buf.gradv;
    P.aux = reinterpret_cast<float4*>(h->buf.aux);
    P.cell = h->cell;
    P.key = h->key;
    P.rank = h->rank;
    P.perm = h->perm;
    P.hist = h->hist;
    P.start = h->start;
    P.bsum = h->bsum;
    P.bbox = h->bbox;
    P.layout = h->layout;
    P.nbr = h->nbr;
    P.nbr_cnt = h->nbr_cnt;
    P.vl = h->vl;
    P.vl_cnt = h->vl_cnt;
    P.nl_cnt = h->nl_cnt;
    P.ovf = h->ovf;
    P.ovf_off = h->ovf_off;
    P.fcell = h->fcell;
    P.xb = h->xb;
    P.sc = h->sc;
    P.ac = h->ac;
    P.jc = solid_jc_ptr(h->solid);
    P.mat = h->solid.mat;
    P.gsym = h->solid.gsym;
    P.irow = h->solid.irow;
    P.inst = h->solid.inst;
    return P;
}

void drop_graph(SphHandle* h) {
    if (h->graph2) { cudaGraphExecDestroy(h->graph2); h->graph2 = nullptr; }
    if (h->graph1) { cudaGraphExecDestroy(h->graph1); h->graph1 = nullptr; }
}

int scan_tiles(const SphHandle* h) { return (int)((h->c.mcap + 1 + kScanTile - 1) / kScanTile); }

// Hands a pending build request to the device (outside any capture: the next step's
// k_layout reads it).
int apply_force(SphHandle* h, cudaStream_t st) {
    if (!h->force_pending) return SPH_OK;
    // any non-zero word asks for a build; a memset node is also capturable
    CK(cudaMemsetAsync(&h->ac->force_build, 1, sizeof(int), st));
    h->force_pending = false;
    return SPH_OK;
}

// The fluid force pass runs its plain instance on standard decks too: its standard one
// measured slower on the 1M dam break (0.455 against 0.414 ms; the gradient pass's standard
// instance gains 0.433 -> 0.387 ms there).
inline int force_shape(const Cst& c) {
    const int s = shape_of(c);
    return s == 2 ? 1 : s;
}

// update_grid_id / counting_sort / the neighbour search of every step
// (particle_system.py:1300-1490): the step-start bins, the candidate lists when the
// displacement bound asks for a build (the sort kernels return at once otherwise), and
// this step's neighbour list.
int rebuild(SphHandle* h, cudaStream_t st) {
    const int nb = blocks_for(h->n);
    Ptr P = make_ptr(h);
    const Cst& c = h->c;
    prof_mark(h, "", st);
    LAUNCH("k_grid_reset", k_grid_reset<<<1, 32, 0, st>>>(P));
    LAUNCH("k_cells", k_cells<<<std::min(nb, kCellsBlocks), kBlock, 0, st>>>(c, P));
    LAUNCH("k_layout", k_layout<<<1, 32, 0, st>>>(c, P));
    int zb = (int)std::min<int64_t>((c.mcap + 2 + kBlock - 1) / kBlock, 148 * 16);
    LAUNCH("k_zero_hist", k_zero_hist<<<zb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_keys", k_keys<<<nb, kBlock, 0, st>>>(c, P));
    int tiles = scan_tiles(h);
    int sb = std::min(tiles, 148 * 8);
    LAUNCH("k_scan_reduce", k_scan_reduce<<<sb, kBlock, 0, st>>>(P));
    LAUNCH("k_scan_bsum", k_scan_bsum<<<1, 1024, 0, st>>>(P));
    LAUNCH("k_scan_apply", k_scan_apply<<<sb, kBlock, 0, st>>>(P));
    LAUNCH("k_scatter", k_scatter<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_stabilise", k_stabilise<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_gather", k_gather<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_gather_back", k_gather_back<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_vlist_build", k_vlist_build<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_nbr_filter", SHAPED(shape_of(c), k_nbr_filter, <<<nb, kBlock, 0, st>>>(c, P)));
    return SPH_OK;
}

int fluid_substep_and_boundary(SphHandle* h, cudaStream_t st) {
    const int nb = blocks_for(h->n);
    const Cst& c = h->c;
    Ptr P = make_ptr(h);
    const int shape = shape_of(c);
    LAUNCH("k_lam", SHAPED(shape, k_lam, <<<nb, kBlock, 0, st>>>(c, P)));
    LAUNCH("k_lamgrad_cont", SHAPED(shape, k_lamgrad_cont, <<<nb, kBlock, 0, st>>>(c, P)));
    LAUNCH("k_eos", k_eos<<<nb, kBlock, 0, st>>>(c, P));
    LAUNCH("k_force", SHAPED(force_shape(c), k_force, <<<nb, kBlock, 0, st>>>(c, P)));
    LAUNCH("k_dt", k_dt<<<1, 32, 0, st>>>(c, P));
    LAUNCH("k_advect", k_advect<<<nb, kBlock, 0, st>>>(c, P));
    if (h->p.pst_enabled) {
        LAUNCH("k_pst", SHAPED(shape, k_pst, <<<nb, kBlock, 0, st>>>(c, P)));
        LAUNCH("k_finish", k_finish<<<nb, kBlock, 0, st>>>(c, P, 3));
    } else {
        LAUNCH("k_finish", k_finish<<<nb, kBlock, 0, st>>>(c, P, 2));
    }
    return SPH_OK;
}

int one_step(SphHandle* h, cudaStream_t st) {
    int r;
    if (h->p.is_solid) {
        if ((r = solid_pre_step(h->c, make_ptr(h), h->solid, st)) != SPH_OK) return r;
    }
    if ((r = rebuild(h, st)) != SPH_OK) return r;
    if (h->p.is_solid)
        return solid_substep_launch(h->c, make_ptr(h), (int)h->n, st,
                                    [&](const char* name) { prof_mark(h, name, st); });
    return fluid_substep_and_boundary(h, st);
}

template <class T> int dalloc(T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    return e == cudaSuccess ? SPH_OK : SPH_ERR_NOMEM;
}

void free_all(SphHandle* h) {
    drop_graph(h);
    for (cudaEvent_t e : h->prof_pool) cudaEventDestroy(e);
    h->prof_pool.clear();
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    void* ptrs[] = {h->cell, h->key, h->rank, h->perm, h->hist, h->start, h->bsum,
                    h->bbox, h->layout, h->nbr, h->nbr_cnt, h->vl, h->vl_cnt, h->nl_cnt, h->ovf, h->ovf_off, h->fcell, h->xb,
                    h->sc, h->ac};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (h->pinned) cudaFreeHost(h->pinned);
    solid_free(h->solid);
}

bool valid_set(const SphFieldSet& s, bool solid) {
    if (!s.pos || !s.vel || !s.x0 || !s.disp || !s.shift || !s.pid) return false;
    if (solid && (!s.sdev || !s.bc || !s.bcdisp || !s.acc)) return false;
    if (solid && (reinterpret_cast<uintptr_t>(s.acc) & 15u) != 0) return false;
    auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    return al(s.pos) && al(s.vel) && al(s.x0) && al(s.disp) && al(s.shift) &&
           (!solid || (al(s.sdev) && al(s.bcdisp) && (reinterpret_cast<uintptr_t>(s.bc) & 7u) == 0));
}

}  // namespace

extern "C" {

int sph_abi_version(void) { return SPH_ABI_VERSION; }
size_t sph_params_size(void) { return sizeof(SphParams); }
size_t sph_scalars_size(void) { return sizeof(SphScalars); }

const char* sph_strerror(int status) {
    switch (status) {
        case SPH_OK: return "ok";
        case SPH_ERR_ARG: return "invalid argument";
        case SPH_ERR_CUDA: return "CUDA runtime error";
        case SPH_ERR_NOMEM: return "device allocation failed";
        case SPH_ERR_UNSUPPORTED: return "option not implemented by libsph_b200";
        case SPH_ERR_NOT_BOUND: return "buffers not bound (sph_bind)";
        case SPH_ERR_NEIGHBOUR_CAP: return "neighbour list overflow (export needs the full list)";
        case SPH_ERR_TIMEOUT: return "bounded device wait ran out";
        case SPH_ERR_SCRATCH_CAP: return "request exceeds the static scratch capacity";
        default: return "unknown status";
    }
}

int sph_params_layout(char* buf, int cap) {
    std::string s;
#define F(name) s += #name "=" + std::to_string(offsetof(SphParams, name)) + ";";
    F(struct_size) F(is_solid) F(two_d) F(axisymmetric) F(plane_strain) F(sym_y) F(sym_z)
    F(walls) F(displacement_positions) F(compensated_volume) F(support_radius)
    F(particle_diameter) F(V0) F(axi_r_min) F(domain_size) F(padding) F(wall_restitution)
    F(density0) F(c0) F(exponent) F(stiffness) F(viscosity) F(CFL) F(delta_sph) F(gravity)
    F(allow_negative_pressure) F(track_visc_work) F(l_eig_tol_lam) F(c_signal) F(dt_pair_mode)
    F(pst_enabled) F(pst_colle) F(pst_ma_mode) F(pst_clamp_disp) F(pst_clamp_vel)
    F(pst_surface_none) F(pst_normal_eigvec) F(pst_ale_momentum) F(pst_R) F(pst_n)
    F(pst_max_shift) F(pst_ma_fixed) F(pst_m_delta) F(pst_lambda_lo) F(pst_lambda_hi)
    F(n_materials) F(mat_rho0) F(mat_K) F(mat_G) F(mat_cp) F(mat_c0) F(mat_delta)
    F(plastic_kind) F(plastic_sy0) F(plastic_H) F(jc_A) F(jc_B) F(jc_n) F(jc_C) F(jc_eps0_dot)
    F(jc_T0) F(jc_Tm) F(jc_m) F(jc_chi) F(mat_cv) F(mat_stiff) F(mat_gamma) F(mat_T0)
    F(axi_conservative_x) F(hg_rate) F(hg_sts_fixed)
    F(kernel_correction) F(l_eig_tol) F(hourglass_alpha) F(hourglass_sts) F(hourglass_sts_cap)
    F(hourglass_sts_safety) F(hg_S) F(hg_W_dx0) F(hg_sts_refresh) F(ale_history) F(transport_e)
    F(ale_diffusion) F(num_constraints) F(ramp_time) F(jc_surrogate) F(jc_surrogate_tol)
    F(q_l2) F(q_cl) F(av_alpha) F(av_beta) F(av_eps) F(hg_sts_rkl) F(objective_none) F(axi_image_signed) F(axi_conservative_r)
    F(delta_pairs_all) F(c0_mixed) F(hg_mixed_impedance)
#undef F
    if (buf && cap > 0) {
        size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
        memcpy(buf, s.data(), k);
        buf[k] = 0;
    }
    return (int)s.size();
}

int sph_create(const SphParams* p, int64_t n_max, SphHandle** out) {
    if (!p || !out || n_max < 0 || n_max > (int64_t)kIdxMask) return SPH_ERR_ARG;
    if (p->struct_size != (int32_t)sizeof(SphParams)) return SPH_ERR_ARG;
    if (!(p->support_radius > 0.0f) || !(p->particle_diameter > 0.0f)) return SPH_ERR_ARG;
    if (p->is_solid && (p->n_materials < 1 || p->n_materials > 4 || p->num_constraints < 0 ||
                        p->num_constraints > 8))
        return SPH_ERR_ARG;
    *out = nullptr;
    SphHandle* h = new (std::nothrow) SphHandle();
    if (!h) return SPH_ERR_NOMEM;
    h->p = *p;
    h->n_max = n_max;
    cudaGetDevice(&h->device);
    // list capacities from the lattice count at this support: the candidates within
    // 1.1 h (1.1^d of the neighbours) with room for twice the lattice density; the
    // neighbour list holds as many, so it cannot overflow while the candidates fit
    double ratio = (double)p->support_radius / (double)p->particle_diameter;
    double est = p->two_d ? M_PI * ratio * ratio * 1.5 : (4.0 / 3.0) * M_PI * ratio * ratio * ratio;
    const double cand_est = est * (p->two_d ? 1.21 : 1.331);
    int Kv = (int)std::ceil((2.0 * cand_est + 16.0) / 32.0) * 32;
    Kv = std::max(64, std::min(Kv, 1024));
    const int K = Kv;
    int64_t mcap = 131072;
    while (mcap < 4 * n_max) mcap <<= 1;
    int lg = 0;
    while ((1ll << lg) < mcap) ++lg;
    h->n = 0;
    fill_constants(h);
    h->c.Kv = Kv;
    h->c.K = K;
    // the overflow pool: as many entries as all lists (a uniform 2x compression beyond
    // the lists' own headroom)
    const size_t ovf_cap = std::min<size_t>((size_t)std::max<int64_t>(n_max, 1) * (size_t)K, 0x7fffffffu);
    h->c.ovf_cap = (unsigned int)ovf_cap;
    h->c.mcap = (int)mcap;
    h->c.mcap_log2 = lg;
    int r = SPH_OK;
    const size_t N = (size_t)std::max<int64_t>(n_max, 1);
    const size_t tiles = (size_t)((mcap + 1 + kScanTile - 1) / kScanTile) + 1;
    if ((r = dalloc(&h->cell, N)) || (r = dalloc(&h->key, N)) ||
        (r = dalloc(&h->rank, N)) || (r = dalloc(&h->perm, N)) ||
        (r = dalloc(&h->hist, (size_t)mcap + 2)) || (r = dalloc(&h->start, (size_t)mcap + 2)) ||
        (r = dalloc(&h->bsum, tiles)) || (r = dalloc(&h->bbox, 8)) ||
        (r = dalloc(&h->layout, 1)) || (r = dalloc(&h->nbr, N * (size_t)K)) ||
        (r = dalloc(&h->nbr_cnt, N)) || (r = dalloc(&h->sc, 1)) || (r = dalloc(&h->ac, 1)) ||
        (r = dalloc(&h->vl, N * (size_t)Kv)) || (r = dalloc(&h->vl_cnt, N)) ||
        (r = dalloc(&h->nl_cnt, N)) ||
        (r = dalloc(&h->ovf, ovf_cap)) || (r = dalloc(&h->ovf_off, N)) ||
        (r = dalloc(&h->fcell, N)) || (r = dalloc(&h->xb, N)) ||
        cudaMallocHost((void**)&h->pinned, sizeof(SphScalars)) != cudaSuccess) {
        if (!r) r = SPH_ERR_NOMEM;
        free_all(h);
        delete h;
        return r;
    }
    if (p->is_solid && ((r = solid_alloc(h->solid, *p, n_max)) != SPH_OK ||
                        (r = solid_sync_rows(h->solid, h->p, h->c)) != SPH_OK)) {
        free_all(h);
        delete h;
        return r;
    }
    SphScalars s0;
    memset(&s0, 0, sizeof(s0));
    // DSPH.py:124-131: the initial step from the CFL on the signal speed
    s0.dt = (float)((double)p->CFL * (double)p->support_radius / (double)p->c_signal);
    DevAccum a0;
    memset(&a0, 0, sizeof(a0));
    if (cudaMemcpy(h->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->ac, &a0, sizeof(a0), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(h->nbr_cnt, 0, N * sizeof(int)) != cudaSuccess ||
        // no lists and no cells until the first build: empty counts, off-grid cells, an
        // empty layout
        cudaMemset(h->vl_cnt, 0, N * sizeof(int)) != cudaSuccess ||
        cudaMemset(h->nl_cnt, 0, N * sizeof(int)) != cudaSuccess ||
        cudaMemset(h->cell, 0xff, N * sizeof(int4)) != cudaSuccess ||
        cudaMemset(h->fcell, 0xff, N * sizeof(int4)) != cudaSuccess ||
        cudaMemset(h->layout, 0, sizeof(GridLayout)) != cudaSuccess) {
        free_all(h);
        delete h;
        return SPH_ERR_CUDA;
    }
    *out = h;
    return SPH_OK;
}

void sph_destroy(SphHandle* h) {
    if (!h) return;
    cudaDeviceSynchronize();
    free_all(h);
    delete h;
}

int sph_bind(SphHandle* h, const SphBuffers* b, int64_t n) {
    if (!h || !b || n < 0 || n > h->n_max) return SPH_ERR_ARG;
    if (!valid_set(b->set[0], h->p.is_solid) || !valid_set(b->set[1], h->p.is_solid)) return SPH_ERR_ARG;
    if ((!h->p.is_solid && !b->acc) || !b->lam || !b->lsym || !b->lgrad || !b->div) return SPH_ERR_ARG;
    if (h->p.is_solid && (!b->gradv || !b->aux)) return SPH_ERR_ARG;
    drop_graph(h);
    h->buf = *b;
    h->n = n;
    h->c.n = (int)n;
    h->parity = 0;
    h->bound = true;
    h->force_pending = true;
    return SPH_OK;
}

int sph_parity(const SphHandle* h) { return h ? h->parity : -1; }

int sph_set_params(SphHandle* h, const SphParams* p) {
    if (!h || !p || p->struct_size != (int32_t)sizeof(SphParams)) return SPH_ERR_ARG;
    if (p->is_solid != h->p.is_solid) return SPH_ERR_ARG;
    if (p->is_solid && (p->n_materials < 1 || p->n_materials > 4)) return SPH_ERR_ARG;
    int K = h->c.K, mcap = h->c.mcap, lg = h->c.mcap_log2, bs = h->c.block, Kv = h->c.Kv;
    unsigned int cap = h->c.ovf_cap;
    h->p = *p;
    fill_constants(h);
    h->c.K = K; h->c.mcap = mcap; h->c.mcap_log2 = lg; h->c.n = (int)h->n; h->c.block = bs;
    h->c.Kv = Kv;
    h->c.ovf_cap = cap;
    h->force_pending = true;
    int r = solid_sync_rows(h->solid, h->p, h->c);
    drop_graph(h);
    return r;
}

int sph_initialize(SphHandle* h, void* stream) {
    if (!h) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    if (h->n == 0) return SPH_OK;
    h->force_pending = true;
    int r = apply_force(h, S(stream));
    if (!r) r = rebuild(h, S(stream));
    if (r) return r;
    CK(cudaGetLastError());
    return SPH_OK;
}

// Captures `steps` consecutive steps into *out (the state stays in field set A, so one
// graph serves any step).
int capture_steps(SphHandle* h, int steps, cudaStream_t st, cudaGraphExec_t* out) {
    if (!h->cap_stream) CK(cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g;
    // finish everything queued on the caller's stream before capturing
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    int r = SPH_OK;
    for (int k = 0; k < steps && r == SPH_OK; ++k) r = one_step(h, h->cap_stream);
    cudaError_t ec = cudaStreamEndCapture(h->cap_stream, &g);
    h->capturing = false;
    if (r != SPH_OK) { if (ec == cudaSuccess) cudaGraphDestroy(g); return r; }
    CK(ec);
    cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    return SPH_OK;
}

int sph_step(SphHandle* h, int nsteps, void* stream) {
    if (!h || nsteps < 0) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    if (h->n == 0 || nsteps == 0) return SPH_OK;
    cudaStream_t st = S(stream);
    if (int r = apply_force(h, st)) return r;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
        // the caller is recording a graph of its own: the steps' kernels go into it
        for (int k = 0; k < nsteps; ++k)
            if (int r = one_step(h, st)) return r;
        return SPH_OK;
    }
    const int pairs = nsteps / 2;
    if (pairs > 0) {
        if (!h->graph2) {
            if (int r = capture_steps(h, 2, st, &h->graph2)) return r;
        }
        for (int k = 0; k < pairs; ++k) CK(cudaGraphLaunch(h->graph2, st));
    }
    if (nsteps & 1) {
        if (h->prof_on) {   // the per-kernel profile times eager launches
            if (int r = one_step(h, st)) return r;
        } else {
            if (!h->graph1) {
                if (int r = capture_steps(h, 1, st, &h->graph1)) return r;
            }
            CK(cudaGraphLaunch(h->graph1, st));
        }
    }
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_run_stage(SphHandle* h, int stage, void* stream) {
    if (!h) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    if (h->n == 0) return SPH_OK;
    cudaStream_t st = S(stream);
    if (int r = apply_force(h, st)) return r;
    const int nb = blocks_for(h->n);
    if (h->p.is_solid) {
        if (stage < SPH_STAGE_SORT || stage > SPH_STAGE_BOUNDARY) return SPH_ERR_ARG;
        int r = SPH_OK;
        if (stage == SPH_STAGE_SORT) {
            r = solid_pre_step(h->c, make_ptr(h), h->solid, st);
            if (!r) r = rebuild(h, st);
        } else {
            r = solid_substep_launch(h->c, make_ptr(h), (int)h->n, st,
                                     [&](const char* name) { prof_mark(h, name, st); }, stage, stage);
        }
        if (r) return r;
        CK(cudaGetLastError());
        return SPH_OK;
    }
    Ptr P = make_ptr(h);
    const Cst& c = h->c;
    switch (stage) {
        case SPH_STAGE_SORT: { int r = rebuild(h, st); if (r) return r; break; }
        case SPH_STAGE_LAM:
            SHAPED(shape_of(c), k_lam, <<<nb, kBlock, 0, st>>>(c, P));
            SHAPED(shape_of(c), k_lamgrad_cont, <<<nb, kBlock, 0, st>>>(c, P));
            break;
        case SPH_STAGE_CONTINUITY: k_eos<<<nb, kBlock, 0, st>>>(c, P); break;
        case SPH_STAGE_FORCES: SHAPED(force_shape(c), k_force, <<<nb, kBlock, 0, st>>>(c, P)); break;
        case SPH_STAGE_DT: k_dt<<<1, 32, 0, st>>>(c, P); break;
        case SPH_STAGE_ADVECT: k_advect<<<nb, kBlock, 0, st>>>(c, P); break;
        case SPH_STAGE_PST:
            if (h->p.pst_enabled) {
                SHAPED(shape_of(c), k_pst, <<<nb, kBlock, 0, st>>>(c, P));
                k_finish<<<nb, kBlock, 0, st>>>(c, P, 1);
            }
            break;
        case SPH_STAGE_BOUNDARY: k_finish<<<nb, kBlock, 0, st>>>(c, P, 2); break;
        default: return SPH_ERR_ARG;
    }
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_set_dt(SphHandle* h, float dt, void* stream) {
    if (!h) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(S(stream)));
    h->pinned->dt = dt;
    CK(cudaMemcpyAsync(&h->sc->dt, &h->pinned->dt, sizeof(float), cudaMemcpyHostToDevice, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
    return SPH_OK;
}

int sph_get_dt(SphHandle* h, float* dt, void* stream) {
    if (!h || !dt) return SPH_ERR_ARG;
    CK(cudaMemcpyAsync(&h->pinned->dt, &h->sc->dt, sizeof(float), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
    *dt = h->pinned->dt;
    return SPH_OK;
}

int sph_get_scalars(SphHandle* h, SphScalars* out, void* stream) {
    if (!h || !out) return SPH_ERR_ARG;
    CK(cudaMemcpyAsync(h->pinned, h->sc, sizeof(SphScalars), cudaMemcpyDeviceToHost, S(stream)));
    CK(cudaStreamSynchronize(S(stream)));
    memcpy(out, h->pinned, sizeof(SphScalars));
    return SPH_OK;
}

int sph_constraints(SphHandle* h, double* force, double* disp, int k, void* stream) {
    if (!h || !h->p.is_solid || h->solid.n_inst > 0 || k < 0 || k > h->p.num_constraints) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    CK(cudaMemcpyAsync(h->pinned, h->sc, sizeof(SphScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int g = 0; g < k; ++g)
        for (int d = 0; d < 3; ++d) {
            if (force) force[3 * g + d] = h->pinned->constraint_force[g][d];
            if (disp) disp[3 * g + d] = h->pinned->constraint_disp[g][d];
        }
    return SPH_OK;
}

int sph_clear_error(SphHandle* h, void* stream) {
    if (!h) return SPH_ERR_ARG;
    CK(cudaMemsetAsync(&h->sc->err, 0, sizeof(int), S(stream)));
    return SPH_OK;
}

int sph_reduce(SphHandle* h, double* out, void* stream) {
    if (!h || !out) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    cudaStream_t st = S(stream);
    CK(cudaMemsetAsync(h->ac->red, 0, sizeof(double) * SPH_RED_COUNT, st));
    if (h->n > 0) {
        Ptr P = make_ptr(h);
        k_reduce<<<blocks_for(h->n), kBlock, 0, st>>>(h->c, P);
        if (h->p.is_solid) solid_reduce_extra(h->c, P, (int)h->n, st);
    }
    CK(cudaMemcpyAsync(out, h->ac->red, sizeof(double) * SPH_RED_COUNT, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH_OK;
}

}  // extern "C"

namespace {
// Largest |x - x_build| over the particles, rounded up, into *dbits (float bits).
__global__ void __launch_bounds__(kBlock) k_disp_since_build(Cst c, Ptr P, unsigned int* dbits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float d = 0.0f;
    if (i < c.n) {
        const float4 p = reinterpret_cast<const float4*>(P.cur.pos)[i];
        if (!(isnan(p.x) || isnan(p.y) || isnan(p.z))) {
            const float4 b = P.xb[i];
            d = norm3(F3{p.x - b.x, p.y - b.y, p.z - b.z}) * (1.0f + 1e-5f);
            if (isnan(d)) d = INFINITY;
        }
    }
    block_max_atomic(d, dbits);
}

// Pair export: one thread per particle counts (off == nullptr, counts to cnt_out) or
// writes its pairs at off[i].  kShift 0: the reference's sweep from the current positions
// against this step's start bins, searched in the coarse table for displacement *dbits;
// kShift 1: the pairs the shift pass evaluates (for_each_pst_neighbour); kShift 2: this
// step's neighbour list as the pair passes read it (for_each_neighbour).
template <int kShift>
__global__ void k_pairs_export(Cst c, Ptr P, const unsigned int* dbits, const int* off, int* cnt_out,
                               int* out_i, int* out_j, int* out_m) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const F3 xi = f3(reinterpret_cast<const float4*>(P.cur.pos)[i]);
    int cnt = 0;
    const int base = off ? off[i] : 0;
    auto emit = [&](int j, int mir) {
        if (off) { out_i[base + cnt] = i; out_j[base + cnt] = j; out_m[base + cnt] = mir; }
        ++cnt;
    };
    auto emit3 = [&](int j, int mir, float4) { emit(j, mir); };
    auto emit5 = [&](int j, int mir, float4, F3, float) { emit(j, mir); };
    if (kShift == 2) {
        for_each_neighbour(c, P, i, emit);
    } else if (kShift == 1) {
        for_each_pst_neighbour<false>(c, P, i, xi, emit5);
    } else if (!(isnan(xi.x) || isnan(xi.y) || isnan(xi.z))) {
        stale_search(c, P, i, xi, cell_of(xi.x, c.h), cell_of(xi.y, c.h), cell_of(xi.z, c.h),
                     __uint_as_float(*dbits), emit3);
    }
    if (!off) cnt_out[i] = cnt;
}

// Counts, then writes, the pairs of one export kernel into host arrays.
template <int kShift>
int export_pairs(SphHandle* h, int32_t* pi, int32_t* pj, int32_t* mir, int64_t cap, int64_t* count,
                 cudaStream_t st) {
    const int n = (int)h->n;
    Ptr P = make_ptr(h);
    int* dcnt = nullptr;
    unsigned int* dbits = nullptr;
    int r = dalloc(&dcnt, n);
    if (!r) r = dalloc(&dbits, 1);
    if (r) { cudaFree(dcnt); return r; }
    std::vector<int> cnt(n);
    cudaMemsetAsync(dbits, 0, sizeof(unsigned int), st);
    k_disp_since_build<<<blocks_for(n), kBlock, 0, st>>>(h->c, P, dbits);
    k_pairs_export<kShift><<<blocks_for(n), kBlock, 0, st>>>(h->c, P, dbits, nullptr, dcnt, nullptr, nullptr,
                                                             nullptr);
    cudaMemcpyAsync(cnt.data(), dcnt, n * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { cudaFree(dcnt); cudaFree(dbits); CK(e); }
    std::vector<int> off(n);
    int64_t tot = 0;
    for (int i = 0; i < n; ++i) { off[i] = (int)tot; tot += cnt[i]; }
    *count = tot;
    int *di = nullptr, *dj = nullptr, *dm = nullptr;
    const size_t m1 = (size_t)std::max<int64_t>(tot, 1);
    if ((r = dalloc(&di, m1)) || (r = dalloc(&dj, m1)) || (r = dalloc(&dm, m1))) {
        cudaFree(dcnt); cudaFree(dbits); cudaFree(di); cudaFree(dj); cudaFree(dm);
        return r;
    }
    cudaMemcpyAsync(dcnt, off.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
    k_pairs_export<kShift><<<blocks_for(n), kBlock, 0, st>>>(h->c, P, dbits, dcnt, nullptr, di, dj, dm);
    int64_t m = std::min<int64_t>(cap, tot);
    if (pi && m > 0) {
        cudaMemcpyAsync(pi, di, m * sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(pj, dj, m * sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(mir, dm, m * sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    e = cudaStreamSynchronize(st);
    cudaFree(dcnt); cudaFree(dbits); cudaFree(di); cudaFree(dj); cudaFree(dm);
    CK(e);
    CK(cudaGetLastError());
    return SPH_OK;
}
}  // namespace

extern "C" int sph_pairs(SphHandle* h, int mode, int32_t* pi, int32_t* pj, int32_t* mir,
                         int64_t cap, int64_t* count, void* stream) {
    if (!h || !count || (mode != 0 && mode != 1)) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    cudaStream_t st = S(stream);
    const int n = (int)h->n;
    *count = 0;
    if (n == 0) return SPH_OK;
    if (mode == 1) return export_pairs<0>(h, pi, pj, mir, cap, count, st);
    return export_pairs<2>(h, pi, pj, mir, cap, count, st);
}

extern "C" int sph_shift_pairs(SphHandle* h, float disp_bound, int32_t* pi, int32_t* pj, int32_t* mir,
                               int64_t cap, int64_t* count, void* stream) {
    if (!h || !count || std::isnan(disp_bound)) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    cudaStream_t st = S(stream);
    *count = 0;
    if (h->n == 0) return SPH_OK;
    // the step's displacement record (since the build, this step's advect, the grips),
    // replaced for this call when a bound is given
    // (a given bound also drops the near lists, which belong to the step's start)
    unsigned int* words[4] = {&h->ac->d_start_bits, &h->ac->max_disp_bits, &h->ac->max_grip_disp_bits,
                              &h->ac->near_m_bits};
    unsigned int saved[4];
    for (int k = 0; k < 4; ++k)
        CK(cudaMemcpyAsync(&saved[k], words[k], sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    unsigned int set[4] = {0u, 0u, 0u, 0u};
    if (disp_bound >= 0.0f) {
        std::memcpy(&set[0], &disp_bound, sizeof(float));
        for (int k = 0; k < 4; ++k)
            CK(cudaMemcpyAsync(words[k], &set[k], sizeof(unsigned int), cudaMemcpyHostToDevice, st));
    }
    const int r = export_pairs<1>(h, pi, pj, mir, cap, count, st);
    for (int k = 0; k < 4; ++k)
        CK(cudaMemcpyAsync(words[k], &saved[k], sizeof(unsigned int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return r;
}

extern "C" int sph_relax_pass(SphHandle* h, float beta, float* residual, float* residual_each,
                              void* stream) {
    if (!h || !residual || !(beta >= 0.0f)) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    cudaStream_t st = S(stream);
    *residual = 0.0f;
    if (h->n == 0) return SPH_OK;
    if (int r = apply_force(h, st)) return r;
    const int nb = blocks_for(h->n);
    if (int r = rebuild(h, st)) return r;
    Ptr P = make_ptr(h);
    const Cst& c = h->c;
    k_lam<0><<<nb, kBlock, 0, st>>>(c, P);
    if (!h->p.pst_normal_eigvec) k_relax_lamgrad<<<nb, kBlock, 0, st>>>(c, P);
    CK(cudaMemsetAsync(&h->ac->relax_max_bits, 0, sizeof(unsigned int), st));
    k_relax<<<nb, kBlock, 0, st>>>(c, P, beta, residual_each);
    unsigned int bits = 0u;
    CK(cudaMemcpyAsync(&bits, &h->ac->relax_max_bits, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(residual, &bits, sizeof(float));
    CK(cudaGetLastError());
    return SPH_OK;
}

extern "C" int sph_relax_move(SphHandle* h, void* stream) {
    if (!h) return SPH_ERR_ARG;
    if (!h->bound) return SPH_ERR_NOT_BOUND;
    if (h->n == 0) return SPH_OK;
    cudaStream_t st = S(stream);
    k_relax_move<<<blocks_for(h->n), kBlock, 0, st>>>(h->c, make_ptr(h));
    CK(cudaGetLastError());
    return SPH_OK;
}

extern "C" int sph_list_stats(SphHandle* h, uint64_t* out, int reset, void* stream) {
    if (!h || !out) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    unsigned long long v[3];
    CK(cudaMemcpyAsync(v, &h->ac->n_steps, sizeof(v), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) out[k] = (uint64_t)v[k];
    if (reset) {
        static const unsigned long long zero[3] = {0ull, 0ull, 0ull};
        CK(cudaMemcpyAsync(&h->ac->n_steps, zero, sizeof(zero), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    return SPH_OK;
}

extern "C" int sph_profile_enable(SphHandle* h, int on) {
    if (!h) return SPH_ERR_ARG;
    h->prof_on = on != 0;
    h->prof_marks.clear();
    h->prof_used = 0;
    return SPH_OK;
}

extern "C" int sph_profile_read(SphHandle* h, char* names, int names_cap, double* ms,
                                int* launches, int cap, int* count) {
    if (!h || !count) return SPH_ERR_ARG;
    CK(cudaDeviceSynchronize());
    std::vector<std::string> nm;
    std::vector<double> tot;
    std::vector<int> cnt;
    for (size_t k = 1; k < h->prof_marks.size(); ++k) {
        const char* name = h->prof_marks[k].first;
        if (!name || !name[0]) continue;  // a sequence start
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, h->prof_marks[k - 1].second, h->prof_marks[k].second) != cudaSuccess)
            continue;
        size_t idx = 0;
        while (idx < nm.size() && nm[idx] != name) ++idx;
        if (idx == nm.size()) { nm.push_back(name); tot.push_back(0.0); cnt.push_back(0); }
        tot[idx] += t;
        cnt[idx] += 1;
    }
    std::string joined;
    int m = (int)std::min<size_t>(nm.size(), (size_t)std::max(cap, 0));
    for (int k = 0; k < m; ++k) {
        if (ms) ms[k] = tot[k];
        if (launches) launches[k] = cnt[k];
        joined += nm[k];
        joined += "\n";
    }
    if (names && names_cap > 0) {
        size_t L = std::min<size_t>(joined.size(), (size_t)names_cap - 1);
        memcpy(names, joined.data(), L);
        names[L] = 0;
    }
    *count = m;
    h->prof_marks.clear();
    h->prof_used = 0;
    return SPH_OK;
}

// ------------------------------------------------------------------ Johnson-Cook surrogate
extern "C" {

namespace {
// Eight independent FMA chains per thread, kFmaIters rounds; the sum is stored so that
// nothing is optimised away.
constexpr int kFmaIters = 4096;
__global__ void __launch_bounds__(256) k_fma_peak(float* out, float a, float b) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int it = 0; it < kFmaIters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 123.456f) out[blockIdx.x & 1023] = s;   // practically never; keeps the chains live
}
}  // namespace

int sph_fma_peak(double* tflops, void* stream) {
    if (!tflops) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* out = nullptr;
    CK(cudaMalloc((void**)&out, 1024 * sizeof(float)));
    const int blocks = sms * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_peak<<<blocks, 256, 0, st>>>(out, 0.999f, 1e-4f);   // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < 10; ++r) k_fma_peak<<<blocks, 256, 0, st>>>(out, 0.999f, 1e-4f);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    CK(e);
    const double flop = 10.0 * blocks * 256.0 * kFmaIters * 8.0 * 2.0;
    *tflops = ms > 0.0f ? flop / (ms * 1e-3) / 1e12 : 0.0;
    return SPH_OK;
}

int sph_mlp_param_count(void) { return kMlpParams; }
int64_t sph_mlp_packed_bytes(void) { return (int64_t)kMlpPackedBytes; }

int sph_mlp_forward(const float* W, const float* X, int64_t n, float* Y, void* stream) {
    if (!W || (n > 0 && (!X || !Y)) || n < 0 || n > INT32_MAX) return SPH_ERR_ARG;
    if (n == 0) return SPH_OK;
    k_mlp_forward<<<(int)((n + 127) / 128), 128, 0, S(stream)>>>(W, reinterpret_cast<const float4*>(X), (int)n, Y);
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_mlp_grad(const float* W, const float* X, const float* T, int64_t n, float* G, double* loss,
                 void* stream) {
    if (!W || !G || !loss || n <= 0 || n > INT32_MAX || !X || !T) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    CK(cudaMemsetAsync(G, 0, sizeof(float) * kMlpParams, st));
    CK(cudaMemsetAsync(loss, 0, sizeof(double), st));
    k_mlp_grad<<<(int)((n + kMlpGradThreads - 1) / kMlpGradThreads), kMlpGradThreads,
                 sizeof(float) * kMlpParams, st>>>(W, reinterpret_cast<const float4*>(X), T, (int)n,
                                                    1.0f / (float)n, G, loss);
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_mlp_adam(float* W, const float* G, float* M, float* V, int64_t step, float lr, void* stream) {
    if (!W || !G || !M || !V || step < 1 || !(lr > 0.0f)) return SPH_ERR_ARG;
    const double b1 = 0.9, b2 = 0.999;
    const float c1 = (float)(1.0 / (1.0 - std::pow(b1, (double)step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow(b2, (double)step)));
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, S(stream)>>>(W, G, M, V, kMlpParams, lr, (float)b1,
                                                                (float)b2, 1e-8f, c1, c2);
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_mlp_pack(const float* W, void* packed, void* stream) {
    if (!W || !packed) return SPH_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(packed) % 16) return SPH_ERR_ARG;
    k_mlp_pack<<<(2 * kMlpPackedHalf + 255) / 256, 256, 0, S(stream)>>>(W, static_cast<__nv_bfloat16*>(packed));
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_mlp_infer_tc(const float* W, const void* packed, const float* X, int64_t n, float* Y, int* err,
                     void* stream) {
    if (!W || !packed || !err || n < 0 || n > INT32_MAX || (n > 0 && (!X || !Y))) return SPH_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(packed) % 16 || reinterpret_cast<uintptr_t>(X) % 16) return SPH_ERR_ARG;
    if (n == 0) return SPH_OK;
    const int tiles = (int)((n + kMlpTileRows - 1) / kMlpTileRows);
    k_mlp_tc<<<std::min(kMlpCtasPerSm * 148, tiles), kMlpTcThreads, 0, S(stream)>>>(
        W, static_cast<const __nv_bfloat16*>(packed), reinterpret_cast<const float4*>(X), (int)n, nullptr, Y, err);
    CK(cudaGetLastError());
    return SPH_OK;
}

int sph_jc_surrogate(SphHandle* h, const float* W, float tol, int enable, void* stream) {
    if (!h || !h->p.is_solid) return SPH_ERR_ARG;
    if (enable && (!W || !(tol > 0.0f))) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    if (enable) {
        int r = solid_jc_alloc(h->solid, h->n_max);
        if (r) return r;
        CK(cudaMemcpyAsync(h->solid.W, W, sizeof(float) * kMlpParams, cudaMemcpyDeviceToDevice, st));
        k_mlp_pack<<<(2 * kMlpPackedHalf + 255) / 256, 256, 0, st>>>(h->solid.W,
                                                                    static_cast<__nv_bfloat16*>(h->solid.packed));
        CK(cudaGetLastError());
        h->p.jc_surrogate_tol = h->c.p.jc_surrogate_tol = tol;
    }
    h->p.jc_surrogate = h->c.p.jc_surrogate = enable ? 1 : 0;
    drop_graph(h);
    return SPH_OK;
}

int sph_jc_log(SphHandle* h, float* rows, int64_t capacity, unsigned long long* count) {
    if (!h || !h->p.is_solid) return SPH_ERR_ARG;
    if (rows && (!count || capacity <= 0 || reinterpret_cast<uintptr_t>(rows) % 16)) return SPH_ERR_ARG;
    h->solid.log = rows;
    h->solid.log_count = rows ? count : nullptr;
    h->solid.log_cap = rows ? capacity : 0;
    drop_graph(h);
    return SPH_OK;
}

int sph_jc_stats(SphHandle* h, uint64_t* out, int reset, void* stream) {
    if (!h || !out || !h->p.is_solid || !h->solid.stats) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    unsigned long long v[4];
    CK(cudaMemcpyAsync(v, h->solid.stats, sizeof(v), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; ++k) out[k] = v[k];
    if (reset) CK(cudaMemsetAsync(h->solid.stats, 0, sizeof(v), st));
    return SPH_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ ensembles and launch shape
extern "C" {

int sph_ensemble_set(SphHandle* h, const SphMatRow* mat, const SphInstRow* inst, int n_inst,
                     const float* dt0, void* stream) {
    if (!h || !h->p.is_solid || n_inst < 0 || n_inst > kMaxInstances) return SPH_ERR_ARG;
    if (n_inst > 0 && (!mat || !inst || !dt0)) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    if (n_inst == 0) {
        h->solid.n_inst = 0;
        int r = solid_sync_rows(h->solid, h->p, h->c);
        drop_graph(h);
        return r;
    }
    for (int k = 0; k < n_inst; ++k)
        if (!(dt0[k] > 0.0f) || !(mat[k].rho0 > 0.0f)) return SPH_ERR_ARG;
    // the instances' time steps carry no viscosity limits
    if (h->p.q_l2 > 0.0f || h->p.av_alpha > 0.0f || h->p.av_beta > 0.0f) return SPH_ERR_UNSUPPORTED;
    std::vector<SphInstState> s0((size_t)n_inst);
    for (int k = 0; k < n_inst; ++k) {
        memset(&s0[k], 0, sizeof(SphInstState));
        s0[k].dt = dt0[k];
        s0[k].sts_stages = 1;
    }
    CK(cudaMemcpyAsync(h->solid.mat, mat, sizeof(SphMatRow) * n_inst, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->solid.irow, inst, sizeof(SphInstRow) * n_inst, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->solid.inst, s0.data(), sizeof(SphInstState) * n_inst, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));           // s0 is a host temporary
    solid_row_flags(mat, n_inst, h->solid.any_plastic, h->solid.all_gamma_one, h->solid.any_jc);
    h->solid.n_inst = n_inst;
    h->c.n_inst = n_inst;
    h->c.any_plastic = h->solid.any_plastic;
    h->c.all_gamma_one = h->solid.all_gamma_one;
    h->c.any_jc = h->solid.any_jc;
    h->c.one_material = 0;
    h->force_pending = true;
    drop_graph(h);
    return SPH_OK;
}

int sph_ensemble_state(SphHandle* h, SphInstState* out, int n_inst, void* stream) {
    if (!h || !out || !h->p.is_solid || n_inst < 1 || n_inst > h->solid.n_inst) return SPH_ERR_ARG;
    cudaStream_t st = S(stream);
    CK(cudaMemcpyAsync(out, h->solid.inst, sizeof(SphInstState) * n_inst, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH_OK;
}

int sph_set_block(SphHandle* h, int threads) {
    if (!h) return SPH_ERR_ARG;
    if (threads == 0) threads = kBlock;
    if (threads < 64 || threads > kBlock || threads % 32) return SPH_ERR_ARG;
    h->c.block = threads;
    drop_graph(h);
    return SPH_OK;
}

}  // extern "C"

// sph_grid.cuh -- cell binning, counting sort with Morton-ordered buckets, the reorder of
// every persistent field, and neighbour enumeration.
//
// Replaces ParticleSystem.update_grid_id / PrefixSumExecutor / counting_sort
// (particle_system.py:1300-1345) and for_all_neighbors (:1348-1490).  The reference
// bins through a spatial hash whose bucket order is random in space; here the buckets
// are the cells of the occupied cell box in compact Morton order, so the sorted particle
// order is spatially coherent and the neighbour gathers of the pair passes stay in L1/L2.
// When the occupied box does not fit the table (a particle far from the rest) the
// rebuild falls back to the reference's hashed table, with its cell-id filter.  Both
// enumerate exactly the reference's neighbour set: j binned in one of the 27 cells
// around i's cell, j != i, |x_i - x_j| < h, plus the mirror sweeps.
#pragma once
#include "sph_device.cuh"

namespace sph {

// ------------------------------------------------------------------ binning
__global__ void k_grid_reset(Ptr P) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        P.bbox[0] = P.bbox[1] = P.bbox[2] = 0x7fffffff;
        P.bbox[3] = P.bbox[4] = P.bbox[5] = (int)0x80000000;
        P.sc->off_grid_num = 0;
        P.sc->off_grid_mass = 0.0;
        P.ac->d_start_bits = 0u;
    }
}

// update_grid_id's first half (particle_system.py:1224-1234, :1304-1316): NaN
// quarantine and the off-grid tally, every particle's cell of size h (the bins of this
// step), the box of occupied coarse cells (used if this step builds), and how far the
// particles moved since the last build.  Grid-stride over at most kCellsBlocks blocks,
// reduced per block: one atomic per block and quantity (per-warp atomics on the box's six
// words serialised at the L2).
constexpr int kCellsBlocks = 148 * 8;
__global__ void __launch_bounds__(kBlock) k_cells(Cst c, Ptr P) {
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff};
    int mx[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
    int offg = 0;
    double offm = 0.0;
    float dst = 0.0f;
    const float4* __restrict__ pos = reinterpret_cast<const float4*>(P.cur.pos);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        const bool nan = isnan(p.x) || isnan(p.y) || isnan(p.z);
        P.fcell[i] = nan ? make_int4(0, 0, 0, -1)
                         : make_int4(cell_of(p.x, c.h), cell_of(p.y, c.h), cell_of(p.z, c.h), 0);
        if (nan) {
            offg += 1;
            offm += (double)P.cur.vel[4 * i + 3];
        } else {
            // coarse cell, for the box of a build
            const int cx = cell_of(p.x, c.hc), cy = cell_of(p.y, c.hc), cz = cell_of(p.z, c.hc);
            mn[0] = min(mn[0], cx); mx[0] = max(mx[0], cx);
            mn[1] = min(mn[1], cy); mx[1] = max(mx[1], cy);
            mn[2] = min(mn[2], cz); mx[2] = max(mx[2], cz);
            const float4 b = P.xb[i];
            // rounded up; a NaN build position (never built) reads as infinitely far
            const float d = norm3(F3{p.x - b.x, p.y - b.y, p.z - b.z}) * (1.0f + 1e-5f);
            dst = fmaxf(dst, isnan(d) ? INFINITY : d);
        }
    }
    __shared__ int s_box[6][32];
    __shared__ float s_d[32];
    __shared__ int s_n[32];
    __shared__ double s_m[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    dst = warp_max(dst);
    offm = warp_sum(offm);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) offg += __shfl_xor_sync(0xffffffffu, offg, o);
    if (lane == 0) {
        for (int a = 0; a < 3; ++a) { s_box[a][wid] = mn[a]; s_box[3 + a][wid] = mx[a]; }
        s_d[wid] = dst; s_n[wid] = offg; s_m[wid] = offm;
    }
    __syncthreads();
    if (wid == 0) {
        const bool in = lane < nw;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int v0 = in ? s_box[a][lane] : 0x7fffffff, v1 = in ? s_box[3 + a][lane] : (int)0x80000000;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                v0 = min(v0, __shfl_xor_sync(0xffffffffu, v0, o));
                v1 = max(v1, __shfl_xor_sync(0xffffffffu, v1, o));
            }
            if (lane == 0) {
                if (v0 != 0x7fffffff) atomicMin(&P.bbox[a], v0);
                if (v1 != (int)0x80000000) atomicMax(&P.bbox[3 + a], v1);
            }
        }
        float d = warp_max(in ? s_d[lane] : 0.0f);
        double m = warp_sum(in ? s_m[lane] : 0.0);
        int g = in ? s_n[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) {
            atomicMax(&P.ac->d_start_bits, __float_as_uint(fmaxf(d, 0.0f)));
            if (g) {
                atomicAdd(&P.sc->off_grid_num, g);
                atomicAdd(&P.sc->off_grid_mass, m);
            }
        }
    }
}

// Decides whether this step builds the candidate lists: when the host asked, when the
// off-grid count changed (the lists hold no quarantined particle), or when the particles'
// displacement since the last build plus the last step's could pass the lists' bound (so
// that the shift pass, after this step's move, can still use them).  A build chooses the
// table: dense Morton over the occupied coarse-cell box if its compact code fits the
// capacity, else the hashed table.
__global__ void k_layout(Cst c, Ptr P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    DevAccum& A = *P.ac;
    const float dstart = __uint_as_float(A.d_start_bits);
    const float pred = __uint_as_float(A.max_disp_bits) + __uint_as_float(A.max_grip_disp_bits);
    A.max_disp_bits = 0u;       // this step's move accumulates from here
    A.max_grip_disp_bits = 0u;
    A.m_min_bits = 0xffffffffu; // filled by this step's advect (fluid)
    A.m_max_bits = 0u;
    A.ovf_used = 0u;
    const int offg = P.sc->off_grid_num;
    const int build = A.force_build || offg != A.off_grid_build || !(dstart + pred <= c.dlim);
    A.n_steps += 1ull;
    A.rebuild = build;
    // the near lists' margin: three times the last step's move (at least h / 1000), and no
    // more than the candidates cover beyond this step's start (2 (dlim - D_start)), so
    // that the shift may use them whenever this step moves particles less than M / 2
    {
        const float ds = build ? 0.0f : dstart;
        float m = fmaxf(3.0f * pred, 1e-3f * c.h);
        m = fminf(m, 2.0f * (c.dlim - ds));
        A.near_m_bits = (m > 0.0f) ? __float_as_uint(m) : 0u;
    }
    if (!build) return;
    A.force_build = 0;
    A.off_grid_build = offg;
    A.d_start_bits = 0u;
    A.n_builds += 1ull;
    GridLayout L;
    int any = P.bbox[0] <= P.bbox[3];
    int tb = 0;
    for (int a = 0; a < 3; ++a) {
        L.cmin[a] = any ? P.bbox[a] : 0;
        L.cmax[a] = any ? P.bbox[3 + a] : 0;
        long long ext = (long long)L.cmax[a] - (long long)L.cmin[a] + 1;
        int b = 0;
        while ((1ll << b) < ext && b < 40) ++b;
        L.bits[a] = b;
        tb += b;
    }
    L.total_bits = tb;
    {
        // the key bits of each axis: x, y, z in turn from the least significant end,
        // each while it has bits left
        unsigned m[3] = {0u, 0u, 0u};
        int pos = 0;
        const int nb = max(L.bits[0], max(L.bits[1], L.bits[2]));
        for (int b = 0; b < nb && pos < 32; ++b)
            for (int a = 0; a < 3; ++a)
                if (b < L.bits[a] && pos < 32) m[a] |= 1u << pos++;
        for (int a = 0; a < 3; ++a) L.mask[a] = m[a];
    }
    if (tb <= c.mcap_log2) {
        L.mode = 0;
        L.nbuckets = 1 << tb;
    } else {
        L.mode = 1;
        L.nbuckets = c.mcap;
        atomicOr(&P.sc->err, SPH_EW_HASHED_GRID);
    }
    *P.layout = L;
}

__global__ void k_zero_hist(Cst c, Ptr P) {
    if (!P.ac->rebuild) return;
    int nb = P.layout->nbuckets + 2;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        P.hist[b] = 0;
}

// Bucket of every particle and its arbitrary slot in the bucket.
__global__ void __launch_bounds__(kBlock) k_keys(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || !P.ac->rebuild) return;
    const GridLayout L = *P.layout;
    const float4 p = reinterpret_cast<const float4*>(P.cur.pos)[i];
    const bool nan = isnan(p.x) || isnan(p.y) || isnan(p.z);
    int key = nan ? L.nbuckets
                  : bucket_of(cell_of(p.x, c.hc), cell_of(p.y, c.hc), cell_of(p.z, c.hc), L, c.mcap);
    P.key[i] = key;
    P.rank[i] = atomicAdd(&P.hist[key], 1);
}

// Exclusive scan of hist[0 .. nbuckets] into start[0 .. nbuckets + 1], three phases.
constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int ws[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        int s = lane < nw ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) ws[lane] = s;
    }
    __syncthreads();
    int base = wid > 0 ? ws[wid - 1] : 0;
    *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void __launch_bounds__(kBlock) k_scan_reduce(Ptr P) {
    if (!P.ac->rebuild) return;
    int nb = P.layout->nbuckets + 1;
    int ntiles = (nb + kScanTile - 1) / kScanTile;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int base = t * kScanTile + threadIdx.x * kScanItems;
        int s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) s += (base + k < nb) ? P.hist[base + k] : 0;
        s = warp_sum(s);
        __shared__ int ws[32];
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            int v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0;
            v = warp_sum(v);
            if (threadIdx.x == 0) P.bsum[t] = v;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) k_scan_bsum(Ptr P) {
    if (!P.ac->rebuild) return;
    int nb = P.layout->nbuckets + 1;
    int ntiles = (nb + kScanTile - 1) / kScanTile;
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < ntiles ? P.bsum[i] : 0;
        int tot;
        int ex = block_exclusive_scan(v, &tot);
        if (i < ntiles) P.bsum[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) k_scan_apply(Ptr P) {
    if (!P.ac->rebuild) return;
    int nb = P.layout->nbuckets + 1;
    int ntiles = (nb + kScanTile - 1) / kScanTile;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int base = t * kScanTile + threadIdx.x * kScanItems;
        int vals[kScanItems];
        int s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            vals[k] = (base + k < nb) ? P.hist[base + k] : 0;
            s += vals[k];
        }
        int tot;
        int ex = block_exclusive_scan(s, &tot) + P.bsum[t];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < nb) P.start[base + k] = ex;
            ex += vals[k];
        }
        if (t == ntiles - 1 && threadIdx.x == blockDim.x - 1) P.start[nb] = ex;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) k_scatter(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || !P.ac->rebuild) return;
    P.perm[P.start[P.key[i]] + P.rank[i]] = i;
}

// Makes the order inside each bucket the previous order (a stable counting sort): the
// particle that drew slot 0 insertion-sorts its bucket's permutation entries.
__global__ void __launch_bounds__(kBlock) k_stabilise(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || !P.ac->rebuild || P.rank[i] != 0) return;
    int k = P.key[i];
    int s = P.start[k], e = P.start[k + 1];
    for (int a = s + 1; a < e; ++a) {
        int v = P.perm[a];
        int b = a - 1;
        while (b >= s && P.perm[b] > v) { P.perm[b + 1] = P.perm[b]; --b; }
        P.perm[b + 1] = v;
    }
}

// Copies every persistent field of particle s in set A to slot d of set B.
__device__ __forceinline__ void copy_particle(const Cst& c, const SphFieldSet& A, int s, const SphFieldSet& B,
                                              int d) {
    reinterpret_cast<float4*>(B.pos)[d] = __ldg(reinterpret_cast<const float4*>(A.pos) + s);
    reinterpret_cast<float4*>(B.vel)[d] = __ldg(reinterpret_cast<const float4*>(A.vel) + s);
    reinterpret_cast<float4*>(B.x0)[d] = __ldg(reinterpret_cast<const float4*>(A.x0) + s);
    reinterpret_cast<float4*>(B.disp)[d] = __ldg(reinterpret_cast<const float4*>(A.disp) + s);
    reinterpret_cast<float4*>(B.shift)[d] = __ldg(reinterpret_cast<const float4*>(A.shift) + s);
    B.pid[d] = __ldg(A.pid + s);
    if (c.p.is_solid) {
        const float4* sa = reinterpret_cast<const float4*>(A.sdev);
        float4* sb = reinterpret_cast<float4*>(B.sdev);
        sb[2 * d] = __ldg(sa + 2 * s);
        sb[2 * d + 1] = __ldg(sa + 2 * s + 1);
        reinterpret_cast<int2*>(B.bc)[d] = __ldg(reinterpret_cast<const int2*>(A.bc) + s);
        reinterpret_cast<float4*>(B.bcdisp)[d] = __ldg(reinterpret_cast<const float4*>(A.bcdisp) + s);
        reinterpret_cast<float4*>(B.acc)[d] = __ldg(reinterpret_cast<const float4*>(A.acc) + s);
    }
}

// A build's reorder, first half: every persistent field into the other buffer set in
// the new order, with each particle's coarse cell and bucket.  The particles stay in the
// first set between builds, so steps that do not build move no field data.
__global__ void __launch_bounds__(kBlock) k_gather(Cst c, Ptr P) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= c.n || !P.ac->rebuild) return;
    const int s = P.perm[d];
    copy_particle(c, P.cur, s, P.nxt, d);
    const float4 p = __ldg(reinterpret_cast<const float4*>(P.cur.pos) + s);
    const bool nan = isnan(p.x) || isnan(p.y) || isnan(p.z);
    P.cell[d] = nan ? make_int4(0, 0, 0, -1)
                    : make_int4(cell_of(p.x, c.hc), cell_of(p.y, c.hc), cell_of(p.z, c.hc), P.key[s]);
}

// Second half: the reordered fields back into the first set, the cells of size h in the
// new order, and the build positions.
__global__ void __launch_bounds__(kBlock) k_gather_back(Cst c, Ptr P) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= c.n || !P.ac->rebuild) return;
    copy_particle(c, P.nxt, d, P.cur, d);
    const float4 p = __ldg(reinterpret_cast<const float4*>(P.nxt.pos) + d);
    const bool nan = isnan(p.x) || isnan(p.y) || isnan(p.z);
    P.fcell[d] = nan ? make_int4(0, 0, 0, -1)
                     : make_int4(cell_of(p.x, c.h), cell_of(p.y, c.h), cell_of(p.z, c.h), 0);
    P.xb[d] = p;
}

// ------------------------------------------------------------------ neighbour enumeration
// The reference bins every step in cells of size h and pairs i with j when j is binned in
// one of the 27 cells around i's cell, j != i and |x_i - x_j| < h; the y, z and corner
// mirror sweeps pair i's image with the particles binned in the y = 0 row, the z = 0 row
// and the corner column (particle_system.py:1348-1490).  Here the pairs come from
// candidate lists: every pair within h + skin at the last build, found over coarse cells
// of h + skin.  While no particle has moved more than dlim since the build, every pair of
// the reference's sweep is in the list, and the list is filtered with the reference's own
// tests: the distance, and the cells of size h (a pair whose axis separations all stay
// well inside h always passes those; one that ends up 2 cells apart in floating point
// does not).

// Candidates of the coarse cell (nx, ny, nz) in bucket b: the bucket's range, filtered on
// the cell id when the table is hashed (collisions share buckets).
template <class F>
__device__ __forceinline__ void bucket_candidates(const Ptr& P, bool hashed, int b, int nx, int ny,
                                                  int nz, F&& f) {
    const int s = __ldg(P.start + b), e = __ldg(P.start + b + 1);
    for (int j = s; j < e; ++j) {
        if (hashed) {
            const int4 cj = __ldg(P.cell + j);
            if (cj.x != nx || cj.y != ny || cj.z != nz) continue;
        }
        f(j);
    }
}

// Every candidate of the coarse table around coarse cell (bx, by, bz), radius w: the real
// sweep (self excluded) with the query point xq, then -- when xq is within hcut of the
// plane -- the mirror sweeps with xq's image over coarse rows rlo..rhi of the mirrored
// axis.  f(j, mirror, pos_j, d2) for d2 < d2cut.
template <class F>
__device__ __forceinline__ void sweep_coarse(const Cst& c, const Ptr& P, const GridLayout& L, int self_idx,
                                             F3 xq, int bx, int by, int bz, int w, int rlo, int rhi,
                                             float d2cut, float hcut, F&& f) {
    const float4* __restrict__ pos = reinterpret_cast<const float4*>(P.cur.pos);
    const bool hashed = L.mode != 0;
    auto cell_b = [&](int mir, F3 xs, int b, int nx, int ny, int nz) {
        bucket_candidates(P, hashed, b, nx, ny, nz, [&](int j) {
            if (mir == 0 && j == self_idx) return;
            const float4 pj = __ldg(pos + j);
            const float d2 = dist2_rn(xs, f3(pj));
            if (d2 < d2cut) f(j, mir, pj, d2);
        });
    };
    auto cell = [&](int mir, F3 xs, int nx, int ny, int nz) {
        const int b = bucket_of(nx, ny, nz, L, c.mcap);
        if (b >= 0) cell_b(mir, xs, b, nx, ny, nz);
    };
    if (!hashed) {
        // the real sweep over the dense table, in the same cell order: x and y dilated once
        // per row, z stepped with dilated_next along the row
        const int z_lo = max(bz - w, L.cmin[2]), z_hi = min(bz + w, L.cmax[2]);
#pragma unroll 1
        for (int o0 = -w; o0 <= w; ++o0) {
            const int nx = bx + o0;
            if (nx < L.cmin[0] || nx > L.cmax[0]) continue;
            const unsigned kx = dilate((unsigned)(nx - L.cmin[0]), L.mask[0]);
#pragma unroll 1
            for (int o1 = -w; o1 <= w; ++o1) {
                const int ny = by + o1;
                if (ny < L.cmin[1] || ny > L.cmax[1] || z_lo > z_hi) continue;
                const unsigned kxy = kx | dilate((unsigned)(ny - L.cmin[1]), L.mask[1]);
                unsigned kz = dilate((unsigned)(z_lo - L.cmin[2]), L.mask[2]);
#pragma unroll 1
                for (int nz = z_lo; nz <= z_hi; ++nz) {
                    cell_b(0, xq, (int)(kxy | kz), nx, ny, nz);
                    kz = dilated_next(kz, L.mask[2]);
                }
            }
        }
    } else {
#pragma unroll 1
        for (int o0 = -w; o0 <= w; ++o0)
#pragma unroll 1
            for (int o1 = -w; o1 <= w; ++o1)
#pragma unroll 1
                for (int o2 = -w; o2 <= w; ++o2) cell(0, xq, bx + o0, by + o1, bz + o2);
    }
    const bool my = c.mirror_y && xq.y < hcut, mz = c.mirror_z && xq.z < hcut;
    if (my) {
        const F3 xm = mirror3(1, xq);
#pragma unroll 1
        for (int o0 = -w; o0 <= w; ++o0)
#pragma unroll 1
            for (int ry = rlo; ry <= rhi; ++ry)
#pragma unroll 1
                for (int o1 = -w; o1 <= w; ++o1) cell(1, xm, bx + o0, ry, bz + o1);
    }
    if (mz) {
        const F3 xm = mirror3(2, xq);
#pragma unroll 1
        for (int o0 = -w; o0 <= w; ++o0)
#pragma unroll 1
            for (int o1 = -w; o1 <= w; ++o1)
#pragma unroll 1
                for (int rz = rlo; rz <= rhi; ++rz) cell(2, xm, bx + o0, by + o1, rz);
    }
    if (my && mz) {
        const F3 xm = mirror3(3, xq);
#pragma unroll 1
        for (int o0 = -w; o0 <= w; ++o0)
#pragma unroll 1
            for (int ry = rlo; ry <= rhi; ++ry)
#pragma unroll 1
                for (int rz = rlo; rz <= rhi; ++rz) cell(3, xm, bx + o0, ry, rz);
    }
}

// The cell test of the reference's sweeps for a pair that passed the distance test: j's
// cell (jx, jy, jz) of size h against the query cell q.  A mirror sweep takes j from the
// y = 0 row (y image), the z = 0 row (z image) or both (corner).
__device__ __forceinline__ bool sweep_cell_ok(int mir, int jx, int jy, int jz, int qx, int qy, int qz) {
    if (abs(jx - qx) > 1) return false;
    if (mir & 1) { if (jy != 0) return false; } else if (abs(jy - qy) > 1) return false;
    if (mir & 2) { if (jz != 0) return false; } else if (abs(jz - qz) > 1) return false;
    return true;
}

// Candidate counts, packed: deep entries in the low half, edge entries in the high half,
// each saturated at 0xffff.  The deep entries sit in rows 0 .. deep-1 of the neighbour
// list (untouched between builds; every step appends its accepted edge entries after
// them), the edge entries in rows 0 .. edge-1 of the candidate list.  More than Kv in all
// means the candidates overflowed and neither is used.
__device__ __forceinline__ int vl_deep(int vc) { return vc & 0xffff; }
__device__ __forceinline__ int vl_edge(int vc) { return (int)((unsigned)vc >> 16); }
__device__ __forceinline__ bool vl_overflow(const Cst& c, int vc) { return vl_deep(vc) + vl_edge(vc) > c.Kv; }

// Builds every particle's candidate list at the build's positions: the coarse 27-cell
// sweep out to h + skin, and the mirror sweeps over coarse rows -1 and 0 (a particle
// that crosses the plane later is binned in row 0 or -1 of size h).  Real entries within
// h - skin are deep: under the bound they stay within h and their cells stay adjacent, so
// every step takes them as they are (they go straight to the neighbour list).  The others
// (edge entries) are tested every step.
__global__ void __launch_bounds__(kBlock) k_vlist_build(Cst c, Ptr P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || !P.ac->rebuild) return;
    const int4 ci = P.cell[i];
    if (ci.w < 0) { P.vl_cnt[i] = 0; return; }
    const GridLayout L = *P.layout;
    const F3 xi = f3(reinterpret_cast<const float4*>(P.cur.pos)[i]);
    int nd = 0, ne = 0;
    const int n = c.n, Kv = c.Kv;
    int* __restrict__ vl = P.vl;
    int* __restrict__ nb = P.nbr;
    sweep_coarse(c, P, L, i, xi, ci.x, ci.y, ci.z, 1, -1, 0, c.d2_skin, c.h + c.skin,
                 [&](int j, int mir, float4, float d2) {
        const bool deep = mir == 0 && d2 < c.d2_deep;
        if (nd + ne < Kv) (deep ? nb + (size_t)nd * n : vl + (size_t)ne * n)[i] = j | (mir << kMirShift);
        if (deep) ++nd; else ++ne;
    });
    if (nd + ne > Kv) atomicOr(&P.sc->err, SPH_EW_CAND_OVERFLOW);
    P.vl_cnt[i] = min(nd, 0xffff) | (min(ne, 0xffff) << 16);
}

// The m stored entries of one particle's k-major list, with the next two entries in
// flight while the current pair is evaluated (the pair passes are bound by the latency
// of the dependent list -> particle gathers).
template <class F>
__device__ __forceinline__ void list_entries(const int* __restrict__ nb, size_t n, int m, F&& f) {
    int e0 = m > 0 ? __ldg(nb) : 0;
    int e1 = m > 1 ? __ldg(nb + n) : 0;
#pragma unroll 2
    for (int k = 0; k < m; ++k) {
        const int e = e0;
        e0 = e1;
        if (k + 2 < m) e1 = __ldg(nb + (size_t)(k + 2) * n);
        f(e);
    }
}
template <bool kPlain = false, class F>
__device__ __forceinline__ void list_pairs(const int* __restrict__ nb, size_t n, int m, F&& f) {
    list_entries(nb, n, m, [&](int e) { f(Shape<kPlain ? 1 : 0>::idx(e), Shape<kPlain ? 1 : 0>::mir(e)); });
}

// Entries 0 .. m-1 of a list made of pieces, with the same two-entry prefetch: at(k)
// loads entry k; f(k, entry).
template <class At, class F>
__device__ __forceinline__ void split_entries(int m, At&& at, F&& f) {
    int e0 = m > 0 ? at(0) : 0;
    int e1 = m > 1 ? at(1) : 0;
#pragma unroll 2
    for (int k = 0; k < m; ++k) {
        const int e = e0;
        e0 = e1;
        if (k + 2 < m) e1 = at(k + 2);
        f(k, e);
    }
}

// The reference's sweep against the bins of this step's start (particle_system.py:
// 1348-1490) for query point xq in cell q of size h, without the candidate lists: the
// coarse table of the last build searched wide enough for displacement D since it, each
// candidate tested for distance at the current positions and for its step-start cell.
// f(j, mirror, pos_j).
template <class F>
__device__ __forceinline__ void stale_search(const Cst& c, const Ptr& P, int i, F3 xq, int qx, int qy, int qz,
                                             float D, F&& f) {
    const int4 bi = P.cell[i];
    if (bi.w < 0) return;
    const GridLayout L = *P.layout;
    // |r| < h now => |r| < h + 2 D at the build => coarse cells at most w apart; a row of
    // size h at the plane (y in [0, h)) lies in coarse rows floor(-D / hc) .. w - 1
    const float wf = ceilf((c.h + 2.0f * D) / c.hc);
    const int w = wf <= 8.0f ? max((int)wf, 1) : 8;
    if (!(wf <= 8.0f)) atomicOr(&P.sc->err, SPH_EW_NBR_DROPPED);
    const float rf = ceilf(D / c.hc);
    const int rlo = -(rf <= 8.0f ? max((int)rf, 1) : 8);
    sweep_coarse(c, P, L, i, xq, bi.x, bi.y, bi.z, w, rlo, w - 1, c.d2_lt, c.h,
                 [&](int j, int mir, float4 pj, float) {
        const int4 fj = __ldg(P.fcell + j);
        if (fj.w >= 0 && sweep_cell_ok(mir, fj.x, fj.y, fj.z, qx, qy, qz)) f(j, mir, pj);
    });
}

// This step's neighbour list (every step; the pair passes read it): after the deep rows,
// the edge entries that pass the reference's own tests at the step-start positions --
// distance, and cells of size h (from the positions, which are the bins).  A particle
// whose candidates overflowed gets all its pairs from the stale-bin search instead; past
// K of those, the rest go in order to a run of the overflow pool (the search runs a
// second time to write it).
template <int kShape>
__global__ void SPH_BOUNDS(SPH_OCC_FILTER) k_nbr_filter(Cst c, Ptr P) {
    using S = Shape<kShape>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int vc = __ldg(P.vl_cnt + i);
    const int4 fi = P.fcell[i];
    int cnt = 0;
    const int n = c.n, K = c.K;
    int* __restrict__ nb = P.nbr;
    const float4* __restrict__ pos = reinterpret_cast<const float4*>(P.cur.pos);
    if (fi.w >= 0 && !vl_overflow(c, vc)) {
        const F3 xi = f3(pos[i]);
        const bool py = xi.y < c.h, pz = xi.z < c.h;
        // the near list: edge candidates this step rejects that lie within h + M (or whose
        // plane is within h + M), the only ones the shift can gain if particles move less
        // than M / 2 during the step
        const float m = __uint_as_float(P.ac->near_m_bits);
        const float hm = c.h + m, d2_near = hm * hm * (1.0f + 1e-5f);
        const bool ny = xi.y < hm, nz = xi.z < hm;
        int nn = 0;
        const int ne = vl_edge(vc);
        cnt = vl_deep(vc);
        // accepted entries go after the deep rows; near ones fill the list from its last
        // row down (deep + accepted + near <= the candidates <= Kv = K rows)
        list_entries(P.vl + i, (size_t)n, ne, [&](int e) {
            const int j = S::idx(e), mir = S::mir(e);
            if (mir && (((mir & 1) && !ny) || ((mir & 2) && !nz))) return;
            const float4 pj = __ldg(pos + j);
            F3 xj = f3(pj);
            if (mir) xj = mirror3(mir, xj);
            const float d2 = dist2_rn(xi, xj);
            if (!(d2 < d2_near)) return;
            if (d2 < c.d2_lt && !(mir && (((mir & 1) && !py) || ((mir & 2) && !pz))) &&
                sweep_cell_ok(mir, cell_of_fast(pj.x, c.h, c.inv_h), cell_of_fast(pj.y, c.h, c.inv_h),
                              cell_of_fast(pj.z, c.h, c.inv_h), fi.x, fi.y, fi.z)) {
                nb[(size_t)cnt * n + i] = e;
                ++cnt;
            } else {
                nb[(size_t)(K - 1 - nn) * n + i] = e;
                ++nn;
            }
        });
        P.nl_cnt[i] = nn;
    } else if (fi.w >= 0) {
        const F3 xi = f3(pos[i]);
        const float D = __uint_as_float(P.ac->d_start_bits);
        stale_search(c, P, i, xi, fi.x, fi.y, fi.z, D, [&](int j, int mir, float4) {
            if (cnt < K) nb[(size_t)cnt * n + i] = j | (mir << kMirShift);
            ++cnt;
        });
        if (cnt > K) {
            atomicOr(&P.sc->err, SPH_EW_NBR_OVERFLOW);
            const unsigned extra = (unsigned)(cnt - K);
            const unsigned base = atomicAdd(&P.ac->ovf_used, extra);
            if (base <= c.ovf_cap && extra <= c.ovf_cap - base) {
                P.ovf_off[i] = (int)base;
                int* __restrict__ run = P.ovf + base;
                int k = 0;
                stale_search(c, P, i, xi, fi.x, fi.y, fi.z, D, [&](int j, int mir, float4) {
                    if (k >= K) run[k - K] = j | (mir << kMirShift);
                    ++k;
                });
            } else {
                atomicOr(&P.sc->err, SPH_EW_NBR_DROPPED);
                cnt = K;
            }
        }
    }
    P.nbr_cnt[i] = cnt;
}

// Calls f(j, mirror, pos_j) for this step's neighbours of i, requesting the next entry's
// position while the current pair is evaluated (the passes stall on that gather).
template <bool kPlain = false, class F>
__device__ __forceinline__ void for_each_neighbour_pos(const Cst& c, const Ptr& P, int i,
                                                       const float4* __restrict__ pos, F&& f) {
    using S = Shape<kPlain ? 1 : 0>;
    const int cnt = __ldg(P.nbr_cnt + i);
    const int m = cnt < c.K ? cnt : c.K;
    const size_t n = (size_t)c.n;
    const int* __restrict__ nb = P.nbr + i;
    int e0 = m > 0 ? __ldg(nb) : 0;
    int e1 = m > 1 ? __ldg(nb + n) : 0;
    float4 p0 = m > 0 ? __ldg(pos + S::idx(e0)) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < m; ++k) {
        const int e = e0;
        const float4 pj = p0;
        e0 = e1;
        if (k + 2 < m) e1 = __ldg(nb + (size_t)(k + 2) * n);
        if (k + 1 < m) p0 = __ldg(pos + S::idx(e0));
        f(S::idx(e), S::mir(e), pj);
    }
    if (cnt > c.K)
        list_pairs<kPlain>(P.ovf + __ldg(P.ovf_off + i), 1, cnt - c.K,
                           [&](int j, int mir) { f(j, mir, __ldg(pos + j)); });
}

// Calls f(j, mirror) for this step's neighbours of i: the list, then any overflow run.
template <bool kPlain = false, class F>
__device__ __forceinline__ void for_each_neighbour(const Cst& c, const Ptr& P, int i, F&& f) {
    const int cnt = __ldg(P.nbr_cnt + i);
    list_pairs<kPlain>(P.nbr + i, (size_t)c.n, cnt < c.K ? cnt : c.K, f);
    if (cnt > c.K) list_pairs<kPlain>(P.ovf + __ldg(P.ovf_off + i), 1, cnt - c.K, f);
}


}  // namespace sph

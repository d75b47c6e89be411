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
    }
}

// update_grid_id's first half: the cell of every particle, NaN quarantine
// (particle_system.py:1224-1234, :1304-1316), and the box of occupied cells.
__global__ void __launch_bounds__(kBlock) k_cells(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff};
    int mx[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
    int offg = 0;
    double offm = 0.0;
    if (i < c.n) {
        float4 p = reinterpret_cast<const float4*>(P.cur.pos)[i];
        bool nan = isnan(p.x) || isnan(p.y) || isnan(p.z);
        int4 cl;
        cl.x = cell_of(p.x, c.h);
        cl.y = cell_of(p.y, c.h);
        cl.z = cell_of(p.z, c.h);
        cl.w = nan ? -1 : 0;
        if (nan) { cl.x = cl.y = cl.z = 0; }
        P.cell_tmp[i] = cl;
        if (nan) {
            offg = 1;
            offm = (double)P.cur.vel[4 * i + 3];
        } else {
            mn[0] = mx[0] = cl.x; mn[1] = mx[1] = cl.y; mn[2] = mx[2] = cl.z;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int v0 = mn[a], v1 = mx[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 = min(v0, __shfl_xor_sync(0xffffffffu, v0, o));
            v1 = max(v1, __shfl_xor_sync(0xffffffffu, v1, o));
        }
        if ((threadIdx.x & 31) == 0) {
            if (v0 != 0x7fffffff) atomicMin(&P.bbox[a], v0);
            if (v1 != (int)0x80000000) atomicMax(&P.bbox[3 + a], v1);
        }
    }
    unsigned any = __ballot_sync(0xffffffffu, offg != 0);
    if (any) {
        int cnt = __popc(any);
        double m = warp_sum(offm);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&P.sc->off_grid_num, cnt);
            atomicAdd(&P.sc->off_grid_mass, m);
        }
    }
}

// Chooses the table: dense Morton over the occupied box if its compact code fits the
// capacity, else the hashed table.
__global__ void k_layout(Cst c, Ptr P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
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
    int nb = P.layout->nbuckets + 2;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        P.hist[b] = 0;
}

// Bucket of every particle and its arbitrary slot in the bucket.
__global__ void __launch_bounds__(kBlock) k_keys(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const GridLayout L = *P.layout;
    int4 cl = P.cell_tmp[i];
    int key = cl.w < 0 ? L.nbuckets : bucket_of(cl.x, cl.y, cl.z, L, c.mcap);
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
    if (i >= c.n) return;
    P.perm[P.start[P.key[i]] + P.rank[i]] = i;
}

// Makes the order inside each bucket the previous order (a stable counting sort): the
// particle that drew slot 0 insertion-sorts its bucket's permutation entries.
__global__ void __launch_bounds__(kBlock) k_stabilise(Cst c, Ptr P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n || P.rank[i] != 0) return;
    int k = P.key[i];
    int s = P.start[k], e = P.start[k + 1];
    for (int a = s + 1; a < e; ++a) {
        int v = P.perm[a];
        int b = a - 1;
        while (b >= s && P.perm[b] > v) { P.perm[b + 1] = P.perm[b]; --b; }
        P.perm[b + 1] = v;
    }
}

// Gathers every persistent field into the other buffer set in the new order.
__global__ void __launch_bounds__(kBlock) k_gather(Cst c, Ptr P) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= c.n) return;
    int s = P.perm[d];
    const SphFieldSet& A = P.cur;
    const SphFieldSet& B = P.nxt;
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
    int4 cl = P.cell_tmp[s];
    cl.w = cl.w < 0 ? -1 : P.key[s];
    P.cell[d] = cl;
}

// ------------------------------------------------------------------ neighbour enumeration
// Candidates of cell (nx, ny, nz) in bucket b: the bucket's range, filtered on the cell
// id when the table is hashed (collisions share buckets).
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

// The y, z and corner mirror sweeps of a particle at xi in cell (cx, cy, cz)
// (particle_system.py:1442-1490): the image of xi against the cells of the y = 0 row,
// the z = 0 row and the corner column; a particle pairs with its own image too.  A sweep
// runs when xi is within hcut of its plane; f(j, mirror, pos_j, d2) gets every candidate
// with d2 < d2cut (the neighbour test uses hcut = h, d2cut = the |r| < h threshold).
template <class F>
__device__ __forceinline__ void enumerate_mirrors_cut(const Cst& c, const Ptr& P, const GridLayout& L,
                                                      F3 xi, int cx, int cy, int cz, float d2cut,
                                                      float hcut, F&& f) {
    const float4* __restrict__ pos = reinterpret_cast<const float4*>(P.cur.pos);
    const bool hashed = L.mode != 0;
    if (c.mirror_y && xi.y < hcut) {
        const F3 xm = mirror3(1, xi);
#pragma unroll 1
        for (int o0 = -1; o0 <= 1; ++o0)
#pragma unroll 1
            for (int o1 = -1; o1 <= 1; ++o1) {
                const int nx = cx + o0, ny = 0, nz = cz + o1;
                const int b = bucket_of(nx, ny, nz, L, c.mcap);
                if (b < 0) continue;
                bucket_candidates(P, hashed, b, nx, ny, nz, [&](int j) {
                    const float4 pj = __ldg(pos + j);
                    const float d2 = dist2_rn(xm, f3(pj));
                    if (d2 < d2cut) f(j, 1, pj, d2);
                });
            }
    }
    if (c.mirror_z && xi.z < hcut) {
        const F3 xm = mirror3(2, xi);
#pragma unroll 1
        for (int o0 = -1; o0 <= 1; ++o0)
#pragma unroll 1
            for (int o1 = -1; o1 <= 1; ++o1) {
                const int nx = cx + o0, ny = cy + o1, nz = 0;
                const int b = bucket_of(nx, ny, nz, L, c.mcap);
                if (b < 0) continue;
                bucket_candidates(P, hashed, b, nx, ny, nz, [&](int j) {
                    const float4 pj = __ldg(pos + j);
                    const float d2 = dist2_rn(xm, f3(pj));
                    if (d2 < d2cut) f(j, 2, pj, d2);
                });
            }
    }
    if (c.mirror_y && c.mirror_z && xi.y < hcut && xi.z < hcut) {
        const F3 xm = mirror3(3, xi);
#pragma unroll 1
        for (int o0 = -1; o0 <= 1; ++o0) {
            const int nx = cx + o0, ny = 0, nz = 0;
            const int b = bucket_of(nx, ny, nz, L, c.mcap);
            if (b < 0) continue;
            bucket_candidates(P, hashed, b, nx, ny, nz, [&](int j) {
                const float4 pj = __ldg(pos + j);
                const float d2 = dist2_rn(xm, f3(pj));
                if (d2 < d2cut) f(j, 3, pj, d2);
            });
        }
    }
}

// Every candidate of a particle at xi whose centre cell is (cx, cy, cz) with d2 < d2cut,
// in the reference's order: the 27 offsets with the last index fastest, then the y, z and
// corner mirror sweeps (particle_system.py:1393-1490).  `self_idx` is excluded from the
// real sweep only.  Positions are read from `pos` (live positions).
template <class F>
__device__ __forceinline__ void enumerate_cut(const Cst& c, const Ptr& P, const GridLayout& L, int self_idx,
                                              F3 xi, int cx, int cy, int cz, float d2cut, float hcut,
                                              F&& f) {
    const float4* __restrict__ pos = reinterpret_cast<const float4*>(P.cur.pos);
    const bool hashed = L.mode != 0;
#pragma unroll 1
    for (int o0 = -1; o0 <= 1; ++o0)
#pragma unroll 1
        for (int o1 = -1; o1 <= 1; ++o1)
#pragma unroll 1
            for (int o2 = -1; o2 <= 1; ++o2) {
                const int nx = cx + o0, ny = cy + o1, nz = cz + o2;
                const int b = bucket_of(nx, ny, nz, L, c.mcap);
                if (b < 0) continue;
                bucket_candidates(P, hashed, b, nx, ny, nz, [&](int j) {
                    if (j == self_idx) return;
                    const float4 pj = __ldg(pos + j);
                    const float d2 = dist2_rn(xi, f3(pj));
                    if (d2 < d2cut) f(j, 0, pj, d2);
                });
            }
    enumerate_mirrors_cut(c, P, L, xi, cx, cy, cz, d2cut, hcut, f);
}

// The neighbours proper: f(j, mirror, pos_j) for |r| < h (bit-exact against the reference).
template <class F>
__device__ __forceinline__ void enumerate_neighbours(const Cst& c, const Ptr& P, const GridLayout& L,
                                                     int self_idx, F3 xi, int cx, int cy, int cz,
                                                     F&& f) {
    enumerate_cut(c, P, L, self_idx, xi, cx, cy, cz, c.d2_lt, c.h,
                  [&](int j, int mir, float4 pj, float) { f(j, mir, pj); });
}

// Builds the neighbour list of every particle from the positions the cells were binned
// at (before advect the live and the binned cell coincide).  Entries beyond K are not
// stored; the count is the true count and the pair passes recover the rest by a direct
// search (for_each_neighbour below).
__global__ void __launch_bounds__(kBlock) k_nbr_build(Cst c, Ptr P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const GridLayout L = *P.layout;
    const int4 ci = P.cell[i];
    if (ci.w < 0) {
        P.nbr_cnt[i] = 0;
        if (c.pst_skin) P.shell_cnt[i] = 0;
        return;
    }
    const F3 xi = f3(reinterpret_cast<const float4*>(P.cur.pos)[i]);
    int cnt = 0;
    const int n = c.n, K = c.K;
    int* __restrict__ nb = P.nbr;
    if (c.pst_skin) {
        // the same sweep out to h + skin: neighbours proper go to the list (in the same
        // order as without the shell), the rest of the shell to the shift's candidates
        int scnt = 0;
        const int Ks = c.Ks;
        int* __restrict__ sb = P.shell;
        enumerate_cut(c, P, L, i, xi, ci.x, ci.y, ci.z, c.d2_skin, c.h + c.skin,
                      [&](int j, int mir, float4, float d2) {
            const bool plane = mir == 0 || (((mir & 1) == 0 || xi.y < c.h) && ((mir & 2) == 0 || xi.z < c.h));
            const int e = j | (d2 < c.d2_deep ? 0 : kRimBit) | (mir << kMirShift);
            if (d2 < c.d2_lt && plane) {
                if (cnt < K) nb[(size_t)cnt * n + i] = e;
                ++cnt;
            } else {
                if (scnt < Ks) sb[(size_t)scnt * n + i] = e;
                ++scnt;
            }
        });
        P.shell_cnt[i] = scnt;
    } else {
        enumerate_neighbours(c, P, L, i, xi, ci.x, ci.y, ci.z, [&](int j, int mir, float4) {
            if (cnt < K) nb[(size_t)cnt * n + i] = j | (mir << kMirShift);
            ++cnt;
        });
    }
    if (cnt > K) atomicOr(&P.sc->err, SPH_EW_NBR_OVERFLOW);
    P.nbr_cnt[i] = cnt;
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
template <class F>
__device__ __forceinline__ void list_pairs(const int* __restrict__ nb, size_t n, int m, F&& f) {
    list_entries(nb, n, m, [&](int e) { f(e & kIdxMask, (int)((unsigned)e >> kMirShift)); });
}

// Calls f(j, mirror) for the stored neighbours of i, then for any beyond the list's
// capacity by re-running the search (same order, first K skipped).
template <class F>
__device__ __forceinline__ void for_each_neighbour(const Cst& c, const Ptr& P, int i, F&& f) {
    const int cnt = __ldg(P.nbr_cnt + i);
    const int m = cnt < c.K ? cnt : c.K;
    list_pairs(P.nbr + i, (size_t)c.n, m, f);
    if (cnt > c.K) {
        const GridLayout L = *P.layout;
        int4 ci = P.cell[i];
        F3 xi = f3(reinterpret_cast<const float4*>(P.cur.pos)[i]);
        int k = 0;
        enumerate_neighbours(c, P, L, i, xi, ci.x, ci.y, ci.z, [&](int j, int mir, float4) {
            if (k >= c.K) f(j, mir);
            ++k;
        });
    }
}

}  // namespace sph

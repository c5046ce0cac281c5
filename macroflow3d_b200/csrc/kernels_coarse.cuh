// kernels_coarse.cuh -- the coarse end of the V-cycle in one thread-block cluster, in FP64.
//
// Same cycle as the one-CTA tail (kernels_tail.cuh) and v_cycle_recursive of the reference
// (src/multigrid/cycle/v_cycle.cu:36-74): in-place GSRB (red = (i+j+k) even, then black;
// gsrb_3d.cu:368-576), residual + 8-child restriction, the coarsest level's sweeps,
// parent-injection prolongation and post-smoothing, with the per-cell weights of
// tail_weights_kernel (x_c = sum_f w_f x_f - bd b_c, r_c = q (x_c - x_GS)).
//
// Everything a level needs stays in shared memory for the whole launch: x with a one-cell
// ghost layer, and b and the eight weights of every cell, stored by colour (the cells of one
// colour of a slab are consecutive, in the order a half-sweep visits them, so a warp reads
// consecutive words).  Levels are placed in two ways:
//   - "clustered" levels (more than CT_LOCAL_MAX cells) are cut into z slabs, one per CTA of
//     the cluster.  The slabs are nested: the planes of a CTA on level l are the children of
//     its planes on level l+1, so restriction and prolongation stay inside the CTA.  A relaxed
//     cell on the first or last plane of a slab is also stored into the neighbouring CTA's
//     ghost plane (distributed shared memory), and a cell on a periodic x / y face into the
//     ghost column or row across the grid, so no copy step is needed; every phase ends with
//     one cluster barrier (release / acquire).
//   - "local" levels (at most CT_LOCAL_MAX cells) run in CTA 0 alone, with CTA barriers: the
//     last clustered restriction writes their right-hand side into CTA 0's shared memory, and
//     the first clustered prolongation reads their correction from there.  The coarsest level,
//     when local and at most 32 cells of each colour, runs in one warp with warp barriers;
//     when local and at most CT_MAP_MAX cells, it is x = M b with its sweeps' map M.
// A periodic axis must have an even count on every level here (a cell and its ghost copy
// then have different colours, so no relaxation reads a value being written).
#pragma once
#include <cstdint>

#include "kernels_tail.cuh"

namespace mf3d {

constexpr int CT_NT = 512;
constexpr int CT_MAX_CLUSTER = 8;   // portable cluster size
constexpr int CT_LOCAL_MAX = 1024;  // levels of at most this many cells run in CTA 0 alone
constexpr int CT_MAX_CELLS = 32768; // largest level the cluster takes (shared memory decides)

// n / d by one 64-bit multiply and a shift: m = ceil(2^40 / d) gives floor(n / d) exactly
// whenever n * d < 2^40 (the error n (m d - 2^40) / (d 2^40) stays below 1 / d).
struct FDiv {
    unsigned long long m;
    int d;
};
inline FDiv make_fdiv(int d) {
    FDiv f;
    f.d = d;
    f.m = ((1ull << 40) + (unsigned long long)d - 1) / (unsigned long long)d;
    return f;
}
__device__ __forceinline__ int fdv(int n, const FDiv& f) {
    return (int)(((unsigned long long)(unsigned)n * f.m) >> 40);
}

struct CLevel {
    int nx, ny, nz, n;
    int per_x, per_y, per_z;
    int clustered; // z slabs over the cluster, else CTA 0 holds the level
    int shift;     // clustered: planes of this level per partition unit, as a power of two
    int pmax;      // planes of the largest slab (clustered) or nz (local)
    int hcap;      // cells of one colour a slab can hold: hx * ny * pmax
    int xoff;      // x (ghost-padded slab) in shared memory (doubles)
    int boff;      // b by colour: [2 hcap]
    int woff;      // weights by colour: [8][2 hcap]
    FDiv fhx, fnx, fny; // (nx + 1) / 2, nx, ny
    const double* w;    // 8 n weights in global memory: w_-x, w_+x, w_-y, w_+y, w_-z, w_+z, bd, q
};

struct CoarseArgs {
    int nlev;  // levels from the first coarse level to the coarsest
    int ncl;   // the first ncl of them are clustered
    int pre, post, coarse_iters;
    int units; // partition units: planes of the level below the last clustered one (or of that
               // level itself when it is the coarsest); CTA r owns units [r U / R, (r+1) U / R)
    // The coarsest level's coarse_iters sweeps from x = 0 are a linear map of its b: when it is
    // local and small, M (n rows in cell order, 2 hcap columns in b's colour order) holds that
    // map (coarse_map_kernel) and the level is solved as x = M b, M staged at moff.
    const double* M;
    int moff;
    CLevel L[TAIL2_MAX_LEVELS];
};
constexpr int CT_MAP_MAX = 64; // coarsest levels of at most this many cells use the map

__device__ __forceinline__ unsigned ct_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned ct_nranks() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// every thread of every CTA of the cluster; shared-memory writes before it (local or remote)
// are visible to every thread after it
__device__ __forceinline__ void ct_cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// the same shared-memory location in CTA `rank` of the cluster, as a generic address (plain
// loads and stores reach it; the cluster barrier's release / acquire orders them)
__device__ __forceinline__ double* ct_remote(const double* p, unsigned rank) {
    unsigned long long r;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"((unsigned long long)p), "r"(rank));
    return reinterpret_cast<double*>(r);
}

// The planes [z0, z1) of one level that a CTA holds, and where its neighbours' ghost planes are.
struct Slab {
    int z0, z1;
    int has_prev, has_next; // a neighbour below / above that keeps a ghost copy of the first /
                            // last plane (the periodic wrap included)
    int prev_np;            // planes of the neighbour below
    double* prev_x;         // the neighbours' x of this level (generic addresses)
    double* next_x;
};

__device__ __forceinline__ Slab ct_slab(const CoarseArgs& a, int l, unsigned rank, unsigned nr, double* sm) {
    const CLevel& L = a.L[l];
    Slab S;
    const double* xs = sm + L.xoff;
    if (!L.clustered) {
        S.z0 = 0;
        S.z1 = L.nz;
        S.has_prev = S.has_next = L.per_z;
        S.prev_np = L.nz;
        S.prev_x = S.next_x = ct_remote(xs, rank);
        return S;
    }
    const int U = a.units, R = (int)nr, r = (int)rank;
    S.z0 = (r * U / R) << L.shift;
    S.z1 = ((r + 1) * U / R) << L.shift;
    const int rp = r > 0 ? r - 1 : R - 1, rn = r + 1 < R ? r + 1 : 0;
    S.has_prev = r > 0 || L.per_z;
    S.has_next = r + 1 < R || L.per_z;
    S.prev_np = (((rp + 1) * U / R) - (rp * U / R)) << L.shift;
    S.prev_x = ct_remote(xs, (unsigned)rp);
    S.next_x = ct_remote(xs, (unsigned)rn);
    return S;
}

// padded slab index of x
__device__ __forceinline__ int ct_P(const CLevel& L, const Slab& S, int i, int j, int k) {
    return (i + 1) + (L.nx + 2) * ((j + 1) + (L.ny + 2) * (k - S.z0 + 1));
}
// colour-ordered slab index of b and the weights: colour (i+j+k) & 1, then the half-sweep
// item (i / 2) + hx * (j + ny * (k - z0))
__device__ __forceinline__ int ct_Q(const CLevel& L, const Slab& S, int i, int j, int k) {
    return ((i + j + k) & 1) * L.hcap + (i >> 1) + L.fhx.d * (j + L.ny * (k - S.z0));
}

// Gauss-Seidel value of a cell from the weights and b in shared memory (the expression of
// tl_gs: w_-x x_-x + w_+x x_+x + w_-y x_-y + w_+y x_+y + w_-z x_-z + w_+z x_+z - bd b)
__device__ __forceinline__ double ct_gs(const CLevel& L, const double* sm, const double* x, int P, int Q) {
    const int sy = L.nx + 2, sz = sy * (L.ny + 2), wc = 2 * L.hcap;
    const double* w = sm + L.woff + Q;
    return w[0] * x[P - 1] + w[wc] * x[P + 1] + w[2 * wc] * x[P - sy] + w[3 * wc] * x[P + sy] +
           w[4 * wc] * x[P - sz] + w[5 * wc] * x[P + sz] - w[6 * wc] * sm[L.boff + Q];
}

// x(i, j, k) = v, and every ghost copy of it: across a periodic x / y face in this slab, and
// in the neighbouring slab's ghost plane
__device__ __forceinline__ void ct_set(const CLevel& L, const Slab& S, double* x, int i, int j, int k, int P,
                                       double v) {
    x[P] = v;
    const int sy = L.nx + 2, sz = sy * (L.ny + 2);
    if (L.per_x) {
        if (i == 0) x[P + L.nx] = v;
        if (i == L.nx - 1) x[P - L.nx] = v;
    }
    if (L.per_y) {
        if (j == 0) x[P + L.ny * sy] = v;
        if (j == L.ny - 1) x[P - L.ny * sy] = v;
    }
    const int p2 = (i + 1) + sy * (j + 1);
    if (k == S.z0 && S.has_prev) S.prev_x[p2 + sz * (S.prev_np + 1)] = v;
    if (k == S.z1 - 1 && S.has_next) S.next_x[p2] = v;
}

// one colour of a GSRB sweep over the slab (col 0: red) by threads [0, nthr)
__device__ __forceinline__ void ct_half(const CLevel& L, const Slab& S, double* sm, double* x, int col, int tid,
                                        int nthr) {
    const int hx = L.fhx.d;
    const int items = hx * L.ny * (S.z1 - S.z0);
    for (int e = tid; e < items; e += nthr) {
        const int row = fdv(e, L.fhx), m = e - row * hx;
        const int kk = fdv(row, L.fny), j = row - kk * L.ny;
        const int k = S.z0 + kk;
        const int i = 2 * m + ((j + k + col) & 1);
        if (i >= L.nx) continue;
        const int P = ct_P(L, S, i, j, k);
        ct_set(L, S, x, i, j, k, P, ct_gs(L, sm, x, P, col * L.hcap + e));
    }
}

constexpr int CT_SYNC_CTA = 0, CT_SYNC_CLUSTER = 1, CT_SYNC_WARP = 2;
__device__ __forceinline__ void ct_sync(int mode) {
    if (mode == CT_SYNC_CLUSTER)
        ct_cluster_sync();
    else if (mode == CT_SYNC_CTA)
        __syncthreads();
    else
        __syncwarp();
}

// `sweeps` GSRB sweeps of one level by threads [0, nthr), each colour followed by a barrier
__device__ __forceinline__ void ct_sweeps(const CLevel& L, const Slab& S, double* sm, double* x, int sweeps, int sync,
                                          int tid, int nthr) {
    for (int sw = 0; sw < sweeps; ++sw)
        for (int col = 0; col < 2; ++col) {
            ct_half(L, S, sm, x, col, tid, nthr);
            ct_sync(sync);
        }
}

// b of the coarse cells whose children are in this slab, into bc (b of the coarse level by
// colour): this CTA's coarse slab (Sc its slab) or CTA 0's b of a local coarse level
__device__ __forceinline__ void ct_restrict(const CLevel& Lf, const Slab& Sf, double* sm, const double* x,
                                            const CLevel& Lc, const Slab& Sc, double* bc, int tid, int nthr) {
    const int ncx = Lc.nx, ncy = Lc.ny;
    const int Kc0 = Sf.z0 / 2;
    const int items = ncx * ncy * ((Sf.z1 - Sf.z0) / 2);
    for (int e = tid; e < items; e += nthr) {
        const int row = fdv(e, Lc.fnx), I = e - row * ncx;
        const int KK = fdv(row, Lc.fny), J = row - KK * ncy;
        const int K = Kc0 + KK;
        double acc = 0.0;
        // children in the order (000,100,010,110,001,101,011,111), restrict_3d.cu:38-49
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dxx = 0; dxx < 2; ++dxx) {
                    const int i = 2 * I + dxx, j = 2 * J + dy, k = 2 * K + dz;
                    const int P = ct_P(Lf, Sf, i, j, k), Q = ct_Q(Lf, Sf, i, j, k);
                    const double xg = ct_gs(Lf, sm, x, P, Q);
                    acc += sm[Lf.woff + 7 * 2 * Lf.hcap + Q] * (x[P] - xg);
                }
        bc[ct_Q(Lc, Sc, I, J, K)] = acc / 8.0;
    }
}

// x += parent's correction for the cells of this slab; xc is the coarse level's x, this CTA's
// slab (first plane kb = z0 / 2) or CTA 0's local level (kb = 0)
__device__ __forceinline__ void ct_prolong(const CLevel& Lf, const Slab& Sf, double* x, const CLevel& Lc,
                                           const double* xc, int kb, int tid, int nthr) {
    const int items = Lf.nx * Lf.ny * (Sf.z1 - Sf.z0);
    const int syc = Lc.nx + 2, szc = syc * (Lc.ny + 2);
    for (int e = tid; e < items; e += nthr) {
        const int row = fdv(e, Lf.fnx), i = e - row * Lf.nx;
        const int kk = fdv(row, Lf.fny), j = row - kk * Lf.ny;
        const int k = Sf.z0 + kk;
        const int P = ct_P(Lf, Sf, i, j, k);
        const int Pc = ((i >> 1) + 1) + syc * ((j >> 1) + 1) + szc * ((k >> 1) - kb + 1);
        ct_set(Lf, Sf, x, i, j, k, P, x[P] + xc[Pc]);
    }
}

// Column q of the coarsest level's map: `iters` GSRB sweeps (tl_smooth, the one-CTA tail's
// sweep) from x = 0 with b = the unit vector of the cell whose colour-ordered index is q.
// One CTA per cell; M (n x 2 hcap, zero-filled by the caller) receives x in cell order.
__global__ void __launch_bounds__(64) coarse_map_kernel(const TailLevel L, const CLevel Lc, int iters,
                                                        double* __restrict__ M) {
    __shared__ double x[1024], b[CT_MAP_MAX];
    const int tid = threadIdx.x, j = blockIdx.x;
    const int np = (L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    for (int e = tid; e < np; e += 64) x[e] = 0.0;
    for (int e = tid; e < L.n; e += 64) b[e] = e == j ? 1.0 : 0.0;
    __syncthreads();
    tl_smooth(L, x, b, iters, tid, 64, false);
    const int ji = j % L.nx, jj = (j / L.nx) % L.ny, jk = j / (L.nx * L.ny);
    const int q = ((ji + jj + jk) & 1) * Lc.hcap + (ji >> 1) + Lc.fhx.d * (jj + L.ny * jk);
    for (int c = tid; c < L.n; c += 64) {
        const int i = c % L.nx, jy = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
        M[(size_t)c * 2 * Lc.hcap + q] = x[tl_pad(L, i, jy, k)];
    }
}

template <class TI, class TO>
__global__ void __launch_bounds__(CT_NT, 1) coarse_cluster_kernel(const __grid_constant__ CoarseArgs a,
                                                                  const TI* __restrict__ b_in, TO* __restrict__ x_out) {
    extern __shared__ __align__(16) double sm[];
    const int tid = threadIdx.x;
    const unsigned rank = ct_rank(), nr = ct_nranks();
    const bool cta0 = rank == 0;
    // ---- every level this CTA holds: x = 0 (ghosts included), its cells' weights; b of the
    // first level ----
    for (int l = 0; l < a.nlev; ++l) {
        const CLevel& L = a.L[l];
        if (!L.clustered && !cta0) continue;
        const int np = (L.nx + 2) * (L.ny + 2) * (L.pmax + 2);
        for (int e = tid; e < np; e += CT_NT) sm[L.xoff + e] = 0.0;
        for (int e = tid; e < 2 * L.hcap; e += CT_NT) sm[L.boff + e] = 0.0; // slots of no cell stay 0
    }
    __syncthreads();
    for (int l = 0; l < a.nlev; ++l) {
        const CLevel& L = a.L[l];
        if (!L.clustered && !cta0) continue;
        const Slab S = ct_slab(a, l, rank, nr, sm);
        const int plane = L.nx * L.ny, cnt = (S.z1 - S.z0) * plane, off = S.z0 * plane, wc = 2 * L.hcap;
        for (int e = tid; e < cnt; e += CT_NT) {
            const int row = fdv(e, L.fnx), i = e - row * L.nx;
            const int kk = fdv(row, L.fny), j = row - kk * L.ny;
            const int Q = ct_Q(L, S, i, j, S.z0 + kk);
#pragma unroll
            for (int f = 0; f < 8; ++f) sm[L.woff + f * wc + Q] = __ldg(L.w + (size_t)f * L.n + off + e);
            if (l == 0) sm[L.boff + Q] = (double)b_in[off + e];
        }
    }
    if (a.M && cta0) {
        const CLevel& L = a.L[a.nlev - 1];
        const int cnt = L.n * 2 * L.hcap;
        for (int e = tid; e < cnt; e += CT_NT) sm[a.moff + e] = __ldg(a.M + e);
    }
    ct_cluster_sync();
    // ---- down: pre-smoothing, residual + restriction; then the coarsest level ----
    // A clustered level runs on every CTA with cluster barriers, a local one on CTA 0 with CTA
    // barriers (the other CTAs go on to the next cluster barrier).
    for (int l = 0; l < a.nlev; ++l) {
        const CLevel& L = a.L[l];
        const bool cl = L.clustered != 0;
        const bool coarsest = l + 1 == a.nlev;
        if (cl || cta0) {
            const Slab S = ct_slab(a, l, rank, nr, sm);
            double* x = sm + L.xoff;
            if (coarsest && a.M) {
                // x = M b (CTA 0, local level): one cell per thread, b's colour order
                const int nc = 2 * L.hcap;
                if (tid < L.n) {
                    const double* m = sm + a.moff + tid * nc;
                    const double* bb = sm + L.boff;
                    double acc0 = 0.0, acc1 = 0.0;
                    for (int q = 0; q < nc; q += 2) {
                        acc0 += m[q] * bb[q];
                        acc1 += m[q + 1] * bb[q + 1];
                    }
                    const int row = fdv(tid, L.fnx), i = tid - row * L.nx;
                    const int k = fdv(row, L.fny), j = row - k * L.ny;
                    ct_set(L, S, x, i, j, k, ct_P(L, S, i, j, k), acc0 + acc1);
                }
                __syncthreads();
            } else {
                // the coarsest level with at most 32 cells of each colour: one warp, warp barriers
                const bool warp = coarsest && !cl && L.fhx.d * L.ny * L.nz <= 32;
                if (!warp || tid < 32)
                    ct_sweeps(L, S, sm, x, coarsest ? a.coarse_iters : a.pre,
                              cl ? CT_SYNC_CLUSTER : (warp ? CT_SYNC_WARP : CT_SYNC_CTA), tid, warp ? 32 : CT_NT);
                if (warp) __syncthreads();
            }
            if (!coarsest) {
                const CLevel& Lc = a.L[l + 1];
                const Slab Sc = ct_slab(a, l + 1, rank, nr, sm);
                const bool to0 = cl && !Lc.clustered; // into CTA 0's local level
                ct_restrict(L, S, sm, x, Lc, Sc, to0 ? ct_remote(sm + Lc.boff, 0) : sm + Lc.boff, tid, CT_NT);
                ct_sync(cl ? CT_SYNC_CLUSTER : CT_SYNC_CTA);
            }
        }
    }
    // ---- up: prolongation + post-smoothing ----
    for (int l = a.nlev - 2; l >= 0; --l) {
        const CLevel& L = a.L[l];
        const CLevel& Lc = a.L[l + 1];
        const bool cl = L.clustered != 0;
        if (cl && !Lc.clustered) ct_cluster_sync(); // CTA 0's local levels are done
        if (cl || cta0) {
            const Slab S = ct_slab(a, l, rank, nr, sm);
            double* x = sm + L.xoff;
            const bool from0 = cl && !Lc.clustered; // from CTA 0's local level
            ct_prolong(L, S, x, Lc, from0 ? ct_remote(sm + Lc.xoff, 0) : sm + Lc.xoff, Lc.clustered ? S.z0 / 2 : 0,
                       tid, CT_NT);
            ct_sync(cl ? CT_SYNC_CLUSTER : CT_SYNC_CTA);
            ct_sweeps(L, S, sm, x, a.post, cl ? CT_SYNC_CLUSTER : CT_SYNC_CTA, tid, CT_NT);
        }
    }
    // ---- the first level's correction ----
    {
        const CLevel& L = a.L[0];
        if (L.clustered || cta0) {
            const Slab S = ct_slab(a, 0, rank, nr, sm);
            const int cnt = L.nx * L.ny * (S.z1 - S.z0);
            for (int e = tid; e < cnt; e += CT_NT) {
                const int row = fdv(e, L.fnx), i = e - row * L.nx;
                const int kk = fdv(row, L.fny), j = row - kk * L.ny;
                const int k = S.z0 + kk;
                x_out[i + L.nx * (j + L.ny * k)] = (TO)sm[L.xoff + ct_P(L, S, i, j, k)];
            }
        }
    }
    // no CTA leaves while another may still store into its shared memory
    ct_cluster_sync();
}

} // namespace mf3d

// mf3d_device.cuh -- device-side data layout and helpers shared by every kernel.
//
// Operator storage ("plus-face form").  The reference recomputes the harmonic mean
// K_f = 2/(1/K_c + 1/K_n) for every face in every kernel
// (src/multigrid/common/mg_conventions.cuh:133, bc_stencil_helpers.cuh:33-271).  Here each
// level stores every face coefficient once:
//   cx[c]  couples cell c with its +x neighbour; at i = nx-1 it holds the xmax boundary
//          coefficient (Dirichlet 2K_c, Neumann 0, periodic harmonic mean with cell 0);
//   bxm[j + ny*k] is the xmin boundary coefficient of cell (0,j,k) (Dirichlet 2K_c,
//          Neumann 0; unused when x is periodic, where cx[nx-1] is the wrap face);
// and likewise cy/bym (plane nx*nz, index i + nx*k) and cz/bzm (plane nx*ny, index i + nx*j).
// The diagonal is the sum of the six face coefficients (doubled at cell 0 when pinned), and a
// boundary neighbour value is 0 unless the axis is periodic.  This is the reference's
// discretisation (src/multigrid/common/mg_conventions.cuh:44-110) with the divisions hoisted
// out of the sweeps.
//
// Coefficients may be stored as double, float or bf16; a bf16 level keeps its coefficients
// scaled by 2^-s and folds 2^s into the level's dx2 / inv_dx2 (the scale cancels in the
// smoother and re-appears in the residual).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mf3d {

enum : int { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_PERIODIC = 2 };

__host__ __device__ __forceinline__ double ld_as_double(double v) { return v; }
__host__ __device__ __forceinline__ double ld_as_double(float v) { return (double)v; }
__device__ __forceinline__ double ld_as_double(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
__device__ __forceinline__ float ld_as_float(double v) { return (float)v; }
__device__ __forceinline__ float ld_as_float(float v) { return v; }
__device__ __forceinline__ float ld_as_float(__nv_bfloat16 v) { return __bfloat162float(v); }

// value of a stored coefficient (double, float or bf16) as the compute type T
template <class T> __device__ __forceinline__ T ld_as_float_or_double(double v) { return (T)v; }
template <class T> __device__ __forceinline__ T ld_as_float_or_double(float v) { return (T)v; }
template <class T> __device__ __forceinline__ T ld_as_float_or_double(__nv_bfloat16 v) {
    return (T)__bfloat162float(v);
}

template <class T> __device__ __forceinline__ T cvt(double v);
template <> __device__ __forceinline__ double cvt<double>(double v) { return v; }
template <> __device__ __forceinline__ float cvt<float>(double v) { return (float)v; }

template <class T, class S> __device__ __forceinline__ T load_as(const S* p, size_t i);
template <> __device__ __forceinline__ double load_as<double, double>(const double* p, size_t i) { return __ldg(p + i); }
template <> __device__ __forceinline__ double load_as<double, float>(const float* p, size_t i) { return (double)__ldg(p + i); }
template <> __device__ __forceinline__ float load_as<float, float>(const float* p, size_t i) { return __ldg(p + i); }
template <> __device__ __forceinline__ float load_as<float, double>(const double* p, size_t i) { return (float)__ldg(p + i); }
template <> __device__ __forceinline__ double load_as<double, __nv_bfloat16>(const __nv_bfloat16* p, size_t i) {
    return (double)__bfloat162float(p[i]);
}
template <> __device__ __forceinline__ float load_as<float, __nv_bfloat16>(const __nv_bfloat16* p, size_t i) {
    return __bfloat162float(p[i]);
}

// One multigrid level's operator, as seen by the kernels.
template <class TC> struct LevelOp {
    int nx, ny, nz;
    int per_x, per_y, per_z; // periodic axes
    int pin;                 // diagonal doubling at cell 0
    double dx2;              // dx^2 (times 2^-s for scaled bf16 coefficients)
    double inv_dx2;          // 1/dx^2 (times 2^s)
    const TC* cx;
    const TC* cy;
    const TC* cz;
    const TC* bxm; // ny*nz
    const TC* bym; // nx*nz
    const TC* bzm; // nx*ny
};

// Wrap a coordinate that may lie one or more cells outside [0,n); returns -1 if the cell is
// outside a non-periodic axis.
__device__ __forceinline__ int wrap_or_out(int i, int n, int periodic) {
    if (i >= 0 && i < n) return i;
    if (!periodic) return -1;
    i %= n;
    return i < 0 ? i + n : i;
}

// The six face coefficients of cell (i,j,k) (all coordinates inside the domain), in the
// order -x,+x,-y,+y,-z,+z, and the diagonal.
template <class T, class TC>
__device__ __forceinline__ void cell_coefs(const LevelOp<TC>& L, int i, int j, int k, size_t c,
                                           T& cxm, T& cxp, T& cym, T& cyp, T& czm, T& czp) {
    const size_t nxy = (size_t)L.nx * L.ny;
    cxp = load_as<T>(L.cx, c);
    cyp = load_as<T>(L.cy, c);
    czp = load_as<T>(L.cz, c);
    if (i > 0) cxm = load_as<T>(L.cx, c - 1);
    else cxm = L.per_x ? load_as<T>(L.cx, c + (L.nx - 1)) : load_as<T>(L.bxm, (size_t)j + (size_t)L.ny * k);
    if (j > 0) cym = load_as<T>(L.cy, c - L.nx);
    else cym = L.per_y ? load_as<T>(L.cy, c + (size_t)(L.ny - 1) * L.nx) : load_as<T>(L.bym, (size_t)i + (size_t)L.nx * k);
    if (k > 0) czm = load_as<T>(L.cz, c - nxy);
    else czm = L.per_z ? load_as<T>(L.cz, c + (size_t)(L.nz - 1) * nxy) : load_as<T>(L.bzm, (size_t)i + (size_t)L.nx * j);
}

// ---------------------------------------------------------------------------------------
// Deterministic grid-wide sum: every block writes its partial, the last block to arrive
// adds the partials in index order.  `ticket` must start at 0; it is reset by the last block.
// ---------------------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red /* NT/32 doubles */) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = tid >> 5, l = tid & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (tid == 0) {
        for (int i = 0; i < NT / 32; ++i) s += red[i];
    }
    __syncthreads();
    return s; // valid on thread 0
}

// Returns true on thread 0 of the last block to finish; `out` then holds the grid sums.
// Blocks may be 1-, 2- or 3-D; NT is the number of threads per block.  `bid` is the block's
// index among the `nblocks` that share the partials (the hardware block index by default; a
// virtual block of one realisation in the batched kernels).
template <int NT, int NV>
__device__ __forceinline__ bool grid_sums(const double (&v)[NV], double* partials, unsigned* ticket,
                                          int nblocks, double (&out)[NV], int bid = -1) {
    __shared__ double red[NT / 32];
    __shared__ bool s_last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (bid < 0) bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    for (int q = 0; q < NV; ++q) {
        double s = block_sum<NT>(v[q], red);
        if (tid == 0) partials[(size_t)q * nblocks + bid] = s;
    }
    if (tid == 0) {
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == (unsigned)nblocks - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    for (int q = 0; q < NV; ++q) {
        double acc = 0.0;
        for (int b = tid; b < nblocks; b += NT) acc += __ldcg(partials + (size_t)q * nblocks + b);
        out[q] = block_sum<NT>(acc, red);
    }
    if (tid == 0) *ticket = 0u;
    return tid == 0;
}

// 3-D launch shape used by the cell kernels: 32 x 8 threads per (x, y) tile, each thread
// marching `zchunk` planes of its column (no integer division per cell).
struct Col3 {
    int i, j, k0, k1;
    bool ok;
};
__device__ __forceinline__ Col3 col3(int nx, int ny, int nz, int zchunk, int bx, int by, int bz) {
    Col3 c;
    c.i = bx * 32 + threadIdx.x;
    c.j = by * 8 + threadIdx.y;
    c.k0 = bz * zchunk;
    c.k1 = min(c.k0 + zchunk, nz);
    c.ok = c.i < nx && c.j < ny;
    return c;
}
__device__ __forceinline__ Col3 col3(int nx, int ny, int nz, int zchunk) {
    return col3(nx, ny, nz, zchunk, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------------------
// Batched launches.  One launch serves several independent realisations ("segments"): the
// virtual blocks of segment s are [off[s], off[s+1]) and a CTA finds its segment by binary
// search.  A virtual block is a 3-D block index (x fastest) of that segment's own grid.
// ---------------------------------------------------------------------------------------
struct VBlk {
    int x, y, z;    // block index in the segment's grid
    int gx, gy, gz; // the segment's grid
    int id, count;  // linear index and number of blocks
};

__device__ __forceinline__ VBlk hw_vblk() {
    VBlk v;
    v.x = blockIdx.x, v.y = blockIdx.y, v.z = blockIdx.z;
    v.gx = gridDim.x, v.gy = gridDim.y, v.gz = gridDim.z;
    v.id = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    v.count = gridDim.x * gridDim.y * gridDim.z;
    return v;
}

__device__ __forceinline__ VBlk make_vblk(int id, int gx, int gy, int gz) {
    VBlk v;
    v.id = id;
    v.gx = gx, v.gy = gy, v.gz = gz;
    v.count = gx * gy * gz;
    v.x = id % gx;
    v.y = (id / gx) % gy;
    v.z = id / (gx * gy);
    return v;
}

// segment of virtual block b: the last s with off[s] <= b (off[0] = 0, off[nseg] = total)
__device__ __forceinline__ int find_seg(const int* __restrict__ off, int nseg, int b) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

} // namespace mf3d

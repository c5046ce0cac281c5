// kernels_tail.cuh -- the coarse end of the V-cycle in one CTA, in FP64.
//
// Every level from `first` down to the coarsest runs inside a single CTA: pre-smoothing,
// residual + restriction, the coarsest level's sweeps, prolongation and post-smoothing, in
// the order of v_cycle_recursive (src/multigrid/cycle/v_cycle.cu:36-74) with in-place GSRB
// (red = (i+j+k) even, then black; gsrb_3d.cu:368-576).
//
// Data: x of every tail level lives in shared memory with a one-cell ghost layer (zero for
// Dirichlet and Neumann faces, a copy of the opposite face for periodic axes), b in shared
// memory, and per cell the weights precomputed by tail_weights_kernel when K is set:
//   w_f = C_f / D (six faces), bd = dx^2 / D, q = D / dx^2,
// so a relaxation is x_c = sum_f w_f x_f - bd * b_c and the residual is r_c = q (x_c - x_GS),
// the reference's (sum_f C_f x_f - b dx^2) / D and b - A x with the division done once.
#pragma once
#include "mf3d_device.cuh"

namespace mf3d {

constexpr int TAIL2_MAX_LEVELS = 8;
constexpr int TAIL2_NT = 512;

struct TailLevel {
    int nx, ny, nz, n;
    int per_x, per_y, per_z, xoff; // xoff: padded x in shared memory (doubles)
    int boff;                      // b in shared memory (doubles)
    int pad;
    const double* w;               // 8 * n: w_-x, w_+x, w_-y, w_+y, w_-z, w_+z, bd, q
};

struct Tail2Args {
    int nlev;
    int pre, post, coarse_iters;
    TailLevel L[TAIL2_MAX_LEVELS];
};

// weights of one tail level from its FP64 face coefficients (pin doubles D at cell 0)
__global__ void tail_weights_kernel(const LevelOp<double> L, double* __restrict__ w) {
    const size_t n = (size_t)L.nx * L.ny * L.nz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % L.nx), j = (int)((c / L.nx) % L.ny), k = (int)(c / ((size_t)L.nx * L.ny));
        double cxm, cxp, cym, cyp, czm, czp;
        cell_coefs<double>(L, i, j, k, c, cxm, cxp, cym, cyp, czm, czp);
        double D = cxm + cxp + cym + cyp + czm + czp;
        if (L.pin && c == 0) D *= 2.0;
        w[0 * n + c] = cxm / D;
        w[1 * n + c] = cxp / D;
        w[2 * n + c] = cym / D;
        w[3 * n + c] = cyp / D;
        w[4 * n + c] = czm / D;
        w[5 * n + c] = czp / D;
        w[6 * n + c] = L.dx2 / D;
        w[7 * n + c] = D * L.inv_dx2;
    }
}

__device__ __forceinline__ int tl_pad(const TailLevel& L, int i, int j, int k) {
    return (i + 1) + (L.nx + 2) * ((j + 1) + (L.ny + 2) * (k + 1));
}

// Gauss-Seidel value of cell (i,j,k) from the current x (padded) and b.
__device__ __forceinline__ double tl_gs(const TailLevel& L, const double* x, const double* b, int i, int j, int k) {
    const int c = i + L.nx * (j + L.ny * k);
    const int P = tl_pad(L, i, j, k);
    const int sy = L.nx + 2, sz = (L.nx + 2) * (L.ny + 2);
    const double* w = L.w;
    const int n = L.n;
    return __ldg(w + 0 * n + c) * x[P - 1] + __ldg(w + 1 * n + c) * x[P + 1] + __ldg(w + 2 * n + c) * x[P - sy] +
           __ldg(w + 3 * n + c) * x[P + sy] + __ldg(w + 4 * n + c) * x[P - sz] + __ldg(w + 5 * n + c) * x[P + sz] -
           __ldg(w + 6 * n + c) * b[c];
}

// copy the periodic faces into the ghost layer (threads [0, nthr))
__device__ __forceinline__ void tl_ghosts(const TailLevel& L, double* x, int tid, int nthr) {
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    if (L.per_x)
        for (int e = tid; e < ny * nz; e += nthr) {
            const int j = e % ny, k = e / ny;
            x[tl_pad(L, -1, j, k)] = x[tl_pad(L, nx - 1, j, k)];
            x[tl_pad(L, nx, j, k)] = x[tl_pad(L, 0, j, k)];
        }
    if (L.per_y)
        for (int e = tid; e < nx * nz; e += nthr) {
            const int i = e % nx, k = e / nx;
            x[tl_pad(L, i, -1, k)] = x[tl_pad(L, i, ny - 1, k)];
            x[tl_pad(L, i, ny, k)] = x[tl_pad(L, i, 0, k)];
        }
    if (L.per_z)
        for (int e = tid; e < nx * ny; e += nthr) {
            const int i = e % nx, j = e / nx;
            x[tl_pad(L, i, j, -1)] = x[tl_pad(L, i, j, nz - 1)];
            x[tl_pad(L, i, j, nz)] = x[tl_pad(L, i, j, 0)];
        }
}

// `sweeps` GSRB sweeps on one level by threads [0, nthr); `warp` selects warp barriers.
__device__ __forceinline__ void tl_smooth(const TailLevel& L, double* x, const double* b, int sweeps, int tid,
                                          int nthr, bool warp) {
    const int hx = (L.nx + 1) >> 1; // cells of one colour per row, at most
    const int items = hx * L.ny * L.nz;
    const bool per = L.per_x | L.per_y | L.per_z;
    for (int it = 0; it < sweeps; ++it)
        for (int col = 0; col < 2; ++col) {
            for (int e = tid; e < items; e += nthr) {
                const int m = e % hx, row = e / hx;
                const int j = row % L.ny, k = row / L.ny;
                const int i = 2 * m + ((j + k + col) & 1);
                if (i < L.nx) x[tl_pad(L, i, j, k)] = tl_gs(L, x, b, i, j, k);
            }
            if (per) {
                if (warp) __syncwarp();
                else __syncthreads();
                tl_ghosts(L, x, tid, nthr);
            }
            if (warp) __syncwarp();
            else __syncthreads();
        }
}

template <class TI, class TO>
__device__ __forceinline__ void tail2_body(const Tail2Args& a, const TI* __restrict__ b_in, TO* __restrict__ x_out) {
    extern __shared__ double sm[];
    const int tid = threadIdx.x;
    // zero every padded x (ghosts included), load b of the top level
    for (int l = 0; l < a.nlev; ++l) {
        const TailLevel& L = a.L[l];
        const int np = (L.nx + 2) * (L.ny + 2) * (L.nz + 2);
        for (int e = tid; e < np; e += TAIL2_NT) sm[L.xoff + e] = 0.0;
    }
    {
        const TailLevel& L = a.L[0];
        for (int c = tid; c < L.n; c += TAIL2_NT) sm[L.boff + c] = (double)b_in[c];
    }
    __syncthreads();
    // ---- down: pre-smoothing, residual + restriction ----
    for (int l = 0; l + 1 < a.nlev; ++l) {
        const TailLevel& L = a.L[l];
        double* x = sm + L.xoff;
        const double* b = sm + L.boff;
        tl_smooth(L, x, b, a.pre, tid, TAIL2_NT, false);
        const TailLevel& Lc = a.L[l + 1];
        double* bc = sm + Lc.boff;
        for (int C = tid; C < Lc.n; C += TAIL2_NT) {
            const int I = C % Lc.nx, J = (C / Lc.nx) % Lc.ny, K = C / (Lc.nx * Lc.ny);
            double acc = 0.0;
            // children in the order (000,100,010,110,001,101,011,111), restrict_3d.cu:38-49
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dxx = 0; dxx < 2; ++dxx) {
                        const int i = 2 * I + dxx, j = 2 * J + dy, k = 2 * K + dz;
                        const int c = i + L.nx * (j + L.ny * k);
                        const double xg = tl_gs(L, x, b, i, j, k);
                        acc += __ldg(L.w + 7 * L.n + c) * (x[tl_pad(L, i, j, k)] - xg);
                    }
            bc[C] = acc / 8.0;
        }
        __syncthreads();
    }
    // ---- coarsest level ----
    {
        const TailLevel& L = a.L[a.nlev - 1];
        const bool warp_only = L.n <= 2048;
        if (!warp_only || tid < 32)
            tl_smooth(L, sm + L.xoff, sm + L.boff, a.coarse_iters, tid, warp_only ? 32 : TAIL2_NT, warp_only);
        __syncthreads();
    }
    // ---- up: prolongation (parent injection) + post-smoothing ----
    for (int l = a.nlev - 2; l >= 0; --l) {
        const TailLevel& L = a.L[l];
        const TailLevel& Lc = a.L[l + 1];
        double* x = sm + L.xoff;
        const double* xc = sm + Lc.xoff;
        for (int c = tid; c < L.n; c += TAIL2_NT) {
            const int i = c % L.nx, j = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
            x[tl_pad(L, i, j, k)] += xc[tl_pad(Lc, i >> 1, j >> 1, k >> 1)];
        }
        __syncthreads();
        if (L.per_x | L.per_y | L.per_z) {
            tl_ghosts(L, x, tid, TAIL2_NT);
            __syncthreads();
        }
        tl_smooth(L, x, sm + L.boff, a.post, tid, TAIL2_NT, false);
    }
    {
        const TailLevel& L = a.L[0];
        for (int c = tid; c < L.n; c += TAIL2_NT) {
            const int i = c % L.nx, j = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
            x_out[c] = (TO)sm[L.xoff + tl_pad(L, i, j, k)];
        }
    }
}

template <class TI, class TO>
__global__ void __launch_bounds__(TAIL2_NT, 1) tail2_kernel(const Tail2Args a, const TI* __restrict__ b_in,
                                                            TO* __restrict__ x_out) {
    tail2_body<TI, TO>(a, b_in, x_out);
}

// One realisation's coarse tail in a batched launch.
template <class TI, class TO> struct TailItem {
    Tail2Args a;
    const TI* b_in;
    TO* x_out;
    const int* stop; // skip when set
};

// The coarse tails of several realisations, one CTA each (the launch's dynamic shared memory
// is the largest of theirs).
template <class TI, class TO>
__global__ void __launch_bounds__(TAIL2_NT, 1) tail2_batch_kernel(const TailItem<TI, TO>* __restrict__ items) {
    const TailItem<TI, TO>& it = items[blockIdx.x];
    if (it.stop && *it.stop) return;
    tail2_body<TI, TO>(it.a, it.b_in, it.x_out);
}

} // namespace mf3d

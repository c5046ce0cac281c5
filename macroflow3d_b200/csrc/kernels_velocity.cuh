// kernels_velocity.cuh -- Darcy face velocities from head, and the discrete mass balance.
//
// One kernel writes all three components (the reference launches 3 interior + 6 boundary
// kernels on the legacy default stream, src/physics/flow/velocity_from_head.cu:601-777).
// Each cell writes its three min-side faces; the plus faces are evaluated only at the max
// boundary, or for the mass balance, so an interior face is computed once.
// Formulas are the reference's: interior q = -[2 K_L K_R / (K_L + K_R)] (h_R - h_L)/dx;
// Dirichlet faces -K_c (h_c - h_bc)/(dx/2) (min side) and -K_c (h_bc - h_c)/(dx/2) (max side);
// Neumann 0; periodic faces use the wrapped neighbour (velocity_from_head.cu:102-381).
#pragma once
#include "kernels_setup.cuh"
#include "mf3d_device.cuh"

namespace mf3d {

// Flux through an interior (or periodic) face from cell L to cell R: -[2 K_L K_R / (K_L + K_R)]
// (h_R - h_L) / d, evaluated with one division (the reference's two differ in rounding only).
__device__ __forceinline__ double flux_lr(double KL, double KR, double HL, double HR, double d) {
    return (2.0 * KL * KR * (HL - HR)) / ((KL + KR) * d);
}

struct VelOut {
    double* U;
    double* V;
    double* W;
    int layout; // 0 compact MAC, 1 padded (nx+1)(ny+1)(nz+1)
};

__device__ __forceinline__ size_t u_idx(int layout, int i, int j, int k, int nx, int ny) {
    return layout ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + i
                  : (size_t)i + (size_t)j * (nx + 1) + (size_t)k * (nx + 1) * ny;
}
__device__ __forceinline__ size_t v_idx(int layout, int i, int j, int k, int nx, int ny) {
    return layout ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + i
                  : (size_t)i + (size_t)j * nx + (size_t)k * nx * (ny + 1);
}
__device__ __forceinline__ size_t w_idx(int layout, int i, int j, int k, int nx, int ny) {
    return layout ? (size_t)k * (ny + 1) * (nx + 1) + (size_t)j * (nx + 1) + i
                  : (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
}

// Flux through the min-side face of cell c along one axis.  `lo` is 1 when the cell is on
// the min boundary of that axis, cw the wrapped neighbour index for periodic, cn the
// in-domain neighbour otherwise.
__device__ __forceinline__ double face_min(const double* H, const double* K, size_t c, size_t cn, size_t cw,
                                           bool lo, int type, double hbc, double d) {
    if (!lo) return flux_lr(K[cn], K[c], H[cn], H[c], d);
    if (type == BC_DIRICHLET) return -K[c] * (H[c] - hbc) / (d * 0.5);
    if (type == BC_PERIODIC) return flux_lr(K[cw], K[c], H[cw], H[c], d);
    return 0.0;
}
__device__ __forceinline__ double face_max_bnd(const double* H, const double* K, size_t c, size_t cw, int type,
                                               double hbc, double d) {
    if (type == BC_DIRICHLET) return -K[c] * (hbc - H[c]) / (d * 0.5);
    if (type == BC_PERIODIC) return flux_lr(K[c], K[cw], H[c], H[cw], d);
    return 0.0;
}

constexpr int VEL_NT = 256;

// Writes U,V,W.  With mb != null also accumulates the mass balance:
// mb[0] = max_c |sum_f q_f A_f| (as ordered bits), mb[1] = Q_in (x=0), mb[2] = Q_out (x=L).
__global__ void __launch_bounds__(VEL_NT) velocity_kernel(int nx, int ny, int nz, double dx,
                                                          const double* __restrict__ H, const double* __restrict__ K,
                                                          BcDev bc, VelOut o, unsigned long long* mb_max,
                                                          double* partials, unsigned* ticket, double* mb_sums,
                                                          int zchunk) {
    const size_t nxy = (size_t)nx * ny;
    double qin = 0.0, qout = 0.0, mx = 0.0;
    const double A = dx * dx;
    const Col3 q = col3(nx, ny, nz, zchunk);
    const int i = q.i, j = q.j;
    for (int k = q.k0; q.ok && k < q.k1; ++k) {
        const size_t c = (size_t)i + (size_t)nx * j + nxy * k;
        const double u0 = face_min(H, K, c, c - 1, c + (nx - 1), i == 0, bc.type[0], bc.value[0], dx);
        const double v0 = face_min(H, K, c, c - nx, c + (size_t)(ny - 1) * nx, j == 0, bc.type[2], bc.value[2], dx);
        const double w0 = face_min(H, K, c, c - nxy, c + (size_t)(nz - 1) * nxy, k == 0, bc.type[4], bc.value[4], dx);
        o.U[u_idx(o.layout, i, j, k, nx, ny)] = u0;
        o.V[v_idx(o.layout, i, j, k, nx, ny)] = v0;
        o.W[w_idx(o.layout, i, j, k, nx, ny)] = w0;
        // plus faces: at the max boundary (written here), and for the mass balance the
        // neighbour's min face, with the same arithmetic as that neighbour's store
        double u1 = 0.0, v1 = 0.0, w1 = 0.0;
        if (i == nx - 1) {
            u1 = face_max_bnd(H, K, c, c - (nx - 1), bc.type[1], bc.value[1], dx);
            o.U[u_idx(o.layout, nx, j, k, nx, ny)] = u1;
        } else if (mb_max) {
            u1 = flux_lr(K[c], K[c + 1], H[c], H[c + 1], dx);
        }
        if (j == ny - 1) {
            v1 = face_max_bnd(H, K, c, c - (size_t)(ny - 1) * nx, bc.type[3], bc.value[3], dx);
            o.V[v_idx(o.layout, i, ny, k, nx, ny)] = v1;
        } else if (mb_max) {
            v1 = flux_lr(K[c], K[c + nx], H[c], H[c + nx], dx);
        }
        if (k == nz - 1) {
            w1 = face_max_bnd(H, K, c, c - (size_t)(nz - 1) * nxy, bc.type[5], bc.value[5], dx);
            o.W[w_idx(o.layout, i, j, nz, nx, ny)] = w1;
        } else if (mb_max) {
            w1 = flux_lr(K[c], K[c + nxy], H[c], H[c + nxy], dx);
        }
        if (mb_max) {
            const double d = ((u1 - u0) + (v1 - v0) + (w1 - w0)) * A;
            mx = fmax(mx, fabs(d));
            if (i == 0) qin += u0 * A;
            if (i == nx - 1) qout += u1 * A;
        }
    }
    if (mb_max) {
        double v[2] = {qin, qout}, out[2];
        // max: non-negative doubles order like their bit patterns
        for (int ofs = 16; ofs > 0; ofs >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, ofs));
        if (threadIdx.x == 0) atomicMax(mb_max, (unsigned long long)__double_as_longlong(mx)); // lane 0 of each warp row
        if (grid_sums<VEL_NT, 2>(v, partials, ticket, gridDim.x * gridDim.y * gridDim.z, out)) {
            mb_sums[0] = out[0];
            mb_sums[1] = out[1];
        }
    }
}

// ---------------------------------------------------------------------------------------
// Velocity diagnostics at cell centres (compute_velocity_diagnostics,
// src/physics/flow/velocity_diagnostics.cu:48-179): the divergence of every cell, and at the
// interior cells (1 <= i <= nx-2, likewise j, k; none when a dimension is below 3) the curl of
// the face-averaged cell velocity by centred differences, its magnitude and the helicity
// u . curl u; zero elsewhere.  Any output may be null.  With stats != null the kernel also
// reduces min / max / sum of the three fields (deterministic: per-block partials combined in
// block order by the last block); stats[9] = min, max, mean of div, |omega|, helicity.
// Column-marching launch (Col3); every velocity value comes through the read-only path, so the
// neighbour columns' reads of one tile hit in L1.
// ---------------------------------------------------------------------------------------
constexpr int VD_NT = 256;

__device__ __forceinline__ void vd_block_reduce(double (&mn)[3], double (&mx)[3], double (&sm)[3], double* red) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int o = 16; o > 0; o >>= 1)
        for (int q = 0; q < 3; ++q) {
            mn[q] = fmin(mn[q], __shfl_down_sync(0xffffffffu, mn[q], o));
            mx[q] = fmax(mx[q], __shfl_down_sync(0xffffffffu, mx[q], o));
            sm[q] += __shfl_down_sync(0xffffffffu, sm[q], o);
        }
    const int w = tid >> 5, l = tid & 31;
    if (l == 0)
        for (int q = 0; q < 3; ++q) {
            red[(3 * q) * (VD_NT / 32) + w] = mn[q];
            red[(3 * q + 1) * (VD_NT / 32) + w] = mx[q];
            red[(3 * q + 2) * (VD_NT / 32) + w] = sm[q];
        }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < 3; ++q) {
            double a = red[(3 * q) * (VD_NT / 32)], b = red[(3 * q + 1) * (VD_NT / 32)], c = 0.0;
            for (int i = 0; i < VD_NT / 32; ++i) {
                a = fmin(a, red[(3 * q) * (VD_NT / 32) + i]);
                b = fmax(b, red[(3 * q + 1) * (VD_NT / 32) + i]);
                c += red[(3 * q + 2) * (VD_NT / 32) + i];
            }
            mn[q] = a, mx[q] = b, sm[q] = c;
        }
    __syncthreads();
}

__global__ void __launch_bounds__(VD_NT) velocity_diag_kernel(int nx, int ny, int nz, double inv_dx, int layout,
                                                              const double* __restrict__ U,
                                                              const double* __restrict__ V,
                                                              const double* __restrict__ W, double* div,
                                                              double* omag, double* hel, double* partials,
                                                              unsigned* ticket, double* stats, int zchunk) {
    __shared__ double red[9 * (VD_NT / 32)];
    __shared__ bool s_last;
    const size_t nxy = (size_t)nx * ny;
    const double inv2 = 0.5 * inv_dx;
    const bool curl = nx >= 3 && ny >= 3 && nz >= 3;
    double mn[3], mx[3], sm[3];
    for (int q = 0; q < 3; ++q) mn[q] = INFINITY, mx[q] = -INFINITY, sm[q] = 0.0;
    const Col3 q = col3(nx, ny, nz, zchunk);
    const int i = q.i, j = q.j;
    auto Uf = [&](int a, int b, int c) { return __ldg(U + u_idx(layout, a, b, c, nx, ny)); };
    auto Vf = [&](int a, int b, int c) { return __ldg(V + v_idx(layout, a, b, c, nx, ny)); };
    auto Wf = [&](int a, int b, int c) { return __ldg(W + w_idx(layout, a, b, c, nx, ny)); };
    auto uc = [&](int a, int b, int c) { return 0.5 * (Uf(a, b, c) + Uf(a + 1, b, c)); };
    auto vc = [&](int a, int b, int c) { return 0.5 * (Vf(a, b, c) + Vf(a, b + 1, c)); };
    auto wc = [&](int a, int b, int c) { return 0.5 * (Wf(a, b, c) + Wf(a, b, c + 1)); };
    for (int k = q.k0; q.ok && k < q.k1; ++k) {
        const size_t c = (size_t)i + (size_t)nx * j + nxy * k;
        const double Ui = Uf(i, j, k), Uip = Uf(i + 1, j, k), Vj = Vf(i, j, k), Vjp = Vf(i, j + 1, k);
        const double Wk = Wf(i, j, k), Wkp = Wf(i, j, k + 1);
        const double d = (Uip - Ui) * inv_dx + (Vjp - Vj) * inv_dx + (Wkp - Wk) * inv_dx;
        double om = 0.0, he = 0.0;
        if (curl && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 2) {
            const double u0 = 0.5 * (Ui + Uip), v0 = 0.5 * (Vj + Vjp), w0 = 0.5 * (Wk + Wkp);
            const double dwdy = (wc(i, j + 1, k) - wc(i, j - 1, k)) * inv2;
            const double dvdz = (vc(i, j, k + 1) - vc(i, j, k - 1)) * inv2;
            const double dudz = (uc(i, j, k + 1) - uc(i, j, k - 1)) * inv2;
            const double dwdx = (wc(i + 1, j, k) - wc(i - 1, j, k)) * inv2;
            const double dvdx = (vc(i + 1, j, k) - vc(i - 1, j, k)) * inv2;
            const double dudy = (uc(i, j + 1, k) - uc(i, j - 1, k)) * inv2;
            const double ox = dwdy - dvdz, oy = dudz - dwdx, oz = dvdx - dudy;
            om = sqrt(ox * ox + oy * oy + oz * oz);
            he = u0 * ox + v0 * oy + w0 * oz;
        }
        if (div) div[c] = d;
        if (omag) omag[c] = om;
        if (hel) hel[c] = he;
        const double f[3] = {d, om, he};
        for (int r = 0; r < 3; ++r) mn[r] = fmin(mn[r], f[r]), mx[r] = fmax(mx[r], f[r]), sm[r] += f[r];
    }
    if (!stats) return;
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    vd_block_reduce(mn, mx, sm, red);
    if (tid == 0) {
        for (int r = 0; r < 3; ++r) {
            partials[(size_t)(3 * r) * nb + bid] = mn[r];
            partials[(size_t)(3 * r + 1) * nb + bid] = mx[r];
            partials[(size_t)(3 * r + 2) * nb + bid] = sm[r];
        }
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == (unsigned)nb - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int r = 0; r < 3; ++r) mn[r] = INFINITY, mx[r] = -INFINITY, sm[r] = 0.0;
    // the last block: partials in block order, each thread a strided subset, then the block
    for (int b = tid; b < nb; b += VD_NT)
        for (int r = 0; r < 3; ++r) {
            mn[r] = fmin(mn[r], __ldcg(partials + (size_t)(3 * r) * nb + b));
            mx[r] = fmax(mx[r], __ldcg(partials + (size_t)(3 * r + 1) * nb + b));
            sm[r] += __ldcg(partials + (size_t)(3 * r + 2) * nb + b);
        }
    vd_block_reduce(mn, mx, sm, red);
    if (tid == 0) {
        const double n = (double)nxy * nz;
        for (int r = 0; r < 3; ++r) {
            stats[3 * r] = mn[r];
            stats[3 * r + 1] = mx[r];
            stats[3 * r + 2] = sm[r] / n;
        }
        *ticket = 0u;
    }
}

} // namespace mf3d

// kernels_setup.cuh -- per-K setup: face coefficients, K coarsening, right-hand side and
// initial guess.  Runs once per conductivity field.
#pragma once
#include "mf3d_device.cuh"

namespace mf3d {

struct BcDev {
    int type[6];
    double value[6];
};

// Harmonic mean exactly as the reference evaluates it
// (src/multigrid/common/mg_conventions.cuh:133-135); symmetric in its arguments bit-for-bit.
__device__ __forceinline__ double hmean_ref(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

template <class TC> __device__ __forceinline__ TC store_coef(double v);
template <> __device__ __forceinline__ double store_coef<double>(double v) { return v; }
template <> __device__ __forceinline__ float store_coef<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ __nv_bfloat16 store_coef<__nv_bfloat16>(double v) {
    return __float2bfloat16_rn((float)v);
}

// Face coefficients of one level from its cell K (FP64), scaled by `scale` (1 unless the
// level stores bf16 with a power-of-two scale).
template <class TC>
__global__ void faces_kernel(int nx, int ny, int nz, const double* __restrict__ K, BcDev bc, double scale,
                             TC* __restrict__ cx, TC* __restrict__ cy, TC* __restrict__ cz,
                             TC* __restrict__ bxm, TC* __restrict__ bym, TC* __restrict__ bzm, int zchunk) {
    const size_t nxy = (size_t)nx * ny;
    const Col3 q = col3(nx, ny, nz, zchunk);
    if (!q.ok) return;
    const int i = q.i, j = q.j;
    for (int k = q.k0; k < q.k1; ++k) {
        const size_t c = (size_t)i + (size_t)nx * j + nxy * k;
        const double Kc = K[c];
        double v;
        // +x face
        if (i < nx - 1) v = hmean_ref(Kc, K[c + 1]);
        else if (bc.type[1] == BC_PERIODIC) v = hmean_ref(Kc, K[c - (nx - 1)]);
        else v = bc.type[1] == BC_DIRICHLET ? 2.0 * Kc : 0.0;
        cx[c] = store_coef<TC>(v * scale);
        if (j < ny - 1) v = hmean_ref(Kc, K[c + nx]);
        else if (bc.type[3] == BC_PERIODIC) v = hmean_ref(Kc, K[c - (size_t)(ny - 1) * nx]);
        else v = bc.type[3] == BC_DIRICHLET ? 2.0 * Kc : 0.0;
        cy[c] = store_coef<TC>(v * scale);
        if (k < nz - 1) v = hmean_ref(Kc, K[c + nxy]);
        else if (bc.type[5] == BC_PERIODIC) v = hmean_ref(Kc, K[c - (size_t)(nz - 1) * nxy]);
        else v = bc.type[5] == BC_DIRICHLET ? 2.0 * Kc : 0.0;
        cz[c] = store_coef<TC>(v * scale);
        // minus boundary faces
        if (i == 0) bxm[(size_t)j + (size_t)ny * k] = store_coef<TC>((bc.type[0] == BC_DIRICHLET ? 2.0 * Kc : 0.0) * scale);
        if (j == 0) bym[(size_t)i + (size_t)nx * k] = store_coef<TC>((bc.type[2] == BC_DIRICHLET ? 2.0 * Kc : 0.0) * scale);
        if (k == 0) bzm[(size_t)i + (size_t)nx * j] = store_coef<TC>((bc.type[4] == BC_DIRICHLET ? 2.0 * Kc : 0.0) * scale);
    }
}

// Geometric mean of the 8 children, src/physics/flow/coarsen_K.cu:15-53 (same order).
__global__ void coarsen_kernel(int NX, int NY, int NZ, const double* __restrict__ Kf, double* __restrict__ Kc,
                               int zchunk) {
    const int Nx = 2 * NX;
    const size_t stride = (size_t)Nx * 2 * NY;
    const Col3 q = col3(NX, NY, NZ, zchunk);
    if (!q.ok) return;
    const int I = q.i, J = q.j;
    for (int Kk = q.k0; Kk < q.k1; ++Kk) {
        const size_t C = (size_t)I + (size_t)NX * J + (size_t)NX * NY * Kk;
        const size_t i000 = (size_t)(2 * I) + (size_t)Nx * (2 * J) + stride * (2 * Kk);
        const size_t i001 = i000 + stride;
        const double ls = log(Kf[i000]) + log(Kf[i000 + 1]) + log(Kf[i000 + Nx]) + log(Kf[i000 + 1 + Nx]) +
                          log(Kf[i001]) + log(Kf[i001 + 1]) + log(Kf[i001 + Nx]) + log(Kf[i001 + 1 + Nx]);
        Kc[C] = exp(ls / 8.0);
    }
}

// b: Dirichlet contributions -2 h_bc K_c / dx^2 (src/physics/flow/rhs_head.cu:21-194, faces
// in the order xmin..zmax); x0: the x-linear guess when both x faces are Dirichlet, else 0
// (src/physics/flow/solve_head.cu:29-73).  x0 may be null.
__global__ void rhs_guess_kernel(int nx, int ny, int nz, double dx, const double* __restrict__ K, BcDev bc,
                                 double* __restrict__ b, double* __restrict__ x0, int zchunk) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const bool lin = bc.type[0] == BC_DIRICHLET && bc.type[1] == BC_DIRICHLET;
    const Col3 q = col3(nx, ny, nz, zchunk);
    if (!q.ok) return;
    const int i = q.i, j = q.j;
    for (int k = q.k0; k < q.k1; ++k) {
        const size_t c = (size_t)i + (size_t)nx * j + (size_t)nx * ny * k;
        const double Kc = K[c];
        double v = 0.0;
        const bool on[6] = {i == 0, i == nx - 1, j == 0, j == ny - 1, k == 0, k == nz - 1};
        for (int f = 0; f < 6; ++f)
            if (on[f] && bc.type[f] == BC_DIRICHLET) v -= 2.0 * bc.value[f] * Kc * inv_dx2;
        b[c] = v;
        if (x0) {
            if (lin) {
                const double t = ((double)i + 0.5) / (double)nx;
                x0[c] = bc.value[0] + (bc.value[1] - bc.value[0]) * t;
            } else {
                x0[c] = 0.0;
            }
        }
    }
}

template <class TO, class TI>
__global__ void convert_kernel(size_t n, const TI* __restrict__ in, TO* __restrict__ out) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        out[c] = (TO)in[c];
}

} // namespace mf3d

// kernels_kfield.cuh -- log-normal K by the randomization (spectral) method.
//
// lnK(x) = sigma / sqrt(N) * sum_m (a_m sin(k_m . x) + b_m cos(k_m . x)) at cell centres,
// K = exp(lnK + ln K_g) (src/physics/stochastic/stochastic.cu:180-260).  Each thread owns a
// run of SEG cells along x; per mode it evaluates sin/cos once and advances the phase along
// the run by a rotation through k_x * dx (angle addition), so the cost per (mode, cell) is a
// handful of FMAs instead of two transcendental calls.
#pragma once
#include "mf3d_device.cuh"

namespace mf3d {

constexpr int KF_SEG = 16;
constexpr int KF_NT = 128;
constexpr int KF_MODES_PER_PASS = 512;

// modes: k1,k2,k3,a,b packed as 5 arrays of n_modes doubles.
__global__ void __launch_bounds__(KF_NT) kfield_kernel(int nx, int ny, int nz, double dx, int n_modes,
                                                       const double* __restrict__ modes, double sigma,
                                                       double log_kg, int want_exp, double* __restrict__ out) {
    __shared__ double sm[7][KF_MODES_PER_PASS];
    const int nseg = (nx + KF_SEG - 1) / KF_SEG;
    const size_t nrows = (size_t)ny * nz;
    const size_t task = blockIdx.x * (size_t)KF_NT + threadIdx.x;
    const bool active = task < nrows * nseg;
    const int seg = active ? (int)(task % nseg) : 0;
    const size_t row = active ? task / nseg : 0;
    const int j = (int)(row % ny), k = (int)(row / ny);
    const int i_start = seg * KF_SEG;
    const double x0 = dx * (i_start + 0.5), y = dx * (j + 0.5), z = dx * (k + 0.5);
    double acc[KF_SEG];
#pragma unroll
    for (int q = 0; q < KF_SEG; ++q) acc[q] = 0.0;
    const double* k1 = modes;
    const double* k2 = modes + n_modes;
    const double* k3 = modes + 2 * (size_t)n_modes;
    const double* am = modes + 3 * (size_t)n_modes;
    const double* bm = modes + 4 * (size_t)n_modes;
    for (int m0 = 0; m0 < n_modes; m0 += KF_MODES_PER_PASS) {
        const int cnt = min(KF_MODES_PER_PASS, n_modes - m0);
        __syncthreads();
        for (int q = threadIdx.x; q < cnt; q += KF_NT) {
            sm[0][q] = k1[m0 + q];
            sm[1][q] = k2[m0 + q];
            sm[2][q] = k3[m0 + q];
            sm[3][q] = am[m0 + q];
            sm[4][q] = bm[m0 + q];
            sincos(k1[m0 + q] * dx, &sm[5][q], &sm[6][q]); // rotation by one cell along x
        }
        __syncthreads();
        if (!active) continue;
        for (int q = 0; q < cnt; ++q) {
            const double ph = sm[0][q] * x0 + sm[1][q] * y + sm[2][q] * z;
            double s, c;
            sincos(ph, &s, &c);
            const double sd = sm[5][q], cd = sm[6][q];
            const double a = sm[3][q], b = sm[4][q];
#pragma unroll
            for (int t = 0; t < KF_SEG; ++t) {
                acc[t] += a * s + b * c;
                const double s2 = s * cd + c * sd;
                c = c * cd - s * sd;
                s = s2;
            }
        }
    }
    if (!active) return;
    const double scale = sigma / sqrt((double)n_modes);
    const size_t base = (size_t)i_start + (size_t)nx * row;
#pragma unroll
    for (int t = 0; t < KF_SEG; ++t) {
        if (i_start + t < nx) {
            const double v = scale * acc[t];
            out[base + t] = want_exp ? exp(v + log_kg) : v;
        }
    }
}

} // namespace mf3d

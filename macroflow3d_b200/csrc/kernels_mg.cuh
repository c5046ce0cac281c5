// kernels_mg.cuh -- multigrid V-cycle kernels.
//
// sweep_kernel: one full red-black Gauss-Seidel sweep (red, then black) of one level in a
// single pass over memory.  A CTA owns a TX x TY column tile and a z range; it marches in z
// keeping a ring of x planes (tile plus halo) in shared memory and runs the stages as a
// wavefront: at step t it loads plane t, updates red cells of plane t-1 (on the tile plus a
// 2- or 1-cell ring), black cells of plane t-2 (on the tile, or tile plus 1 when the
// residual follows) and, in RESID mode, the residual of plane t-3 (tile) which is restricted
// to the coarse right-hand side in pairs of planes.  The sweep is out of place (x_in ->
// x_out): a neighbouring CTA's halo is always read from x_in, so tiles never race.
//
// Reference semantics: one call equals gsrb_smooth_3d(iters=1) (src/multigrid/smoothers/
// gsrb_3d.cu:368-576: red = (i+j+k) even first, each colour reads only the other colour),
// optionally preceded by prolong_3d_add (prolong_3d.cu:520-621, parent injection) and
// followed by compute_residual_3d + restrict_3d (residual_3d.cu:378-502, restrict_3d.cu:12-53).
#pragma once
#include "mf3d_device.cuh"

namespace mf3d {

enum : int { M_ZERO = 1, M_PROLONG = 2, M_RESID = 4, M_DOT = 8 };

constexpr int SW_TX = 32;
constexpr int SW_TY = 8;
constexpr int SW_NT = 256;

template <class T, class TC, class TB> struct SweepArgs {
    LevelOp<TC> L;
    const TB* b;       // right-hand side of this level
    const T* x_in;     // ignored with M_ZERO
    T* x_out;          // swept x
    const T* e_c;      // coarse correction (M_PROLONG), coarse dims ncx, ncy
    int ncx, ncy;
    T* b_coarse;       // restricted residual (M_RESID)
    int zchunk;        // planes per CTA (even)
    double* dot_partials; // M_DOT: <r64, x_out> summed over the grid into *dot_out
    unsigned* dot_ticket;
    double* dot_out;
    const double* r64;    // FP64 residual for M_DOT
    const int* stop;      // batched launches: the realisation's stop flag (skip when set)
};

__device__ __forceinline__ int pmod(int a, int m) {
    int r = a % m;
    return r < 0 ? r + m : r;
}

template <class T, class TC, class TB, int MODE>
__device__ __forceinline__ void sweep_body(const SweepArgs<T, TC, TB>& a, const VBlk& vb) {
    constexpr bool ZERO = (MODE & M_ZERO) != 0;
    constexpr bool PROL = (MODE & M_PROLONG) != 0;
    constexpr bool RESID = (MODE & M_RESID) != 0;
    constexpr bool DOT = (MODE & M_DOT) != 0;
    constexpr int NS = RESID ? 3 : 2; // stages: red, black[, residual]
    constexpr int H = NS;             // x halo
    constexpr int SX = SW_TX + 2 * H, SY = SW_TY + 2 * H;
    constexpr int NPL = NS + 2;       // live planes t-NS-1 .. t
    __shared__ T xs[NPL][SY][SX];
    __shared__ T rs[RESID ? 2 : 1][SW_TY][SW_TX];

    const LevelOp<TC>& L = a.L;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const size_t nxy = (size_t)nx * ny;
    const int i0 = vb.x * SW_TX, j0 = vb.y * SW_TY;
    const int z0 = vb.z * a.zchunk;
    const int z1 = min(z0 + a.zchunk, nz);
    const int tid = threadIdx.x;
    const T dx2 = (T)L.dx2;
    double dot_acc = 0.0;

    // ---- one cell update, shared by the red and black stages ----
    auto relax = [&](int li, int lj, int gi, int gj, int gp, int sl, int slm, int slp) {
        const size_t c = (size_t)gi + (size_t)nx * gj + nxy * gp;
        T cxm, cxp, cym, cyp, czm, czp;
        cell_coefs<T>(L, gi, gj, gp, c, cxm, cxp, cym, cyp, czm, czp);
        T D = cxm + cxp + cym + cyp + czm + czp;
        if (L.pin && c == 0) D *= (T)2;
        const T s = cxp * xs[sl][lj][li + 1] + cxm * xs[sl][lj][li - 1] + cyp * xs[sl][lj + 1][li] +
                    cym * xs[sl][lj - 1][li] + czp * xs[slp][lj][li] + czm * xs[slm][lj][li];
        const T bv = load_as<T>(a.b, c);
        xs[sl][lj][li] = (s - bv * dx2) / D;
    };

    const int zlo = z0 - NS, zhi = z1 - 1 + NS;
    for (int t = zlo; t <= zhi; ++t) {
        // ---------------- load plane t (tile + halo H) ----------------
        {
            const int sl = pmod(t, NPL);
            const int gp = wrap_or_out(t, nz, L.per_z);
            for (int e = tid; e < SX * SY; e += SW_NT) {
                const int li = e % SX, lj = e / SX;
                const int gi = wrap_or_out(i0 - H + li, nx, L.per_x);
                const int gj = wrap_or_out(j0 - H + lj, ny, L.per_y);
                T v = (T)0;
                if (gp >= 0 && gi >= 0 && gj >= 0) {
                    const size_t c = (size_t)gi + (size_t)nx * gj + nxy * gp;
                    if (!ZERO) v = a.x_in[c];
                    if (PROL)
                        v += a.e_c[(size_t)(gi >> 1) + (size_t)a.ncx * ((size_t)(gj >> 1) + (size_t)a.ncy * (gp >> 1))];
                }
                xs[sl][lj][li] = v;
            }
        }
        __syncthreads();

        // ---------------- red at plane p = t-1 on tile + (NS-1) ----------------
        {
            const int p = t - 1;
            constexpr int hr = NS - 1;
            const int gp = wrap_or_out(p, nz, L.per_z);
            if (p >= z0 - hr && p <= z1 - 1 + hr && gp >= 0) {
                const int sl = pmod(p, NPL), slm = pmod(p - 1, NPL), slp = pmod(p + 1, NPL);
                constexpr int PW = (SW_TX + 2 * hr) / 2, PH = SW_TY + 2 * hr;
                for (int e = tid; e < PW * PH; e += SW_NT) {
                    const int r = e / PW, pr = e % PW;
                    const int iu0 = i0 - hr + 2 * pr, ju = j0 - hr + r; // unwrapped coords
                    const int iu = iu0 + ((iu0 + ju + p) & 1);          // red: (i+j+k) even
                    const int gi = wrap_or_out(iu, nx, L.per_x);
                    const int gj = wrap_or_out(ju, ny, L.per_y);
                    if (gi < 0 || gj < 0) continue;
                    relax(iu - i0 + H, ju - j0 + H, gi, gj, gp, sl, slm, slp);
                }
            }
        }
        __syncthreads();

        // ---------------- black at plane q = t-2 on tile + (NS-2) ----------------
        {
            const int q = t - 2;
            constexpr int hb = NS - 2;
            const int gq = wrap_or_out(q, nz, L.per_z);
            if (q >= z0 - hb && q <= z1 - 1 + hb && gq >= 0) {
                const int sl = pmod(q, NPL), slm = pmod(q - 1, NPL), slp = pmod(q + 1, NPL);
                constexpr int PW = (SW_TX + 2 * hb) / 2, PH = SW_TY + 2 * hb;
                for (int e = tid; e < PW * PH; e += SW_NT) {
                    const int r = e / PW, pr = e % PW;
                    const int iu0 = i0 - hb + 2 * pr, ju = j0 - hb + r;
                    const int iu = iu0 + (((iu0 + ju + q) & 1) ^ 1); // black: (i+j+k) odd
                    const int gi = wrap_or_out(iu, nx, L.per_x);
                    const int gj = wrap_or_out(ju, ny, L.per_y);
                    if (gi < 0 || gj < 0) continue;
                    const int li = iu - i0 + H, lj = ju - j0 + H;
                    relax(li, lj, gi, gj, gq, sl, slm, slp);
                }
            }
            __syncthreads();
            // write the finished plane q (red and black) for the tile
            if (q >= z0 && q < z1) {
                const int sl = pmod(q, NPL);
                for (int e = tid; e < SW_TX * SW_TY; e += SW_NT) {
                    const int li = e % SW_TX, lj = e / SW_TX;
                    const int gi = i0 + li, gj = j0 + lj;
                    if (gi >= nx || gj >= ny) continue;
                    const size_t c = (size_t)gi + (size_t)nx * gj + nxy * q;
                    const T v = xs[sl][lj + H][li + H];
                    a.x_out[c] = v;
                    if (DOT) dot_acc += __ldg(a.r64 + c) * (double)v;
                }
            }
        }

        // ---------------- residual at plane s = t-3, restriction per plane pair ----------------
        if (RESID) {
            const int s = t - 3;
            if (s >= z0 && s < z1) {
                const int sl = pmod(s, NPL), slm = pmod(s - 1, NPL), slp = pmod(s + 1, NPL);
                const T inv_dx2 = (T)L.inv_dx2;
                for (int e = tid; e < SW_TX * SW_TY; e += SW_NT) {
                    const int li = e % SW_TX, lj = e / SW_TX;
                    const int gi = i0 + li, gj = j0 + lj;
                    T rv = (T)0;
                    if (gi < nx && gj < ny) {
                        const size_t c = (size_t)gi + (size_t)nx * gj + nxy * s;
                        T cxm, cxp, cym, cyp, czm, czp;
                        cell_coefs<T>(L, gi, gj, s, c, cxm, cxp, cym, cyp, czm, czp);
                        T D = cxm + cxp + cym + cyp + czm + czp;
                        if (L.pin && c == 0) D *= (T)2;
                        const int Li = li + H, Lj = lj + H;
                        const T sum = cxp * xs[sl][Lj][Li + 1] + cxm * xs[sl][Lj][Li - 1] +
                                      cyp * xs[sl][Lj + 1][Li] + cym * xs[sl][Lj - 1][Li] +
                                      czp * xs[slp][Lj][Li] + czm * xs[slm][Lj][Li];
                        rv = load_as<T>(a.b, c) - (sum - D * xs[sl][Lj][Li]) * inv_dx2;
                    }
                    rs[(s - z0) & 1][lj][li] = rv;
                }
                if (((s - z0) & 1) == 1) {
                    __syncthreads();
                    const int ncx = nx >> 1, ncy = ny >> 1;
                    for (int e = tid; e < (SW_TX / 2) * (SW_TY / 2); e += SW_NT) {
                        const int ci = e % (SW_TX / 2), cj = e / (SW_TX / 2);
                        const int I = (i0 >> 1) + ci, J = (j0 >> 1) + cj;
                        if (I >= ncx || J >= ncy) continue;
                        const int fi = 2 * ci, fj = 2 * cj;
                        T acc = (T)0;
                        acc += rs[0][fj][fi];
                        acc += rs[0][fj][fi + 1];
                        acc += rs[0][fj + 1][fi];
                        acc += rs[0][fj + 1][fi + 1];
                        acc += rs[1][fj][fi];
                        acc += rs[1][fj][fi + 1];
                        acc += rs[1][fj + 1][fi];
                        acc += rs[1][fj + 1][fi + 1];
                        a.b_coarse[(size_t)I + (size_t)ncx * J + (size_t)ncx * ncy * (s >> 1)] = acc / (T)8;
                    }
                }
            }
        }
        __syncthreads();
    }

    if (DOT) {
        double v[1] = {dot_acc}, out[1];
        if (grid_sums<SW_NT, 1>(v, a.dot_partials, a.dot_ticket, vb.count, out, vb.id)) *a.dot_out = out[0];
    }
}

template <class T, class TC, class TB, int MODE>
__global__ void __launch_bounds__(SW_NT) sweep_kernel(const SweepArgs<T, TC, TB> a) {
    sweep_body<T, TC, TB, MODE>(a, hw_vblk());
}

// The same sweep for several realisations in one launch: segment s (args[s], its block grid
// dims[s]) owns the CTAs [off[s], off[s+1]); realisations whose solve has stopped are skipped.
template <class T, class TC, class TB, int MODE>
__global__ void __launch_bounds__(SW_NT) sweep_batch_kernel(const SweepArgs<T, TC, TB>* __restrict__ args,
                                                            const int4* __restrict__ dims, const int* __restrict__ off,
                                                            int nseg) {
    const int s = find_seg(off, nseg, blockIdx.x);
    const SweepArgs<T, TC, TB>& a = args[s];
    if (a.stop && *a.stop) return;
    const int4 d = dims[s];
    sweep_body<T, TC, TB, MODE>(a, make_vblk(blockIdx.x - off[s], d.x, d.y, d.z));
}

// x_out = x_in + P e_c  (or P e_c when x_in is null): the prolongation alone, for levels
// configured with zero post-smoothing sweeps.
template <class T>
__global__ void prolong_kernel(int nx, int ny, int nz, const T* x_in, const T* e_c, T* x_out) {
    const size_t n = (size_t)nx * ny * nz;
    const int ncx = nx >> 1, ncy = ny >> 1;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        T v = e_c[(size_t)(i >> 1) + (size_t)ncx * ((size_t)(j >> 1) + (size_t)ncy * (k >> 1))];
        if (x_in) v += x_in[c];
        x_out[c] = v;
    }
}

// b_coarse = R b (restriction of the right-hand side itself): the residual of a zero guess,
// for levels configured with zero pre-smoothing sweeps.
template <class T, class TB>
__global__ void restrict_kernel(int ncx, int ncy, int ncz, const TB* fine, T* coarse) {
    const size_t n = (size_t)ncx * ncy * ncz;
    const int nx = 2 * ncx;
    const size_t nxy = (size_t)nx * 2 * ncy;
    for (size_t C = blockIdx.x * (size_t)blockDim.x + threadIdx.x; C < n; C += (size_t)gridDim.x * blockDim.x) {
        const int I = (int)(C % ncx), J = (int)((C / ncx) % ncy), K = (int)(C / ((size_t)ncx * ncy));
        const size_t f = (size_t)(2 * I) + (size_t)nx * (2 * J) + nxy * (2 * K);
        T acc = (T)0;
        acc += (T)fine[f];
        acc += (T)fine[f + 1];
        acc += (T)fine[f + nx];
        acc += (T)fine[f + nx + 1];
        acc += (T)fine[f + nxy];
        acc += (T)fine[f + nxy + 1];
        acc += (T)fine[f + nxy + nx];
        acc += (T)fine[f + nxy + nx + 1];
        coarse[C] = acc / (T)8;
    }
}

} // namespace mf3d

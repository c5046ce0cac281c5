// kernels_resid.cuh -- residual and 2:1 restriction of a staged level, in one pass.
//
// r = b - A x at every fine cell (the smoother's operator: the pinned cell's diagonal doubled,
// src/multigrid/smoothers/residual_3d.cu:365-368) and b_coarse = the mean of the 8 children
// (src/multigrid/transfer/restrict_3d.cu, cell-centred full weighting), for the levels whose
// last pre-smoothing sweep runs as a plain sweep.
//
// 2.5-D blocking as in pmatvec_dot_kernel (kernels_pcg.cuh): a CTA of 256 threads owns a
// 16 x 16 column tile and marches an even z chunk; each thread stages, by cp.async into a ring
// of RR_NS shared-memory slots, its own cell's x, b and +x/+y/+z faces RR_NS - 1 planes ahead, and
// three warps stage the tile's x ring and its -x/-y faces.  A warp covers two rows of 16
// cells, so the 2 x 2 children of a coarse cell in a plane are summed by two shuffles and the
// two planes of a coarse cell in a register.  x of the plane below and the -z face are
// carried in registers.  Non-periodic axes only read zeros beyond the faces (the ghost value
// of the homogeneous correction problem); periodic axes wrap.
#pragma once
#include <cstddef>

#include "kernels_pcg.cuh"

namespace mf3d {

#ifndef MF3D_RR_MINB
#define MF3D_RR_MINB 4 // resident CTAs per SM the register budget is cut for
#endif
#ifndef MF3D_RR_PERSM
#define MF3D_RR_PERSM 8 // CTAs launched per SM (z chunks sized to match)
#endif
#ifndef MF3D_RR_NS
#define MF3D_RR_NS 4 // staged planes: the one applied, the next, RR_NS - 2 in flight
#endif
constexpr int RR_T = 16, RR_NS = MF3D_RR_NS;

template <class T, class TC> struct RrSlot {
    T x[RR_T + 2][RR_T + 2];  // tile and its one-cell ring
    T b[RR_T][RR_T];
    TC cx[RR_T][RR_T + 1];    // +x faces at column tx+1; column 0: the -x faces at i0
    TC cy[RR_T + 1][RR_T];    // +y faces at row ty+1; row 0: the -y faces at j0
    TC cz[RR_T][RR_T];        // +z faces
};
template <class T, class TC> constexpr size_t rr_smem_bytes() { return RR_NS * sizeof(RrSlot<T, TC>); }

template <class T, class TC>
__global__ void __launch_bounds__(256, MF3D_RR_MINB)
    resid_restrict_staged_kernel(const LevelOp<TC> L, const T* __restrict__ x, const T* __restrict__ b,
                                 T* __restrict__ b_coarse, int zchunk) {
    static_assert(sizeof(T) >= 4 && sizeof(TC) >= 4, "cp.async moves 4 or 8 bytes per thread");
    using Slot = RrSlot<T, TC>;
    extern __shared__ __align__(16) unsigned char rr_sm[];
    RrSlot<T, TC>* slot = reinterpret_cast<RrSlot<T, TC>*>(rr_sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tx = lane & 15, ty = 2 * warp + (lane >> 4);
    const int nx = L.nx, ny = L.ny, nz = L.nz, ncx = nx >> 1, ncy = ny >> 1;
    const size_t nxy = (size_t)nx * ny;
    const int i0 = blockIdx.x * RR_T, j0 = blockIdx.y * RR_T, i = i0 + tx, j = j0 + ty;
    const int k0 = blockIdx.z * zchunk, k1 = min(k0 + zchunk, nz);
    const bool own = i < nx && j < ny;
    const T inv_dx2 = (T)L.inv_dx2;
    auto xy_of = [&](int ii, int jj, long long& g) {
        const int a = wrap_or_out(ii, nx, L.per_x), c = wrap_or_out(jj, ny, L.per_y);
        g = (long long)a + (long long)nx * c;
        return a >= 0 && c >= 0;
    };
    const size_t cO = own ? (size_t)i + (size_t)nx * j : 0;
    const int fO = (ty + 1) * (RR_T + 2) + tx + 1;
    // Extra staging role, warp-uniform: warp 0 the ring rows below / above the tile, warp 1
    // the ring columns left / right, warp 2 the -x faces of the first column / the -y faces of
    // the first row.
    int kindE = 0, fE = 0;
    long long gE = 0;
    bool okE = false;
    const TC* cb = L.cx;
    size_t cs = 0;
    {
        const int h = lane >> 4, m = lane & 15;
        if (warp == 0) {
            kindE = 1;
            fE = (h ? RR_T + 1 : 0) * (RR_T + 2) + m + 1;
            okE = xy_of(i0 + m, h ? j0 + RR_T : j0 - 1, gE);
        } else if (warp == 1) {
            kindE = 1;
            fE = (m + 1) * (RR_T + 2) + (h ? RR_T + 1 : 0);
            okE = xy_of(h ? i0 + RR_T : i0 - 1, j0 + m, gE);
        } else if (warp == 2) {
            kindE = 2;
            if (!h) { // -x face of cell (i0, j0 + m)
                const int jj = j0 + m;
                okE = jj < ny;
                fE = (int)offsetof(Slot, cx) + m * (RR_T + 1) * (int)sizeof(TC);
                if (i0 > 0) cb = L.cx + (i0 - 1) + (size_t)nx * jj, cs = nxy;
                else if (L.per_x) cb = L.cx + (nx - 1) + (size_t)nx * jj, cs = nxy;
                else cb = L.bxm + jj, cs = (size_t)ny;
            } else { // -y face of cell (i0 + m, j0)
                const int ii = i0 + m;
                okE = ii < nx;
                fE = (int)offsetof(Slot, cy) + m * (int)sizeof(TC);
                if (j0 > 0) cb = L.cy + ii + (size_t)nx * (j0 - 1), cs = nxy;
                else if (L.per_y) cb = L.cy + ii + (size_t)nx * (ny - 1), cs = nxy;
                else cb = L.bym + ii, cs = (size_t)nx;
            }
            if (!okE) cb = L.cx, cs = 0;
        }
    }
    long long gO;
    const bool okO = xy_of(i, j, gO);
    // one commit group per plane kk: x of the staged cells; b and the faces for kk < k1
    auto issue = [&](int kk) {
        if (kk <= k1) {
            RrSlot<T, TC>& S = slot[(unsigned)(kk - k0) % RR_NS];
            const int kz = wrap_or_out(kk, nz, L.per_z);
            const long long zo = (long long)nxy * (kz < 0 ? 0 : kz);
            const bool okx = okO && kz >= 0;
            pmv_cp<(int)sizeof(T)>(&S.x[0][0] + fO, x + (okx ? (size_t)(gO + zo) : 0), okx);
            if (kindE == 1) {
                const bool ok = okE && kz >= 0;
                pmv_cp<(int)sizeof(T)>(&S.x[0][0] + fE, x + (ok ? (size_t)(gE + zo) : 0), ok);
            }
            if (kk < k1) {
                if (own) {
                    const size_t c = cO + nxy * kk;
                    pmv_cp<(int)sizeof(T)>(&S.b[ty][tx], b + c, true);
                    pmv_cp<(int)sizeof(TC)>(&S.cx[ty][tx + 1], L.cx + c, true);
                    pmv_cp<(int)sizeof(TC)>(&S.cy[ty + 1][tx], L.cy + c, true);
                    pmv_cp<(int)sizeof(TC)>(&S.cz[ty][tx], L.cz + c, true);
                }
                if (kindE == 2) pmv_cp<(int)sizeof(TC)>(reinterpret_cast<unsigned char*>(&S) + fE, cb + cs * kk, okE);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    T xb = (T)0, czm = (T)0;
    size_t c = cO + nxy * k0;
    if (own) { // x below the first plane and the first plane's -z face, read directly
        const int kb = wrap_or_out(k0 - 1, nz, L.per_z);
        if (kb >= 0) xb = __ldg(x + cO + nxy * kb);
        czm = k0 > 0 ? load_as<T>(L.cz, c - nxy)
                     : (L.per_z ? load_as<T>(L.cz, c + (size_t)(nz - 1) * nxy) : load_as<T>(L.bzm, cO));
    }
    const bool writer = own && !(tx & 1) && !(ty & 1);
    const size_t cc0 = (size_t)(i >> 1) + (size_t)ncx * (size_t)(j >> 1);
#pragma unroll
    for (int q = 0; q < RR_NS - 1; ++q) issue(k0 + q);
    T accz = (T)0;
    for (int k = k0; k < k1; ++k, c += nxy) {
        // this thread's copies of plane k+1 have landed; the barrier publishes everyone's
        // copies of plane k and frees the slot of plane k-1
        asm volatile("cp.async.wait_group %0;" ::"n"(RR_NS - 3) : "memory");
        __syncthreads();
        issue(k + RR_NS - 1);
        const unsigned u = (unsigned)(k - k0);
        const RrSlot<T, TC>& S = slot[u % RR_NS];
        const T* X = &S.x[0][0];
        const T xt = (&slot[(u + 1) % RR_NS].x[0][0])[fO];
        const T xc = X[fO], xw = X[fO - 1], xe = X[fO + 1], xs = X[fO - (RR_T + 2)], xn = X[fO + (RR_T + 2)];
        const T cxp = (T)S.cx[ty][tx + 1], cxm = (T)S.cx[ty][tx];
        const T cyp = (T)S.cy[ty + 1][tx], cym = (T)S.cy[ty][tx];
        const T czp = (T)S.cz[ty][tx];
        T D = cxm + cxp + cym + cyp + czm + czp;
        if (L.pin && own && c == 0) D *= (T)2;
        const T sum = cxp * xe + cxm * xw + cyp * xn + cym * xs + czp * xt + czm * xb;
        T r = own ? S.b[ty][tx] - (sum - D * xc) * inv_dx2 : (T)0;
        r += __shfl_xor_sync(0xffffffffu, r, 1);  // x pair
        r += __shfl_xor_sync(0xffffffffu, r, 16); // y pair (rows 2w, 2w+1)
        if (!(k & 1)) {
            accz = r;
        } else {
            accz += r;
            if (writer) b_coarse[cc0 + (size_t)ncx * ncy * (size_t)(k >> 1)] = accz / (T)8;
        }
        xb = xc;
        czm = czp;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

} // namespace mf3d

// kernels_resid.cuh -- residual and 2:1 restriction of a staged level, in one pass.
//
// r = b - A x at every fine cell (the smoother's operator: the pinned cell's diagonal doubled,
// src/multigrid/smoothers/residual_3d.cu:365-368) and b_coarse = the mean of the 8 children
// (src/multigrid/transfer/restrict_3d.cu, cell-centred full weighting), for the levels whose
// last pre-smoothing sweep runs as a plain sweep.
//
// 2.5-D blocking as in pmatvec_dot_kernel (kernels_pcg.cuh): a CTA of 256 threads owns a
// 32 x 16 column tile and marches an even z chunk.  Each thread owns an x-pair of cells (the
// two x children of a coarse cell; fine levels have even nx, so a pair starts on an 8-byte
// FP32 / 16-byte FP64 boundary) and stages, by one cp.async per array into a ring of RR_NS
// shared-memory slots, the pair's x, b and +x/+y/+z faces RR_NS - 1 planes ahead; three
// warps stage the tile's x ring and its -x/-y faces.  A warp covers two rows of 16 pairs, so
// a coarse cell's 2 x 2 children in a plane are one register sum and one shuffle, and its two
// planes a register carry.  x of the plane below and the -z faces are carried in registers.
// Non-periodic axes read zeros beyond the faces (the ghost value of the homogeneous
// correction problem); periodic axes wrap.
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
constexpr int RR_TX = 32, RR_TY = 16, RR_NS = MF3D_RR_NS;
constexpr int RR_XW = RR_TX + 4; // x row: pad, -x ring cell, 32 cells, +x ring cell, pad

template <class T, class TC> struct RrSlot {
    T x[RR_TY + 2][RR_XW];      // cell i0 + q at column q + 2; row 0 / RR_TY + 1: the y ring
    T b[RR_TY][RR_TX];
    TC cx[RR_TY][RR_TX + 2];    // +x face of cell i0 + q at column q + 2; column 1: -x faces at i0
    TC cy[RR_TY + 1][RR_TX];    // +y faces at row ty + 1; row 0: the -y faces at j0
    TC cz[RR_TY][RR_TX];        // +z faces
};
template <class T, class TC> constexpr size_t rr_smem_bytes() { return RR_NS * sizeof(RrSlot<T, TC>); }

// one value / two consecutive values of type E at p, as T
template <class T, class E> __device__ __forceinline__ T rr_one(const E* p) {
    if constexpr (std::is_same<E, __nv_bfloat16>::value) return (T)__bfloat162float(*p);
    else return (T)*p;
}
template <class T, class E> __device__ __forceinline__ void rr_pair(const E* p, T& a, T& b) {
    a = rr_one<T>(p);
    b = rr_one<T>(p + 1);
}

// One CTA's work: tile (bx, by) of 32 x 16 cells, z chunk bz.
template <class T, class TC>
__device__ __forceinline__ void resid_restrict_body(const LevelOp<TC>& L, const T* __restrict__ x,
                                                    const T* __restrict__ b, T* __restrict__ b_coarse, int zchunk,
                                                    int bx, int by, int bz) {
    // cp.async moves 4, 8 or 16 bytes per copy: a pair of BF16 faces is one 4-byte copy, and the
    // single -x face of a row (kind 3 below) is loaded one plane ahead and stored by hand
    static_assert(sizeof(T) >= 4 && (sizeof(TC) >= 4 || std::is_same<TC, __nv_bfloat16>::value),
                  "FP64 / FP32 coefficients, or BF16 coefficients with FP32 vectors");
    using Slot = RrSlot<T, TC>;
    constexpr int ST = (int)sizeof(T), SC = (int)sizeof(TC);
    extern __shared__ __align__(16) unsigned char rr_sm[];
    Slot* slot = reinterpret_cast<Slot*>(rr_sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tx = lane & 15, ty = 2 * warp + (lane >> 4); // pair tx of row ty
    const int nx = L.nx, ny = L.ny, nz = L.nz, ncx = nx >> 1, ncy = ny >> 1;
    const size_t nxy = (size_t)nx * ny;
    const int i0 = bx * RR_TX, j0 = by * RR_TY, i = i0 + 2 * tx, j = j0 + ty;
    const int k0 = bz * zchunk, k1 = min(k0 + zchunk, nz);
    const bool own = i < nx && j < ny; // both cells of the pair (nx even)
    const T inv_dx2 = (T)L.inv_dx2;
    auto xy_of = [&](int ii, int jj, long long& g) {
        const int a = wrap_or_out(ii, nx, L.per_x), c = wrap_or_out(jj, ny, L.per_y);
        g = (long long)a + (long long)nx * c;
        return a >= 0 && c >= 0;
    };
    const size_t cO = own ? (size_t)i + (size_t)nx * j : 0;
    const int fO = (ty + 1) * RR_XW + 2 + 2 * tx; // the pair's x in a slot
    // Extra staging role, warp-uniform kind: warp 0 the ring rows below / above the tile (x
    // pairs), warp 1 the ring columns left / right (single x), warp 2 the -x faces of the
    // first column (single) / the -y faces of the first row (pairs).
    int kindE = 0, fE = 0; // 1: x pair, 2: single x, 3: single face, 4: face pair (fE in bytes)
    long long gE = 0;
    bool okE = false;
    const TC* cb = L.cx;
    size_t cs = 0;
    {
        const int h = lane >> 4, m = lane & 15;
        if (warp == 0) {
            kindE = 1;
            fE = ((h ? RR_TY + 1 : 0) * RR_XW + 2 + 2 * m) * ST;
            okE = xy_of(i0 + 2 * m, h ? j0 + RR_TY : j0 - 1, gE);
        } else if (warp == 1) {
            kindE = 2;
            fE = ((m + 1) * RR_XW + (h ? RR_TX + 2 : 1)) * ST;
            okE = xy_of(h ? i0 + RR_TX : i0 - 1, j0 + m, gE);
        } else if (warp == 2) {
            if (!h) { // -x face of cell (i0, j0 + m)
                kindE = 3;
                const int jj = j0 + m;
                okE = jj < ny;
                fE = (int)offsetof(Slot, cx) + (m * (RR_TX + 2) + 1) * SC;
                if (i0 > 0) cb = L.cx + (i0 - 1) + (size_t)nx * jj, cs = nxy;
                else if (L.per_x) cb = L.cx + (nx - 1) + (size_t)nx * jj, cs = nxy;
                else cb = L.bxm + jj, cs = (size_t)ny;
            } else { // -y faces of cells (i0 + 2m, j0), (i0 + 2m + 1, j0)
                kindE = 4;
                const int ii = i0 + 2 * m;
                okE = ii < nx;
                fE = (int)offsetof(Slot, cy) + 2 * m * SC;
                if (j0 > 0) cb = L.cy + ii + (size_t)nx * (j0 - 1), cs = nxy;
                else if (L.per_y) cb = L.cy + ii + (size_t)nx * (ny - 1), cs = nxy;
                else cb = L.bym + ii, cs = (size_t)nx;
            }
            if (!okE) cb = L.cx, cs = 0;
        }
    }
    long long gO;
    const bool okO = xy_of(i, j, gO);
    TC face_next = TC(0.0f); // SC == 2, kind 3: the -x face of plane kk + 1, loaded at issue(kk)
    if constexpr (SC == 2) {
        if (kindE == 3 && okE && k0 < k1) face_next = cb[cs * (size_t)k0];
    }
    // one commit group per plane kk: x of the staged cells; b and the faces for kk < k1
    auto issue = [&](int kk) {
        if (kk <= k1) {
            Slot& S = slot[(unsigned)(kk - k0) % RR_NS];
            unsigned char* Sb = reinterpret_cast<unsigned char*>(&S);
            const int kz = wrap_or_out(kk, nz, L.per_z);
            const long long zo = (long long)nxy * (kz < 0 ? 0 : kz);
            const bool okx = okO && kz >= 0;
            pmv_cp<2 * ST>(&S.x[0][0] + fO, x + (okx ? (size_t)(gO + zo) : 0), okx);
            if (kindE == 1 || kindE == 2) {
                const bool ok = okE && kz >= 0;
                const T* src = x + (ok ? (size_t)(gE + zo) : 0);
                if (kindE == 1) pmv_cp<2 * ST>(Sb + fE, src, ok);
                else pmv_cp<ST>(Sb + fE, src, ok);
            }
            if (kk < k1) {
                if (own) {
                    const size_t c = cO + nxy * kk;
                    pmv_cp<2 * ST>(&S.b[ty][2 * tx], b + c, true);
                    pmv_cp<2 * SC>(&S.cx[ty][2 + 2 * tx], L.cx + c, true);
                    pmv_cp<2 * SC>(&S.cy[ty + 1][2 * tx], L.cy + c, true);
                    pmv_cp<2 * SC>(&S.cz[ty][2 * tx], L.cz + c, true);
                }
                if (kindE == 3) {
                    if constexpr (SC == 2) { // store the face fetched one plane ago, fetch the next
                        *reinterpret_cast<TC*>(Sb + fE) = okE ? face_next : TC(0.0f);
                        if (okE && kk + 1 < k1) face_next = cb[cs * (size_t)(kk + 1)];
                    } else {
                        pmv_cp<SC>(Sb + fE, cb + cs * kk, okE);
                    }
                } else if (kindE == 4) {
                    pmv_cp<2 * SC>(Sb + fE, cb + cs * kk, okE);
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    T xb0 = (T)0, xb1 = (T)0, czm0 = (T)0, czm1 = (T)0;
    size_t c = cO + nxy * k0;
    if (own) { // x below the first plane and the first plane's -z faces, read directly
        const int kb = wrap_or_out(k0 - 1, nz, L.per_z);
        if (kb >= 0) rr_pair<T>(x + cO + nxy * kb, xb0, xb1);
        if (k0 > 0) {
            czm0 = load_as<T>(L.cz, c - nxy), czm1 = load_as<T>(L.cz, c - nxy + 1);
        } else if (L.per_z) {
            czm0 = load_as<T>(L.cz, c + (size_t)(nz - 1) * nxy), czm1 = load_as<T>(L.cz, c + (size_t)(nz - 1) * nxy + 1);
        } else {
            czm0 = load_as<T>(L.bzm, cO), czm1 = load_as<T>(L.bzm, cO + 1);
        }
    }
    const bool writer = own && !(ty & 1);
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
        const Slot& S = slot[u % RR_NS];
        const T* X = &S.x[0][0] + fO;
        T xt0, xt1, xc0, xc1, xs0, xs1, xn0, xn1;
        rr_pair<T>(&slot[(u + 1) % RR_NS].x[0][0] + fO, xt0, xt1);
        rr_pair<T>(X, xc0, xc1);
        rr_pair<T>(X - RR_XW, xs0, xs1);
        rr_pair<T>(X + RR_XW, xn0, xn1);
        const T xw0 = X[-1], xe1 = X[2];
        T cxm0 = rr_one<T>(&S.cx[ty][1 + 2 * tx]), cxp0, cxp1, cym0, cym1, cyp0, cyp1, czp0, czp1, b0, b1;
        rr_pair<T>(&S.cx[ty][2 + 2 * tx], cxp0, cxp1);
        rr_pair<T>(&S.cy[ty][2 * tx], cym0, cym1);
        rr_pair<T>(&S.cy[ty + 1][2 * tx], cyp0, cyp1);
        rr_pair<T>(&S.cz[ty][2 * tx], czp0, czp1);
        rr_pair<T>(&S.b[ty][2 * tx], b0, b1);
        // cell i (its +x neighbour is cell i+1, whose -x face is cxp0)
        T D0 = cxm0 + cxp0 + cym0 + cyp0 + czm0 + czp0;
        if (L.pin && own && c == 0) D0 *= (T)2;
        const T s0 = cxp0 * xc1 + cxm0 * xw0 + cyp0 * xn0 + cym0 * xs0 + czp0 * xt0 + czm0 * xb0;
        const T D1 = cxp0 + cxp1 + cym1 + cyp1 + czm1 + czp1;
        const T s1 = cxp1 * xe1 + cxp0 * xc0 + cyp1 * xn1 + cym1 * xs1 + czp1 * xt1 + czm1 * xb1;
        T r = own ? (b0 - (s0 - D0 * xc0) * inv_dx2) + (b1 - (s1 - D1 * xc1) * inv_dx2) : (T)0;
        r += __shfl_xor_sync(0xffffffffu, r, 16); // y pair (rows 2w, 2w+1)
        if (!(k & 1)) {
            accz = r;
        } else {
            accz += r;
            if (writer) b_coarse[cc0 + (size_t)ncx * ncy * (size_t)(k >> 1)] = accz / (T)8;
        }
        xb0 = xc0, xb1 = xc1;
        czm0 = czp0, czm1 = czp1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

template <class T, class TC>
__global__ void __launch_bounds__(256, MF3D_RR_MINB)
    resid_restrict_staged_kernel(const LevelOp<TC> L, const T* __restrict__ x, const T* __restrict__ b,
                                 T* __restrict__ b_coarse, int zchunk) {
    resid_restrict_body<T, TC>(L, x, b, b_coarse, zchunk, blockIdx.x, blockIdx.y, blockIdx.z);
}

// The residual + restriction of several realisations in one launch: realisation s owns the
// CTAs [off[s], off[s+1]) (its gx x gy x gz grid); realisations whose solve has stopped are
// skipped.
template <class T, class TC> struct RrItem {
    LevelOp<TC> L;
    const T* x;
    const T* b;
    T* out;
    int zchunk, gx, gy, gz;
    const int* stop;
};
template <class T, class TC>
__global__ void __launch_bounds__(256, MF3D_RR_MINB)
    resid_restrict_batch_kernel(const RrItem<T, TC>* __restrict__ items, const int* __restrict__ off, int nseg) {
    const int s = find_seg(off, nseg, blockIdx.x);
    const RrItem<T, TC>& it = items[s];
    if (it.stop && *it.stop) return; // that realisation's solve has finished (CTA-uniform)
    const int v = blockIdx.x - __ldg(off + s);
    resid_restrict_body<T, TC>(it.L, it.x, it.b, it.out, it.zchunk, v % it.gx, (v / it.gx) % it.gy,
                               v / (it.gx * it.gy));
}

} // namespace mf3d

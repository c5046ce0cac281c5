// kernels_sweep_tma.cuh -- the fused red-black sweep with its operands staged by TMA.
//
// Same algorithm as sweep_kernel (kernels_mg.cuh): one full red-black Gauss-Seidel sweep of
// a level (red = (i+j+k) even first), optionally preceded by the prolongation of a coarse
// correction and followed by residual + restriction, in one pass over memory.
//
// Schedule.  A CTA owns a TX x TY column tile and marches a z range; at step t it updates
//   red   cells of plane t   on the tile plus an RR-cell ring,
//   black cells of plane t-1 on the tile plus an RB = RR-1 ring,
//   the residual of plane t-2 on the tile (RESID), restricted to the coarse right-hand side
//   one step later, per pair of planes, and writes plane t-2 (now final) to global memory.
// Every thread owns one pair of x-adjacent cells (one red, one black in every plane) in
// every stage; the black cell of plane t-1 lies in the column of the red cell of plane t.
// Every value a stage reads from another thread was written before the previous step's
// barrier: ONE __syncthreads per plane.
//
// Instruction economy.  The pairs of a warp all lie in rows of one parity, so the offset of
// the red cell inside the pair, (row + t) & 1, is the same for the whole warp; the march is
// unrolled by two and each step is compiled for its offset, with no per-cell selects.  The
// stages compute unconditionally and predicate only their stores.  A pair's coefficients of
// plane t are read from shared memory once; the black cell's ones are kept in registers for
// the next step (double-buffered by the unrolling), and RESID keeps the whole pair for the
// residual two steps later.  The -x and -y faces of the pair come from one precomputed
// shared-memory offset each, which points at the staged boundary faces on the min faces.
//
// Staging.  Two rings fed by cp.async.bulk.tensor.3d; thread 0 issues the copies and waits
// on their mbarriers (bounded) at the end of the step before the one that reads them, so the
// step barrier publishes the landed planes:
//   x ring (NRX slots): planes t+1 .. t-2 are live at step t; plane t+1 is the red stage's
//     upper z neighbour (corrected by the coarse correction in PROLONG mode), plane t holds
//     the red updates, t-1 the black updates, t-2 the residual's reads and the output;
//   coefficient ring (NRC slots): b, cx, cy, cz of plane t, plus the -x faces of the box rows
//     and the -y faces of the box columns when the tile touches those boundaries; for plane -1
//     the -z faces take the place of cz.
// Boxes start at x = i0 - HX with HX * sizeof(element) a multiple of 16 bytes (TMA's rule
// for the innermost coordinate); y and z may start outside the grid, where TMA fills zeros:
// the ghost value of a Dirichlet or Neumann face for x.  Periodic axes are served by
// sweep_kernel instead.
//
// Work split.  One CTA per (tile, z chunk), tiles fastest, sized so that all CTAs are
// resident at once (MINB per SM): neighbouring tiles then march the same planes together and
// the halo rows one CTA stages are still in L2 when its neighbours stage them.
#pragma once
#include <cuda.h>

#include <type_traits>

#include "kernels_mg.cuh"

namespace mf3d {

struct TmaMaps {
    CUtensorMap x, b, cx, cy, cz; // 3-D, box BX x BY x 1
    CUtensorMap bxm, bym, bzm;    // 2-D boundary-face planes: BYP x 1, BX x 1, BX x BY
};

template <class T, class TC> struct TmaGeom {
    static constexpr int lcm_elts() {
        const int a = 16 / (int)sizeof(T), c = 16 / (int)sizeof(TC);
        return a > c ? a : c; // both are powers of two
    }
    static constexpr int hx(int H) { return ((H + lcm_elts() - 1) / lcm_elts()) * lcm_elts(); }
};

template <class T, class TC> struct TmaSweepArgs {
    LevelOp<TC> L;
    T* x_out;
    const T* e_c; // coarse correction (M_PROLONG)
    int ncx, ncy;
    T* b_coarse;       // M_RESID
    const double* r64; // M_DOT: <r64, x_out>
    double* dot_partials;
    unsigned* dot_ticket;
    double* dot_out;
    int zchunk; // planes per CTA (even)
    int* err;   // set to 1 when an mbarrier wait gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <class T, class TC, int MODE> struct TmaSweepCfg {
    static constexpr bool ZERO = (MODE & M_ZERO) != 0;
    static constexpr bool PROL = (MODE & M_PROLONG) != 0;
    static constexpr bool RESID = (MODE & M_RESID) != 0;
    static constexpr int RR = RESID ? 2 : 1; // red ring
    static constexpr int RB = RR - 1;        // black ring
    static constexpr int H = RR + 1;         // x halo read by the red ring
    static constexpr int HX = TmaGeom<T, TC>::hx(H);
    static constexpr int TX = 32, TY = sizeof(T) == 8 ? 8 : 16;
    static constexpr int BX = TX + 2 * HX, BY = TY + 2 * H;
    // pair items cover columns [i0-2, i0+TX+2) and rows [j0-RI, j0+TY+RI); PROLONG corrects
    // the whole x halo, so its items reach ring H.  Half the warps take the even rows, half
    // the odd ones.
    static constexpr int RI = PROL ? H : RR;
    static constexpr int IPW = TX / 2 + 2, IH = TY + 2 * RI;
    static_assert(IH % 2 == 0, "rows come in parity pairs");
    static constexpr int IPC = IPW * (IH / 2); // items per parity class
    static constexpr int WPC = (IPC + 31) / 32;
    static constexpr int NT = 2 * 32 * WPC;
    static_assert(RI <= H && HX >= 2 && HX >= H, "pair items and their reads must stay inside the box");
    static constexpr size_t align128(size_t v) { return (v + 127) & ~(size_t)127; }
    static constexpr size_t XB = (size_t)BX * BY * sizeof(T), CB = (size_t)BX * BY * sizeof(TC);
    static constexpr size_t XS = align128(XB), CA = align128(CB);
    // -x boundary faces of the box rows, from row j0 - BYS (BYS * sizeof(TC) a multiple of 16)
    static constexpr int AL = 16 / (int)sizeof(TC);
    static constexpr int BYS = ((4 + AL - 1) / AL) * AL;
    static constexpr int BYP = ((TY + BYS + 4 + AL - 1) / AL) * AL;
    static_assert(BYS >= H, "boundary rows must cover the halo");
    static constexpr size_t BXMB = (size_t)BYP * sizeof(TC), BYMB = (size_t)BX * sizeof(TC);
    // coefficient slot: b, cx, cy, cz, bxm, bym
    static constexpr size_t C_CX = XS, C_CY = XS + CA, C_CZ = XS + 2 * CA, C_BXM = XS + 3 * CA;
    static constexpr size_t C_BYM = C_BXM + align128(BXMB);
    static constexpr size_t CS = C_BYM + align128(BYMB);
    static constexpr size_t RS = RESID ? align128(3 * (size_t)TX * TY * sizeof(T)) : 0;
    static constexpr int MINB = 2; // CTAs per SM
    static constexpr size_t BUDGET = 110 * 1024;
    static constexpr int NRX = 7; // 4 live x planes + 3 in flight
    static constexpr int NRC_FIT = (int)((BUDGET - 256 - align128((size_t)BX * sizeof(T) + 16) - RS - NRX * XS) / CS);
    static constexpr int NRC = NRC_FIT < 8 ? NRC_FIT : 8;
    static_assert(NRC >= 3, "coefficient ring too small");
    // the x ring starts one guard row in: unpredicated neighbour reads of the edge items may
    // reach one box row before the first slot (they are never used)
    static constexpr size_t OFF_X = 256 + align128((size_t)BX * sizeof(T) + 16);
    static constexpr size_t OFF_C = OFF_X + NRX * XS, OFF_R = OFF_C + NRC * CS;
    static constexpr size_t SMEM = OFF_R + RS;
};

template <class T> __device__ __forceinline__ void lds_pair(const T* p, T& a, T& b);
template <> __device__ __forceinline__ void lds_pair<float>(const float* p, float& a, float& b) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x;
    b = v.y;
}
template <> __device__ __forceinline__ void lds_pair<double>(const double* p, double& a, double& b) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x;
    b = v.y;
}
template <class T> __device__ __forceinline__ void st_pair(T* p, T a, T b);
template <> __device__ __forceinline__ void st_pair<float>(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
}
template <> __device__ __forceinline__ void st_pair<double>(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
template <class T, class TC> __device__ __forceinline__ void lds_pair_as(const TC* p, T& a, T& b) {
    if constexpr (std::is_same<TC, __nv_bfloat16>::value) {
        const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
        a = (T)v.x;
        b = (T)v.y;
    } else if constexpr (std::is_same<TC, T>::value) {
        lds_pair<T>(p, a, b);
    } else {
        a = (T)p[0];
        b = (T)p[1];
    }
}

// The black cell's coefficients of one plane, kept for the next step.
template <class T> struct CellCoef {
    T b, cxp, cxm, cyp, cym, czp;
};
// A pair's coefficients of one plane (RESID keeps them for the residual).
template <class T> struct PairCoef {
    T b0, b1, cx0, cx1, cy0, cy1, cz0, cz1, cxl, cyd0, cyd1;
};

template <class T, class TC, int MODE>
__global__ void __launch_bounds__(TmaSweepCfg<T, TC, MODE>::NT, TmaSweepCfg<T, TC, MODE>::MINB)
    sweep_tma_kernel(const __grid_constant__ TmaMaps maps, const TmaSweepArgs<T, TC> a) {
    using C = TmaSweepCfg<T, TC, MODE>;
    constexpr bool ZERO = C::ZERO, PROL = C::PROL, RESID = C::RESID;
    constexpr bool DOT = (MODE & M_DOT) != 0;
    constexpr int TX = C::TX, TY = C::TY, BX = C::BX, H = C::H, HX = C::HX, RR = C::RR, RB = C::RB;
    constexpr int NRX = C::NRX, NRC = C::NRC;
    extern __shared__ __align__(128) unsigned char sweep_sm[];
    uint64_t* barx = reinterpret_cast<uint64_t*>(sweep_sm);
    uint64_t* barc = barx + NRX;
    T* rsb = reinterpret_cast<T*>(sweep_sm + C::OFF_R);
    auto xsl = [&](int s) { return reinterpret_cast<T*>(sweep_sm + C::OFF_X + C::XS * s); };
    auto cbase = [&](int s) { return sweep_sm + C::OFF_C + C::CS * s; };

    const LevelOp<TC>& L = a.L;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const size_t nxy = (size_t)nx * ny;
    const int tid = threadIdx.x;
    const T dx2 = (T)L.dx2, inv_dx2 = (T)L.inv_dx2;
    auto divide = [](T num, T den) -> T {
        if constexpr (sizeof(T) == 4) return __fdividef(num, den); // preconditioner: 2-ulp division
        else return num / den;
    };
    auto tc = [](TC v) -> T { return ld_as_float_or_double<T>(v); };

    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY, ntiles = ntx * nty;

    if (tid == 0) {
        for (int s = 0; s < NRX + NRC; ++s) mbar_init(&barx[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // ring bookkeeping.  Every thread tracks the planes staged so far (qx, qc) and the slots of
    // the planes it reads; thread 0 alone issues the copies and waits for them (phases in
    // phx / phc).
    unsigned qx = 0, qc = 0;
    int xi_slot = 0, ci_slot = 0, xw_slot = 0, cw_slot = 0; // thread 0: next slot to issue / wait
    unsigned phx = 0u, phc = 0u;
    double dot_acc = 0.0;
    bool fail = false;
    auto nxt_x = [](int s) { return s + 1 == NRX ? 0 : s + 1; };
    auto nxt_c = [](int s) { return s + 1 == NRC ? 0 : s + 1; };
    auto wait_x = [&]() { // thread 0
        const bool ok = mbar_wait(&barx[xw_slot], (phx >> xw_slot) & 1u);
        phx ^= 1u << xw_slot;
        xw_slot = nxt_x(xw_slot);
        return ok;
    };
    auto wait_c = [&]() {
        const bool ok = mbar_wait(&barc[cw_slot], (phc >> cw_slot) & 1u);
        phc ^= 1u << cw_slot;
        cw_slot = nxt_c(cw_slot);
        return ok;
    };

    // ---- this thread's pair within a tile (tile-independent part) ----
    const int cls = tid / (32 * C::WPC);        // row parity class of the warp
    const int idx = tid - cls * (32 * C::WPC);  // item within the class
    const bool iv = idx < C::IPC;
    const int rr_ = iv ? idx / C::IPW : 0, ic = iv ? idx - rr_ * C::IPW : 1;
    const int ir = 2 * rr_ + ((cls + C::RI) & 1); // item row, 0 .. IH-1; gj & 1 == cls
    const int e = (ir - C::RI + H) * BX + (2 * ic - 2 + HX); // box element of the pair's left cell

    // CTA b: tile b % ntiles, z chunk b / ntiles (tiles fastest, so neighbouring tiles march
    // the same planes at the same time and share their halo rows in L2)
    for (int b = blockIdx.x; b < ntiles * ((nz + a.zchunk - 1) / a.zchunk) && !fail; b += gridDim.x) {
        // ---------------- one z chunk of one tile ----------------
        const int tile = b % ntiles;
        const int z0 = (b / ntiles) * a.zchunk;
        const int z1 = min(nz, z0 + a.zchunk);
        const int i0 = (tile % ntx) * TX, j0 = (tile / ntx) * TY;
        const int t0 = z0 - RR;      // first red plane
        const int pl0 = t0 - 1;      // first plane staged
        const int cl1 = z1 + RR - 1; // last coefficient plane (last red plane)
        const int xl1 = cl1 + 1;     // last x plane (its upper neighbour)
        // last step: plane z1 - 1 is written at step z1 + 1 and its residual pair restricted at
        // step z1 + 2; the count of steps is made even for the two-step unrolling
        int t1 = RESID ? z1 + 2 : z1 + 1;
        if ((t1 - pl0 + 1) & 1) ++t1;
        const bool bnd_x = i0 == 0, bnd_y = j0 == 0;
        int xi_plane = pl0, ci_plane = pl0; // thread 0: next plane to issue
        int xw_plane = pl0, cw_plane = pl0; // thread 0: next plane to wait for
        auto issue_x = [&]() {
            mbar_expect_tx(&barx[xi_slot], (unsigned)C::XB);
            tma_load_3d(xsl(xi_slot), &maps.x, i0 - HX, j0 - H, xi_plane, &barx[xi_slot]);
            xi_slot = nxt_x(xi_slot);
            ++xi_plane;
        };
        auto issue_c = [&]() {
            uint64_t* bar = &barc[ci_slot];
            unsigned char* cs = cbase(ci_slot);
            mbar_expect_tx(bar, (unsigned)(C::XB + 3 * C::CB + (bnd_x ? C::BXMB : 0) + (bnd_y ? C::BYMB : 0)));
            tma_load_3d(cs, &maps.b, i0 - HX, j0 - H, ci_plane, bar);
            tma_load_3d(cs + C::C_CX, &maps.cx, i0 - HX, j0 - H, ci_plane, bar);
            tma_load_3d(cs + C::C_CY, &maps.cy, i0 - HX, j0 - H, ci_plane, bar);
            if (ci_plane == -1) // the -z boundary faces stand in for plane -1's +z faces
                tma_load_2d(cs + C::C_CZ, &maps.bzm, i0 - HX, j0 - H, bar);
            else
                tma_load_3d(cs + C::C_CZ, &maps.cz, i0 - HX, j0 - H, ci_plane, bar);
            if (bnd_x) tma_load_2d(cs + C::C_BXM, &maps.bxm, j0 - C::BYS, ci_plane, bar);
            if (bnd_y) tma_load_2d(cs + C::C_BYM, &maps.bym, i0 - HX, ci_plane, bar);
            ci_slot = nxt_c(ci_slot);
            ++ci_plane;
        };
        if (tid == 0) {
            if (!ZERO)
                while (xi_plane <= xl1 && xi_plane < pl0 + NRX) issue_x();
            while (ci_plane <= cl1 && ci_plane < pl0 + NRC) issue_c();
            // the first step reads x planes pl0 and pl0 + 1 and coefficient plane pl0
            bool ok = true;
            if (!ZERO) {
                ok = wait_x();
                ++xw_plane;
                if (ok) {
                    ok = wait_x();
                    ++xw_plane;
                }
            }
            if (ok) {
                ok = wait_c();
                ++cw_plane;
            }
            fail = !ok;
        }
        fail = __syncthreads_or(fail) != 0;
        // slots of x planes t+1, t, t-1, t-2 and of coefficient plane t (the same in every thread)
        int sxp = nxt_x((int)(qx % NRX)), sx0 = (int)(qx % NRX), sx1 = 0, sx2 = 0;
        int scc = (int)(qc % NRC);

        // ---- the pair in this tile ----
        const int gi = i0 - 2 + 2 * ic, gj = j0 - C::RI + ir;
        const bool rowg = iv && gj >= 0 && gj < ny;
        const bool g0 = rowg && gi >= 0 && gi < nx, g1 = rowg && gi + 1 >= 0 && gi + 1 < nx;
        auto in_ring = [&](int i, int r) {
            return iv && gj >= j0 - r && gj < j0 + TY + r && i >= i0 - r && i < i0 + TX + r;
        };
        const bool rr0 = in_ring(gi, RR), rr1 = in_ring(gi + 1, RR);
        const bool rb0 = in_ring(gi, RB), rb1 = in_ring(gi + 1, RB);
        const bool tl0 = in_ring(gi, 0) && g0, tl1 = in_ring(gi + 1, 0) && g1;
        const bool pin_pair = L.pin && gi == 0 && gj == 0;
        // byte offsets in a coefficient slot of the left cell's -x face and the pair's -y faces
        const int off_cxl = (gi == 0) ? (int)C::C_BXM + (gj - (j0 - C::BYS)) * (int)sizeof(TC)
                                      : (int)C::C_CX + (e - 1) * (int)sizeof(TC);
        const int off_cyd = (gj == 0) ? (int)C::C_BYM + (gi - (i0 - HX)) * (int)sizeof(TC)
                                      : (int)C::C_CY + (e - BX) * (int)sizeof(TC);
        const int ncx = a.ncx;
        const size_t ncxy = (size_t)a.ncx * a.ncy;
        const bool restricts = RESID && tl0 && ((gj - j0) & 1) == 0 && gj + 1 < ny;
        // output item: VEC consecutive cells of one tile row (nx is a multiple of VEC)
        constexpr int VEC = 16 / (int)sizeof(T), VPR = TX / VEC;
        const int vr = tid / VPR, vc = tid - vr * VPR;
        const bool vo_ok = tid < VPR * TY && j0 + vr < ny && i0 + VEC * vc < nx;
        const int vo_e = (vr + H) * BX + HX + VEC * vc;
        const size_t vo_g = (size_t)(i0 + VEC * vc) + (size_t)nx * (j0 + vr);

        // the pair's x_old in plane p (slot s) plus, in PROLONG mode, the coarse correction,
        // stored back so that the neighbours read the corrected plane
        auto own_x = [&](int p, int s, T& va, T& vb) {
            va = (T)0;
            vb = (T)0;
            T* xs = xsl(s);
            if (!ZERO) lds_pair<T>(xs + e, va, vb);
            if (PROL) {
                if (p >= 0 && p < nz && g0) { // nx is even: one coarse cell per pair
                    const T ev = a.e_c[(size_t)(gi >> 1) + (size_t)ncx * (gj >> 1) + ncxy * (size_t)(p >> 1)];
                    va += ev;
                    vb += ev;
                }
                if (iv) st_pair<T>(xs + e, va, vb);
            }
        };
        auto restrict_pair = [&](int s1, int rs0, int rs1) { // coarse plane s1 >> 1 from s1 - 1, s1
            const T* r0 = rsb + rs0 * TX * TY;
            const T* r1 = rsb + rs1 * TX * TY;
            const int f = (gj - j0) * TX + (gi - i0);
            T acc = (T)0;
            acc += r0[f];
            acc += r0[f + 1];
            acc += r0[f + TX];
            acc += r0[f + TX + 1];
            acc += r1[f];
            acc += r1[f + 1];
            acc += r1[f + TX];
            acc += r1[f + TX + 1];
            a.b_coarse[(size_t)(gi >> 1) + (size_t)ncx * (gj >> 1) + ncxy * (size_t)(s1 >> 1)] = acc / (T)8;
        };

        // carried state: the black cell's coefficients of the previous plane (cbA / cbB), the
        // red cell's +z face of two planes back (czA / czB), and in RESID the whole pair of
        // planes t-1, t-2 (c1, c2), cz of plane t-3 and the pair's final x of plane t-3
        CellCoef<T> cbA{}, cbB{};
        T czA = 0, czB = 0;
        PairCoef<T> c1{}, c2{};
        T cz3a = 0, cz3b = 0, x3a = 0, x3b = 0;
        int rslot = 0; // rsb slot of residual plane t-2 ((t - 2 - z0) mod 3)

        // one step of the march; O: offset of the red cell of plane t in the pair (compile time)
        auto step = [&](auto Oc, int t, CellCoef<T>& cb_in, CellCoef<T>& cb_out, T& cz_io) {
            constexpr int O = decltype(Oc)::value;
            // -------- refill the slots freed by the previous step (thread 0) --------
            if (tid == 0) {
                if (!ZERO && t - 3 >= pl0 && xi_plane <= xl1) issue_x();
                if (t - 1 >= pl0 && ci_plane <= cl1) issue_c();
            }
            const bool in_z = t >= 0 && t < nz;
            // -------- the pair's x in plane t+1 (and t at the start), corrected --------
            T xpa = 0, xpb = 0;
            if (t == pl0) {
                T d0, d1;
                own_x(t, sx0, d0, d1);
            }
            if (t + 1 <= xl1) own_x(t + 1, sxp, xpa, xpb);
            // -------- coefficients of plane t --------
            PairCoef<T> c0;
            {
                const unsigned char* cs = cbase(scc);
                lds_pair<T>(reinterpret_cast<const T*>(cs) + e, c0.b0, c0.b1);
                lds_pair_as<T, TC>(reinterpret_cast<const TC*>(cs + C::C_CX) + e, c0.cx0, c0.cx1);
                lds_pair_as<T, TC>(reinterpret_cast<const TC*>(cs + C::C_CY) + e, c0.cy0, c0.cy1);
                lds_pair_as<T, TC>(reinterpret_cast<const TC*>(cs + C::C_CZ) + e, c0.cz0, c0.cz1);
                lds_pair_as<T, TC>(reinterpret_cast<const TC*>(cs + off_cyd), c0.cyd0, c0.cyd1);
                c0.cxl = tc(*reinterpret_cast<const TC*>(cs + off_cxl));
            }
            // -------- red, plane t, cell O --------
            T vred;
            {
                const T cxp = O ? c0.cx1 : c0.cx0, cxm = O ? c0.cx0 : c0.cxl;
                const T cyp = O ? c0.cy1 : c0.cy0, cym = O ? c0.cyd1 : c0.cyd0;
                const T czp = O ? c0.cz1 : c0.cz0, czm = cb_in.czp; // cz(t-1) of this cell
                T D = cxm + cxp + cym + cyp + czm + czp;
                if (pin_pair && O == 0 && t == 0) D *= (T)2;
                T s = (T)0;
                T* xs = xsl(sx0);
                if (!ZERO) {
                    const T xr = xs[e + O + 1], xl = xs[e + O - 1];
                    s = cxp * xr + cxm * xl + cyp * xs[e + O + BX] + cym * xs[e + O - BX] + czp * (O ? xpb : xpa) +
                        czm * xsl(sx1)[e + O];
                }
                const bool live = t >= t0 && t <= cl1 && (O ? rr1 : rr0);
                vred = (in_z && (O ? g1 : g0)) ? divide(s - (O ? c0.b1 : c0.b0) * dx2, D) : (T)0;
                if (live) xs[e + O] = vred;
                // the black cell of plane t (the other one) is updated at the next step
                if (O == 0) cb_out = CellCoef<T>{c0.b1, c0.cx1, c0.cx0, c0.cy1, c0.cyd1, c0.cz1};
                else cb_out = CellCoef<T>{c0.b0, c0.cx0, c0.cxl, c0.cy0, c0.cyd0, c0.cz0};
            }
            // -------- black, plane t-1, cell O --------
            {
                const int q = t - 1;
                const T czm = cz_io; // cz(t-2) of this cell: the red cell's +z face two steps back
                const T D = cb_in.cxm + cb_in.cxp + cb_in.cym + cb_in.cyp + czm + cb_in.czp;
                T* xs = xsl(sx1);
                const T xr = xs[e + O + 1], xl = xs[e + O - 1];
                const T s = cb_in.cxp * xr + cb_in.cxm * xl + cb_in.cyp * xs[e + O + BX] + cb_in.cym * xs[e + O - BX] +
                            cb_in.czp * vred + czm * xsl(sx2)[e + O];
                const bool live = q >= z0 - RB && q < z1 + RB && (O ? rb1 : rb0);
                const T v = (q >= 0 && q < nz && (O ? g1 : g0)) ? divide(s - cb_in.b * dx2, D) : (T)0;
                if (live) xs[e + O] = v;
            }
            cz_io = O ? c0.cz1 : c0.cz0; // for the black stage two steps on
            // -------- plane t-2 is final: write the tile, 16 bytes per thread --------
            if (t - 2 >= z0 && t - 2 < z1 && vo_ok) {
                const T* xs = xsl(sx2);
                const size_t cg = vo_g + nxy * (size_t)(t - 2);
                if constexpr (sizeof(T) == 4) {
                    const float4 v = *reinterpret_cast<const float4*>(xs + vo_e);
                    *reinterpret_cast<float4*>(a.x_out + cg) = v;
                    if (DOT) {
                        const double2 r0 = __ldg(reinterpret_cast<const double2*>(a.r64 + cg));
                        const double2 r1 = __ldg(reinterpret_cast<const double2*>(a.r64 + cg + 2));
                        dot_acc += r0.x * (double)v.x + r0.y * (double)v.y + r1.x * (double)v.z + r1.y * (double)v.w;
                    }
                } else {
                    const double2 v = *reinterpret_cast<const double2*>(xs + vo_e);
                    *reinterpret_cast<double2*>(a.x_out + cg) = v;
                    if (DOT) {
                        const double2 r0 = __ldg(reinterpret_cast<const double2*>(a.r64 + cg));
                        dot_acc += r0.x * (double)v.x + r0.y * (double)v.y;
                    }
                }
            }
            if constexpr (RESID) {
                // -------- residual, plane t-2 (smoother's pin convention) --------
                const int sp = t - 2;
                const T* xs = xsl(sx2);
                T x2a, x2b, x1a, x1b, ua, ub, da, db;
                lds_pair<T>(xs + e, x2a, x2b);
                lds_pair<T>(xsl(sx1) + e, x1a, x1b);
                lds_pair<T>(xs + e + BX, ua, ub);
                lds_pair<T>(xs + e - BX, da, db);
                const T xl = xs[e - 1], xr = xs[e + 2];
                T ra, rb;
                {
                    const T cxp = c2.cx0, cxm = c2.cxl, cyp = c2.cy0, cym = c2.cyd0, czp = c2.cz0, czm = cz3a;
                    T D = cxm + cxp + cym + cyp + czm + czp;
                    if (pin_pair && sp == 0) D *= (T)2;
                    const T sum = cxp * x2b + cxm * xl + cyp * ua + cym * da + czp * x1a + czm * x3a;
                    ra = c2.b0 - (sum - D * x2a) * inv_dx2;
                }
                {
                    const T cxp = c2.cx1, cxm = c2.cx0, cyp = c2.cy1, cym = c2.cyd1, czp = c2.cz1, czm = cz3b;
                    const T D = cxm + cxp + cym + cyp + czm + czp;
                    const T sum = cxp * xr + cxm * x2a + cyp * ub + cym * db + czp * x1b + czm * x3b;
                    rb = c2.b1 - (sum - D * x2b) * inv_dx2;
                }
                if (sp >= z0 && sp < z1 && (tl0 || tl1))
                    st_pair<T>(rsb + rslot * TX * TY + (gj - j0) * TX + (gi - i0), tl0 ? ra : (T)0, tl1 ? rb : (T)0);
                // -------- restriction of planes (t-4, t-3), finished before the last barrier --------
                const int s1 = t - 3;
                if (restricts && s1 > z0 && s1 < z1 && ((s1 - z0) & 1) == 1)
                    restrict_pair(s1, rslot == 0 ? 1 : rslot - 1 == 0 ? 2 : rslot - 2, rslot == 0 ? 2 : rslot - 1);
                if (sp >= z0) rslot = rslot == 2 ? 0 : rslot + 1;
                x3a = x2a;
                x3b = x2b;
                cz3a = c2.cz0;
                cz3b = c2.cz1;
                c2 = c1;
                c1 = c0;
            }
            // -------- thread 0: wait for the planes of the next step --------
            if (tid == 0 && t < t1) {
                bool ok = true;
                if (!ZERO && xw_plane <= xl1) {
                    ok = wait_x();
                    ++xw_plane;
                }
                if (ok && cw_plane <= cl1) {
                    ok = wait_c();
                    ++cw_plane;
                }
                fail = !ok;
            }
            // generic-proxy writes to the rings are ordered before the TMA writes that reuse
            // the slots; the barrier completes the hand-off and the plane exchange
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            fail = __syncthreads_or(fail) != 0;
            sx2 = sx1;
            sx1 = sx0;
            sx0 = sxp;
            sxp = nxt_x(sxp);
            scc = nxt_c(scc);
        };

        using Z = std::integral_constant<int, 0>;
        using I = std::integral_constant<int, 1>;
        for (int t = pl0; t < t1 && !fail; t += 2) {
            // red offset of plane t: (gj + t) & 1 = (cls + t) & 1, uniform in the warp
            if (((cls + t) & 1) == 0) step(Z{}, t, cbB, cbA, czA);
            else step(I{}, t, cbB, cbA, czA);
            if (fail) break;
            if (((cls + t) & 1) == 0) step(I{}, t + 1, cbA, cbB, czB);
            else step(Z{}, t + 1, cbA, cbB, czB);
        }
        if (fail) {
            // drain this CTA's copies in flight (bounded waits), then leave
            if (tid == 0) {
                atomicExch(a.err, 1);
                while (xw_plane < xi_plane) {
                    (void)wait_x();
                    ++xw_plane;
                }
                while (cw_plane < ci_plane) {
                    (void)wait_c();
                    ++cw_plane;
                }
            }
            break;
        }
        if (!ZERO) qx += (unsigned)(xl1 - pl0 + 1);
        qc += (unsigned)(cl1 - pl0 + 1);
    }

    if (DOT && !fail) {
        double v[1] = {dot_acc}, out[1];
        if (grid_sums<C::NT, 1>(v, a.dot_partials, a.dot_ticket, gridDim.x, out)) *a.dot_out = out[0];
    }
}

} // namespace mf3d

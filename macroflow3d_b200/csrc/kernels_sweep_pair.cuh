// kernels_sweep_pair.cuh -- one red-black Gauss-Seidel sweep, x-pairs of cells per thread.
//
// Same result as sweep_kernel (kernels_mg.cuh) and gsrb_smooth_3d(iters = 1) of the reference
// (src/multigrid/smoothers/gsrb_3d.cu:368-576): red = (i+j+k) even first, each colour reading
// only the other colour, optionally preceded by the prolongation of a coarse correction
// (prolong_3d_add, prolong_3d.cu:520-621: x += e of the parent cell) and with <r64, x_out>
// summed for the preconditioned CG (M_DOT).
//
// Schedule.  A CTA owns a 32 x 16 column tile and marches a z chunk [z0, z1).  Every thread of
// the 8 tile warps owns an x-pair of cells (2m, 2m+1) of one row.  In plane t the red cell of
// the pair is 2m + o with o = (j + t) & 1; in plane t-1 the same column holds a black cell.  At
// step t the thread therefore
//   - relaxes its red cell of plane t from old black values,
//   - relaxes the black cell of plane t-1 in the same column from the red values of planes
//     t-2, t-1 (published at the previous step) and t (just computed),
//   - writes plane t-1, now final, as one pair (red value of the last step, black value now).
// Only red values go through shared memory (one store per thread and step); a thread keeps
// the old x of its own column for planes t-1 .. t+1, its last two red values and the
// coefficient pairs of the last plane in registers.  ONE barrier per plane.
//
// The black updates next to the tile need the red values of the one-cell ring around it, so
// two more warps relax the red cells of that ring (without storing them): warp 8 the ring
// rows below and above the tile (x-pairs), warp 9 the ring columns left and right (one cell
// each, relaxed in the planes where it is red).  x is staged with a two-cell ring for them.
//
// Periodic axes must be a whole number of tiles (x: 32 cells, y: 16), so that the ring of a
// tile is the wrapped neighbour of its edge.
//
// Staging.  Every thread copies, by cp.async into rings of shared-memory slots, the x pair(s)
// it owns and their b / face coefficients; the ring warps also stage the outer x rows, the
// corner pairs and the boundary faces the tile needs.  x plane p and the coefficients of
// plane p - 1 form one commit group, issued SP_D planes ahead, so the coefficients arrive
// exactly one step before their use.  Cells beyond a non-periodic face are staged as zeros
// (the ghost value); the -x / -y / -z faces of the first cells come from the boundary-face
// planes bxm / bym / bzm; periodic axes wrap.  With M_PROLONG the stager adds the coarse
// correction to the pairs it staged before the barrier that publishes them.
#pragma once
#include <cstddef>

#include "kernels_mg.cuh"
#include "kernels_pcg.cuh"

namespace mf3d {

constexpr int SP_TX = 32, SP_TY = 16;     // tile (cells)
constexpr int SP_PX = SP_TX / 2;          // pairs per tile row
constexpr int SP_W = SP_TX + 4;           // slot row pitch: columns i0-2 .. i0+TX+1
constexpr int SP_XR = SP_TY + 4;          // x rows j0-2 .. j0+TY+1
constexpr int SP_CR = SP_TY + 2;          // b, cx, cz rows j0-1 .. j0+TY
constexpr int SP_YR = SP_TY + 3;          // cy rows j0-2 .. j0+TY
constexpr int SP_NT = 320;                // 8 tile warps + ring rows + ring columns
#ifndef MF3D_SP_D
#define MF3D_SP_D 3 // planes staged ahead of the one the red stage reads
#endif
constexpr int SP_D = MF3D_SP_D;
constexpr int SP_NSX = SP_D + 2; // x planes t-1 .. t+D
constexpr int SP_NSC = SP_D;     // coefficient planes t .. t+D-1

template <class T> struct SpXSlot {
    T x[SP_XR][SP_W];
};
template <class T, class TC> struct SpCSlot {
    T b[SP_CR][SP_W];
    TC cx[SP_CR][SP_W];
    TC cy[SP_YR][SP_W];
    TC cz[SP_CR][SP_W];
};
template <class T, class TC> constexpr size_t sp_smem_bytes() {
    return SP_NSX * sizeof(SpXSlot<T>) + SP_NSC * sizeof(SpCSlot<T, TC>);
}
// resident CTAs per SM the register budget is cut for
template <class T> constexpr int sp_minb() { return sizeof(T) == 8 ? 2 : 3; }

template <class T, class TC> struct SpArgs {
    LevelOp<TC> L;
    const T* x_in; // ignored with M_ZERO
    const T* b;
    T* x_out;
    const T* e_c; // coarse correction (M_PROLONG), coarse dims ncx, ncy
    int ncx, ncy;
    const double* r64; // M_DOT: <r64, x_out> into *dot_out
    double* dot_partials;
    unsigned* dot_ticket;
    double* dot_out;
    int zchunk; // planes per work item
};

template <class T> struct P2 {
    T a, b; // cells 2m, 2m+1
    __device__ __forceinline__ T at(int o) const { return o ? b : a; }
};
template <class T> __device__ __forceinline__ P2<T> sp_ld2(const T* p) {
    if constexpr (sizeof(T) == 8) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        return P2<T>{(T)v.x, (T)v.y};
    } else {
        const float2 v = *reinterpret_cast<const float2*>(p);
        return P2<T>{(T)v.x, (T)v.y};
    }
}
template <class T> __device__ __forceinline__ void sp_st2(T* p, T a, T b) {
    if constexpr (sizeof(T) == 8) *reinterpret_cast<double2*>(p) = make_double2(a, b);
    else *reinterpret_cast<float2*>(p) = make_float2(a, b);
}
template <class T> __device__ __forceinline__ void sp_stg2(T* p, T a, T b) {
    if constexpr (sizeof(T) == 8) *reinterpret_cast<double2*>(p) = make_double2(a, b);
    else *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

template <class T, class TC, int MODE>
__global__ void __launch_bounds__(SP_NT, sp_minb<T>()) sweep_pair_kernel(const SpArgs<T, TC> a) {
    static_assert(sizeof(T) == sizeof(TC) && sizeof(T) >= 4, "FP64 or FP32 vectors with coefficients of the same type");
    constexpr bool ZERO = (MODE & M_ZERO) != 0, PROL = (MODE & M_PROLONG) != 0, DOT = (MODE & M_DOT) != 0;
    static_assert((MODE & M_RESID) == 0, "the residual runs in a kernel of its own");
    constexpr int ST = (int)sizeof(T), W = SP_W;
    using XS = SpXSlot<T>;
    using CS = SpCSlot<T, TC>;
    extern __shared__ __align__(16) unsigned char sp_sm[];
    XS* xsl = reinterpret_cast<XS*>(sp_sm);
    CS* csl = reinterpret_cast<CS*>(sp_sm + SP_NSX * sizeof(XS));

    const LevelOp<TC>& L = a.L;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const size_t nxy = (size_t)nx * ny;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntx = (nx + SP_TX - 1) / SP_TX, ntiles = ntx * ((ny + SP_TY - 1) / SP_TY);
    const int total = ntiles * ((nz + a.zchunk - 1) / a.zchunk);
    const T dx2 = (T)L.dx2;
    auto divide = [](T num, T den) -> T {
        if constexpr (sizeof(T) == 4) return __fdividef(num, den); // preconditioner: 2-ulp division
        else return num / den;
    };
    // role 0: tile pair (red + black + output); 1: ring-row pair (red); 2: ring-column cell (red)
    const int role = warp < 8 ? 0 : (warp == 8 ? 1 : 2);
    const int hi = lane >> 4, lo = lane & 15;
    double dot_acc = 0.0;

    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        __syncthreads(); // the previous item's reads of the slots are done
        const int tile = item % ntiles;
        const int z0 = (item / ntiles) * a.zchunk, z1 = min(z0 + a.zchunk, nz);
        const int i0 = (tile % ntx) * SP_TX, j0 = (tile / ntx) * SP_TY;
        // ---- this thread's pair (first cell pi, row pj; both may lie outside the grid) ----
        int pj, pi, side = -1;
        if (role == 0) pj = j0 + 2 * warp + hi, pi = i0 + 2 * lo;
        else if (role == 1) pj = hi ? j0 + SP_TY : j0 - 1, pi = i0 + 2 * lo;
        else side = hi, pj = j0 + lo, pi = hi ? i0 + SP_TX : i0 - 2;
        // tile pairs lie inside [0, n) or beyond a partial tile's edge (never wrapped: a periodic
        // axis is a whole number of tiles); ring pairs wrap on periodic axes
        const int wi = role == 0 ? (pi < nx ? pi : -1) : wrap_or_out(pi, nx, L.per_x);
        const int wj = role == 0 ? (pj < ny ? pj : -1) : wrap_or_out(pj, ny, L.per_y);
        const bool pin_xy = wi >= 0 && wj >= 0; // both cells (nx is even)
        const long long gxy = pin_xy ? (long long)wi + (long long)nx * wj : 0;
        const int fx = (pj - j0 + 2) * W + (pi - i0 + 2); // x slot; cy slot too
        const int fc = fx - W;                            // b, cx, cz slots (rows from j0-1)
        // secondary x pair: ring-row warp the outer rows, ring-column lanes 0/1/16/17 the corners
        int sj = 0, si = 0;
        bool has2 = false;
        if (role == 1) has2 = true, sj = hi ? j0 + SP_TY + 1 : j0 - 2, si = pi;
        else if (role == 2 && (lo == 0 || lo == 1)) has2 = true, sj = lo ? j0 + SP_TY : j0 - 1, si = pi;
        const int wi2 = wrap_or_out(si, nx, L.per_x), wj2 = wrap_or_out(sj, ny, L.per_y);
        const bool pin2 = has2 && wi2 >= 0 && wj2 >= 0;
        const long long gxy2 = pin2 ? (long long)wi2 + (long long)nx * wj2 : 0;
        const int fx2 = (sj - j0 + 2) * W + (si - i0 + 2);
        // coefficient copies beyond the primary pair's b, cx, cy, cz:
        //   cx of a corner pair (ring-column lanes 0 / 1: rows j0-1, j0+TY, left side)
        //   cy of the row below the ring row (ring-row lanes 0-15) or of a corner (ring-column
        //   lanes 0 / 16: row j0-1)
        const bool cx2 = role == 2 && side == 0 && (lo == 0 || lo == 1);
        const bool cy2 = (role == 1 && !hi) || (role == 2 && lo == 0);
        const int cy2j = role == 1 ? j0 - 2 : j0 - 1;
        const int wcy2 = wrap_or_out(cy2j, ny, L.per_y);
        // primary cx: at the -x boundary (pair -2, -1 of a non-periodic axis) the -x faces bxm
        const bool cx_bnd = pi == -2 && !L.per_x;
        const bool cx2_bnd = cx_bnd; // corners share the column
        // primary cy / corner cy: on row -1 of a non-periodic axis the -y faces bym
        const bool cy_bnd = pj == -1 && !L.per_y;
        const bool cy2_bnd = cy2j == -1 && !L.per_y;

        const int P0 = z0 - 2;               // first x plane staged
        const int XL = z1 + 1, CL = z1;      // last x plane, last coefficient plane
        auto xslot = [&](int p) -> XS& { return xsl[(unsigned)(p - P0) % SP_NSX]; };
        auto cslot = [&](int p) -> CS& { return csl[(unsigned)(p - P0) % SP_NSC]; };

        // one commit group: x plane p and the coefficients of plane p - 1
        auto issue = [&](int p) {
            if (!ZERO && p <= XL) {
                const int kz = wrap_or_out(p, nz, L.per_z);
                const size_t ko = nxy * (size_t)(kz < 0 ? 0 : kz);
                XS& S = xslot(p);
                const bool ok = pin_xy && kz >= 0;
                pmv_cp<2 * ST>(&S.x[0][0] + fx, a.x_in + (ok ? (size_t)gxy + ko : 0), ok);
                if (has2) {
                    const bool ok2 = pin2 && kz >= 0;
                    pmv_cp<2 * ST>(&S.x[0][0] + fx2, a.x_in + (ok2 ? (size_t)gxy2 + ko : 0), ok2);
                }
            }
            const int q = p - 1;
            if (q >= P0 && q <= CL) {
                const int kz = wrap_or_out(q, nz, L.per_z);
                const bool kin = kz >= 0;
                const size_t ko = nxy * (size_t)(kin ? kz : 0);
                CS& C = cslot(q);
                const bool ok = pin_xy && kin;
                const size_t g = ok ? (size_t)gxy + ko : 0;
                pmv_cp<2 * ST>(&C.b[0][0] + fc, a.b + g, ok);
                if (cx_bnd) { // -x faces of cell (0, pj): one value into the column of cell -1
                    const bool okb = wj >= 0 && kin;
                    pmv_cp<ST>(&C.cx[0][0] + fc + 1, L.bxm + (okb ? (size_t)wj + (size_t)ny * kz : 0), okb);
                } else {
                    pmv_cp<2 * ST>(&C.cx[0][0] + fc, L.cx + g, ok);
                }
                if (cy_bnd) { // -y faces of the pair's cells in row 0
                    const bool okb = wi >= 0 && kin;
                    pmv_cp<2 * ST>(&C.cy[0][0] + fx, L.bym + (okb ? (size_t)wi + (size_t)nx * kz : 0), okb);
                } else {
                    pmv_cp<2 * ST>(&C.cy[0][0] + fx, L.cy + g, ok);
                }
                if (q == -1 && !L.per_z) { // the -z faces of plane 0 stand in for plane -1's +z faces
                    pmv_cp<2 * ST>(&C.cz[0][0] + fc, L.bzm + (pin_xy ? (size_t)gxy : 0), pin_xy);
                } else {
                    pmv_cp<2 * ST>(&C.cz[0][0] + fc, L.cz + g, ok);
                }
                if (cx2) {
                    const int fcc = (sj - j0 + 1) * W + (si - i0 + 2);
                    if (cx2_bnd) {
                        const bool okb = wj2 >= 0 && kin;
                        pmv_cp<ST>(&C.cx[0][0] + fcc + 1, L.bxm + (okb ? (size_t)wj2 + (size_t)ny * kz : 0), okb);
                    } else {
                        const bool ok2 = pin2 && kin;
                        pmv_cp<2 * ST>(&C.cx[0][0] + fcc, L.cx + (ok2 ? (size_t)gxy2 + ko : 0), ok2);
                    }
                }
                if (cy2) {
                    const int fyy = (cy2j - j0 + 2) * W + (pi - i0 + 2);
                    if (cy2_bnd) {
                        const bool okb = wi >= 0 && kin;
                        pmv_cp<2 * ST>(&C.cy[0][0] + fyy, L.bym + (okb ? (size_t)wi + (size_t)nx * kz : 0), okb);
                    } else {
                        const bool ok2 = wi >= 0 && wcy2 >= 0 && kin;
                        pmv_cp<2 * ST>(&C.cy[0][0] + fyy,
                                       L.cy + (ok2 ? (size_t)wi + (size_t)nx * wcy2 + ko : 0), ok2);
                    }
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        // coarse correction of a pair (both cells share the parent) in plane p
        auto corr = [&](bool in_xy, int ii, int jj, int p) -> T {
            if (!PROL) return (T)0;
            const int kz = wrap_or_out(p, nz, L.per_z);
            if (!in_xy || kz < 0) return (T)0;
            return __ldg(a.e_c + (size_t)(ii >> 1) + (size_t)a.ncx * ((size_t)(jj >> 1) + (size_t)a.ncy * (size_t)(kz >> 1)));
        };
        // x pair of plane p staged at offset f, with the correction added (and written back for
        // the other threads when `publish`)
        auto take = [&](int p, int f, T e, bool publish) -> P2<T> {
            T* s = &xslot(p).x[0][0] + f;
            P2<T> v{(T)0, (T)0};
            if constexpr (!ZERO) v = sp_ld2<T>(s);
            if constexpr (PROL) {
                v.a += e;
                v.b += e;
                if (publish) sp_st2<T>(s, v.a, v.b);
            }
            return v;
        };

        // ---- prologue: x planes P0, P0+1 and the coefficients of plane P0 ----
#pragma unroll
        for (int q = 0; q <= SP_D; ++q) issue(P0 + q);
        asm volatile("cp.async.wait_group %0;" ::"n"(SP_D - 1) : "memory");
        __syncthreads();
        P2<T> xprev = take(P0, fx, corr(pin_xy, wi, wj, P0), false);
        P2<T> xcur = take(P0 + 1, fx, corr(pin_xy, wi, wj, P0 + 1), true);
        if (has2) (void)take(P0 + 1, fx2, corr(pin2, wi2, wj2, P0 + 1), true);
        T en = corr(pin_xy, wi, wj, P0 + 2), en2 = has2 ? corr(pin2, wi2, wj2, P0 + 2) : (T)0;
        P2<T> czp1 = sp_ld2<TC>(&cslot(P0).cz[0][0] + fc); // +z faces of plane t-1 (-z of plane t)
        P2<T> czp2{(T)0, (T)0};                           // +z faces of plane t-2
        // carried coefficients of plane t-1 (the black stage)
        P2<T> b1{}, cx1{}, cy1{}, cyd1{};
        T cxl1 = 0;
        T red1 = 0, red2 = 0; // red values of planes t-1 and t-2 in this column
        double2 r64n = make_double2(0.0, 0.0);

        for (int t = z0 - 1; t <= z1; ++t) {
            // this thread's copies of x plane t+1 and coefficients of plane t have landed; the
            // barrier publishes everyone's and the red values of plane t-1, and frees the slots
            // of x plane t-2 and coefficient plane t-1
            asm volatile("cp.async.wait_group %0;" ::"n"(SP_D - 2) : "memory");
            __syncthreads();
            issue(t + SP_D);
            const int o = (pj + t) & 1;
            // ---- x of plane t+1 (own column, and the pairs this thread staged for the others) ----
            const P2<T> xnext = take(t + 1, fx, en, true);
            if (has2) (void)take(t + 1, fx2, en2, true);
            if constexpr (PROL) {
                en = corr(pin_xy, wi, wj, t + 2);
                if (has2) en2 = corr(pin2, wi2, wj2, t + 2);
            }
            // ---- coefficients of plane t ----
            const CS& C = cslot(t);
            const P2<T> b0 = sp_ld2<T>(&C.b[0][0] + fc), cx0 = sp_ld2<TC>(&C.cx[0][0] + fc);
            const P2<T> cy0 = sp_ld2<TC>(&C.cy[0][0] + fx), cyd0 = sp_ld2<TC>(&C.cy[0][0] + fx - W);
            const P2<T> cz0 = sp_ld2<TC>(&C.cz[0][0] + fc);
            const T cxl0 = (T)(&C.cx[0][0])[fc - 1];
            // ---- red cell pi + o of plane t, from old black values ----
            T* X0 = &xslot(t).x[0][0];
            const int kt = wrap_or_out(t, nz, L.per_z);
            const bool red_in = pin_xy && kt >= 0 && (role != 2 || o != side);
            T red;
            {
                T xin = (T)0, xout = (T)0, xs_ = (T)0, xn_ = (T)0, xt = (T)0, xb = (T)0;
                if constexpr (!ZERO || PROL) {
                    xin = xcur.at(1 - o);
                    xout = X0[fx - 1 + 3 * o];
                    xs_ = X0[fx - W + o];
                    xn_ = X0[fx + W + o];
                    xt = xnext.at(o);
                    xb = xprev.at(o);
                }
                const T xw = o ? xin : xout, xe = o ? xout : xin;
                const T cxp = cx0.at(o), cxm = o ? cx0.a : cxl0;
                const T cyp = cy0.at(o), cym = cyd0.at(o), czp = cz0.at(o), czm = czp1.at(o);
                T D = cxm + cxp + cym + cyp + czm + czp;
                if (L.pin && kt == 0 && wi == 0 && wj == 0 && o == 0) D *= (T)2; // cell 0 is red
                const T s = cxp * xe + cxm * xw + cyp * xn_ + cym * xs_ + czp * xt + czm * xb;
                red = red_in ? divide(s - b0.at(o) * dx2, D) : (T)0;
            }
            if (role != 2 || o != side) X0[fx + o] = red;
            // ---- black cell pi + o of plane t-1 from red values; plane t-1 is then final ----
            if (role == 0) {
                const int q = t - 1;
                const bool out_q = q >= z0 && q < z1 && pin_xy;
                if (out_q) {
                    const T* X1 = &xslot(q).x[0][0];
                    const T xout = X1[fx - 1 + 3 * o], xs_ = X1[fx - W + o], xn_ = X1[fx + W + o];
                    const T xw = o ? red1 : xout, xe = o ? xout : red1;
                    const T cxp = cx1.at(o), cxm = o ? cx1.a : cxl1;
                    const T cyp = cy1.at(o), cym = cyd1.at(o), czp = czp1.at(o), czm = czp2.at(o);
                    const T D = cxm + cxp + cym + cyp + czm + czp;
                    const T s = cxp * xe + cxm * xw + cyp * xn_ + cym * xs_ + czp * red + czm * red2;
                    const T blk = divide(s - b1.at(o) * dx2, D);
                    const T va = o ? red1 : blk, vb = o ? blk : red1;
                    const size_t c = (size_t)gxy + nxy * (size_t)q;
                    sp_stg2<T>(a.x_out + c, va, vb);
                    if constexpr (DOT) dot_acc += r64n.x * (double)va + r64n.y * (double)vb;
                }
                if constexpr (DOT) { // r64 of plane t, for the output of plane t at the next step
                    const bool out_t = t >= z0 && t < z1 && pin_xy;
                    r64n = out_t ? __ldg(reinterpret_cast<const double2*>(a.r64 + (size_t)gxy + nxy * (size_t)t))
                                 : make_double2(0.0, 0.0);
                }
            }
            // ---- carry to the next plane ----
            red2 = red1;
            red1 = red;
            xprev = xcur;
            xcur = xnext;
            b1 = b0, cx1 = cx0, cy1 = cy0, cyd1 = cyd0, cxl1 = cxl0;
            czp2 = czp1;
            czp1 = cz0;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    if constexpr (DOT) {
        double v[1] = {dot_acc}, out[1];
        if (grid_sums<SP_NT, 1>(v, a.dot_partials, a.dot_ticket, gridDim.x, out)) *a.dot_out = out[0];
    }
}

} // namespace mf3d

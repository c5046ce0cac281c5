// kernels_sweep_pair.cuh -- one red-black Gauss-Seidel sweep, x-pairs of cells per thread.
//
// Same result as sweep_kernel (kernels_mg.cuh) and gsrb_smooth_3d(iters = 1) of the reference
// (src/multigrid/smoothers/gsrb_3d.cu:368-576): red = (i+j+k) even first, each colour reading
// only the other colour, optionally preceded by the prolongation of a coarse correction
// (prolong_3d_add, prolong_3d.cu:520-621: x += e of the parent cell) and with <r64, x_out>
// summed for the preconditioned CG (M_DOT).
//
// Schedule.  A CTA owns a 32 x 16 column tile and marches a z chunk [z0, z1).  Every thread of
// the 8 tile warps owns an x-pair of cells (2m, 2m+1) of one row (a warp covers rows r and
// r+2, so the red offset is the same for the whole warp).  In plane t the red cell of the pair
// is 2m + O with O = (j + t) & 1; in plane t-1 the same column holds a black cell.  At step t
// the thread therefore
//   - relaxes its red cell of plane t from old black values,
//   - relaxes the black cell of plane t-1 in the same column from the red values of planes
//     t-2, t-1 (published at the previous step) and t (just computed),
//   - writes plane t-1, now final, as one pair (red value of the last step, black value now).
// Only red values go through shared memory (one store per thread and step); a thread keeps
// the old x of its own column for planes t-1 .. t+1, its last two red values and the
// coefficients of the last plane in registers.  ONE barrier per plane.
//
// The black updates next to the tile need the red values of the one-cell ring around it, so
// two more warps relax the red cells of that ring (without storing them): warp 8 the ring
// rows below and above the tile (x-pairs), warp 9 the ring columns left and right (one cell
// each, relaxed in the planes where it is red).  x is staged with a two-cell ring for them.
//
// Staging, two forms (template parameter TM):
//   TMA (non-periodic grids whose rows are 16-byte multiples): one thread copies each plane's
//     x box and coefficient boxes (tile plus ring, zero-filled beyond the grid: the ghost
//     value) with cp.async.bulk.tensor, and the -x / -y / -z boundary faces of the first cells
//     from the boundary-face planes bxm / bym / bzm; one full mbarrier per group, waited on by
//     that thread (bounded) before the step barrier.
//   cp.async (periodic axes, which must then be a whole number of tiles): every thread copies
//     its own x pair(s) and their coefficients; the ring warps also stage the outer rows,
//     corners and boundary faces; wrapped coordinates on periodic axes.
// x plane p and the coefficients of plane p - 1 form one group, issued SP_D planes ahead, so
// the coefficients arrive one step before their use.  With M_PROLONG each thread adds the
// coarse correction to the pairs it owns (and the ring warps to the outer pairs) before the
// barrier that publishes them.
#pragma once
#include <cuda.h>

#include <cstddef>
#include <type_traits>

#include "kernels_mg.cuh"
#include "kernels_pcg.cuh"
#include "kernels_sweep_tma.cuh"

namespace mf3d {

constexpr int SP_TX = 32, SP_TY = 16; // tile of one x-pair per thread (cells); FP32 TMA tiles are 64 wide
constexpr int SP_XR = SP_TY + 4;      // x rows j0-2 .. j0+TY+1
constexpr int SP_CR = SP_TY + 2;      // b, cx, cz rows j0-1 .. j0+TY
constexpr int SP_YR = SP_TY + 3;      // cy rows j0-2 .. j0+TY
constexpr int SP_NT = 320;            // 8 tile warps + ring rows + ring columns
// the thread that issues the TMA copies and waits for them: lane 0 of the ring-column warp,
// whose relaxation work per plane is the smallest
constexpr int SP_PROD = SP_NT - 32;
#ifndef MF3D_SP_D
#define MF3D_SP_D 3 // planes staged ahead of the one the red stage reads
#endif
constexpr int SP_D = MF3D_SP_D;
constexpr int SP_NSX = SP_D + 2; // x planes t-1 .. t+D
constexpr int SP_NSC = SP_D;     // coefficient planes t .. t+D-1

// Shared-memory layout of one precision and staging form.  Columns i0-HX .. i0+TX+HX-1 (a TMA
// box starts on a 16-byte boundary, for the narrower of the vector and coefficient types);
// every array of a slot starts on a 128-byte boundary.
template <class T, class TC, bool TM> struct SpGeom {
    static constexpr int ST = (int)sizeof(T), SC = (int)sizeof(TC);
    static constexpr int SMIN = ST < SC ? ST : SC;
    // x-pairs per thread: two (a quad of cells) with FP32 vectors and TMA staging, where one
    // pair per thread would move too few bytes per plane step; one otherwise
    static constexpr int NP = (ST == 4 && TM) ? 2 : 1;
    static constexpr int TX = SP_TX * NP; // tile width (cells)
    static constexpr int HX = TM ? 16 / SMIN : 2;
    static constexpr int W = TX + 2 * HX;
    static constexpr int BXS = TM ? 16 / SC : 2; // the -x face buffer starts at row j0 - BXS
    static constexpr int BXN = SP_TY + 2 * BXS;
    static constexpr size_t a128(size_t v) { return (v + 127) & ~(size_t)127; }
    static constexpr size_t XSB = a128((size_t)SP_XR * W * ST); // x slot
    // coefficient slot: b (vector type), then cx, cy, cz and the -x faces (bxm) and -y faces
    // (bym) of a tile on the grid's min faces (TMA form), in the coefficient type
    static constexpr size_t BB = a128((size_t)SP_CR * W * ST);
    static constexpr size_t CB = a128((size_t)SP_CR * W * SC), CYB = a128((size_t)SP_YR * W * SC);
    static constexpr size_t OB = 0, OCX = BB, OCY = BB + CB, OCZ = BB + CB + CYB, OBX = BB + 2 * CB + CYB;
    static constexpr size_t OBY = OBX + a128((size_t)BXN * SC);
    static constexpr size_t CSB = OBY + a128((size_t)W * SC);
    static constexpr size_t SMEM = SP_NSX * XSB + SP_NSC * CSB + 128; // + alignment of the base
};
template <class T, class TC, bool TM> constexpr size_t sp_smem_bytes() { return SpGeom<T, TC, TM>::SMEM; }
template <class T, class TC, bool TM> constexpr int sp_tx() { return SpGeom<T, TC, TM>::TX; }
// resident CTAs per SM the register budget is cut for
template <class T, class TC, bool TM> constexpr int sp_minb() {
    return (sizeof(T) == 8 || SpGeom<T, TC, TM>::NP == 2) ? 2 : 3;
}

struct SpMaps;
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
    int* err;   // set to 1 when a staging wait gives up (TMA form)
    const int* stop; // batched launches: the realisation's stop flag (its items are skipped)
    // batched launches, the launch-wide argument only: work items [seg_off[s], seg_off[s+1])
    // belong to realisation segment s, whose arguments and tensor maps are seg_args[s] and
    // seg_maps[s] (device memory, 64-byte aligned)
    const int* seg_off;
    const SpArgs* seg_args;
    const SpMaps* seg_maps;
    int nseg, total;
};

// Tensor maps of the TMA form: x / b / cx / cz / cy boxes of W x (XR | CR | CR | CR | YR) x 1;
// bxm (ny x nz) box BXN x 1, bym (nx x nz) box W x 1, bzm (nx x ny) box W x CR.
struct SpMaps {
    CUtensorMap x, b, cx, cy, cz, bxm, bym, bzm;
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
// a coefficient pair (cells 2m, 2m+1) in the vector type
template <class T, class TC> __device__ __forceinline__ P2<T> sp_ldc(const TC* p) {
    if constexpr (std::is_same<TC, __nv_bfloat16>::value) {
        const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
        return P2<T>{(T)v.x, (T)v.y};
    } else {
        return sp_ld2<T>(reinterpret_cast<const T*>(p));
    }
}
template <class T, class TC> __device__ __forceinline__ T sp_c1(const TC* p) {
    if constexpr (std::is_same<TC, __nv_bfloat16>::value) return (T)__bfloat162float(*p);
    else return (T)*p;
}
template <class T> __device__ __forceinline__ void sp_st2(T* p, T a, T b) {
    if constexpr (sizeof(T) == 8) *reinterpret_cast<double2*>(p) = make_double2(a, b);
    else *reinterpret_cast<float2*>(p) = make_float2(a, b);
}
template <class T> __device__ __forceinline__ void sp_stg2(T* p, T a, T b) { sp_st2<T>(p, a, b); }

// cp.async of B bytes (4, 8 or 16) to a shared address; `ok` false reads nothing and zero-fills.
// 16-byte copies bypass L1 (.cg): staged data is never re-read through L1, and allocating it
// there measured 1.5x slower (FP64 plain sweep at 256^3: 0.363 ms with .ca, 0.246 ms with .cg).
template <int B> __device__ __forceinline__ void sp_cp(uint32_t dst, const char* src, bool ok) {
    if constexpr (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(B), "r"(ok ? B : 0)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(B), "r"(ok ? B : 0)
                     : "memory");
}

// BATCH: one launch sweeps the same level depth of several realisations (TMA form); the
// CTAs walk the concatenated (tile, z chunk) items of every realisation whose solve is running.
template <class T, class TC, int MODE, bool TM, bool BATCH = false>
__global__ void __launch_bounds__(SP_NT, (sp_minb<T, TC, TM>()))
    sweep_pair_kernel(const __grid_constant__ SpMaps maps0, const SpArgs<T, TC> a0) {
    static_assert(!BATCH || TM, "batched launches use the TMA form");
    static_assert((std::is_same<T, TC>::value && sizeof(T) >= 4) ||
                      (std::is_same<T, float>::value && std::is_same<TC, __nv_bfloat16>::value && TM),
                  "FP64 or FP32 vectors with coefficients of the same type, or FP32 / BF16 with TMA staging");
    constexpr bool ZERO = (MODE & M_ZERO) != 0, PROL = (MODE & M_PROLONG) != 0, DOT = (MODE & M_DOT) != 0;
    static_assert((MODE & M_RESID) == 0, "the residual runs in a kernel of its own");
    // the producer thread; FP64 prolongation sweeps keep it in tile warp 0 (measured faster
    // there: 0.181 against 0.193 ms at 256^3, where the other sweeps gain 5-9% in warp 9)
    constexpr int PROD = (PROL && sizeof(T) == 8) ? 0 : SP_PROD;
    using G = SpGeom<T, TC, TM>;
    constexpr int ST = G::ST, SC = G::SC, W = G::W, HX = G::HX, NP = G::NP, TX = G::TX;
    constexpr int QS = 32; // cells between the pairs of one lane (16 lanes x one pair each)
    extern __shared__ __align__(128) unsigned char sp_sm_raw[];
    // slots start on a 128-byte boundary of the shared window (TMA destinations)
    unsigned char* const sp_sm =
        sp_sm_raw + ((128u - ((uint32_t)__cvta_generic_to_shared(sp_sm_raw) & 127u)) & 127u);
    __shared__ __align__(8) uint64_t sp_full[SP_NSX]; // TMA form: one full barrier per group (x slot)
    T* const xs0 = reinterpret_cast<T*>(sp_sm); // x slot s at xs0 + s * XE
    constexpr int XE = (int)(G::XSB / ST), CE = (int)(G::CSB / ST);
    T* const cs0 = reinterpret_cast<T*>(sp_sm + SP_NSX * G::XSB); // coefficient slot s at cs0 + s * CE
    // arrays in a coefficient slot, in elements
    constexpr int OB = (int)(G::OB / ST), OCX = (int)(G::OCX / ST), OCY = (int)(G::OCY / ST);
    constexpr int OCZ = (int)(G::OCZ / ST), OBX = (int)(G::OBX / ST), OBY = (int)(G::OBY / ST);
    // the coefficient-typed arrays of slot s start at cof(s); their offsets in that type
    // (the cp.async form, where the types agree, uses the offsets above from cs0)
    constexpr int OCYc = (int)((G::OCY - G::OCX) / SC), OCZc = (int)((G::OCZ - G::OCX) / SC);
    constexpr int OBXc = (int)((G::OBX - G::OCX) / SC), OBYc = (int)((G::OBY - G::OCX) / SC);
    auto cof = [&](int sl) -> TC* {
        return reinterpret_cast<TC*>(reinterpret_cast<unsigned char*>(cs0 + sl * CE) + G::OCX);
    };
    const uint32_t xs0_u = (uint32_t)__cvta_generic_to_shared(xs0), cs0_u = (uint32_t)__cvta_generic_to_shared(cs0);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // work items of the launch: one realisation's, or (BATCH) every segment's
    const int gtotal = BATCH ? a0.total
                             : ((a0.L.nx + TX - 1) / TX) * ((a0.L.ny + SP_TY - 1) / SP_TY) *
                                   ((a0.L.nz + a0.zchunk - 1) / a0.zchunk);
    auto divide = [](T num, T den) -> T {
        if constexpr (sizeof(T) == 4) return __fdividef(num, den); // preconditioner: 2-ulp division
        else return num / den;
    };
    // role 0: tile pair (red + black + output); 1: ring-row pair (red); 2: ring-column cell (red)
    const int role = warp < 8 ? 0 : (warp == 8 ? 1 : 2);
    const int hi = lane >> 4, lo = lane & 15;
    // tile warps cover rows {r, r+2}: the red offset o = (j + t) & 1 is the same for the whole warp
    const int tyr = 4 * (warp >> 1) + (warp & 1) + 2 * hi;
    auto nxs = [](int s) { return s + 1 == SP_NSX ? 0 : s + 1; };
    auto ncs = [](int s) { return s + 1 == SP_NSC ? 0 : s + 1; };
    double dot_acc = 0.0;
    // TMA form: the producer thread issues every copy and waits on the groups' barriers
    unsigned phase = 0u; // producer: parity of the next wait, per barrier
    bool fail = false;
    if constexpr (TM) {
        if (tid == PROD) {
            for (int k = 0; k < SP_NSX; ++k) mbar_init(&sp_full[k], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }

    for (int gitem = blockIdx.x; gitem < gtotal && !fail; gitem += gridDim.x) {
        int sg = 0, item = gitem, nitems = gtotal; // segment, item within it, its item count
        if constexpr (BATCH) {
            sg = find_seg(a0.seg_off, a0.nseg, gitem);
            const int o = __ldg(a0.seg_off + sg);
            item = gitem - o;
            nitems = __ldg(a0.seg_off + sg + 1) - o;
        }
        const SpArgs<T, TC>& a = BATCH ? a0.seg_args[sg] : a0;
        const SpMaps& maps = BATCH ? a0.seg_maps[sg] : maps0;
        if constexpr (BATCH) {
            if (a.stop && *a.stop) continue; // that realisation's solve has finished (CTA-uniform)
        }
        const LevelOp<TC>& L = a.L;
        const int nx = L.nx, ny = L.ny, nz = L.nz;
        const size_t nxy = (size_t)nx * ny;
        const int ntx = (nx + TX - 1) / TX, ntiles = ntx * ((ny + SP_TY - 1) / SP_TY);
        const T dx2 = (T)L.dx2;
        if constexpr (TM) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads(); // the previous item's reads (and generic writes) of the slots are done
        if constexpr (BATCH) {
            if (tid == PROD) {
                // tensor maps read from global memory, written there by a host copy: the acquire
                // has system scope (a narrower scope may leave the TMA unit a stale descriptor
                // cached for the same address)
                const CUtensorMap* mp[8] = {&maps.x, &maps.b, &maps.cx, &maps.cy, &maps.cz, &maps.bxm, &maps.bym, &maps.bzm};
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(mp[k]) : "memory");
            }
        }
        const int tile = item % ntiles;
        const int z0 = (item / ntiles) * a.zchunk, z1 = min(z0 + a.zchunk, nz);
        const int i0 = (tile % ntx) * TX, j0 = (tile / ntx) * SP_TY;
        const int P0 = z0 - 2;          // first x plane staged
        const int XL = z1 + 1, CL = z1; // last x plane, last coefficient plane
        // slots: x plane p in (p - P0) mod SP_NSX, coefficient plane q in (q - P0) mod SP_NSC.
        // A group holds x plane p and coefficient plane p - 1; it is empty past both ends.
        auto real = [&](int p) { return (!ZERO && p <= XL) || (p - 1 >= P0 && p - 1 <= CL); };
        auto zin = [&](int t) { return (t >= 0 && t < nz) || L.per_z; };
        auto zzero = [&](int t) { return t == 0 || (L.per_z && t == nz); }; // plane t is plane 0
        // coarse correction of a pair (both cells share the parent) in plane p
        auto corr = [&](bool in_xy, int ii, int jj, int p) -> T {
            if (!PROL) return (T)0;
            const int kz = wrap_or_out(p, nz, L.per_z);
            if (!in_xy || kz < 0) return (T)0;
            return __ldg(a.e_c + (size_t)(ii >> 1) + (size_t)a.ncx * ((size_t)(jj >> 1) + (size_t)a.ncy * (size_t)(kz >> 1)));
        };
        // x pair staged at f of slot sx, with the correction added and written back for the others
        auto take = [&](int sx, int f, T e) -> P2<T> {
            T* sp = xs0 + sx * XE + f;
            P2<T> v{(T)0, (T)0};
            if constexpr (!ZERO) v = sp_ld2<T>(sp);
            if constexpr (PROL) {
                v.a += e;
                v.b += e;
                sp_st2<T>(sp, v.a, v.b);
            }
            return v;
        };
        int sxi = 0, sci = SP_NSC - 1; // slots of the next group's x plane and coefficient plane
        int next_wait = P0;            // the producer (TMA form): the next group to wait for
        // slots of the planes the first step (t = z0 - 1) reads: x t-1, t, t+1; coefficients t
        int sxm = 0, sx0 = 1, sx1 = 2, sc0 = 1;
        auto advance = [&]() { // the issue slots advance as the groups are issued
            sxm = sx0, sx0 = sx1, sx1 = nxs(sx1);
            sc0 = ncs(sc0);
        };
        // ---- TMA form: the producer's copies of group p and its waits ----
        auto tma_issue = [&](int p) {
            if constexpr (TM) {
                if (tid == PROD && real(p)) {
                    const int q = p - 1;
                    const bool dox = !ZERO && p <= XL, doc = q >= P0 && q <= CL;
                    uint64_t* bar = &sp_full[sxi];
                    unsigned bytes = 0;
                    if (dox) bytes += (unsigned)(SP_XR * W * ST);
                    if (doc) bytes += (unsigned)(SP_CR * W * ST + (2 * SP_CR + SP_YR) * W * SC + (i0 == 0 ? G::BXN * SC : 0) +
                                                 (j0 == 0 ? W * SC : 0));
                    mbar_expect_tx(bar, bytes);
                    if (dox) tma_load_3d(xs0 + sxi * XE, &maps.x, i0 - HX, j0 - 2, p, bar);
                    if (doc) {
                        T* C = cs0 + sci * CE;
                        TC* Cc = cof(sci);
                        tma_load_3d(C, &maps.b, i0 - HX, j0 - 1, q, bar);
                        tma_load_3d(Cc, &maps.cx, i0 - HX, j0 - 1, q, bar);
                        tma_load_3d(Cc + OCYc, &maps.cy, i0 - HX, j0 - 2, q, bar);
                        if (q == -1) // the -z faces of plane 0 stand in for plane -1's +z faces
                            tma_load_2d(Cc + OCZc, &maps.bzm, i0 - HX, j0 - 1, bar);
                        else
                            tma_load_3d(Cc + OCZc, &maps.cz, i0 - HX, j0 - 1, q, bar);
                        if (i0 == 0) tma_load_2d(Cc + OBXc, &maps.bxm, j0 - G::BXS, q, bar);
                        if (j0 == 0) tma_load_2d(Cc + OBYc, &maps.bym, i0 - HX, q, bar);
                    }
                }
            }
        };
        // the producer waits for group p (x slot s); the barrier publishes it (and this step's red
        // values); false when a wait gave up
        auto sync_step = [&](int p, int s) -> bool {
            if constexpr (TM) {
                bool bad = false;
                if (tid == PROD && real(p)) {
                    bad = !mbar_wait(&sp_full[s], (phase >> s) & 1u);
                    if (!bad) phase ^= 1u << s;
                }
                if (tid == PROD && !bad) next_wait = p + 1;
                // generic writes to the slots (red values, corrections) before later TMA writes
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                return !bar_red_or(1, SP_NT, bad);
            } else {
                asm volatile("cp.async.wait_group %0;" ::"n"(SP_D - 2) : "memory");
                asm volatile("bar.sync 0;" ::: "memory");
                return true;
            }
        };
        // the first two groups (x planes P0, P0 + 1, coefficients of plane P0)
        auto sync_prologue = [&]() -> bool {
            if constexpr (TM) {
                bool bad = false;
                if (tid == PROD) {
                    for (int p = P0; p <= P0 + 1 && !bad; ++p) {
                        if (real(p)) {
                            const int s = p - P0;
                            bad = !mbar_wait(&sp_full[s], (phase >> s) & 1u);
                            if (bad) break;
                            phase ^= 1u << s;
                        }
                        next_wait = p + 1;
                    }
                }
                return !bar_red_or(1, SP_NT, bad);
            } else {
                asm volatile("cp.async.wait_group %0;" ::"n"(SP_D - 1) : "memory");
                asm volatile("bar.sync 0;" ::: "memory");
                return true;
            }
        };
        // after a failed wait: the producer waits (bounded) for the groups it issued and nobody
        // waited for yet, so that no copy is in flight when the CTA leaves
        auto drain = [&](int p_last) {
            if constexpr (TM) {
                if (tid == PROD) {
                    atomicExch(a.err, 1);
                    for (int p = next_wait; p <= p_last; ++p) {
                        if (!real(p)) continue;
                        const int s = (p - P0) % SP_NSX;
                        (void)mbar_wait(&sp_full[s], (phase >> s) & 1u);
                        phase ^= 1u << s;
                    }
                }
            }
        };
        // the copies of one pair: x of plane p at fx, b / cx / cy / cz of plane p - 1 (cy at fx,
        // the others at fx - W); boundary planes wrap (periodic z), are zero, or take the -z faces
        // bzm for plane -1; `cxb` / `cyb`: the pair is the one left of x = 0 / below y = 0 of a
        // non-periodic axis, whose cx / cy stand for the boundary faces bxm / bym
        auto issue_pair = [&](int p, uint32_t xo, uint32_t co, bool pin, long long g, int wi_, int wj_, int fx_,
                              bool cxb, bool cyb, bool want_x, bool want_c) {
            const int q = p - 1;
            const bool dox = !ZERO && want_x && p <= XL, doc = want_c && q >= P0 && q <= CL;
            if (p >= 1 && p < nz && !cxb && !cyb) { // interior planes: one offset for all arrays
                const long long off = (g + (long long)nxy * p) * ST;
                if (dox) sp_cp<2 * ST>(xo + fx_ * ST, reinterpret_cast<const char*>(a.x_in) + (pin ? off : 0), pin);
                if (doc) {
                    const long long oq = pin ? off - (long long)nxy * ST : 0;
                    const uint32_t fcb = co + (fx_ - W) * ST;
                    sp_cp<2 * ST>(fcb + OB * ST, reinterpret_cast<const char*>(a.b) + oq, pin);
                    sp_cp<2 * ST>(fcb + OCX * ST, reinterpret_cast<const char*>(L.cx) + oq, pin);
                    sp_cp<2 * ST>(co + (OCY + fx_) * ST, reinterpret_cast<const char*>(L.cy) + oq, pin);
                    sp_cp<2 * ST>(fcb + OCZ * ST, reinterpret_cast<const char*>(L.cz) + oq, pin);
                }
                return;
            }
            T* X = reinterpret_cast<T*>(sp_sm + (xo - xs0_u));
            T* Cb = reinterpret_cast<T*>(sp_sm + (co - xs0_u));
            // (boundary planes and boundary tiles only: the L1-allocating copy is fine here)
            const int fc_ = fx_ - W;
            if (dox) {
                const int kz = wrap_or_out(p, nz, L.per_z);
                const bool ok = pin && kz >= 0;
                pmv_cp<2 * ST>(X + fx_, a.x_in + (ok ? (size_t)g + nxy * (size_t)kz : 0), ok);
            }
            if (doc) {
                const int kz = wrap_or_out(q, nz, L.per_z);
                const bool kin = kz >= 0;
                const bool ok = pin && kin;
                const size_t gq = ok ? (size_t)g + nxy * (size_t)kz : 0;
                pmv_cp<2 * ST>(Cb + OB + fc_, a.b + gq, ok);
                if (cxb) { // -x face of cell (0, wj_): one value into the column of cell -1
                    const bool okb = wj_ >= 0 && kin;
                    pmv_cp<ST>(Cb + OCX + fc_ + 1, L.bxm + (okb ? (size_t)wj_ + (size_t)ny * kz : 0), okb);
                } else {
                    pmv_cp<2 * ST>(Cb + OCX + fc_, L.cx + gq, ok);
                }
                if (cyb) { // -y faces of the pair's cells in row 0
                    const bool okb = wi_ >= 0 && kin;
                    pmv_cp<2 * ST>(Cb + OCY + fx_, L.bym + (okb ? (size_t)wi_ + (size_t)nx * kz : 0), okb);
                } else {
                    pmv_cp<2 * ST>(Cb + OCY + fx_, L.cy + gq, ok);
                }
                if (q == -1 && !L.per_z) { // the -z faces of plane 0 stand in for plane -1's +z faces
                    pmv_cp<2 * ST>(Cb + OCZ + fc_, L.bzm + (pin ? (size_t)g : 0), pin);
                } else {
                    pmv_cp<2 * ST>(Cb + OCZ + fc_, L.cz + gq, ok);
                }
            }
        };
        auto slot_u = [&](int sx, int sc, uint32_t& xo, uint32_t& co) {
            xo = xs0_u + (uint32_t)(sx * XE * ST);
            co = cs0_u + (uint32_t)(sc * CE * ST);
        };

        if (role == 0) {
            // =============== tile pairs: red of plane t and black of plane t-1 ===============
            // NP pairs per thread in one row: pair q starts at cell i0 + 2 lo + QS q, so that the
            // 16 lanes of a row read and write consecutive pairs
            const int pj = j0 + tyr, pi0 = i0 + 2 * lo;
            const int wj = pj < ny ? pj : -1; // never wrapped
            const int fx = (pj - j0 + 2) * W + (pi0 - i0 + HX), fc = fx - W;
            bool pin[NP];
            long long gxy[NP];
            int cxl_off[NP], cyd_off[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const int pi = pi0 + QS * q;
                pin[q] = pi < nx && wj >= 0;
                gxy[q] = pin[q] ? (long long)pi + (long long)nx * wj : 0;
                // the -x face of cell pi - 1 and the -y faces of the pair: from the boundary-face
                // buffers where the TMA form stages them, else from the cx / cy slots
                cxl_off[q] = (TM && i0 == 0 && pi == 0) ? OBXc + (pj - j0 + G::BXS) : fc + QS * q - 1;
                cyd_off[q] = (TM && j0 == 0 && pj == 0) ? OBYc + (pi - i0 + HX) : OCYc + fx + QS * q - W;
            }
            auto issue = [&](int p) {
                if constexpr (TM) {
                    tma_issue(p);
                } else {
                    uint32_t xo, co;
                    slot_u(sxi, sci, xo, co);
                    issue_pair(p, xo, co, pin[0], gxy[0], pi0, wj, fx, false, false, true, true);
                    asm volatile("cp.async.commit_group;" ::: "memory");
                }
                sxi = nxs(sxi);
                sci = ncs(sci);
            };
#pragma unroll
            for (int q = 0; q <= SP_D; ++q) issue(P0 + q);
            if (!sync_prologue()) {
                drain(P0 + SP_D);
                fail = true;
                break;
            }
            const int wpar = warp & 1; // parity of this warp's rows (j0 is even)
            const int O0 = (wpar + z0 - 1) & 1;
            // carried, per pair: A = x(t).at(1-O), B = x(t-1).at(O), the red values of planes t-1
            // (column 1-O) and t-2 (column O), the black cell's coefficients of plane t-1
            // (column O), cz of planes t-1 and t-2
            T A[NP], B[NP], red1[NP], red2[NP], kb[NP], kxp[NP], kxm[NP], kyp[NP], kym[NP], en[NP];
            P2<T> czp1[NP], czp2[NP];
            double2 r64n[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const int pi = pi0 + QS * q;
                const P2<T> xp0 = take(0, fx + QS * q, corr(pin[q], pi, wj, P0)); // x(P0): own column only
                const P2<T> xp1 = take(1, fx + QS * q, corr(pin[q], pi, wj, P0 + 1)); // x(P0 + 1), published
                en[q] = corr(pin[q], pi, wj, P0 + 2); // correction of the pair in plane t + 1
                czp1[q] = sp_ldc<T, TC>(cof(0) + OCZc + fc + QS * q);
                czp2[q] = P2<T>{(T)0, (T)0};
                A[q] = O0 ? xp1.a : xp1.b;
                B[q] = O0 ? xp0.b : xp0.a;
                red1[q] = red2[q] = kb[q] = kxp[q] = kxm[q] = kyp[q] = kym[q] = (T)0;
                r64n[q] = make_double2(0.0, 0.0);
            }

            auto step = [&](auto Oc, int t) {
                constexpr int O = decltype(Oc)::value;
                issue(t + SP_D);
                const T* C = cs0 + sc0 * CE;
                const TC* Cc = cof(sc0);
                T* X0 = xs0 + sx0 * XE;
                const T* X1 = xs0 + sxm * XE;
                const int q_out = t - 1;
                const bool out_ok = q_out >= z0 && q_out < z1;
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const int f = fx + QS * q, g = fc + QS * q;
                    // ---- x of plane t+1 (own column; published for the neighbours with PROL) ----
                    T xnO;
                    if constexpr (PROL) {
                        const P2<T> v = take(sx1, f, en[q]);
                        xnO = O ? v.b : v.a;
                        en[q] = corr(pin[q], pi0 + QS * q, wj, t + 2);
                    } else if constexpr (ZERO) {
                        xnO = (T)0;
                    } else {
                        xnO = xs0[sx1 * XE + f + O];
                    }
                    // ---- coefficients of plane t ----
                    const P2<T> b2 = sp_ld2<T>(C + OB + g), cx2p = sp_ldc<T, TC>(Cc + g);
                    const P2<T> cy2p = sp_ldc<T, TC>(Cc + OCYc + f), cyd2 = sp_ldc<T, TC>(Cc + cyd_off[q]);
                    const P2<T> cz2 = sp_ldc<T, TC>(Cc + OCZc + g);
                    const T cxl = sp_c1<T, TC>(Cc + cxl_off[q]);
                    // ---- red cell pi + O of plane t, from old black values ----
                    T red = (T)0;
                    {
                        T xout = (T)0, xsv = (T)0, xnv = (T)0;
                        if constexpr (!ZERO || PROL) {
                            xout = X0[f - 1 + 3 * O];
                            xsv = X0[f - W + O];
                            xnv = X0[f + W + O];
                        }
                        const T xw = O ? A[q] : xout, xe = O ? xout : A[q];
                        const T cxp = O ? cx2p.b : cx2p.a, cxm = O ? cx2p.a : cxl;
                        const T cyp = O ? cy2p.b : cy2p.a, cym = O ? cyd2.b : cyd2.a;
                        const T czp = O ? cz2.b : cz2.a, czm = O ? czp1[q].b : czp1[q].a;
                        T D = cxm + cxp + cym + cyp + czm + czp;
                        if (O == 0 && L.pin && pi0 + QS * q == 0 && pj == 0 && zzero(t)) D *= (T)2; // cell 0 is red
                        const T sum = cxp * xe + cxm * xw + cyp * xnv + cym * xsv + czp * xnO + czm * B[q];
                        const T bb = O ? b2.b : b2.a;
                        if (pin[q] && zin(t)) red = divide(sum - bb * dx2, D);
                    }
                    X0[f + O] = red;
                    // ---- black cell pi + O of plane t-1 from red values; plane t-1 is then final ----
                    if (out_ok && pin[q]) {
                        const T xout = X1[f - 1 + 3 * O], xsv = X1[f - W + O], xnv = X1[f + W + O];
                        const T xw = O ? red1[q] : xout, xe = O ? xout : red1[q];
                        const T kzp = O ? czp1[q].b : czp1[q].a, kzm = O ? czp2[q].b : czp2[q].a;
                        const T D = kxm[q] + kxp[q] + kym[q] + kyp[q] + kzm + kzp;
                        const T sum = kxp[q] * xe + kxm[q] * xw + kyp[q] * xnv + kym[q] * xsv + kzp * red + kzm * red2[q];
                        const T blk = divide(sum - kb[q] * dx2, D);
                        const T va = O ? red1[q] : blk, vb = O ? blk : red1[q];
                        sp_stg2<T>(a.x_out + (size_t)gxy[q] + nxy * (size_t)q_out, va, vb);
                        if constexpr (DOT) dot_acc += r64n[q].x * (double)va + r64n[q].y * (double)vb;
                    }
                    if constexpr (DOT) { // r64 of plane t, for the output of plane t at the next step
                        const bool out_t = t >= z0 && t < z1 && pin[q];
                        r64n[q] = out_t ? __ldg(reinterpret_cast<const double2*>(a.r64 + (size_t)gxy[q] + nxy * (size_t)t))
                                        : make_double2(0.0, 0.0);
                    }
                    // ---- carry to the next plane (red offset 1 - O) ----
                    B[q] = A[q];
                    A[q] = xnO;
                    red2[q] = red1[q];
                    red1[q] = red;
                    kb[q] = O ? b2.a : b2.b;
                    kxp[q] = O ? cx2p.a : cx2p.b;
                    kxm[q] = O ? cxl : cx2p.a;
                    kyp[q] = O ? cy2p.a : cy2p.b;
                    kym[q] = O ? cyd2.a : cyd2.b;
                    czp2[q] = czp1[q];
                    czp1[q] = cz2;
                }
            };
            using Z = std::integral_constant<int, 0>;
            using I = std::integral_constant<int, 1>;
            for (int t = z0 - 1; t <= z1; ++t) {
                // x plane t+1 and the coefficients of plane t have landed; the barrier publishes
                // them and the red values of plane t-1, and frees the slots of x plane t-2 and
                // coefficient plane t-1
                if (!sync_step(t + 1, sx1)) {
                    drain(t + SP_D - 1);
                    fail = true;
                    break;
                }
                if (((wpar + t) & 1) == 0) step(Z{}, t);
                else step(I{}, t);
                advance();
            }
        } else {
            // =============== ring pairs / cells: red of plane t only ===============
            // ring-row lanes: NP pairs side by side; ring-column lanes: one cell (its side pair)
            int pj, pi0, side = -1;
            if (role == 1) pj = hi ? j0 + SP_TY : j0 - 1, pi0 = i0 + 2 * lo;
            else side = hi, pj = j0 + lo, pi0 = hi ? i0 + TX : i0 - 2;
            const int npair = role == 1 ? NP : 1;
            const int wj = wrap_or_out(pj, ny, L.per_y);
            const int fx = (pj - j0 + 2) * W + (pi0 - i0 + HX), fc = fx - W;
            // second x pair(s): the ring-row warp the outer rows, ring-column lanes 0/1 of each
            // side the corner pairs (rows j0-1, j0+TY)
            int sj = 0;
            bool has2 = false;
            if (role == 1) has2 = true, sj = hi ? j0 + SP_TY + 1 : j0 - 2;
            else if (lo == 0 || lo == 1) has2 = true, sj = lo ? j0 + SP_TY : j0 - 1;
            const int wj2 = wrap_or_out(sj, ny, L.per_y);
            const int fx2 = (sj - j0 + 2) * W + (pi0 - i0 + HX);
            // coefficients beyond the pair's own (cp.async form): cx of the left corner pairs
            // (ring-column lanes 0 / 1 of the left side: the -x faces of the ring-row cells at
            // i0), cy of the row below the ring row (ring-row lanes 0-15) and of row j0-1 beside
            // the tile (ring-column lanes 0 / 16: the -y faces of the ring-column cells at j0)
            const bool cx2 = role == 2 && side == 0 && has2;
            const bool cy2 = (role == 1 && !hi) || (role == 2 && lo == 0);
            const int cy2j = role == 1 ? j0 - 2 : j0 - 1;
            const int wcy2 = wrap_or_out(cy2j, ny, L.per_y);
            const bool cy_bnd = pj == -1 && !L.per_y;
            const bool cy2_bnd = cy2j == -1 && !L.per_y;
            const int fyy = (cy2j - j0 + 2) * W + (pi0 - i0 + HX);
            int wi[NP], cxl_off[NP], cyd_off[NP];
            bool pin[NP], pin2[NP], cx_bnd[NP];
            long long gxy[NP], gxy2[NP], gcy2[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const int pi = pi0 + QS * q;
                wi[q] = wrap_or_out(pi, nx, L.per_x);
                pin[q] = q < npair && wi[q] >= 0 && wj >= 0;
                gxy[q] = pin[q] ? (long long)wi[q] + (long long)nx * wj : 0;
                pin2[q] = q < npair && has2 && wi[q] >= 0 && wj2 >= 0;
                gxy2[q] = pin2[q] ? (long long)wi[q] + (long long)nx * wj2 : 0;
                gcy2[q] = (wi[q] >= 0 && wcy2 >= 0) ? (long long)wi[q] + (long long)nx * wcy2 : 0;
                cx_bnd[q] = pi == -2 && !L.per_x;
                cxl_off[q] = (TM && i0 == 0 && pi == 0) ? OBXc + (pj - j0 + G::BXS) : fc + QS * q - 1;
                cyd_off[q] = (TM && j0 == 0 && pj == 0) ? OBYc + (pi - i0 + HX) : OCYc + fx + QS * q - W;
            }
            auto issue = [&](int p) {
                if constexpr (!TM) { // (one pair per lane: NP == 1 in this form)
                    uint32_t xo, co;
                    slot_u(sxi, sci, xo, co);
                    issue_pair(p, xo, co, pin[0], gxy[0], wi[0], wj, fx, cx_bnd[0], cy_bnd, true, true);
                    if (has2) { // x of the second pair; cx of a corner pair
                        issue_pair(p, xo, co, pin2[0], gxy2[0], wi[0], wj2, fx2, false, false, true, false);
                        if (cx2) { // only cx of plane p - 1 (b, cy, cz of the corner are not read)
                            const int q = p - 1;
                            if (q >= P0 && q <= CL) {
                                T* Cb = reinterpret_cast<T*>(sp_sm + (co - xs0_u));
                                const int kz = wrap_or_out(q, nz, L.per_z);
                                const bool kin = kz >= 0;
                                if (cx_bnd[0]) {
                                    const bool okb = wj2 >= 0 && kin;
                                    pmv_cp<ST>(Cb + OCX + fx2 - W + 1, L.bxm + (okb ? (size_t)wj2 + (size_t)ny * kz : 0), okb);
                                } else {
                                    const bool ok2 = pin2[0] && kin;
                                    pmv_cp<2 * ST>(Cb + OCX + fx2 - W,
                                                   L.cx + (ok2 ? (size_t)gxy2[0] + nxy * (size_t)kz : 0), ok2);
                                }
                            }
                        }
                    }
                    if (cy2) { // cy of plane p - 1 in row cy2j
                        const int q = p - 1;
                        if (q >= P0 && q <= CL) {
                            T* Cb = reinterpret_cast<T*>(sp_sm + (co - xs0_u));
                            const int kz = wrap_or_out(q, nz, L.per_z);
                            const bool kin = kz >= 0;
                            if (cy2_bnd) {
                                const bool okb = wi[0] >= 0 && kin;
                                pmv_cp<2 * ST>(Cb + OCY + fyy, L.bym + (okb ? (size_t)wi[0] + (size_t)nx * kz : 0), okb);
                            } else {
                                const bool ok2 = wi[0] >= 0 && wcy2 >= 0 && kin;
                                pmv_cp<2 * ST>(Cb + OCY + fyy, L.cy + (ok2 ? (size_t)gcy2[0] + nxy * (size_t)kz : 0), ok2);
                            }
                        }
                    }
                    asm volatile("cp.async.commit_group;" ::: "memory");
                } else {
                    tma_issue(p); // (the producer thread may be in this role)
                }
                sxi = nxs(sxi);
                sci = ncs(sci);
            };
#pragma unroll
            for (int q = 0; q <= SP_D; ++q) issue(P0 + q);
            if (!sync_prologue()) {
                drain(P0 + SP_D);
                fail = true;
                break;
            }
            P2<T> xprev[NP], xcur[NP], czp1[NP];
            T en[NP], en2[NP];
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                // (a ring-column lane has one pair: its slot neighbour belongs to the tile, and the
                // correction written back by take() must not touch it)
                xprev[q] = xcur[q] = czp1[q] = P2<T>{(T)0, (T)0};
                en[q] = en2[q] = (T)0;
                if (q >= npair) continue;
                xprev[q] = take(0, fx + QS * q, corr(pin[q], wi[q], wj, P0));
                xcur[q] = take(1, fx + QS * q, corr(pin[q], wi[q], wj, P0 + 1));
                if (has2) (void)take(1, fx2 + QS * q, corr(pin2[q], wi[q], wj2, P0 + 1));
                en[q] = corr(pin[q], wi[q], wj, P0 + 2);
                en2[q] = has2 ? corr(pin2[q], wi[q], wj2, P0 + 2) : (T)0;
                czp1[q] = sp_ldc<T, TC>(cof(0) + OCZc + fc + QS * q);
            }
            for (int t = z0 - 1; t <= z1; ++t) {
                if (!sync_step(t + 1, sx1)) {
                    drain(t + SP_D - 1);
                    fail = true;
                    break;
                }
                issue(t + SP_D);
                const int o = (pj + t) & 1;
                const T* C = cs0 + sc0 * CE;
                const TC* Cc = cof(sc0);
                T* X0 = xs0 + sx0 * XE;
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    if (q >= npair) break;
                    const int f = fx + QS * q, g = fc + QS * q;
                    const P2<T> xnext = take(sx1, f, en[q]);
                    if (has2) (void)take(sx1, fx2 + QS * q, en2[q]);
                    if constexpr (PROL) {
                        en[q] = corr(pin[q], wi[q], wj, t + 2);
                        if (has2) en2[q] = corr(pin2[q], wi[q], wj2, t + 2);
                    }
                    const P2<T> b2 = sp_ld2<T>(C + OB + g), cx2p = sp_ldc<T, TC>(Cc + g);
                    const P2<T> cy2p = sp_ldc<T, TC>(Cc + OCYc + f), cyd2 = sp_ldc<T, TC>(Cc + cyd_off[q]);
                    const P2<T> cz2 = sp_ldc<T, TC>(Cc + OCZc + g);
                    const T cxl = sp_c1<T, TC>(Cc + cxl_off[q]);
                    if (role == 1 || o != side) { // a ring-column cell is relaxed where it is red
                        T xout = (T)0, xsv = (T)0, xnv = (T)0;
                        if constexpr (!ZERO || PROL) {
                            xout = X0[f - 1 + 3 * o];
                            xsv = X0[f - W + o];
                            xnv = X0[f + W + o];
                        }
                        const T xin = xcur[q].at(1 - o);
                        const T xw = o ? xin : xout, xe = o ? xout : xin;
                        const T cxp = cx2p.at(o), cxm = o ? cx2p.a : cxl;
                        const T cyp = cy2p.at(o), cym = cyd2.at(o), czp = cz2.at(o), czm = czp1[q].at(o);
                        T D = cxm + cxp + cym + cyp + czm + czp;
                        if (L.pin && wi[q] == 0 && wj == 0 && o == 0 && zzero(t)) D *= (T)2;
                        const T sum = cxp * xe + cxm * xw + cyp * xnv + cym * xsv + czp * xnext.at(o) +
                                      czm * xprev[q].at(o);
                        T red = (T)0;
                        if (pin[q] && zin(t)) red = divide(sum - b2.at(o) * dx2, D);
                        X0[f + o] = red;
                    }
                    xprev[q] = xcur[q];
                    xcur[q] = xnext;
                    czp1[q] = cz2;
                }
                advance();
            }
        }
        if constexpr (!TM) asm volatile("cp.async.wait_all;" ::: "memory");
        if constexpr (BATCH && DOT) {
            // this item's share of <r64, x_out>; the last item of the realisation adds the
            // items' partials in index order (deterministic)
            __shared__ double sp_red[SP_NT / 32];
            double v = dot_acc;
            dot_acc = 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) sp_red[warp] = v;
            __syncthreads();
            if (tid == 0 && !fail) {
                double sum = 0.0;
                for (int w = 0; w < SP_NT / 32; ++w) sum += sp_red[w];
                a.dot_partials[item] = sum;
                __threadfence();
                if (atomicAdd(a.dot_ticket, 1u) == (unsigned)nitems - 1) {
                    __threadfence();
                    double acc = 0.0;
                    for (int i = 0; i < nitems; ++i) acc += __ldcg(a.dot_partials + i);
                    *a.dot_out = acc;
                    *a.dot_ticket = 0u;
                }
            }
            __syncthreads();
        }
    }
    if constexpr (DOT && !BATCH) {
        double v[1] = {dot_acc}, out[1];
        if (grid_sums<SP_NT, 1>(v, a0.dot_partials, a0.dot_ticket, gridDim.x, out)) *a0.dot_out = out[0];
    }
}

} // namespace mf3d

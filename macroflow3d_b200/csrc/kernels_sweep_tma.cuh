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
// Every thread owns one quad: four x-consecutive cells starting on a 16-byte boundary of the
// staged box, two red and two black in every plane.  The black cells of plane t-1 lie in the
// columns of the red cells of plane t.  All loads, the output and the residual move 16 bytes
// per access.  Every value a stage reads from another thread was written before the previous
// step's barrier: ONE __syncthreads per plane.
//
// Instruction economy.  The quads of a warp all lie in rows of one parity, so the offset of
// the red cells inside the quad, (row + t) & 1, is the same for the whole warp; the march is
// unrolled by two and each step is compiled for its offset.  Stages compute unconditionally
// and predicate only their stores.  Without RESID the black cells' coefficients of plane t
// are kept in registers for the next step (double-buffered by the unrolling); RESID keeps
// three coefficient planes staged instead and reads the black stage's and the residual's
// coefficients from them.  The -x and -y faces of a quad come from one precomputed
// shared-memory offset each, which points at the staged boundary faces on the min faces.
//
// Staging.  Two rings fed by cp.async.bulk.tensor.3d; thread 0 issues the copies and waits
// on their mbarriers (bounded) at the end of the step before the one that reads them, so the
// step barrier publishes the landed planes:
//   x ring (NRX slots): planes t+1 .. t-2 are live at step t (box rows j0-H .. j0+TY+H-1);
//   coefficient ring (NRC slots, LC live): b, cx, cz (rows j0-RR ..), cy (rows j0-H ..), the
//     -x faces of the box rows and the -y faces of the box columns when the tile touches
//     those boundaries; for plane -1 the -z faces take the place of cz.
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
    const int* stop; // batched launches: the realisation's stop flag (its items are skipped)
    // batched launches, the launch-wide argument only: work items [seg_off[s], seg_off[s+1])
    // belong to realisation segment s, whose arguments and tensor maps are seg_args[s] and
    // seg_maps[s] (device memory, 64-byte aligned)
    const int* seg_off;
    const TmaSweepArgs* seg_args;
    const TmaMaps* seg_maps;
    int nseg, total;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false if it gave up after `tries` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int tries = 1 << 22) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < tries; ++it) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Barrier `id` among the first `n` threads of the CTA, OR-reducing a flag.
__device__ __forceinline__ bool bar_red_or(int id, int n, bool v) {
    unsigned r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}"
                 : "=r"(r)
                 : "r"((unsigned)v), "r"(id), "r"(n)
                 : "memory");
    return r != 0;
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
    static constexpr int TX = 64, TY = 8;
    // quads start on 4-element boundaries of the box (16 bytes of T) and on TMA's alignment
    static constexpr int HXA = TmaGeom<T, TC>::lcm_elts() > 4 ? TmaGeom<T, TC>::lcm_elts() : 4;
    static constexpr int HX = ((4 + HXA - 1) / HXA) * HXA;
    static constexpr int BX = TX + 2 * HX;
    static constexpr int BY = TY + 2 * H;       // x box rows, from j0 - H
    static constexpr int BYC = TY + 2 * RR;     // b, cx, cz box rows, from j0 - RR
    static constexpr int BYY = TY + 2 * RR + 1; // cy box rows, from j0 - H
    // quads cover columns [i0-4, i0+TX+4) and rows [j0-2, j0+TY+2) (ring 2 in every mode, so
    // that the layout is the same; rows beyond the live ring compute nothing they store).
    // The NMQ interior quads of a row lie in NMQ consecutive lanes; MW warps of interior
    // quads per row parity, then one warp with the 2 edge quads of every row (both parities),
    // then the producer warp.
    static constexpr int NQ = TX / 4 + 2, NMQ = TX / 4, Q0 = HX - 4;
    static constexpr int RI = 2;
    static constexpr int IH = TY + 2 * RI, NRW = IH / 2;
    static_assert(RR <= RI && (!PROL || H <= RI) && H <= 4, "quad rows cover the live rings inside the box");
    static_assert((NMQ * NRW) % 32 == 0 && 4 * NRW <= 32, "interior quads fill whole warps, edge quads one");
    static constexpr int MW = NMQ * NRW / 32;
    static constexpr int NCONS = (2 * MW + 1) * 32; // consumer threads; one producer warp follows
    static constexpr int NT = NCONS + 32;
    static constexpr size_t align128(size_t v) { return (v + 127) & ~(size_t)127; }
    static constexpr size_t XB = (size_t)BX * BY * sizeof(T);
    static constexpr size_t BB = (size_t)BX * BYC * sizeof(T), CCB = (size_t)BX * BYC * sizeof(TC);
    static constexpr size_t CYB = (size_t)BX * BYY * sizeof(TC);
    static constexpr size_t XS = align128(XB);
    // -x boundary faces of the box rows, from row j0 - BYS (BYS * sizeof(TC) a multiple of 16)
    static constexpr int AL = 16 / (int)sizeof(TC);
    static constexpr int BYS = ((4 + AL - 1) / AL) * AL;
    static constexpr int BYP = ((TY + BYS + 4 + AL - 1) / AL) * AL;
    static_assert(BYS >= H, "boundary rows must cover the halo");
    static constexpr size_t BXMB = (size_t)BYP * sizeof(TC), BYMB = (size_t)BX * sizeof(TC);
    // coefficient slot: b, cx, cy, cz, bxm, bym
    static constexpr size_t C_CX = align128(BB), C_CY = C_CX + align128(CCB), C_CZ = C_CY + align128(CYB);
    static constexpr size_t C_BXM = C_CZ + align128(CCB), C_BYM = C_BXM + align128(BXMB);
    static constexpr size_t CS = C_BYM + align128(BYMB);
    static constexpr unsigned C_TX = (unsigned)(BB + 2 * CCB + CYB); // bytes of one plane without boundaries
    static constexpr size_t RS = RESID ? align128(3 * (size_t)TX * TY * sizeof(T)) : 0;
    // two CTAs per SM in FP32 (one CTA's barrier waits overlap the other's work); one in FP64
    static constexpr int MINB = sizeof(T) == 8 ? 1 : 2;
    static constexpr size_t BUDGET = MINB == 2 ? 112 * 1024 : 225 * 1024;
    static constexpr int LC = RESID ? 3 : 1; // coefficient planes read at step t: t .. t-LC+1
    // the x ring starts one guard row in: neighbour reads of edge quads may reach one box row
    // before the first slot (they are never used)
    static constexpr size_t GUARD = align128((size_t)BX * sizeof(T) + 16);
    static constexpr int NRX = 7; // 4 live x planes + 3 in flight
    static constexpr int NRC_FIT = (int)((BUDGET - 256 - GUARD - RS - NRX * XS) / CS);
    static constexpr int NRC = NRC_FIT < 8 ? NRC_FIT : 8;
    static_assert(NRC >= LC + 2 && 2 * (NRX + NRC) * 8 <= 256, "coefficient ring: two planes in flight");
    static constexpr size_t OFF_X = 256 + GUARD;
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

// Four consecutive values; lane k of a quad.
template <class T> struct Q4 {
    T v[4];
};
template <class T, class E> __device__ __forceinline__ Q4<T> ldq(const E* p) {
    Q4<T> q;
    if constexpr (std::is_same<E, float>::value) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        q.v[0] = (T)a.x, q.v[1] = (T)a.y, q.v[2] = (T)a.z, q.v[3] = (T)a.w;
    } else if constexpr (std::is_same<E, double>::value) {
        const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
        q.v[0] = (T)a.x, q.v[1] = (T)a.y, q.v[2] = (T)b.x, q.v[3] = (T)b.y;
    } else {
        const uint2 raw = *reinterpret_cast<const uint2*>(p);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
        q.v[0] = (T)a.x, q.v[1] = (T)a.y, q.v[2] = (T)b.x, q.v[3] = (T)b.y;
    }
    return q;
}
template <class T> __device__ __forceinline__ void stq(T* p, const Q4<T>& q) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2(q.v[0], q.v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(q.v[2], q.v[3]);
    }
}
// A quad's coefficients of one plane: b, the +x/+y/+z faces, the -y faces and the -x face
// of cell 0 (the -x face of cell k > 0 is cx[k-1]).
template <class T> struct QuadCoef {
    Q4<T> b, cx, cy, cz, cyd;
    T cxl;
};
// The two black cells' coefficients (cells O and O+2 of the next plane's quad), kept for the
// next step.
template <class T> struct BlackCoef {
    T b[2], cxp[2], cxm[2], cyp[2], cym[2], czp[2];
};

// BATCH: one launch sweeps the same level depth of several realisations; the persistent CTAs
// walk the concatenated (tile, z chunk) items of every realisation whose solve is running.
template <class T, class TC, int MODE, bool BATCH = false>
__global__ void __launch_bounds__(TmaSweepCfg<T, TC, MODE>::NT, TmaSweepCfg<T, TC, MODE>::MINB)
    sweep_tma_kernel(const __grid_constant__ TmaMaps maps0, const TmaSweepArgs<T, TC> a0) {
    using C = TmaSweepCfg<T, TC, MODE>;
    constexpr bool ZERO = C::ZERO, PROL = C::PROL, RESID = C::RESID;
    constexpr bool DOT = (MODE & M_DOT) != 0;
    constexpr int TX = C::TX, TY = C::TY, BX = C::BX, H = C::H, HX = C::HX, RR = C::RR, RB = C::RB;
    constexpr int NRX = C::NRX, NRC = C::NRC, LC = C::LC;
    extern __shared__ __align__(128) unsigned char sweep_sm[];
    // "full" barriers (a plane landed) of the x and coefficient rings, then "empty" barriers
    // (the consumers released a slot)
    uint64_t* barx = reinterpret_cast<uint64_t*>(sweep_sm);
    uint64_t* barc = barx + NRX;
    uint64_t* emx = barc + NRC;
    uint64_t* emc = emx + NRX;
    // planes issued so far by the producer (read by the consumers only to drain after a failure)
    volatile int* issued = reinterpret_cast<volatile int*>(sweep_sm + 2 * 8 * (NRX + NRC));
    T* rsb = reinterpret_cast<T*>(sweep_sm + C::OFF_R);
    auto xsl = [&](int s) { return reinterpret_cast<T*>(sweep_sm + C::OFF_X + C::XS * s); };
    auto cbase = [&](int s) { return sweep_sm + C::OFF_C + C::CS * s; };

    const int tid = threadIdx.x;
    auto divide = [](T num, T den) -> T {
        if constexpr (sizeof(T) == 4) return __fdividef(num, den); // preconditioner: 2-ulp division
        else return num / den;
    };
    auto tc = [](TC v) -> T { return ld_as_float_or_double<T>(v); };

    if (tid == 0) {
        for (int s = 0; s < 2 * (NRX + NRC); ++s) mbar_init(&barx[s], 1);
        issued[0] = issued[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // ring bookkeeping.  Every thread tracks the planes staged so far (qx, qc) and the slots of
    // the planes it reads.  The producer warp's lane 0 issues the copies, each into a slot the
    // consumers released; consumer thread 0 waits for the landed planes (phases in phx / phc)
    // at the end of the step before the one that reads them, and releases the slots of the
    // planes no longer read.
    const bool producer = tid >= C::NCONS;
    unsigned qx = 0, qc = 0;
    int xw_slot = 0, cw_slot = 0, rx_slot = 0, rc_slot = 0; // consumer thread 0: next to wait / release
    unsigned phx = 0u, phc = 0u;
    double dot_acc = 0.0;
    bool fail = false;
    auto nxt_x = [](int s) { return s + 1 == NRX ? 0 : s + 1; };
    auto nxt_c = [](int s) { return s + 1 == NRC ? 0 : s + 1; };
    auto prv_c = [](int s) { return s == 0 ? NRC - 1 : s - 1; };
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
    auto release_x = [&]() {
        mbar_arrive(&emx[rx_slot]);
        rx_slot = nxt_x(rx_slot);
    };
    auto release_c = [&]() {
        mbar_arrive(&emc[rc_slot]);
        rc_slot = nxt_c(rc_slot);
    };

    // ---- this thread's quad within a tile (tile-independent part) ----
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NRW = C::NRW, NMQ = C::NMQ, MW = C::MW;
    int cls = 0, rq = 0, qc_ = 1;
    bool iv = false, mainq = false;
    if (warp < 2 * MW) { // interior quads of one row parity
        cls = warp / MW;
        const int idx = (warp - cls * MW) * 32 + lane;
        iv = mainq = true;
        rq = idx / NMQ;
        qc_ = 1 + idx % NMQ;
    } else if (warp == 2 * MW && lane < 4 * NRW) { // edge quads: lanes by parity, then row
        cls = lane >= 2 * NRW;
        const int k = lane - cls * 2 * NRW;
        iv = true;
        rq = k >> 1;
        qc_ = (k & 1) ? C::NQ - 1 : 0;
    }
    // the quads left and right of an interior quad are the neighbouring lanes, except at the
    // ends of a row; the edge warp (both parities, diverging on the red offset) reads them
    const bool fb_l = !(mainq && qc_ >= 2), fb_r = !(mainq && qc_ <= C::NQ - 3);
    const bool edge_warp = warp >= 2 * MW; // uniform in a warp
    auto from_left = [&](T v) { return edge_warp ? v : __shfl_up_sync(0xffffffffu, v, 1); };
    auto from_right = [&](T v) { return edge_warp ? v : __shfl_down_sync(0xffffffffu, v, 1); };
    const int ir = 2 * rq + ((cls + C::RI) & 1); // quad row, 0 .. IH-1; gj & 1 == cls
    const int e = (ir - C::RI + H) * BX + C::Q0 + 4 * qc_;     // x (and cy) box element of cell 0
    const int eC = e - (H - RR) * BX;                          // b, cx, cz box element of cell 0

    // Work item b of a level (nitems items): tile b % ntiles, z chunk b / ntiles (tiles
    // fastest, so neighbouring tiles march the same planes at the same time and share their
    // halo rows in L2).
    auto run_item = [&](const TmaSweepArgs<T, TC>& a, const TmaMaps& maps, const int b, const int nitems) {
        const LevelOp<TC>& L = a.L;
        const int nx = L.nx, ny = L.ny, nz = L.nz;
        const size_t nxy = (size_t)nx * ny;
        const T dx2 = (T)L.dx2, inv_dx2 = (T)L.inv_dx2;
        const int ntx = (nx + TX - 1) / TX, ntiles = ntx * ((ny + TY - 1) / TY);
        (void)nitems;
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
        if (producer) {
            // ---- producer: both rings in order of need (x plane p is read one step before
            // coefficient plane p), each copy into a slot the consumers have released ----
            if (tid == C::NCONS) {
                if constexpr (BATCH) {
                    // tensor maps read from global memory, written there by a host copy: the
                    // acquire has system scope (a narrower scope may leave the TMA unit a stale
                    // descriptor cached for the same address)
                    const CUtensorMap* mp[8] = {&maps.x, &maps.b, &maps.cx, &maps.cy, &maps.cz,
                                                &maps.bxm, &maps.bym, &maps.bzm};
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(mp[k]) : "memory");
                }
                auto issue_x = [&](int p) {
                    const unsigned n = qx + (unsigned)(p - pl0);
                    const int s = (int)(n % NRX);
                    if (n >= (unsigned)NRX && !mbar_wait(&emx[s], ((n / NRX) - 1) & 1u)) return false;
                    mbar_expect_tx(&barx[s], (unsigned)C::XB);
                    tma_load_3d(xsl(s), &maps.x, i0 - HX, j0 - H, p, &barx[s]);
                    return true;
                };
                auto issue_c = [&](int p) {
                    const unsigned n = qc + (unsigned)(p - pl0);
                    const int s = (int)(n % NRC);
                    if (n >= (unsigned)NRC && !mbar_wait(&emc[s], ((n / NRC) - 1) & 1u)) return false;
                    uint64_t* bar = &barc[s];
                    unsigned char* cs = cbase(s);
                    mbar_expect_tx(bar, C::C_TX + (bnd_x ? (unsigned)C::BXMB : 0u) + (bnd_y ? (unsigned)C::BYMB : 0u));
                    tma_load_3d(cs, &maps.b, i0 - HX, j0 - RR, p, bar);
                    tma_load_3d(cs + C::C_CX, &maps.cx, i0 - HX, j0 - RR, p, bar);
                    tma_load_3d(cs + C::C_CY, &maps.cy, i0 - HX, j0 - H, p, bar);
                    if (p == -1) // the -z boundary faces stand in for plane -1's +z faces
                        tma_load_2d(cs + C::C_CZ, &maps.bzm, i0 - HX, j0 - RR, bar);
                    else
                        tma_load_3d(cs + C::C_CZ, &maps.cz, i0 - HX, j0 - RR, p, bar);
                    if (bnd_x) tma_load_2d(cs + C::C_BXM, &maps.bxm, j0 - C::BYS, p, bar);
                    if (bnd_y) tma_load_2d(cs + C::C_BYM, &maps.bym, i0 - HX, p, bar);
                    return true;
                };
                int px = ZERO ? xl1 + 1 : pl0, pc = pl0;
                while (!fail && (px <= xl1 || pc <= cl1)) {
                    if (px <= xl1 && (pc > cl1 || px <= pc + 1)) {
                        fail = !issue_x(px);
                        if (!fail) issued[0] = issued[0] + 1;
                        ++px;
                    } else {
                        fail = !issue_c(pc);
                        if (!fail) issued[1] = issued[1] + 1;
                        ++pc;
                    }
                }
                if (fail) atomicExch(a.err, 1);
            }
            if (!ZERO) qx += (unsigned)(xl1 - pl0 + 1);
            qc += (unsigned)(cl1 - pl0 + 1);
            return;
        }
        // ---- consumers ----
        int xw_plane = pl0, cw_plane = pl0; // thread 0: next plane to wait for
        int xr_plane = pl0, cr_plane = pl0; // thread 0: next plane to release
        if (tid == 0) {
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
        fail = bar_red_or(1, C::NCONS, fail);
        // slots of x planes t+1, t, t-1, t-2 and of coefficient planes t, t-1, t-2 (the same in
        // every thread)
        int sxp = nxt_x((int)(qx % NRX)), sx0 = (int)(qx % NRX), sx1 = 0, sx2 = 0;
        int sc0 = (int)(qc % NRC);

        // ---- the quad in this tile ----
        const int gi = i0 - 4 + 4 * qc_, gj = j0 - C::RI + ir;
        // per-cell flags, bit k for cell k: in grid (G), red ring (R), black ring (K), tile (T)
        unsigned fg = 0u, fr = 0u, fk = 0u, ft = 0u;
        {
            const bool rowg = iv && gj >= 0 && gj < ny;
            auto in_ring = [&](int i, int r) {
                return iv && gj >= j0 - r && gj < j0 + TY + r && i >= i0 - r && i < i0 + TX + r;
            };
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = gi + k;
                const bool g = rowg && i >= 0 && i < nx;
                fg |= (unsigned)g << k;
                fr |= (unsigned)in_ring(i, RR) << k;
                fk |= (unsigned)in_ring(i, RB) << k;
                ft |= (unsigned)(g && in_ring(i, 0)) << k;
            }
        }
        const bool pin_quad = L.pin && gi == 0 && gj == 0;
        const bool tileq = (ft & 1u) != 0; // nx is a multiple of 4: a tile quad is all in or out
        const bool restricts = RESID && tileq && ((gj - j0) & 1) == 0 && gj + 1 < ny;
        // byte offsets in a coefficient slot of cell 0's -x face and the quad's -y faces
        const int off_cxl = (gi == 0) ? (int)C::C_BXM + (gj - (j0 - C::BYS)) * (int)sizeof(TC)
                                      : (int)C::C_CX + (eC - 1) * (int)sizeof(TC);
        const int off_cyd = (gj == 0) ? (int)C::C_BYM + (gi - (i0 - HX)) * (int)sizeof(TC)
                                      : (int)C::C_CY + (e - BX) * (int)sizeof(TC);
        const int ncx = a.ncx;
        const size_t ncxy = (size_t)a.ncx * a.ncy;
        const size_t gq = (size_t)(gi > 0 ? gi : 0) + (size_t)nx * (gj > 0 ? gj : 0); // column of cell 0

        auto load_coef = [&](int s) {
            const unsigned char* cs = cbase(s);
            QuadCoef<T> c;
            c.b = ldq<T>(reinterpret_cast<const T*>(cs) + eC);
            c.cx = ldq<T>(reinterpret_cast<const TC*>(cs + C::C_CX) + eC);
            c.cy = ldq<T>(reinterpret_cast<const TC*>(cs + C::C_CY) + e);
            c.cz = ldq<T>(reinterpret_cast<const TC*>(cs + C::C_CZ) + eC);
            c.cyd = ldq<T>(reinterpret_cast<const TC*>(cs + off_cyd));
            c.cxl = from_left(c.cx.v[3]); // the left quad's last +x face
            if (fb_l || gi == 0) c.cxl = tc(*reinterpret_cast<const TC*>(cs + off_cxl));
            return c;
        };
        auto cz_of = [&](int s) { return ldq<T>(reinterpret_cast<const TC*>(cbase(s) + C::C_CZ) + eC); };
        // coarse correction of the quad in plane p (cells 0-1 and 2-3 share coarse cells)
        auto load_ev = [&](int p, T& e0, T& e1) {
            e0 = e1 = (T)0;
            if (!PROL || !(p >= 0 && p < nz && (fg & 1u))) return;
            const T* src = a.e_c + (size_t)(gi >> 1) + (size_t)ncx * (gj >> 1) + ncxy * (size_t)(p >> 1);
            e0 = src[0];
            if (fg & 4u) e1 = src[1];
        };
        auto restrict_quad = [&](int s1, int rs0, int rs1) { // coarse plane s1 >> 1 from s1 - 1, s1
            const T* r0 = rsb + rs0 * TX * TY + (gj - j0) * TX + (gi - i0);
            const T* r1 = rsb + rs1 * TX * TY + (gj - j0) * TX + (gi - i0);
            const Q4<T> a0 = ldq<T>(r0), a1 = ldq<T>(r0 + TX), b0 = ldq<T>(r1), b1 = ldq<T>(r1 + TX);
            T o[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                T acc = (T)0;
                acc += a0.v[2 * h];
                acc += a0.v[2 * h + 1];
                acc += a1.v[2 * h];
                acc += a1.v[2 * h + 1];
                acc += b0.v[2 * h];
                acc += b0.v[2 * h + 1];
                acc += b1.v[2 * h];
                acc += b1.v[2 * h + 1];
                o[h] = acc / (T)8;
            }
            T* dst = a.b_coarse + (size_t)(gi >> 1) + (size_t)ncx * (gj >> 1) + ncxy * (size_t)(s1 >> 1);
            dst[0] = o[0];
            dst[1] = o[1];
        };

        // carried state (non-RESID): the black cells' coefficients of the previous plane and the
        // red cells' +z faces of two planes back; RESID: cz of plane t-3 and the final x of t-3
        BlackCoef<T> cbA{}, cbB{};
        T czA[2] = {0, 0}, czB[2] = {0, 0};
        Q4<T> cz3{}, x3{};
        T evA0 = 0, evA1 = 0; // PROLONG: correction of plane t+2, loaded one step ahead
        int rslot = 0;        // rsb slot of residual plane t-2 ((t - 2 - z0) mod 3)

        // one step of the march; O: offset of the first red cell of plane t in the quad
        auto step = [&](auto Oc, int t, BlackCoef<T>& cb_in, BlackCoef<T>& cb_out, T (&cz_io)[2]) {
            constexpr int O = decltype(Oc)::value;
            const bool in_z = t >= 0 && t < nz;
            const int q = t - 1, sp = t - 2;
            T* xs0 = xsl(sx0);
            T* xs1 = xsl(sx1);
            T* xs2 = xsl(sx2);
            const int sc1 = prv_c(sc0), sc2 = prv_c(sc1);
            // ======== loads of the red and black stages ========
            Q4<T> xp{};
            T ev0, ev1;
            if (t == pl0) { // the first plane: its x_old, corrected
                T f0, f1;
                load_ev(t, f0, f1);
                if (PROL && iv) {
                    Q4<T> v = ZERO ? Q4<T>{} : ldq<T>(xs0 + e);
                    v.v[0] += f0, v.v[1] += f0, v.v[2] += f1, v.v[3] += f1;
                    stq<T>(xs0 + e, v);
                }
                load_ev(t + 1, ev0, ev1);
            } else {
                ev0 = evA0, ev1 = evA1;
            }
            if (PROL) load_ev(t + 2, evA0, evA1);
            if (t + 1 <= xl1) {
                if (!ZERO) xp = ldq<T>(xsl(sxp) + e);
                xp.v[0] += ev0, xp.v[1] += ev0, xp.v[2] += ev1, xp.v[3] += ev1;
            }
            const QuadCoef<T> c0 = load_coef(sc0);
            Q4<T> x0{}, x0u{}, x0d{};
            T x0o = 0;
            if (!ZERO) {
                x0 = ldq<T>(xs0 + e);
                x0u = ldq<T>(xs0 + e + BX);
                x0d = ldq<T>(xs0 + e - BX);
                x0o = O ? from_right(x0.v[0]) : from_left(x0.v[3]);
                if (O ? fb_r : fb_l) x0o = O ? xs0[e + 4] : xs0[e - 1];
            }
            const Q4<T> x1 = ldq<T>(xs1 + e), x1u = ldq<T>(xs1 + e + BX), x1d = ldq<T>(xs1 + e - BX);
            T x1o = O ? from_right(x1.v[0]) : from_left(x1.v[3]);
            if (O ? fb_r : fb_l) x1o = O ? xs1[e + 4] : xs1[e - 1];
            const Q4<T> x2 = ldq<T>(xs2 + e);
            // coefficients of the black cells (plane t-1) and the +z faces of planes t-1, t-2
            T bb[2], bxp[2], bxm[2], byp[2], bym_[2], bzp[2], bzm_[2], rzm[2];
            if constexpr (RESID) {
                const QuadCoef<T> c1 = load_coef(sc1);
                const Q4<T> z2 = cz_of(sc2);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = O + 2 * h;
                    bb[h] = c1.b.v[k];
                    bxp[h] = c1.cx.v[k];
                    bxm[h] = k == 0 ? c1.cxl : c1.cx.v[k - 1];
                    byp[h] = c1.cy.v[k];
                    bym_[h] = c1.cyd.v[k];
                    bzp[h] = c1.cz.v[k];
                    bzm_[h] = z2.v[k];
                    rzm[h] = c1.cz.v[k];
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    bb[h] = cb_in.b[h];
                    bxp[h] = cb_in.cxp[h];
                    bxm[h] = cb_in.cxm[h];
                    byp[h] = cb_in.cyp[h];
                    bym_[h] = cb_in.cym[h];
                    bzp[h] = cb_in.czp[h];
                    bzm_[h] = cz_io[h];
                    rzm[h] = cb_in.czp[h];
                }
            }
            double2 r64a = make_double2(0.0, 0.0), r64b = make_double2(0.0, 0.0);
            const bool out_t = sp >= z0 && sp < z1 && tileq;
            const size_t cg_out = gq + nxy * (size_t)(sp > 0 ? sp : 0);
            if (DOT && out_t) {
                r64a = __ldg(reinterpret_cast<const double2*>(a.r64 + cg_out));
                r64b = __ldg(reinterpret_cast<const double2*>(a.r64 + cg_out + 2));
            }
            // ======== arithmetic ========
            T vred[2], vblk[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = O + 2 * h; // cell of the quad
                // red, plane t
                {
                    const T cxp = c0.cx.v[k], cxm = k == 0 ? c0.cxl : c0.cx.v[k - 1];
                    const T cyp = c0.cy.v[k], cym = c0.cyd.v[k], czp = c0.cz.v[k], czm = rzm[h];
                    T D = cxm + cxp + cym + cyp + czm + czp;
                    if (k == 0 && t == 0 && pin_quad) D *= (T)2;
                    T s = (T)0;
                    if (!ZERO) {
                        const T xl = k == 0 ? x0o : x0.v[k - 1], xr = k == 3 ? x0o : x0.v[k + 1];
                        s = cxp * xr + cxm * xl + cyp * x0u.v[k] + cym * x0d.v[k] + czp * xp.v[k] + czm * x1.v[k];
                    }
                    vred[h] = (in_z && ((fg >> k) & 1u)) ? divide(s - c0.b.v[k] * dx2, D) : (T)0;
                }
                // black, plane t-1
                {
                    const T D = bxm[h] + bxp[h] + bym_[h] + byp[h] + bzm_[h] + bzp[h];
                    const T xl = k == 0 ? x1o : x1.v[k - 1], xr = k == 3 ? x1o : x1.v[k + 1];
                    const T s = bxp[h] * xr + bxm[h] * xl + byp[h] * x1u.v[k] + bym_[h] * x1d.v[k] + bzp[h] * vred[h] +
                                bzm_[h] * x2.v[k];
                    vblk[h] = (q >= 0 && q < nz && ((fg >> k) & 1u)) ? divide(s - bb[h] * dx2, D) : (T)0;
                }
            }
            if constexpr (!RESID) {
                // the black cells of plane t (cells 1-O, 3-O) are updated at the next step
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = (1 - O) + 2 * h;
                    cb_out.b[h] = c0.b.v[k];
                    cb_out.cxp[h] = c0.cx.v[k];
                    cb_out.cxm[h] = k == 0 ? c0.cxl : c0.cx.v[k - 1];
                    cb_out.cyp[h] = c0.cy.v[k];
                    cb_out.cym[h] = c0.cyd.v[k];
                    cb_out.czp[h] = c0.cz.v[k];
                    cz_io[h] = c0.cz.v[O + 2 * h]; // for the black stage two steps on
                }
            }
            // ======== stores of the red and black stages ========
            const bool red_live = t >= t0 && t <= cl1, blk_live = q >= z0 - RB && q < z1 + RB;
            // whole quads: the cells not updated are written back with the values just read
            // (zero in ZERO mode, where nothing reads them before they are updated)
            constexpr unsigned OM = (1u << O) | (4u << O);
            if (red_live && (fr & OM)) {
                Q4<T> w = x0;
                if ((fr >> O) & 1u) w.v[O] = vred[0];
                if ((fr >> (O + 2)) & 1u) w.v[O + 2] = vred[1];
                stq<T>(xs0 + e, w);
            }
            if (blk_live && (fk & OM)) {
                Q4<T> w = x1;
                if ((fk >> O) & 1u) w.v[O] = vblk[0];
                if ((fk >> (O + 2)) & 1u) w.v[O + 2] = vblk[1];
                stq<T>(xs1 + e, w);
            }
            if (PROL && iv && t + 1 <= xl1) stq<T>(xsl(sxp) + e, xp);
            // -------- plane t-2 is final: write the tile --------
            if (out_t) {
                stq<T>(a.x_out + cg_out, x2);
                if constexpr (DOT)
                    dot_acc += r64a.x * (double)x2.v[0] + r64a.y * (double)x2.v[1] + r64b.x * (double)x2.v[2] +
                               r64b.y * (double)x2.v[3];
            }
            if constexpr (RESID) {
                // -------- residual, plane t-2 (smoother's pin convention) --------
                const QuadCoef<T> c2 = load_coef(sc2);
                const Q4<T> x2u = ldq<T>(xs2 + e + BX), x2d = ldq<T>(xs2 + e - BX);
                T x2l = from_left(x2.v[3]), x2r = from_right(x2.v[0]);
                if (fb_l) x2l = xs2[e - 1];
                if (fb_r) x2r = xs2[e + 4];
                Q4<T> x1f = x1; // final x of plane t-1
                x1f.v[O] = vblk[0];
                x1f.v[O + 2] = vblk[1];
                // the black cells of plane t-2 were relaxed last, with their red neighbours final:
                // their residual is zero (to rounding) by construction, so only the red cells
                // (O, O+2, the red offset of plane t-2 equals that of plane t) are evaluated
                Q4<T> r{};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = O + 2 * h;
                    const T cxp = c2.cx.v[k], cxm = k == 0 ? c2.cxl : c2.cx.v[k - 1];
                    const T cyp = c2.cy.v[k], cym = c2.cyd.v[k], czp = c2.cz.v[k], czm = cz3.v[k];
                    T D = cxm + cxp + cym + cyp + czm + czp;
                    if (k == 0 && sp == 0 && pin_quad) D *= (T)2;
                    const T xl = k == 0 ? x2l : x2.v[k - 1], xr = k == 3 ? x2r : x2.v[k + 1];
                    const T sum = cxp * xr + cxm * xl + cyp * x2u.v[k] + cym * x2d.v[k] + czp * x1f.v[k] + czm * x3.v[k];
                    r.v[k] = c2.b.v[k] - (sum - D * x2.v[k]) * inv_dx2;
                }
                if (sp >= z0 && sp < z1 && tileq) stq<T>(rsb + rslot * TX * TY + (gj - j0) * TX + (gi - i0), r);
                // -------- restriction of planes (t-4, t-3), finished before the last barrier --------
                const int s1 = t - 3;
                if (restricts && s1 > z0 && s1 < z1 && ((s1 - z0) & 1) == 1)
                    restrict_quad(s1, rslot == 0 ? 1 : rslot - 1 == 0 ? 2 : rslot - 2, rslot == 0 ? 2 : rslot - 1);
                if (sp >= z0) rslot = rslot == 2 ? 0 : rslot + 1;
                x3 = x2;
                cz3 = c2.cz;
            }
        };
        // the end of a step, common to both offsets: thread 0 waits for the planes of the next
        // step; the barrier publishes them and the plane exchange; the next step's slots
        auto sync_step = [&](int t) {
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
            fail = bar_red_or(1, C::NCONS, fail);
            sx2 = sx1;
            sx1 = sx0;
            sx0 = sxp;
            sxp = nxt_x(sxp);
            sc0 = nxt_c(sc0);
        };

        // the start of a step: thread 0 releases the slots no longer read
        auto release_step = [&](int t) {
            if (tid == 0) {
                if (!ZERO && t - 3 >= pl0 && xr_plane <= xl1) {
                    release_x();
                    ++xr_plane;
                }
                if (t - LC >= pl0 && cr_plane <= cl1) {
                    release_c();
                    ++cr_plane;
                }
            }
        };

        using Z = std::integral_constant<int, 0>;
        using I = std::integral_constant<int, 1>;
        for (int t = pl0; t < t1 && !fail; t += 2) {
            // red offset of plane t: (gj + t) & 1 = (cls + t) & 1, uniform in a warp of interior
            // quads; the edge warp holds both parities and runs both offsets in turn
            const bool even = ((cls + t) & 1) == 0;
            release_step(t);
            if (even) step(Z{}, t, cbB, cbA, czA);
            else step(I{}, t, cbB, cbA, czA);
            sync_step(t);
            if (fail) break;
            release_step(t + 1);
            if (even) step(I{}, t + 1, cbA, cbB, czB);
            else step(Z{}, t + 1, cbA, cbB, czB);
            sync_step(t + 1);
        }
        if (fail) {
            // drain the copies issued and not yet waited for (bounded waits), then leave
            if (tid == 0) {
                atomicExch(a.err, 1);
                const int nx_done = (int)qx + (xw_plane - pl0), nc_done = (int)qc + (cw_plane - pl0);
                for (int k = nx_done; k < issued[0]; ++k) (void)wait_x();
                for (int k = nc_done; k < issued[1]; ++k) (void)wait_c();
            }
            return;
        }
        // release the planes still held, so that the producer can reuse their slots
        if (tid == 0) {
            if (!ZERO)
                for (; xr_plane <= xl1; ++xr_plane) release_x();
            for (; cr_plane <= cl1; ++cr_plane) release_c();
        }
        if (!ZERO) qx += (unsigned)(xl1 - pl0 + 1);
        qc += (unsigned)(cl1 - pl0 + 1);
        if constexpr (BATCH && DOT) {
            // this item's share of <r64, x_out>, summed by the consumers alone (the producer
            // warp is already issuing the next item); the last item of the realisation adds
            // the items' partials in index order
            __shared__ double item_red[C::NCONS / 32];
            double v = dot_acc;
            dot_acc = 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) item_red[warp] = v;
            asm volatile("bar.sync 2, %0;" ::"r"(C::NCONS) : "memory");
            if (tid == 0) {
                double sum = 0.0;
                for (int w = 0; w < C::NCONS / 32; ++w) sum += item_red[w];
                a.dot_partials[b] = sum;
                __threadfence();
                if (atomicAdd(a.dot_ticket, 1u) == (unsigned)nitems - 1) {
                    __threadfence();
                    double acc = 0.0;
                    for (int i = 0; i < nitems; ++i) acc += __ldcg(a.dot_partials + i);
                    *a.dot_out = acc;
                    *a.dot_ticket = 0u;
                }
            }
            asm volatile("bar.sync 2, %0;" ::"r"(C::NCONS) : "memory");
        }
    };

    if constexpr (BATCH) {
        for (int b = blockIdx.x; b < a0.total && !fail; b += gridDim.x) {
            const int sg = find_seg(a0.seg_off, a0.nseg, b);
            const TmaSweepArgs<T, TC>& A = a0.seg_args[sg];
            if (A.stop && *A.stop) continue; // that realisation's solve has finished
            const int o = __ldg(a0.seg_off + sg);
            run_item(A, a0.seg_maps[sg], b - o, __ldg(a0.seg_off + sg + 1) - o);
        }
    } else {
        const int ntiles = ((a0.L.nx + TX - 1) / TX) * ((a0.L.ny + TY - 1) / TY);
        const int total = ntiles * ((a0.L.nz + a0.zchunk - 1) / a0.zchunk);
        for (int b = blockIdx.x; b < total && !fail; b += gridDim.x) run_item(a0, maps0, b, total);
        if (DOT) { // every thread, the producer warp included (grid_sums synchronises the CTA)
            double v[1] = {dot_acc}, out[1];
            if (grid_sums<C::NT, 1>(v, a0.dot_partials, a0.dot_ticket, gridDim.x, out)) *a0.dot_out = out[0];
        }
    }
}

} // namespace mf3d

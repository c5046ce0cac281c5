// kernels_sweep_tma.cuh -- the fused red-black sweep with every operand staged by TMA.
//
// Same algorithm as sweep_kernel (kernels_mg.cuh): a CTA owns a 32 x 8 column tile and a z
// range and runs red (plane t-1), black (plane t-2) and optionally residual+restriction
// (plane t-3) as a wavefront.  Here x_in, b and the three face-coefficient arrays of every
// plane arrive in a shared-memory ring through cp.async.bulk.tensor.3d, issued by one thread
// PF planes ahead of use and tracked by one mbarrier per ring slot, so the stages read only
// shared memory and the march is not bound by global-load latency.  Each thread owns fixed
// cells in every stage (their shared-memory offsets are computed once), ring slots advance
// incrementally, and every stage is one pass with no integer division.
//
// Tile boxes start at x = i0 - HX with HX * sizeof(element) a multiple of 16 bytes (the TMA
// alignment rule for the innermost coordinate); y and z may start outside the grid, where
// TMA fills zeros, which is exactly the ghost value of a Dirichlet or Neumann face.
// Periodic axes are served by sweep_kernel instead.
#pragma once
#include <cuda.h>

#include "kernels_mg.cuh"

namespace mf3d {

struct TmaMaps {
    CUtensorMap x, b, cx, cy, cz;
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
    T* b_coarse; // M_RESID
    int zchunk;
    const double* r64; // M_DOT: <r64, x_out>
    double* dot_partials;
    unsigned* dot_ticket;
    double* dot_out;
    int* err; // set to 1 when an mbarrier wait gives up
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

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <class T, class TC, int MODE> struct TmaSweepCfg {
    static constexpr bool RESID = (MODE & M_RESID) != 0;
    static constexpr int NS = RESID ? 3 : 2;
    static constexpr int H = NS;
    static constexpr int HX = TmaGeom<T, TC>::hx(H);
    // 32 x 16 tiles (512 threads) in FP32, 32 x 8 (256 threads) in FP64 to fit the ring
    static constexpr int TY = sizeof(T) == 8 ? 8 : 16;
    static constexpr int NT = SW_TX * TY;
    static constexpr int BX = SW_TX + 2 * HX, BY = TY + 2 * H;
    static constexpr int PLANE = BX * BY;      // elements per array plane
    static constexpr int FIX = (PLANE + NT - 1) / NT; // fix-up elements per thread
    static constexpr size_t XB = (size_t)PLANE * sizeof(T), CB = (size_t)PLANE * sizeof(TC);
    static constexpr size_t align128(size_t v) { return (v + 127) & ~(size_t)127; }
    static constexpr size_t OB = align128(XB), OC = align128(CB);
    static constexpr size_t SLOT = OB * 2 + OC * 3; // x, b, cx, cy, cz
    static constexpr size_t RS = RESID ? align128(2 * SW_TX * TY * sizeof(T)) : 0;
    // ring slots: NS + 2 planes are live, the rest (PF) are in flight; one CTA per SM takes
    // as many slots as 200 KB of shared memory hold (at most 16)
    static constexpr int NR_FIT = (int)((200 * 1024 - 128 - RS) / SLOT);
    static constexpr int NR = NR_FIT < 16 ? NR_FIT : 16;
    static constexpr int PF = NR - NS - 2;
    static_assert(PF >= 2, "ring too small");
    static constexpr size_t SMEM = 128 /* barriers */ + SLOT * NR + RS;
};

template <class T, class TC, int MODE>
__global__ void __launch_bounds__(TmaSweepCfg<T, TC, MODE>::NT) sweep_tma_kernel(const __grid_constant__ TmaMaps maps,
                                                                             const TmaSweepArgs<T, TC> a) {
    using C = TmaSweepCfg<T, TC, MODE>;
    constexpr int TY = C::TY, NT = C::NT;
    constexpr bool ZERO = (MODE & M_ZERO) != 0;
    constexpr bool PROL = (MODE & M_PROLONG) != 0;
    constexpr bool RESID = C::RESID;
    constexpr bool DOT = (MODE & M_DOT) != 0;
    constexpr int NS = C::NS, H = C::H, HX = C::HX, BX = C::BX, NR = C::NR, PF = C::PF;
    // all ring accesses are 32-bit offsets from the shared array, so they stay shared-space
    // loads (the dynamic shared window starts 1 KB aligned; every slot offset is 128-aligned)
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t* bars = (uint64_t*)smraw;
    constexpr int RING = 128;
    T* rsb = (T*)(smraw + RING + C::SLOT * NR);

    const LevelOp<TC>& L = a.L;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const size_t nxy = (size_t)nx * ny;
    const int i0 = blockIdx.x * SW_TX, j0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * a.zchunk;
    const int z1 = min(z0 + a.zchunk, nz);
    const int tid = threadIdx.x;
    const T dx2 = (T)L.dx2;
    const int zlo = z0 - NS, zhi = z1 - 1 + NS;

    // slot s: x at ring + SLOT*s, b at +OB, cx at +2*OB, cy at +2*OB+OC, cz at +2*OB+2*OC
    auto X = [&](int s) { return (T*)(smraw + RING + C::SLOT * s); };
    auto B = [&](int s) { return (T*)(smraw + RING + C::SLOT * s + C::OB); };
    auto CX = [&](int s) { return (TC*)(smraw + RING + C::SLOT * s + 2 * C::OB); };
    auto CY = [&](int s) { return (TC*)(smraw + RING + C::SLOT * s + 2 * C::OB + C::OC); };
    auto CZ = [&](int s) { return (TC*)(smraw + RING + C::SLOT * s + 2 * C::OB + 2 * C::OC); };
    constexpr unsigned TX_BYTES = (unsigned)(2 * C::XB + 3 * C::CB);

    auto issue = [&](int t, int s) { // thread 0 only; plane t into slot s
        mbar_expect_tx(&bars[s], ZERO ? TX_BYTES - (unsigned)C::XB : TX_BYTES);
        if (!ZERO) tma_load_3d(X(s), &maps.x, i0 - HX, j0 - H, t, &bars[s]);
        tma_load_3d(B(s), &maps.b, i0 - HX, j0 - H, t, &bars[s]);
        tma_load_3d(CX(s), &maps.cx, i0 - HX, j0 - H, t, &bars[s]);
        tma_load_3d(CY(s), &maps.cy, i0 - HX, j0 - H, t, &bars[s]);
        tma_load_3d(CZ(s), &maps.cz, i0 - HX, j0 - H, t, &bars[s]);
    };

    if (tid == 0) {
        for (int s = 0; s < NR; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < PF && zlo + q <= zhi; ++q) issue(zlo + q, q);

    // ---- fixed per-thread work items ----
    constexpr int hr = NS - 1, hb = NS - 2;
    constexpr int RPW = (SW_TX + 2 * hr) / 2, RPH = TY + 2 * hr;
    constexpr int BPW = (SW_TX + 2 * hb) / 2, BPH = TY + 2 * hb;
    static_assert(RPW * RPH <= NT && BPW * BPH <= NT, "one red and one black item per thread");
    // red item: pair (r_iu0, r_iu0+1) in row r_ju
    const int r_iu0 = i0 - hr + 2 * (tid % RPW), r_ju = j0 - hr + tid / RPW;
    const bool r_ok = tid < RPW * RPH && r_ju >= 0 && r_ju < ny;
    const int r_e0 = (r_ju - j0 + H) * BX + (r_iu0 - i0 + HX);
    const int r_par = (r_iu0 + r_ju) & 1;
    // black item
    const int b_iu0 = i0 - hb + 2 * (tid % BPW), b_ju = j0 - hb + tid / BPW;
    const bool b_ok = tid < BPW * BPH && b_ju >= 0 && b_ju < ny;
    const int b_e0 = (b_ju - j0 + H) * BX + (b_iu0 - i0 + HX);
    const int b_par = (b_iu0 + b_ju) & 1;
    // output / residual item
    const int o_li = tid % SW_TX, o_lj = tid / SW_TX; // NT == SW_TX * TY
    const int o_gi = i0 + o_li, o_gj = j0 + o_lj;
    const bool o_ok = o_gi < nx && o_gj < ny;
    const int o_e = (o_lj + H) * BX + o_li + HX;
    const size_t o_c0 = (size_t)o_gi + (size_t)nx * o_gj;
    // fix-up items (zero input / prolongation): region elements tid + k*SW_NT
    int f_e[C::FIX];
    long long f_cb[C::FIX]; // coarse column index, -1 when outside the grid
#pragma unroll
    for (int k = 0; k < C::FIX; ++k) {
        const int e = tid + k * NT;
        f_e[k] = e < C::PLANE ? e : -1;
        const int gi = i0 - HX + e % BX, gj = j0 - H + e / BX;
        f_cb[k] = (e < C::PLANE && gi >= 0 && gi < nx && gj >= 0 && gj < ny)
                      ? (long long)(gi >> 1) + (long long)a.ncx * (gj >> 1)
                      : -1;
    }
    const size_t ncxy = (size_t)a.ncx * a.ncy;

    double dot_acc = 0.0;
    unsigned phase = 0u; // bit s: parity of the next wait on slot s (tracked by thread 0)

    // slot byte offsets of planes t, t-1, ..., t-4 for the current step
    int pb[5];
    auto set_bases = [&](int sl_t) {
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            int v = sl_t - d;
            if (v < 0) v += NR;
            pb[d] = RING + (int)C::SLOT * v;
        }
    };
    auto Xp = [&](int d) { return (T*)(smraw + pb[d]); };
    auto Bp = [&](int d) { return (T*)(smraw + pb[d] + C::OB); };
    auto CXp = [&](int d) { return (TC*)(smraw + pb[d] + 2 * C::OB); };
    auto CYp = [&](int d) { return (TC*)(smraw + pb[d] + 2 * C::OB + C::OC); };
    auto CZp = [&](int d) { return (TC*)(smraw + pb[d] + 2 * C::OB + 2 * C::OC); };
    auto divide = [](T num, T den) -> T {
        if constexpr (sizeof(T) == 4) return __fdividef(num, den); // preconditioner: 2-ulp division
        else return num / den;
    };

    // relaxation of cell (iu, ju, pl) at plane-local element e; d: age of plane pl in the ring
    auto relax = [&](int iu, int ju, int pl, int e, int d) {
        T* x = Xp(d);
        const TC* cx = CXp(d);
        const TC* cy = CYp(d);
        const T cxp = ld_as_float_or_double<T>(cx[e]);
        const T cyp = ld_as_float_or_double<T>(cy[e]);
        const T czp = ld_as_float_or_double<T>(CZp(d)[e]);
        const T cxm = iu > 0 ? ld_as_float_or_double<T>(cx[e - 1]) : load_as<T>(L.bxm, (size_t)ju + (size_t)ny * pl);
        const T cym = ju > 0 ? ld_as_float_or_double<T>(cy[e - BX]) : load_as<T>(L.bym, (size_t)iu + (size_t)nx * pl);
        const T czm = pl > 0 ? ld_as_float_or_double<T>(CZp(d + 1)[e]) : load_as<T>(L.bzm, (size_t)iu + (size_t)nx * ju);
        T D = cxm + cxp + cym + cyp + czm + czp;
        if (L.pin && (iu | ju | pl) == 0) D *= (T)2;
        const T s = cxp * x[e + 1] + cxm * x[e - 1] + cyp * x[e + BX] + cym * x[e - BX] + czp * Xp(d - 1)[e] +
                    czm * Xp(d + 1)[e];
        x[e] = divide(s - Bp(d)[e] * dx2, D);
    };

    int sl_t = 0; // slot of plane t
    for (int t = zlo; t <= zhi; ++t) {
        // ---- thread 0 waits for plane t, refills the ring; the others sleep at the barrier ----
        bool ok = true;
        if (tid == 0) {
            // refill first: plane t-1+PF reuses the slot of plane t-NS-3, which no thread reads
            // in step t-1 (its oldest plane is t-NS-2) and whose last generic-proxy writes were
            // fenced before the barriers of step t-1
            if (t > zlo && t - 1 + PF <= zhi) {
                int s2 = sl_t - 1 + PF;
                if (s2 >= NR) s2 -= NR;
                issue(t - 1 + PF, s2);
            }
            ok = mbar_wait(&bars[sl_t], (phase >> sl_t) & 1u);
            phase ^= 1u << sl_t;
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(a.err, 1);
            return;
        }
        set_bases(sl_t);
        // ---- zero input / prolongation on the freshly landed x plane ----
        if (ZERO || PROL) {
            T* x = Xp(0);
            const bool in_z = t >= 0 && t < nz;
            const size_t cz_off = ncxy * (size_t)(t >> 1);
#pragma unroll
            for (int k = 0; k < C::FIX; ++k) {
                if (f_e[k] < 0) continue;
                T v = (T)0;
                if (in_z && f_cb[k] >= 0) {
                    if (!ZERO) v = x[f_e[k]];
                    if (PROL) v += a.e_c[(size_t)f_cb[k] + cz_off];
                }
                x[f_e[k]] = v;
            }
            __syncthreads();
        }
        // ---- red at plane p = t-1 (tile + hr) ----
        {
            const int p = t - 1;
            if (r_ok && p >= z0 - hr && p <= z1 - 1 + hr && p >= 0 && p < nz) {
                const int off = (r_par + p) & 1;
                const int iu = r_iu0 + off;
                if (iu >= 0 && iu < nx) relax(iu, r_ju, p, r_e0 + off, 1);
            }
        }
        __syncthreads();
        // ---- black at plane q = t-2 (tile + hb), then write the finished plane ----
        const int q = t - 2;
        if (b_ok && q >= z0 - hb && q <= z1 - 1 + hb && q >= 0 && q < nz) {
            const int off = ((b_par + q) & 1) ^ 1;
            const int iu = b_iu0 + off;
            if (iu >= 0 && iu < nx) relax(iu, b_ju, q, b_e0 + off, 2);
        }
        __syncthreads();
        if (q >= z0 && q < z1 && o_ok) {
            const size_t c = o_c0 + nxy * q;
            const T v = Xp(2)[o_e];
            a.x_out[c] = v;
            if (DOT) dot_acc += __ldg(a.r64 + c) * (double)v;
        }
        // ---- residual at plane s = t-3, restriction per pair of planes ----
        if (RESID) {
            const int s = t - 3;
            if (s >= z0 && s < z1) {
                T rv = (T)0;
                if (o_ok) {
                    const int e = o_e;
                    const T* x = Xp(3);
                    const TC* cx = CXp(3);
                    const TC* cy = CYp(3);
                    const T cxp = ld_as_float_or_double<T>(cx[e]);
                    const T cyp = ld_as_float_or_double<T>(cy[e]);
                    const T czp = ld_as_float_or_double<T>(CZp(3)[e]);
                    const T cxm = o_gi > 0 ? ld_as_float_or_double<T>(cx[e - 1]) : load_as<T>(L.bxm, (size_t)o_gj + (size_t)ny * s);
                    const T cym = o_gj > 0 ? ld_as_float_or_double<T>(cy[e - BX]) : load_as<T>(L.bym, (size_t)o_gi + (size_t)nx * s);
                    const T czm = s > 0 ? ld_as_float_or_double<T>(CZp(4)[e]) : load_as<T>(L.bzm, o_c0);
                    T D = cxm + cxp + cym + cyp + czm + czp;
                    if (L.pin && (o_gi | o_gj | s) == 0) D *= (T)2;
                    const T sum = cxp * x[e + 1] + cxm * x[e - 1] + cyp * x[e + BX] + cym * x[e - BX] +
                                  czp * Xp(2)[e] + czm * Xp(4)[e];
                    rv = Bp(3)[e] - (sum - D * x[e]) * (T)L.inv_dx2;
                }
                rsb[((s - z0) & 1) * SW_TX * TY + tid] = rv;
                if (((s - z0) & 1) == 1) {
                    __syncthreads();
                    const int ncx = nx >> 1, ncy = ny >> 1;
                    if (tid < (SW_TX / 2) * (TY / 2)) {
                        const int ci = tid % (SW_TX / 2), cj = tid / (SW_TX / 2);
                        const int I = (i0 >> 1) + ci, J = (j0 >> 1) + cj;
                        if (I < ncx && J < ncy) {
                            const T* r0 = rsb;
                            const T* r1 = rsb + SW_TX * TY;
                            const int f = 2 * cj * SW_TX + 2 * ci;
                            T acc = (T)0;
                            acc += r0[f];
                            acc += r0[f + 1];
                            acc += r0[f + SW_TX];
                            acc += r0[f + SW_TX + 1];
                            acc += r1[f];
                            acc += r1[f + 1];
                            acc += r1[f + SW_TX];
                            acc += r1[f + SW_TX + 1];
                            a.b_coarse[(size_t)I + (size_t)ncx * J + (size_t)ncx * ncy * (s >> 1)] = acc / (T)8;
                        }
                    }
                }
            }
        }
        // generic-proxy writes to the ring are ordered before the TMA writes that reuse the
        // slot; the barrier at the top of the next step completes the hand-off
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        sl_t = (sl_t + 1 == NR) ? 0 : sl_t + 1;
    }

    if (DOT) {
        double v[1] = {dot_acc}, out[1];
        const int nblocks = gridDim.x * gridDim.y * gridDim.z;
        if (grid_sums<NT, 1>(v, a.dot_partials, a.dot_ticket, nblocks, out)) *a.dot_out = out[0];
    }
}

} // namespace mf3d

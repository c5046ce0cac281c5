// kernels_pcg.cuh -- fine-level operator and the device-resident PCG iteration.
//
// The reference's PCG (src/numerics/solvers/pcg.cuh:95-185) does two or three blocking
// host reductions per iteration.  Here every scalar lives in a PcgState in device memory,
// reductions are deterministic grid sums finished by the last CTA, and the CTA that
// finishes the x/r update also evaluates the stopping test and sets the CUDA-graph `while`
// condition, so a whole solve is one graph launch with no host round trip.
#pragma once
#include <cstddef>

#include "mf3d_device.cuh"

namespace mf3d {

struct PcgState {
    double rho_new;   // <r_k, z_k>
    double rho_old;   // <r_{k-1}, z_{k-1}>
    double gamma;     // <r_k, z_{k-1}>  (flexible / Polak-Ribiere beta)
    double pAp;       // <p_k, A p_k>
    double rr;        // ||r_k||^2 (recurrence residual)
    double bb;        // ||b||^2
    double r0sq;      // ||r_0||^2
    double rr_true;   // ||b - A x||^2 after the loop
    double ref_norm;  // denominator of the stopping test (||r_0|| or ||b||)
    double rtol;
    double final_res; // ||r|| at the last check
    double alpha, beta;
    int iter, max_iter, check_every, flexible;
    int converged, status, stop, body_count;
    int solver;                    // MF3D_SOLVER_*: 0 PCG_MG, 1 standalone MG, 2 plain CG
    unsigned long long t_start_ns; // %globaltimer at the start of the solve
    unsigned long long budget_ns;  // device-time limit of one solve
};

enum : int { PCG_OK = 0, PCG_BREAKDOWN = 1, PCG_NONFINITE = 2, PCG_TIMEOUT = 3 };
enum : int { SOLVE_PCG_MG = 0, SOLVE_MG = 1, SOLVE_CG = 2 }; // the ABI's MF3D_SOLVER_* codes

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr int PK_NT = 256;

// y = A x with the reference operator (src/numerics/operators/varcoeff_laplacian.cu:38-239):
// y_c = (sum_f C_f x_f - D_c x_c) / dx^2, and with the pin the diagonal at cell 0 grows by
// the coefficients of its in-domain faces only (varcoeff_laplacian.cu:225-229).
// With pin_full the whole diagonal is doubled instead, the smoother's and residual's
// convention (src/multigrid/smoothers/residual_3d.cu:365-368), used by the standalone MG solver.
template <class TC>
__device__ __forceinline__ double apply_A_cell(const LevelOp<TC>& L, const double* __restrict__ x, int i,
                                               int j, int k, size_t c, bool pin_full = false) {
    const size_t nxy = (size_t)L.nx * L.ny;
    double cxm, cxp, cym, cyp, czm, czp;
    cell_coefs<double>(L, i, j, k, c, cxm, cxp, cym, cyp, czm, czp);
    const double xc = __ldg(x + c);
    const double xw = i > 0 ? __ldg(x + c - 1) : (L.per_x ? __ldg(x + c + L.nx - 1) : 0.0);
    const double xe = i < L.nx - 1 ? __ldg(x + c + 1) : (L.per_x ? __ldg(x + c - (L.nx - 1)) : 0.0);
    const double xs = j > 0 ? __ldg(x + c - L.nx) : (L.per_y ? __ldg(x + c + (size_t)(L.ny - 1) * L.nx) : 0.0);
    const double xn = j < L.ny - 1 ? __ldg(x + c + L.nx) : (L.per_y ? __ldg(x + c - (size_t)(L.ny - 1) * L.nx) : 0.0);
    const double xb = k > 0 ? __ldg(x + c - nxy) : (L.per_z ? __ldg(x + c + (size_t)(L.nz - 1) * nxy) : 0.0);
    const double xt = k < L.nz - 1 ? __ldg(x + c + nxy) : (L.per_z ? __ldg(x + c - (size_t)(L.nz - 1) * nxy) : 0.0);
    double D = cxm + cxp + cym + cyp + czm + czp;
    if (L.pin && c == 0) {
        if (pin_full) D *= 2.0;
        else D += (L.nx > 1 ? cxp : 0.0) + (L.ny > 1 ? cyp : 0.0) + (L.nz > 1 ? czp : 0.0);
    }
    const double s = cxp * xe + cxm * xw + cyp * xn + cym * xs + czp * xt + czm * xb;
    return (s - D * xc) * L.inv_dx2;
}

// r = b - A x, with ||r||^2 and ||b||^2.  mode 0 (start of solve): fills r0sq, rr, bb,
// ref_norm and resets the counters; mode 1 (end of solve): fills rr_true, r is scratch.
template <class TC>
__device__ __forceinline__ void residual_body(const LevelOp<TC>& L, const double* __restrict__ x,
                                              const double* __restrict__ b, double* __restrict__ r, PcgState* st,
                                              double* partials, unsigned* ticket, int mode, int ref_is_b,
                                              float* __restrict__ r32, cudaGraphConditionalHandle cond,
                                              int use_cond, int zchunk, const VBlk& vb) {
    const bool mg = st->solver == SOLVE_MG;
    const bool first = vb.id == 0 && threadIdx.x == 0 && threadIdx.y == 0;
    if (mode == 2 && st->stop) { // standalone MG: finished before this cycle
        if (use_cond && first) cudaGraphSetConditional(cond, 0u);
        return;
    }
    if (mode == 2 && first) {
        // loop bound independent of the reductions (see xr_update_kernel)
        const int bc = atomicAdd(&st->body_count, 1) + 1;
        const bool over_time = global_ns() - st->t_start_ns > st->budget_ns;
        if (bc > st->max_iter + 1 || over_time) {
            if (over_time) st->status = PCG_TIMEOUT;
            st->stop = 1;
            if (use_cond) cudaGraphSetConditional(cond, 0u);
        }
    }
    double srr = 0.0, sbb = 0.0;
    const Col3 q = col3(L.nx, L.ny, L.nz, zchunk, vb.x, vb.y, vb.z);
    if (q.ok) {
        const size_t nxy = (size_t)L.nx * L.ny;
        for (int k = q.k0; k < q.k1; ++k) {
            const size_t c = (size_t)q.i + (size_t)L.nx * q.j + nxy * k;
            const double bv = b[c];
            const double rv = bv + (-1.0) * apply_A_cell(L, x, q.i, q.j, k, c, mg);
            r[c] = rv;
            if (r32) r32[c] = (float)rv;
            srr += rv * rv;
            sbb += bv * bv;
        }
    }
    double v[2] = {srr, sbb}, out[2];
    if (grid_sums<PK_NT, 2>(v, partials, ticket, vb.count, out, vb.id)) {
        if (mode == 0) {
            st->r0sq = out[0];
            st->rr = out[0];
            st->bb = out[1];
            st->ref_norm = ref_is_b ? sqrt(out[1]) : sqrt(out[0]);
            st->final_res = sqrt(out[0]);
            st->iter = 0;
            st->converged = 0;
            st->status = PCG_OK;
            st->rho_new = st->rho_old = st->gamma = st->pAp = 0.0;
            st->alpha = st->beta = 0.0;
            if (st->solver == SOLVE_MG) {
                // mg_solve has no early exit (src/multigrid/cycle/v_cycle.cu:90-113)
                st->stop = st->max_iter <= 0 ? 1 : 0;
            } else {
                // the reference returns at once when ||r0|| is (near) zero (pcg.cuh:122-127, cg.cuh:61-66)
                const double r0 = sqrt(out[0]);
                const bool done = st->solver == SOLVE_CG ? r0 <= st->rtol * r0 : r0 < 1e-15;
                st->stop = (done || st->max_iter <= 0) ? 1 : 0;
                if (done) st->converged = 1;
                st->rho_new = st->solver == SOLVE_CG ? out[0] : 0.0; // plain CG: rho = <r, r>
            }
            if (!isfinite(out[0])) { st->status = PCG_NONFINITE; st->stop = 1; }
            st->t_start_ns = global_ns();
        } else if (mode == 2) {
            // one standalone-MG cycle done: x updated, r = b - A x recomputed (v_cycle.cu:100-112)
            const int it = st->iter + 1;
            st->iter = it;
            st->rr = out[0];
            const double rn = sqrt(out[0]);
            st->final_res = rn;
            int stop = 0;
            if (rn / st->ref_norm < st->rtol) {
                st->converged = 1;
                stop = 1;
            }
            if (!isfinite(out[0])) {
                st->status = PCG_NONFINITE;
                stop = 1;
            }
            if (it >= st->max_iter) stop = 1;
            // a stop that the first block decided in this launch (body cap or time budget) stands
            if (*reinterpret_cast<volatile int*>(&st->stop)) stop = 1;
            st->stop = stop;
            if (use_cond) cudaGraphSetConditional(cond, stop ? 0u : 1u);
        } else {
            st->rr_true = out[0];
        }
    }
}

template <class TC>
__global__ void __launch_bounds__(PK_NT) residual_kernel(const LevelOp<TC> L, const double* __restrict__ x,
                                                         const double* __restrict__ b, double* __restrict__ r,
                                                         PcgState* st, double* partials, unsigned* ticket,
                                                         int mode, int ref_is_b, float* __restrict__ r32,
                                                         cudaGraphConditionalHandle cond, int use_cond, int zchunk) {
    residual_body<TC>(L, x, b, r, st, partials, ticket, mode, ref_is_b, r32, cond, use_cond, zchunk, hw_vblk());
}

// The search-direction update p = z + beta p (beta = 0 on the first iteration, where p = z
// exactly; Fletcher-Reeves rho_new / rho_old, or the flexible Polak-Ribiere form
// (rho_new - gamma) / rho_old) fused with Ap = A p and <p, Ap>: p_new is formed once per cell
// from z and p_old and written once, instead of written by one kernel and re-read by the
// next.  p_old and p_new live in two buffers that swap by iteration parity (pcg_pbuf_in /
// pcg_pbuf_out): no CTA overwrites a value that another still reads.
//
// 2.5-D blocking: a CTA of 32 x 8 threads owns a 32 x 8 column tile and marches a z chunk.
// Every thread stages, by cp.async into a ring of PMV_NS shared-memory slots, the z and p_old
// of its own cell (and of the ring cells beside the tile that it is assigned) and its cell's
// +x/+y/+z faces (the threads on the -x/-y edges also the -x/-y faces), PMV_NS - 1 planes ahead of
// the plane it applies: those copies are in flight while the CTA computes.  From a landed
// slot each thread forms p_new of the cells it staged into a double-buffered slab (tile plus
// one-cell ring); the stencil reads its x/y neighbours from the slab, its -z/+z values and
// its -z face from registers.  One barrier per plane.  Cells outside a non-periodic axis are
// staged as zeros (the operator's ghost value, p_new = 0); periodic axes wrap.  The stencil
// arithmetic per cell is that of apply_A_cell.
__device__ __forceinline__ const double* pcg_pbuf_in(int iter, const double* p0, const double* p1) {
    return (iter & 1) ? p1 : p0;
}
__device__ __forceinline__ double* pcg_pbuf_out(int iter, double* p0, double* p1) { return (iter & 1) ? p0 : p1; }

#ifndef MF3D_PMATVEC_MINB
#define MF3D_PMATVEC_MINB 3 // resident CTAs per SM the register budget is cut for (72 registers)
#endif
#ifndef MF3D_PMATVEC_PERSM
#define MF3D_PMATVEC_PERSM 8 // CTAs launched per SM (z chunks sized to match)
#endif
#ifndef MF3D_PMATVEC_NS
#define MF3D_PMATVEC_NS 4 // staged planes: the one applied, the next, PMV_NS - 2 in flight
#endif
constexpr int PMV_TX = 32, PMV_TY = 8, PMV_NS = MF3D_PMATVEC_NS;

template <class TZ> struct PmvSlot {
    TZ z[PMV_TY + 2][PMV_TX + 2];     // tile and ring, row 0 / column 0 at j0-1 / i0-1
    double p[PMV_TY + 2][PMV_TX + 2]; // p_old, same layout
    double cx[PMV_TY][PMV_TX + 1];    // +x faces at column tx+1; column 0: the -x faces at i0
    double cy[PMV_TY + 1][PMV_TX];    // +y faces at row ty+1; row 0: the -y faces at j0
    double cz[PMV_TY][PMV_TX];        // +z faces
};
template <class TZ> constexpr size_t pmv_smem_bytes() {
    return PMV_NS * sizeof(PmvSlot<TZ>) + 2 * sizeof(double) * (PMV_TY + 2) * (PMV_TX + 2);
}

// cp.async of B bytes (4 or 8); zeros when !ok (nothing is read then)
template <int B> __device__ __forceinline__ void pmv_cp(void* dst, const void* src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "n"(B), "r"(ok ? B : 0)
                 : "memory");
}

// One virtual block (32 x 8 column tile, one z chunk) of one realisation; `sm` is the CTA's
// dynamic shared memory (pmv_smem_bytes<TZ>()).  Every thread of the CTA calls it with the
// same arguments; a CTA that runs several blocks in turn separates them with the barrier at
// the top.
template <class TZ>
__device__ __forceinline__ void pmatvec_body(const LevelOp<double>& L, const TZ* __restrict__ z, double* p0,
                                             double* p1, double* __restrict__ Ap, PcgState* st, double* partials,
                                             unsigned* ticket, int zchunk, const VBlk& vb, unsigned char* sm) {
    constexpr int W = PMV_TX + 2; // slab / staged-plane row pitch
    PmvSlot<TZ>* slot = reinterpret_cast<PmvSlot<TZ>*>(sm);
    double* slab = reinterpret_cast<double*>(sm + PMV_NS * sizeof(PmvSlot<TZ>)); // [2][PMV_TY + 2][W]
    __syncthreads(); // the previous block's reads of the slots and the slab are done
    const PcgState s = *st;
    if (s.stop) return;
    const bool first = s.iter == 0;
    const double beta = first ? 0.0 : (s.rho_new - (s.flexible ? s.gamma : 0.0)) / s.rho_old;
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (vb.id == 0 && tx == 0 && ty == 0) st->beta = beta;
    const double* __restrict__ pin = pcg_pbuf_in(s.iter, p0, p1);
    double* __restrict__ pout = pcg_pbuf_out(s.iter, p0, p1);
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const size_t nxy = (size_t)nx * ny;
    const int i0 = vb.x * PMV_TX, j0 = vb.y * PMV_TY, i = i0 + tx, j = j0 + ty;
    const int k0 = vb.z * zchunk, k1 = min(k0 + zchunk, nz);
    const bool own = i < nx && j < ny;
    // Staging roles, fixed for the whole march: the thread's own cell, and at most one more
    // (warp-uniform kind): warp 0 the ring row below the tile, warp PMV_TY-1 the row above,
    // warp 1 lanes 0-15 the ring columns left and right, warp 1 lanes 16-23 the -x faces of
    // the tile's first column, warp 2 the -y faces of its first row.
    auto xy_of = [&](int ii, int jj, long long& g) {
        const int a = wrap_or_out(ii, nx, L.per_x), b = wrap_or_out(jj, ny, L.per_y);
        g = (long long)a + (long long)nx * b;
        return a >= 0 && b >= 0;
    };
    long long gO, gE = 0;
    const bool okO = xy_of(i, j, gO);
    const int fO = (ty + 1) * W + tx + 1;
    int kindE = 0, fE = 0; // 1: a ring cell at slab index fE; 2: a face into slot offset fE
    bool okE = false;
    const double* cb = L.cx; // kind 2: face of plane kk at cb + cs * kk
    size_t cs = 0;
    if (ty == 0 || ty == PMV_TY - 1) {
        kindE = 1;
        const int jj = ty == 0 ? j0 - 1 : j0 + PMV_TY;
        fE = (ty == 0 ? 0 : PMV_TY + 1) * W + tx + 1;
        okE = xy_of(i, jj, gE);
    } else if (ty == 1 && tx < 16) {
        kindE = 1;
        const int side = tx >> 3, row = tx & 7;
        fE = (row + 1) * W + (side ? PMV_TX + 1 : 0);
        okE = xy_of(side ? i0 + PMV_TX : i0 - 1, j0 + row, gE);
    } else if (ty == 1 && tx < 16 + PMV_TY) {
        kindE = 2;
        const int row = tx - 16, jj = j0 + row;
        okE = jj < ny;
        fE = (int)offsetof(PmvSlot<TZ>, cx) + row * (PMV_TX + 1) * 8;
        if (i0 > 0) cb = L.cx + (i0 - 1) + (size_t)nx * jj, cs = nxy;
        else if (L.per_x) cb = L.cx + (nx - 1) + (size_t)nx * jj, cs = nxy;
        else cb = L.bxm + jj, cs = (size_t)ny;
    } else if (ty == 2) {
        kindE = 2;
        okE = i < nx;
        fE = (int)offsetof(PmvSlot<TZ>, cy) + tx * 8;
        if (j0 > 0) cb = L.cy + i + (size_t)nx * (j0 - 1), cs = nxy;
        else if (L.per_y) cb = L.cy + i + (size_t)nx * (ny - 1), cs = nxy;
        else cb = L.bym + i, cs = (size_t)nx;
    }
    if (!okE && kindE == 2) cb = L.cx, cs = 0;
    const size_t cO = own ? (size_t)i + (size_t)nx * j : 0; // own cell in plane 0
    auto pval = [&](TZ zr, double pr) -> double {
        const double zv = (double)zr;
        return first ? zv : 1.0 * zv + beta * pr;
    };
    // one commit group per plane: z and p_old of the staged cells, the faces of the own cell
    auto issue = [&](int kk) {
        if (kk <= k1) {
            PmvSlot<TZ>& S = slot[(unsigned)(kk - k0) % PMV_NS];
            const int kz = wrap_or_out(kk, nz, L.per_z);
            const long long zo = (long long)nxy * (kz < 0 ? 0 : kz);
            const bool okO_k = okO && kz >= 0;
            const size_t g = okO_k ? (size_t)(gO + zo) : 0;
            pmv_cp<(int)sizeof(TZ)>(&S.z[0][0] + fO, z + g, okO_k);
            pmv_cp<8>(&S.p[0][0] + fO, pin + g, okO_k && !first);
            if (kindE == 1) {
                const bool ok = okE && kz >= 0;
                const size_t ge = ok ? (size_t)(gE + zo) : 0;
                pmv_cp<(int)sizeof(TZ)>(&S.z[0][0] + fE, z + ge, ok);
                pmv_cp<8>(&S.p[0][0] + fE, pin + ge, ok && !first);
            }
            if (kk < k1) {
                if (own) {
                    const size_t c = cO + nxy * kk;
                    pmv_cp<8>(&S.cx[ty][tx + 1], L.cx + c, true);
                    pmv_cp<8>(&S.cy[ty + 1][tx], L.cy + c, true);
                    pmv_cp<8>(&S.cz[ty][tx], L.cz + c, true);
                }
                if (kindE == 2) pmv_cp<8>(reinterpret_cast<unsigned char*>(&S) + fE, cb + cs * kk, okE);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // p_new of the staged cells of the plane in S, into the slab D; returns the own cell's
    auto form = [&](const PmvSlot<TZ>& S, double* D) -> double {
        const double v = pval((&S.z[0][0])[fO], (&S.p[0][0])[fO]);
        D[fO] = v;
        if (kindE == 1) D[fE] = pval((&S.z[0][0])[fE], (&S.p[0][0])[fE]);
        return v;
    };
    constexpr int SLAB = (PMV_TY + 2) * W;
    double acc = 0.0, pb = 0.0, czm = 0.0;
    size_t c = cO + nxy * k0;
    if (own) { // the -z neighbour and the -z face of the first plane, read directly
        const int kb = wrap_or_out(k0 - 1, nz, L.per_z);
        if (kb >= 0) {
            const size_t g = cO + nxy * kb;
            pb = pval(__ldg(z + g), first ? 0.0 : __ldg(pin + g));
        }
        czm = k0 > 0 ? __ldg(L.cz + c - nxy)
                     : (L.per_z ? __ldg(L.cz + c + (size_t)(nz - 1) * nxy) : __ldg(L.bzm + cO));
    }
#pragma unroll
    for (int q = 0; q < PMV_NS - 1; ++q) issue(k0 + q);
    asm volatile("cp.async.wait_group %0;" ::"n"(PMV_NS - 2) : "memory");
    double pc = form(slot[0], slab);
    for (int k = k0; k < k1; ++k, c += nxy) {
        // this thread's copies of plane k+1 have landed; the barrier publishes everyone's
        // copies of plane k and the slab of plane k, and frees the slot of plane k-1
        asm volatile("cp.async.wait_group %0;" ::"n"(PMV_NS - 3) : "memory");
        __syncthreads();
        issue(k + PMV_NS - 1);
        const unsigned u = (unsigned)(k - k0);
        const PmvSlot<TZ>& S = slot[u % PMV_NS];
        const double* P = slab + (u & 1u) * SLAB;
        const double pt = form(slot[(u + 1) % PMV_NS], slab + ((u + 1) & 1u) * SLAB);
        if (own) {
            const double cxp = S.cx[ty][tx + 1], cxm = S.cx[ty][tx];
            const double cyp = S.cy[ty + 1][tx], cym = S.cy[ty][tx];
            const double czp = S.cz[ty][tx];
            const double pw = P[fO - 1], pe = P[fO + 1], ps = P[fO - W], pn = P[fO + W];
            double D = cxm + cxp + cym + cyp + czm + czp;
            if (L.pin && c == 0) D += (nx > 1 ? cxp : 0.0) + (ny > 1 ? cyp : 0.0) + (nz > 1 ? czp : 0.0);
            const double sum = cxp * pe + cxm * pw + cyp * pn + cym * ps + czp * pt + czm * pb;
            const double y = (sum - D * pc) * L.inv_dx2;
            Ap[c] = y;
            pout[c] = pc;
            acc += pc * y;
            czm = czp;
        }
        pb = pc;
        pc = pt;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    double v[1] = {acc}, out[1];
    if (grid_sums<PMV_TX * PMV_TY, 1>(v, partials, ticket, vb.count, out, vb.id)) st->pAp = out[0];
}

template <class TZ>
__global__ void __launch_bounds__(PMV_TX * PMV_TY, MF3D_PMATVEC_MINB)
    pmatvec_dot_kernel(const LevelOp<double> L, const TZ* __restrict__ z, double* p0, double* p1,
                       double* __restrict__ Ap, PcgState* st, double* partials, unsigned* ticket, int zchunk) {
    extern __shared__ __align__(16) unsigned char pmv_sm[];
    pmatvec_body<TZ>(L, z, p0, p1, Ap, st, partials, ticket, zchunk, hw_vblk(), pmv_sm);
}

// x += alpha p; r -= alpha Ap (alpha = rho_new / pAp); ||r||^2 and, for the flexible form,
// gamma = <r_{k+1}, z_k>.  The last CTA runs the stopping test of pcg.cuh:156-164 and sets
// the graph's while condition.
template <class TZ>
__device__ __forceinline__ void xr_update_body(size_t n, double* __restrict__ x, const double* __restrict__ p,
                                               double* __restrict__ r, const double* __restrict__ Ap,
                                               const TZ* __restrict__ z, PcgState* st, double* partials,
                                               unsigned* ticket, cudaGraphConditionalHandle cond, int use_cond,
                                               float* __restrict__ r32, int blk, int nblk) {
    const PcgState s = *st;
    if (blk == 0 && threadIdx.x == 0) {
        // Loop bound that does not depend on the reductions: a body count and a device-time
        // budget, both checked by one thread, so no failure elsewhere can keep the loop alive.
        const int bc = atomicAdd(&st->body_count, 1) + 1;
        const bool over_time = global_ns() - s.t_start_ns > s.budget_ns;
        if (bc > s.max_iter + 1 || over_time) {
            if (over_time) st->status = PCG_TIMEOUT;
            st->stop = 1;
            if (use_cond) cudaGraphSetConditional(cond, 0u);
        }
    }
    if (s.stop) { // converged or failed before this iteration: leave x, r alone and end the loop
        if (use_cond && blk == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
        return;
    }
    const double alpha = s.rho_new / s.pAp;
    double srr = 0.0, sg = 0.0;
    // two cells per thread and pass (16-byte loads and stores); the vectors come from whole
    // allocations, so a pair starts on a 16-byte boundary; an odd last cell goes to thread 0
    auto cell = [&](size_t c) {
        x[c] = x[c] + alpha * p[c];
        const double rv = r[c] + (-alpha) * Ap[c];
        r[c] = rv;
        if (r32) r32[c] = (float)rv;
        srr += rv * rv;
        if (s.flexible) sg += rv * (double)z[c];
    };
    const size_t n2 = n >> 1;
    for (size_t c2 = blk * (size_t)PK_NT + threadIdx.x; c2 < n2; c2 += (size_t)nblk * PK_NT) {
        double2 xv = reinterpret_cast<const double2*>(x)[c2];
        const double2 pv = reinterpret_cast<const double2*>(p)[c2];
        double2 rv = reinterpret_cast<const double2*>(r)[c2];
        const double2 av = reinterpret_cast<const double2*>(Ap)[c2];
        xv.x = xv.x + alpha * pv.x;
        xv.y = xv.y + alpha * pv.y;
        rv.x = rv.x + (-alpha) * av.x;
        rv.y = rv.y + (-alpha) * av.y;
        reinterpret_cast<double2*>(x)[c2] = xv;
        reinterpret_cast<double2*>(r)[c2] = rv;
        if (r32) reinterpret_cast<float2*>(r32)[c2] = make_float2((float)rv.x, (float)rv.y);
        srr += rv.x * rv.x;
        srr += rv.y * rv.y;
        if (s.flexible) {
            double z0, z1;
            if constexpr (sizeof(TZ) == 8) {
                const double2 zv = reinterpret_cast<const double2*>(z)[c2];
                z0 = zv.x, z1 = zv.y;
            } else {
                const float2 zv = reinterpret_cast<const float2*>(z)[c2];
                z0 = (double)zv.x, z1 = (double)zv.y;
            }
            sg += rv.x * z0;
            sg += rv.y * z1;
        }
    }
    if ((n & 1) && blk == 0 && threadIdx.x == 0) cell(n - 1);
    double v[2] = {srr, sg}, out[2];
    if (grid_sums<PK_NT, 2>(v, partials, ticket, nblk, out, blk)) {
        const int it = s.iter + 1;
        st->iter = it;
        st->alpha = alpha;
        st->rr = out[0];
        st->gamma = out[1];
        st->rho_old = s.rho_new;
        if (s.solver == SOLVE_CG) st->rho_new = out[0]; // plain CG: rho = <r, r> for the next beta
        int stop = 0;
        if (!isfinite(out[0]) || !isfinite(s.pAp) || !isfinite(alpha)) {
            st->status = PCG_NONFINITE;
            stop = 1;
        } else if (s.pAp == 0.0) {
            st->status = PCG_BREAKDOWN;
            stop = 1;
        }
        if ((it % s.check_every) == 0 || it >= s.max_iter) {
            const double rn = sqrt(out[0]);
            st->final_res = rn;
            // pcg.cuh:158-160 tests ||r||/||r0|| < rtol; cg.cuh:142-150 tests ||r|| <= rtol ||r0||
            if (s.solver == SOLVE_CG ? rn <= s.rtol * s.ref_norm : rn / s.ref_norm < s.rtol) {
                st->converged = 1;
                stop = 1;
            }
        }
        if (it >= s.max_iter) stop = 1;
        // a stop that block 0 decided in this launch (body cap or time budget) stands: its store
        // precedes its arrival at the grid sum, which precedes this block's
        if (*reinterpret_cast<volatile int*>(&st->stop)) stop = 1;
        st->stop = stop;
        if (use_cond) cudaGraphSetConditional(cond, stop ? 0u : 1u);
    }
}

template <class TZ>
__global__ void __launch_bounds__(PK_NT) xr_update_kernel(size_t n, double* __restrict__ x, const double* __restrict__ p,
                                                          double* __restrict__ r, const double* __restrict__ Ap,
                                                          const TZ* __restrict__ z, PcgState* st,
                                                          double* partials, unsigned* ticket,
                                                          cudaGraphConditionalHandle cond, int use_cond,
                                                          float* __restrict__ r32, const double* p_alt) {
    // p_alt: the second search-direction buffer of pmatvec_dot_kernel (p is then the first);
    // this iteration's direction is the one that kernel wrote
    if (p_alt) p = (st->iter & 1) ? p : p_alt;
    xr_update_body<TZ>(n, x, p, r, Ap, z, st, partials, ticket, cond, use_cond, r32, blockIdx.x, gridDim.x);
}

// Sets the while condition before the loop from the state left by residual_kernel(mode 0).
__global__ void loop_gate_kernel(const PcgState* st, cudaGraphConditionalHandle cond) {
    cudaGraphSetConditional(cond, st->stop ? 0u : 1u);
}

// Standalone MG: x += z (the V-cycle of the current residual) unless the loop has stopped.
template <class TZ>
__global__ void __launch_bounds__(PK_NT) mg_xupdate_kernel(size_t n, double* __restrict__ x, const TZ* __restrict__ z,
                                                           const PcgState* st) {
    if (st->stop) return;
    for (size_t c = blockIdx.x * (size_t)PK_NT + threadIdx.x; c < n; c += (size_t)gridDim.x * PK_NT)
        x[c] = x[c] + (double)z[c];
}

// Re-opens a finished state so the iteration kernels can be timed in isolation (diagnostics).
__global__ void pcg_reopen_kernel(PcgState* st) {
    st->stop = 0;
    st->body_count = 0;
    st->iter = 1;
    st->rtol = 0.0; // never converges while being timed
    st->t_start_ns = global_ns();
}

// PCG state initialisation (host-given controls).
__global__ void pcg_init_kernel(PcgState* st, int max_iter, int check_every, int flexible, double rtol,
                                unsigned long long budget_ns, int solver) {
    st->solver = solver;
    st->max_iter = max_iter;
    st->body_count = 0;
    st->budget_ns = budget_ns;
    st->check_every = check_every > 0 ? check_every : 1;
    st->flexible = flexible;
    st->rtol = rtol;
    st->stop = 0;
}

} // namespace mf3d

// kernels_pcg.cuh -- fine-level operator and the device-resident PCG iteration.
//
// The reference's PCG (src/numerics/solvers/pcg.cuh:95-185) does two or three blocking
// host reductions per iteration.  Here every scalar lives in a PcgState in device memory,
// reductions are deterministic grid sums finished by the last CTA, and the CTA that
// finishes the x/r update also evaluates the stopping test and sets the CUDA-graph `while`
// condition, so a whole solve is one graph launch with no host round trip.
#pragma once
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

// p = z + beta p; beta = 0 on the first iteration, Fletcher-Reeves rho_new/rho_old, or the
// flexible Polak-Ribiere form (rho_new - gamma)/rho_old.
template <class TZ>
__device__ __forceinline__ void pupdate_body(size_t n, const TZ* __restrict__ z, double* __restrict__ p, PcgState* st,
                                             int blk, int nblk) {
    const PcgState s = *st;
    if (s.stop) return;
    const double beta = s.iter == 0 ? 0.0 : (s.rho_new - (s.flexible ? s.gamma : 0.0)) / s.rho_old;
    if (blk == 0 && threadIdx.x == 0) st->beta = beta;
    if (s.iter == 0) { // p = z exactly: whatever p held before must not leak in through 0 * p
        for (size_t c = blk * (size_t)PK_NT + threadIdx.x; c < n; c += (size_t)nblk * PK_NT) p[c] = (double)z[c];
        return;
    }
    for (size_t c = blk * (size_t)PK_NT + threadIdx.x; c < n; c += (size_t)nblk * PK_NT)
        p[c] = 1.0 * (double)z[c] + beta * p[c];
}

template <class TZ>
__global__ void __launch_bounds__(PK_NT) pupdate_kernel(size_t n, const TZ* __restrict__ z, double* __restrict__ p,
                                                        PcgState* st) {
    pupdate_body<TZ>(n, z, p, st, blockIdx.x, gridDim.x);
}

// Ap = A p and <p, Ap>.
template <class TC>
__device__ __forceinline__ void matvec_dot_body(const LevelOp<TC>& L, const double* __restrict__ p,
                                                double* __restrict__ Ap, PcgState* st, double* partials,
                                                unsigned* ticket, int zchunk, const VBlk& vb) {
    if (st->stop) return;
    double acc = 0.0;
    const Col3 q = col3(L.nx, L.ny, L.nz, zchunk, vb.x, vb.y, vb.z);
    if (q.ok) {
        const size_t nxy = (size_t)L.nx * L.ny;
        for (int k = q.k0; k < q.k1; ++k) {
            const size_t c = (size_t)q.i + (size_t)L.nx * q.j + nxy * k;
            const double y = apply_A_cell(L, p, q.i, q.j, k, c);
            Ap[c] = y;
            acc += __ldg(p + c) * y;
        }
    }
    double v[1] = {acc}, out[1];
    if (grid_sums<PK_NT, 1>(v, partials, ticket, vb.count, out, vb.id)) st->pAp = out[0];
}

template <class TC>
__global__ void __launch_bounds__(PK_NT) matvec_dot_kernel(const LevelOp<TC> L, const double* __restrict__ p,
                                                           double* __restrict__ Ap, PcgState* st,
                                                           double* partials, unsigned* ticket, int zchunk) {
    matvec_dot_body<TC>(L, p, Ap, st, partials, ticket, zchunk, hw_vblk());
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
    for (size_t c = blk * (size_t)PK_NT + threadIdx.x; c < n; c += (size_t)nblk * PK_NT) {
        x[c] = x[c] + alpha * p[c];
        const double rv = r[c] + (-alpha) * Ap[c];
        r[c] = rv;
        if (r32) r32[c] = (float)rv;
        srr += rv * rv;
        if (s.flexible) sg += rv * (double)z[c];
    }
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
                                                          float* __restrict__ r32) {
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

// kernels_batch.cuh -- PCG kernels of a batch of independent realisations.
//
// The reference's ensemble loop (src/runtime/ensemble/EnsembleRunner.cu:259-317) calls
// solve_head once per realisation, each solve a chain of small launches on its own grid.
// Here one launch serves every realisation of the batch: the realisations are segments of
// the launch's virtual blocks (find_seg), each segment runs the single-solve kernel body on
// its own grid, PCG state, partials and tickets, and a realisation whose solve has stopped
// (converged, failed or out of iterations) skips its segment.  The kernels are persistent:
// a grid of a few CTAs per SM walks the virtual blocks.
#pragma once
#include "kernels_pcg.cuh"

namespace mf3d {

// One realisation's fine-level PCG vectors and reduction scratch.
struct PcgItem {
    LevelOp<double> L;
    double* x;
    const double* b;
    double* r;
    double* p;  // search directions: p and p2 alternate by iteration (pmatvec_body)
    double* p2;
    double* Ap;
    const void* z;  // preconditioned residual, the V-cycle's type
    float* r32;     // FP32 copy of r for a mixed-precision V-cycle, or null
    PcgState* st;
    double* partials;
    unsigned* tickets; // 16 tickets: [2] residual, [3] matvec, [4] x/r update, [8..] V-cycle
    int* err;          // the V-cycle's TMA pipeline error flag
    size_t n;
    int zchunk, cgx, cgy, cgz; // column launch shape of the cell kernels
    int n1;                    // blocks of the streaming kernels
};

// Batch-wide loop control: a body count and a device-time budget, so that the loop ends
// whatever the reductions do.
struct BatchCtl {
    int bodies, cap;
    unsigned long long t_start, budget;
};

struct CopyItem {
    const double* src;
    double* dst;
    size_t n;
};

// PCG state initialisation of every realisation (one thread each); tickets cleared.
__global__ void batch_init_kernel(const PcgItem* __restrict__ items, int R, BatchCtl* ctl, int max_iter,
                                  int check_every, int flexible, double rtol, unsigned long long budget, int solver,
                                  int cap) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        PcgState* st = items[r].st;
        st->solver = solver;
        st->max_iter = max_iter;
        st->body_count = 0;
        st->budget_ns = budget;
        st->check_every = check_every > 0 ? check_every : 1;
        st->flexible = flexible;
        st->rtol = rtol;
        st->stop = 0;
        for (int k = 0; k < 16; ++k) items[r].tickets[k] = 0u;
    }
    if (threadIdx.x == 0) {
        ctl->bodies = 0;
        ctl->cap = cap;
        ctl->budget = budget;
        ctl->t_start = global_ns();
    }
}

// Loop gate: the while condition is 1 while any realisation is still iterating.  In the loop
// (in_loop = 1) it also counts the bodies; past the cap or the time budget every running
// realisation is stopped with status PCG_TIMEOUT.  any_out (optional) receives the condition.
__global__ void batch_gate_kernel(const PcgItem* __restrict__ items, int R, BatchCtl* ctl,
                                  cudaGraphConditionalHandle cond, int use_cond, int in_loop, int* any_out) {
    __shared__ int any, over;
    if (threadIdx.x == 0) {
        any = 0;
        over = 0;
        if (in_loop) {
            const int b = ++ctl->bodies;
            over = (b > ctl->cap || global_ns() - ctl->t_start > ctl->budget) ? 1 : 0;
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        PcgState* st = items[r].st;
        if (st->stop) continue;
        if (over) {
            st->status = PCG_TIMEOUT;
            st->stop = 1;
        } else {
            atomicOr(&any, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
        if (any_out) *any_out = any;
    }
}

// dst = src for every item (one segment per realisation)
__global__ void __launch_bounds__(PK_NT) batch_copy_kernel(const CopyItem* __restrict__ items,
                                                           const int* __restrict__ off, int nseg, int total) {
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int s = find_seg(off, nseg, b);
        const CopyItem it = items[s];
        const int o = __ldg(off + s), cnt = __ldg(off + s + 1) - o;
        for (size_t c = (size_t)(b - o) * PK_NT + threadIdx.x; c < it.n; c += (size_t)cnt * PK_NT) it.dst[c] = it.src[c];
    }
}

// r = b - A x with norms: mode 0 at the start of the solves, 1 (true residual) at the end.
__global__ void __launch_bounds__(PK_NT) batch_residual_kernel(const PcgItem* __restrict__ items,
                                                               const int* __restrict__ off, int nseg, int total,
                                                               int mode, int ref_is_b) {
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int s = find_seg(off, nseg, b);
        const PcgItem& it = items[s];
        const VBlk vb = make_vblk(b - __ldg(off + s), it.cgx, it.cgy, it.cgz);
        residual_body<double>(it.L, it.x, it.b, mode == 0 ? it.r : it.Ap, it.st, it.partials, it.tickets + 2, mode,
                              ref_is_b, mode == 0 ? it.r32 : nullptr, 0, 0, it.zchunk, vb);
    }
}

// p = z + beta p, Ap = A p and <p, Ap> (pmatvec_body) for every running realisation; dynamic
// shared memory pmv_smem_bytes<TZ>()
template <class TZ>
__global__ void __launch_bounds__(PMV_TX * PMV_TY, MF3D_PMATVEC_MINB)
    batch_pmatvec_kernel(const PcgItem* __restrict__ items, const int* __restrict__ off, int nseg, int total) {
    extern __shared__ __align__(16) unsigned char bpmv_sm[];
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int s = find_seg(off, nseg, b);
        const PcgItem& it = items[s];
        const VBlk vb = make_vblk(b - __ldg(off + s), it.cgx, it.cgy, it.cgz);
        pmatvec_body<TZ>(it.L, (const TZ*)it.z, it.p, it.p2, it.Ap, it.st, it.partials, it.tickets + 3, it.zchunk, vb,
                         bpmv_sm);
    }
}

template <class TZ>
__global__ void __launch_bounds__(PK_NT) batch_xr_update_kernel(const PcgItem* __restrict__ items,
                                                                const int* __restrict__ off, int nseg, int total) {
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int s = find_seg(off, nseg, b);
        const PcgItem& it = items[s];
        if (it.st->stop) continue;
        const int o = __ldg(off + s);
        const double* p = pcg_pbuf_out(it.st->iter, it.p, it.p2); // this iteration's direction
        xr_update_body<TZ>(it.n, it.x, p, it.r, it.Ap, (const TZ*)it.z, it.st, it.partials, it.tickets + 4, 0, 0,
                           it.r32, b - o, __ldg(off + s + 1) - o);
    }
}

// every realisation's PCG state and pipeline error flag into one array (one copy back to the
// host); the error flags are cleared
__global__ void batch_states_kernel(const PcgItem* __restrict__ items, int R, PcgState* __restrict__ out,
                                    int* __restrict__ errs) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        out[r] = *items[r].st;
        errs[r] = *items[r].err;
        *items[r].err = 0;
    }
}

} // namespace mf3d

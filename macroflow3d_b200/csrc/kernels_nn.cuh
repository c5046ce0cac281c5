// kernels_nn.cuh -- kernels of the learned warm start: a small 3-D convolutional
// encoder-decoder (BF16 activations and weights, FP32 accumulation) whose output is the PCG
// initial guess.  No counterpart in the reference, whose initial guess is the x-linear head
// (src/physics/flow/solve_head.cu:29-73).
//
// Layout: activations are voxel-major with channels innermost ("NDHWC"): element (v, c) at
// v * C + c, v = i + nx (j + ny k).  Weights of a 3x3x3 convolution are [cout][27][cin] with
// tap t = (dz+1)*9 + (dy+1)*3 + (dx+1).
//
// conv3d_tc_kernel: implicit GEMM on the 5th-generation tensor cores.  D[v][co] =
// sum_{t, ci} X[v + off(t)][ci] W[co][t][ci]: M = 128 voxels per tile, N = cout, K = 27 cin
// in steps of 16 channels.  Per tap, the CTA gathers the 128 x cin activation tile (zero
// outside the grid) and the cout x cin weight tile into shared memory in the canonical
// K-major, non-swizzled UMMA layout (8-row x 16-byte core matrices; the two 8-channel halves
// of a 16-channel step 128 bytes apart, 8-row groups 256 bytes apart), one thread issues the
// cin/16 tcgen05.mma of the tap into a TMEM accumulator (128 lanes x cout FP32 columns) and
// commits them to the tap's mbarrier, and the CTA gathers the next tap into the other buffer
// meanwhile.  The epilogue reads TMEM with tcgen05.ld (warp w owns lanes 32w..32w+31), adds
// the bias, applies ReLU or a ReLU-derivative mask, and stores BF16 or FP32.  The data
// gradient of a convolution is the same kernel on the output gradient with the weights
// flipped in the taps and transposed in the channels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels_pcg.cuh"

namespace mf3d {
namespace nn {

constexpr int CONV_NT = 128;   // 4 warps: one TMEM lane quarter each
constexpr int CONV_TM = 128;   // voxels per tile (UMMA M)
constexpr int CONV_MAXC = 128; // channel limit (multiples of 16)

// ---- tcgen05 helpers ------------------------------------------------------------------
__device__ __forceinline__ uint32_t sm_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D(tmem) (+)= A(smem desc) * B(smem desc)^T, kind::f16 (BF16 inputs, FP32 accumulate)
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}
// arrive on an mbarrier once every tcgen05.mma this thread issued before has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sm_u32(bar))
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void nn_mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_u32(bar)), "r"(count) : "memory");
}
// bounded wait on an mbarrier phase; false when it gave up
__device__ __forceinline__ bool nn_mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t a = sm_u32(bar);
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

// Shared-memory matrix descriptor of a K-major, non-swizzled operand tile: start address,
// leading byte offset (between the two 8-element K halves) 128 B, stride byte offset (between
// 8-row groups) 256 B, descriptor version 1 (sm_100), layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// byte offset of (row, k) in a K-major tile of `rows` rows and 16 K-columns
__device__ __forceinline__ uint32_t kmajor_off(int row, int khalf) {
    return (uint32_t)((row >> 3) * 256 + khalf * 128 + (row & 7) * 16);
}

struct ConvArgs {
    const __nv_bfloat16* x; // [V][cin]
    const __nv_bfloat16* w; // [cout][27][cin]
    const float* bias;      // [cout] or null
    void* y;                // [V][cout], BF16 or FP32
    const __nv_bfloat16* mask; // [V][cout] or null: y *= (mask > 0)
    int nx, ny, nz, cin, cout;
    int relu, y_f32;
    int* err; // set when an mbarrier wait gives up
};

// shared memory of conv3d_tc_kernel for (cin, cout): two buffers of (A 128 x cin, B cout x cin)
__host__ __device__ constexpr size_t conv_smem(int cin, int cout) {
    return 2 * ((size_t)CONV_TM * cin * 2 + (size_t)cout * cin * 2) + 64;
}
__host__ __device__ constexpr uint32_t tmem_cols(int cout) {
    return cout <= 32 ? 32u : cout <= 64 ? 64u : cout <= 128 ? 128u : 256u;
}

__global__ void __launch_bounds__(CONV_NT) conv3d_tc_kernel(const ConvArgs a) {
    extern __shared__ __align__(1024) unsigned char nn_sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cin = a.cin, cout = a.cout;
    const size_t abytes = (size_t)CONV_TM * cin * 2, bbytes = (size_t)cout * cin * 2;
    unsigned char* buf[2] = {nn_sm, nn_sm + abytes + bbytes};
    uint64_t* bars = reinterpret_cast<uint64_t*>(nn_sm + 2 * (abytes + bbytes)); // 2 mbarriers
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    const uint32_t ncols = tmem_cols(cout);
    if (warp == 0) {
        tmem_alloc(tmem_slot, ncols);
        tmem_relinquish();
    }
    if (tid == 0) {
        nn_mbar_init(&bars[0], 1);
        nn_mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long V = (long long)nx * ny * nz;
    const int ntiles = (int)((V + CONV_TM - 1) / CONV_TM);
    const uint32_t idesc = idesc_bf16(CONV_TM, cout);
    const int ksteps = cin / 16;
    unsigned phase[2] = {0u, 0u};
    int pending[2] = {0, 0}; // commits issued and not yet waited for, per buffer
    bool fail = false;

    for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
        const long long v = (long long)tile * CONV_TM + tid; // this thread's row
        const bool vin = v < V;
        int vi = 0, vj = 0, vk = 0;
        if (vin) {
            vi = (int)(v % nx);
            vj = (int)((v / nx) % ny);
            vk = (int)(v / ((long long)nx * ny));
        }
        for (int t = 0; t < 27 && !fail; ++t) {
            const int b = t & 1;
            // the buffer's previous MMAs must have finished reading it
            if (pending[b]) {
                if (!nn_mbar_wait(&bars[b], phase[b])) fail = true;
                phase[b] ^= 1u;
                pending[b] = 0;
            }
            if (__syncthreads_or(fail)) {
                fail = true;
                break;
            }
            const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dxo = t % 3 - 1;
            // ---- A: this thread's voxel row, cin channels of its neighbour at tap t ----
            {
                const int ii = vi + dxo, jj = vj + dy, kk = vk + dz;
                const bool ok = vin && ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz;
                const uint4* src = ok ? reinterpret_cast<const uint4*>(a.x + ((size_t)ii + (size_t)nx * ((size_t)jj + (size_t)ny * kk)) * cin)
                                      : nullptr;
                unsigned char* A = buf[b];
                for (int c = 0; c < cin / 8; ++c) {
                    const uint4 val = ok ? __ldg(src + c) : make_uint4(0u, 0u, 0u, 0u);
                    *reinterpret_cast<uint4*>(A + (size_t)(c >> 1) * (CONV_TM * 32) + kmajor_off(tid, c & 1)) = val;
                }
            }
            // ---- B: the weights of tap t ----
            {
                unsigned char* B = buf[b] + abytes;
                const int chunks = cout * (cin / 8);
                for (int q = tid; q < chunks; q += CONV_NT) {
                    const int n = q / (cin / 8), c = q % (cin / 8);
                    const uint4 val = __ldg(reinterpret_cast<const uint4*>(a.w + ((size_t)n * 27 + t) * cin) + c);
                    *reinterpret_cast<uint4*>(B + (size_t)(c >> 1) * (cout * 32) + kmajor_off(n, c & 1)) = val;
                }
            }
            // generic-proxy writes to shared memory, then visible to the tensor core
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const uint32_t abase = sm_u32(buf[b]), bbase = sm_u32(buf[b] + abytes);
                for (int s = 0; s < ksteps; ++s)
                    umma_bf16(tmem, kmajor_desc(abase + s * (CONV_TM * 32)), kmajor_desc(bbase + s * (cout * 32)),
                              idesc, (t > 0 || s > 0) ? 1u : 0u);
                umma_commit(&bars[b]);
            }
            pending[b] = 1;
        }
        // ---- epilogue: wait for the last MMAs, then TMEM -> registers -> global ----
        for (int b = 0; b < 2; ++b)
            if (pending[b]) {
                if (!nn_mbar_wait(&bars[b], phase[b])) fail = true;
                phase[b] ^= 1u;
                pending[b] = 0;
            }
        fail = __syncthreads_or(fail);
        if (fail) break;
        tc_fence_after();
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < cout; c0 += 16) {
            float acc[16];
            tmem_ld16(lane_base + (uint32_t)c0, acc);
            if (vin) {
                if (a.bias)
#pragma unroll
                    for (int i = 0; i < 16; ++i) acc[i] += __ldg(a.bias + c0 + i);
                if (a.relu)
#pragma unroll
                    for (int i = 0; i < 16; ++i) acc[i] = fmaxf(acc[i], 0.f);
                if (a.mask) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask + (size_t)v * cout + c0);
                    const uint4 m0 = __ldg(mp), m1 = __ldg(mp + 1);
                    const __nv_bfloat16* mb0 = reinterpret_cast<const __nv_bfloat16*>(&m0);
                    const __nv_bfloat16* mb1 = reinterpret_cast<const __nv_bfloat16*>(&m1);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        if (!(__bfloat162float(mb0[i]) > 0.f)) acc[i] = 0.f;
                        if (!(__bfloat162float(mb1[i]) > 0.f)) acc[8 + i] = 0.f;
                    }
                }
                if (a.y_f32) {
                    float4* yp = reinterpret_cast<float4*>(static_cast<float*>(a.y) + (size_t)v * cout + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) yp[i] = make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);
                } else {
                    __align__(16) __nv_bfloat16 o[16];
#pragma unroll
                    for (int i = 0; i < 16; ++i) o[i] = __float2bfloat16(acc[i]);
                    uint4* yp = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.y) + (size_t)v * cout + c0);
                    yp[0] = reinterpret_cast<const uint4*>(o)[0];
                    yp[1] = reinterpret_cast<const uint4*>(o)[1];
                }
            }
        }
        // every warp has read its lanes before the next tile's MMAs overwrite them
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (fail) {
        if (tid == 0) atomicExch(a.err, 1);
        // wait (bounded) for MMAs still in flight before the accumulator is released
        for (int b = 0; b < 2; ++b)
            if (pending[b]) (void)nn_mbar_wait(&bars[b], phase[b]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// ---- weight gradient (CUDA cores, FP32): dW[co][t][ci] = sum_v dY[v][co] X[v + off(t)][ci] ----
// One CTA per (tap, voxel chunk); the CTA's partial goes to part[chunk][co][t][ci] and
// wgrad_reduce_kernel adds the chunks in order (deterministic).
constexpr int WG_NT = 256;
constexpr int WG_VOX = 32; // voxels staged per step
__global__ void __launch_bounds__(WG_NT) wgrad_kernel(const __nv_bfloat16* __restrict__ x,
                                                      const __nv_bfloat16* __restrict__ dy, float* __restrict__ part,
                                                      int nx, int ny, int nz, int cin, int cout, int vox_per_chunk) {
    __shared__ float sx[WG_VOX][CONV_MAXC];
    __shared__ float sd[WG_VOX][CONV_MAXC];
    const int t = blockIdx.x, chunk = blockIdx.y;
    const int dz = t / 9 - 1, dyo = (t / 3) % 3 - 1, dxo = t % 3 - 1;
    const long long V = (long long)nx * ny * nz;
    const long long v0 = (long long)chunk * vox_per_chunk, v1 = min(V, v0 + vox_per_chunk);
    // thread -> (co, ci) pairs: cout * cin outputs, WG_NT threads
    const int npair = cout * cin;
    float acc[32]; // cout * cin <= 32 * WG_NT
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.f;
    for (long long vb = v0; vb < v1; vb += WG_VOX) {
        __syncthreads();
        for (int e = threadIdx.x; e < WG_VOX * cin; e += WG_NT) {
            const int q = e / cin, c = e % cin;
            const long long v = vb + q;
            float val = 0.f;
            if (v < v1) {
                const int i = (int)(v % nx) + dxo, j = (int)((v / nx) % ny) + dyo, k = (int)(v / ((long long)nx * ny)) + dz;
                if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz)
                    val = __bfloat162float(x[((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)) * cin + c]);
            }
            sx[q][c] = val;
        }
        for (int e = threadIdx.x; e < WG_VOX * cout; e += WG_NT) {
            const int q = e / cout, c = e % cout;
            const long long v = vb + q;
            sd[q][c] = v < v1 ? __bfloat162float(dy[(size_t)v * cout + c]) : 0.f;
        }
        __syncthreads();
        int k = 0;
        for (int p = threadIdx.x; p < npair; p += WG_NT, ++k) {
            const int co = p / cin, ci = p % cin;
            float s = 0.f;
#pragma unroll 8
            for (int q = 0; q < WG_VOX; ++q) s += sd[q][co] * sx[q][ci];
            acc[k] += s;
        }
    }
    int k = 0;
    for (int p = threadIdx.x; p < npair; p += WG_NT, ++k) {
        const int co = p / cin, ci = p % cin;
        part[((size_t)chunk * cout + co) * 27 * cin + (size_t)t * cin + ci] = acc[k];
    }
}

// dw (+)= sum over chunks of the partials, in chunk order (deterministic); used for the
// weight and the bias partials
__global__ void wgrad_reduce_kernel(const float* __restrict__ part, int nchunks, size_t n, float* __restrict__ dw,
                                    int accumulate) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < nchunks; ++c) s += part[(size_t)c * n + e];
        dw[e] = accumulate ? dw[e] + s : s;
    }
}

// bias gradient partials: part[chunk][co] = sum over the chunk's voxels of dY[v][co]
__global__ void bgrad_kernel(const __nv_bfloat16* __restrict__ dy, float* __restrict__ part, long long V, int cout,
                             int vox_per_chunk) {
    __shared__ float red[256];
    const int chunk = blockIdx.x;
    const long long v0 = (long long)chunk * vox_per_chunk, v1 = min(V, v0 + vox_per_chunk);
    for (int co = 0; co < cout; ++co) {
        float s = 0.f;
        for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) s += __bfloat162float(dy[(size_t)v * cout + co]);
        red[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(size_t)chunk * cout + co] = red[0];
        __syncthreads();
    }
}

// W'[ci][t][co] = W[co][26 - t][ci]: the data gradient as a forward convolution
__global__ void flip_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt, int cin,
                                    int cout) {
    const int n = cout * 27 * cin;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int co = e / (27 * cin), t = (e / cin) % 27, ci = e % cin;
        wt[((size_t)ci * 27 + (26 - t)) * cout + co] = w[e];
    }
}

// ---- pooling, upsampling with concatenation, and their gradients (C channels) ----
// average of the 8 children; fine grid (nx, ny, nz) even
__global__ void pool_kernel(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, int nx, int ny,
                            int nz, int C) {
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const size_t n = (size_t)cx * cy * cz * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t P = e / C;
        const int I = (int)(P % cx), J = (int)((P / cx) % cy), K = (int)(P / ((size_t)cx * cy));
        float s = 0.f;
        for (int d = 0; d < 8; ++d) {
            const int i = 2 * I + (d & 1), j = 2 * J + ((d >> 1) & 1), k = 2 * K + (d >> 2);
            s += __bfloat162float(x[((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)) * C + c]);
        }
        y[e] = __float2bfloat16(s * 0.125f);
    }
}
// dx_acc[child] += dy[parent] / 8
__global__ void pool_bwd_kernel(const __nv_bfloat16* __restrict__ dy, float* __restrict__ dx_acc, int nx, int ny,
                                int nz, int C) {
    const size_t n = (size_t)nx * ny * nz * C;
    const int cx = nx / 2, cy = ny / 2;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t v = e / C;
        const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((size_t)nx * ny));
        const size_t P = (size_t)(i >> 1) + (size_t)cx * ((size_t)(j >> 1) + (size_t)cy * (k >> 1));
        dx_acc[e] += 0.125f * __bfloat162float(dy[P * C + c]);
    }
}
// cat[v] = (coarse[parent(v)] (Ca channels), skip[v] (Cb channels)); fine grid (nx, ny, nz)
__global__ void upcat_kernel(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                             __nv_bfloat16* __restrict__ cat, int nx, int ny, int nz, int Ca, int Cb) {
    const int C = Ca + Cb, cx = nx / 2, cy = ny / 2;
    const size_t n = (size_t)nx * ny * nz * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t v = e / C;
        if (c < Ca) {
            const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((size_t)nx * ny));
            const size_t P = (size_t)(i >> 1) + (size_t)cx * ((size_t)(j >> 1) + (size_t)cy * (k >> 1));
            cat[e] = coarse[P * Ca + c];
        } else {
            cat[e] = skip[v * Cb + (c - Ca)];
        }
    }
}
// gradient of upcat: dcoarse[P] = sum over the 8 children of dcat[child][0:Ca];
// dskip_acc[v] += dcat[v][Ca:]
__global__ void upcat_bwd_coarse_kernel(const __nv_bfloat16* __restrict__ dcat, float* __restrict__ dcoarse,
                                        int nx, int ny, int nz, int Ca, int Cb) {
    const int C = Ca + Cb, cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const size_t n = (size_t)cx * cy * cz * Ca;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % Ca);
        const size_t P = e / Ca;
        const int I = (int)(P % cx), J = (int)((P / cx) % cy), K = (int)(P / ((size_t)cx * cy));
        float s = 0.f;
        for (int d = 0; d < 8; ++d) {
            const int i = 2 * I + (d & 1), j = 2 * J + ((d >> 1) & 1), k = 2 * K + (d >> 2);
            s += __bfloat162float(dcat[((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)) * C + c]);
        }
        dcoarse[e] = s;
    }
}
__global__ void upcat_bwd_skip_kernel(const __nv_bfloat16* __restrict__ dcat, float* __restrict__ dskip_acc,
                                      size_t V, int Ca, int Cb) {
    const int C = Ca + Cb;
    const size_t n = V * Cb;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t v = e / Cb;
        dskip_acc[e] += __bfloat162float(dcat[v * C + Ca + (e % Cb)]);
    }
}
// g = bf16(acc * (act > 0)) (the ReLU derivative of a layer whose output gradient was summed
// from two paths in FP32)
__global__ void mask_to_bf16_kernel(const float* __restrict__ acc, const __nv_bfloat16* __restrict__ act,
                                    __nv_bfloat16* __restrict__ g, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        g[e] = __float2bfloat16(__bfloat162float(act[e]) > 0.f ? acc[e] : 0.f);
}
__global__ void bf16_to_f32_kernel(const __nv_bfloat16* __restrict__ a, float* __restrict__ b, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        b[e] = __bfloat162float(a[e]);
}

// ---- network input, output and loss ----
// input channels: 0 lnK / 2, 1 the x-linear head guess - 1/2 (centred), 2..15 zero.
// h_lin = h_w + (h_e - h_w) (i + 1/2) / nx (init_head_guess, solve_head.cu:56-73)
// from lnK (training data, FP32) or from K (the solver's input, FP64: lnK = log K)
template <class TIN, bool FROM_K>
__global__ void nn_input_kernel(const TIN* __restrict__ src, __nv_bfloat16* __restrict__ in, int nx, int ny, int nz,
                                double hw, double he) {
    const size_t V = (size_t)nx * ny * nz;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < V; v += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % nx);
        const double hl = hw + (he - hw) * (i + 0.5) / nx;
        const double lnk = FROM_K ? log((double)src[v]) : (double)src[v];
        __align__(16) __nv_bfloat16 o[16];
        o[0] = __float2bfloat16((float)(0.5 * lnk));
        o[1] = __float2bfloat16((float)(hl - 0.5 * (hw + he)));
        for (int c = 2; c < 16; ++c) o[c] = __float2bfloat16(0.f);
        reinterpret_cast<uint4*>(in + v * 16)[0] = reinterpret_cast<const uint4*>(o)[0];
        reinterpret_cast<uint4*>(in + v * 16)[1] = reinterpret_cast<const uint4*>(o)[1];
    }
}
// x0 = h_lin + scale * out[v][0]
__global__ void nn_output_kernel(const float* __restrict__ out, double* __restrict__ x0, int nx, int ny, int nz,
                                 double hw, double he, double scale) {
    const size_t V = (size_t)nx * ny * nz;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < V; v += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % nx);
        const double hl = hw + (he - hw) * (i + 0.5) / nx;
        x0[v] = hl + scale * (double)out[v * 16];
    }
}
// loss = mean over voxels of (out[v][0] - (h - h_lin)/scale)^2; dout (BF16, 16 channels) =
// d loss / d out; per-block partial sums of the squared error in part[blockIdx.x]
__global__ void nn_loss_kernel(const float* __restrict__ out, const float* __restrict__ h,
                               __nv_bfloat16* __restrict__ dout, float* __restrict__ part, int nx, int ny, int nz,
                               double hw, double he, double inv_scale) {
    __shared__ float red[256];
    const size_t V = (size_t)nx * ny * nz;
    float s = 0.f;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < V; v += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % nx);
        const double hl = hw + (he - hw) * (i + 0.5) / nx;
        const float target = (float)((h[v] - hl) * inv_scale);
        const float d = out[v * 16] - target;
        s += d * d;
        __align__(16) __nv_bfloat16 o[16];
        o[0] = __float2bfloat16(2.f * d / (float)V);
        for (int c = 1; c < 16; ++c) o[c] = __float2bfloat16(0.f);
        reinterpret_cast<uint4*>(dout + v * 16)[0] = reinterpret_cast<const uint4*>(o)[0];
        reinterpret_cast<uint4*>(dout + v * 16)[1] = reinterpret_cast<const uint4*>(o)[1];
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Adam (Kingma & Ba 2015) on FP32 master weights; the BF16 copy the kernels read is refreshed.
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v2, size_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, float gscale) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float gg = g[e] * gscale;
        const float mm = b1 * m[e] + (1.f - b1) * gg;
        const float vv = b2 * v2[e] + (1.f - b2) * gg * gg;
        m[e] = mm;
        v2[e] = vv;
        const float wn = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        w[e] = wn;
        if (wb) wb[e] = __float2bfloat16(wn);
    }
}

} // namespace nn
} // namespace mf3d

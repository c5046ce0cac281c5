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
// bounded wait on an mbarrier phase; false when it gave up.  Each try suspends the thread for
// up to 2 us unless the phase completes first (fewer spinning instructions); at most `tries`.
__device__ __forceinline__ bool nn_mbar_wait(uint64_t* bar, unsigned parity, int tries = 1 << 20) {
    const uint32_t a = sm_u32(bar);
    for (int it = 0; it < tries; ++it) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity), "r"(2000u)
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
    return cout <= 32 ? 32u : cout <= 64 ? 64u : cout <= 128 ? 128u : cout <= 256 ? 256u : 512u;
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

// ---- conv3d_brick_kernel: the same convolution with the halo staged once per plane ----
// A CTA owns a 16 x 16 voxel brick (two 8 x 16 UMMA M-tiles) and marches it through a z
// range.  Producer warps stage each input plane of the brick plus a one-voxel halo
// (18 x 18 voxels x cin) into a ring of 4 plane slots with cp.async (zero fill outside the
// grid), one region per 8-channel half so that every tap's A operand is the same K-major
// canonical layout at a shifted start address: rows of 8 voxels along x at 16 bytes, 8-row
// groups (y) 18 x 16 = 288 bytes apart, the two channel halves of a 16-channel K-step one
// region (18 x 18 x 16 = 5184 bytes) apart.  The weights of all 27 taps stay in shared memory.
// One thread issues the 27 x cin/16 x 2 MMAs of an output plane into one of two TMEM
// accumulator buffers and commits them; four epilogue warps drain the other buffer
// meanwhile (bias, ReLU or mask, BF16 / FP32 store).  Every wait is bounded.
constexpr int BR_MAXNP = 8;                    // input plane slots, at most
constexpr int BR_PROD = 4, BR_EPI = 4;         // producer and epilogue warps
constexpr int BR_NT = (BR_PROD + 1 + BR_EPI) * 32;
// Brick geometry: A UMMA M-tiles of 8 x 16 voxels side by side in x (brick 8A x 16), a ring of
// NP input plane slots, each (8A + 2) x 18 voxels x cin channels, one region per 8 channels.
__host__ __device__ constexpr int brick_region(int A) { return (8 * A + 2) * 18 * 16; }
__host__ __device__ constexpr size_t brick_slot_bytes(int A, int cin) { return (size_t)brick_region(A) * (cin / 8); }
__host__ __device__ constexpr size_t brick_smem(int A, int NP, int cin, int coutp) {
    return (size_t)27 * coutp * cin * 2 + NP * brick_slot_bytes(A, cin) + 256;
}
__host__ __device__ constexpr uint32_t brick_tmem_cols(int A, int coutp) { return tmem_cols(2 * A * coutp); }

// K-major descriptor with explicit leading / stride byte offsets
__device__ __forceinline__ uint64_t kdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void nn_mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_u32(bar)) : "memory");
}

struct BrickArgs {
    int A, NP;        // M-tiles per brick row, input plane slots
    int co0, coutp;   // the output channels [co0, co0 + coutp) of a.cout computed by this launch
    int zchunk;       // planes per brick
};

template <int A>
__global__ void __launch_bounds__(BR_NT, 1) conv3d_brick_kernel(const ConvArgs a, const BrickArgs g) {
    extern __shared__ __align__(1024) unsigned char br_sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cin = a.cin, ctot = a.cout, nhg = cin / 8;
    const int NP = g.NP, co0 = g.co0, coutp = g.coutp, zchunk = g.zchunk;
    const int W = 8 * A + 2;                       // slot width in voxels
    const int REG = brick_region(A);               // bytes of one 8-channel region
    const size_t SLOT = brick_slot_bytes(A, cin);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    unsigned char* wsm = br_sm;                                   // weights: [t][hg][coutp] x 16 B
    unsigned char* slots = br_sm + (size_t)27 * coutp * cin * 2;  // NP plane slots
    uint64_t* bars = reinterpret_cast<uint64_t*>(slots + NP * SLOT);
    uint64_t* full = bars;                 // [NP] plane staged (BR_PROD*32 arrivals)
    uint64_t* empty = bars + BR_MAXNP;     // [NP] plane no longer read (MMA commit)
    uint64_t* tfull = bars + 2 * BR_MAXNP; // [2] accumulator ready (MMA commit)
    uint64_t* tempty = tfull + 2;          // [2] accumulator drained (BR_EPI*32 arrivals)
    uint64_t* drain = tempty + 2;          // [1] every MMA of the CTA done (teardown)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    int* s_fail = reinterpret_cast<int*>(tmem_slot + 1);
    const uint32_t ncols = brick_tmem_cols(A, coutp);
    const int mma_warp = BR_PROD;

    // weights of every tap (output channels co0..) in the canonical B layout: rows co at
    // 16 B, 8-row groups 128 B apart, one region of coutp rows per 8 input channels
    for (int q = tid; q < 27 * coutp * nhg; q += BR_NT) {
        const int t = q / (coutp * nhg), r = q % (coutp * nhg), n = r / nhg, hg = r % nhg;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(a.w + ((size_t)(co0 + n) * 27 + t) * cin) + hg);
        *reinterpret_cast<uint4*>(wsm + ((size_t)(t * nhg + hg) * coutp + n) * 16) = v;
    }
    if (warp == mma_warp) {
        tmem_alloc(tmem_slot, ncols);
        tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < NP; ++i) {
            nn_mbar_init(&full[i], BR_PROD * 32);
            nn_mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            nn_mbar_init(&tfull[i], 1);
            nn_mbar_init(&tempty[i], BR_EPI * 32);
        }
        nn_mbar_init(drain, 1);
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // weights -> tensor core
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int bw = 8 * A;
    const int bx = (nx + bw - 1) / bw, by = (ny + 15) / 16, nzc = (nz + zchunk - 1) / zchunk;
    const int nbricks = bx * by * nzc;
    bool fail = false;

    if (warp < BR_PROD) {
        // ---------------- producers: the brick's input planes, in order ----------------
        // The copies of plane p are committed as one group; the previous plane's group is then
        // waited for, fenced towards the tensor core's proxy and announced, so that one plane's
        // copies are always in flight while the previous one is published.
        unsigned pc = 0;          // planes staged so far (ring position)
        const int K = NP - 3;     // planes whose copies stay in flight (3 slots are being read)
        int pend[BR_MAXNP] = {}, np_ = 0, ph = 0; // committed, not yet announced slots (oldest at ph)
        const int nchunk = nhg * W * 18;
        // wait until at most n copy groups of this thread are pending
        auto wait_groups = [](int n) {
            switch (n) {
            case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
            case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
            case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
            case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
            case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
            default: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
            }
        };
        // announce the oldest pending plane once its copies have landed
        auto publish_oldest = [&]() {
            wait_groups(np_ - 1);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // generic -> async proxy
            nn_mbar_arrive(&full[pend[ph]]);
            ph = (ph + 1) % BR_MAXNP;
            --np_;
        };
        for (int br = blockIdx.x; br < nbricks && !fail; br += gridDim.x) {
            const int col = br % (bx * by), zc = br / (bx * by);
            const int x0 = (col % bx) * bw, y0 = (col / bx) * 16;
            const int z0 = zc * zchunk, z1 = min(nz, z0 + zchunk);
            for (int p = z0 - 1; p <= z1 && !fail; ++p, ++pc) {
                const int sl = (int)(pc % NP);
                if (pc >= (unsigned)NP) { // one lane per warp waits for the slot, the warp follows
                    bool ok = lane == 0 ? nn_mbar_wait(&empty[sl], ((pc / NP) - 1) & 1u) : true;
                    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                    if (!ok) {
                        fail = true;
                        break;
                    }
                }
                const uint32_t base = sm_u32(slots + (size_t)sl * SLOT);
                const bool pin = p >= 0 && p < nz;
                for (int q = tid; q < nchunk; q += BR_PROD * 32) {
                    const int hg = q / (W * 18), r = q % (W * 18), yy = r / W, xx = r % W;
                    const int gx = x0 - 1 + xx, gy = y0 - 1 + yy;
                    const bool ok = pin && gx >= 0 && gx < nx && gy >= 0 && gy < ny;
                    const __nv_bfloat16* src = ok ? a.x + (((size_t)p * ny + gy) * nx + gx) * cin + hg * 8 : a.x;
                    cp_async16(base + (uint32_t)(hg * REG + r * 16), src, ok);
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
                pend[(ph + np_) % BR_MAXNP] = sl;
                ++np_;
                while (np_ > K) publish_oldest();
            }
        }
        while (np_ > 0) publish_oldest(); // the last planes
        if (fail) atomicExch(s_fail, 1);
    } else if (warp == mma_warp) {
        // ---------------- MMA issuer (one thread) ----------------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(CONV_TM, coutp);
            const uint64_t bbase = kdesc(sm_u32(wsm), (uint32_t)(coutp * 16), 128u);
            unsigned pc = 0, pw = 0; // planes waited for, output planes done
            for (int br = blockIdx.x; br < nbricks && !fail; br += gridDim.x) {
                const int zc = br / (bx * by);
                const int z0 = zc * zchunk, z1 = min(nz, z0 + zchunk);
                const unsigned pfirst = pc; // ring position of plane z0 - 1
                for (int k = 0; k < 2 && !fail; ++k, ++pc)
                    if (!nn_mbar_wait(&full[pc % NP], (pc / NP) & 1u)) fail = true;
                for (int z = z0; z < z1 && !fail; ++z, ++pw) {
                    if (!nn_mbar_wait(&full[pc % NP], (pc / NP) & 1u)) { // plane z + 1
                        fail = true;
                        break;
                    }
                    ++pc;
                    const int tb = (int)(pw & 1u);
                    if (pw >= 2 && !nn_mbar_wait(&tempty[tb], ((pw / 2) - 1) & 1u)) {
                        fail = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dacc = tmem + (uint32_t)(tb * A * coutp);
                    // descriptors differ only in their start address (bits 0-13, in 16-byte
                    // units): one base per operand, offsets added
                    for (int dz = -1; dz <= 1; ++dz) {
                        const unsigned pr = pfirst + (unsigned)(z - z0 + 1 + dz); // ring position of plane z + dz
                        const uint64_t abase = kdesc(sm_u32(slots + (size_t)(pr % NP) * SLOT), (uint32_t)REG,
                                                     (uint32_t)(W * 16));
                        const int tz = (dz + 1) * 9;
                        for (int s2 = 0; s2 < cin / 16; ++s2) {
                            const uint64_t a_s = abase + (uint64_t)(2 * s2 * (REG >> 4));
                            const uint64_t b_s = bbase + (uint64_t)(2 * s2 * coutp);
#pragma unroll
                            for (int tyx = 0; tyx < 9; ++tyx) {
                                const int dy = tyx / 3, dx = tyx % 3; // 0..2: offsets + 1
                                const uint64_t bd = b_s + (uint64_t)((tz + tyx) * nhg * coutp);
                                // every tile's first product of the plane overwrites its accumulator
                                const uint32_t acc = (dz > -1 || s2 > 0 || tyx > 0) ? 1u : 0u;
#pragma unroll
                                for (int j = 0; j < A; ++j)
                                    umma_bf16(dacc + (uint32_t)(j * coutp), a_s + (uint64_t)(dy * W + dx + 8 * j), bd,
                                              idesc, acc);
                            }
                        }
                    }
                    umma_commit(&tfull[tb]);
                    // plane z - 1 is read by no later output plane of this brick
                    umma_commit(&empty[(pfirst + (unsigned)(z - z0)) % NP]);
                }
                if (!fail) { // the brick's last two planes (z1 - 1, z1) are released too
                    umma_commit(&empty[(pfirst + (unsigned)(z1 - z0)) % NP]);
                    umma_commit(&empty[(pfirst + (unsigned)(z1 - z0 + 1)) % NP]);
                }
            }
            if (fail) atomicExch(s_fail, 1);
        }
    } else {
        // ---------------- epilogue warps: TMEM -> registers -> global ----------------
        const int q = warp & 3;      // TMEM lane quarter this warp may access
        const int m = q * 32 + lane; // row of an M-tile: x = m % 8, y = m / 8
        unsigned pw = 0;
        for (int br = blockIdx.x; br < nbricks && !fail; br += gridDim.x) {
            const int col = br % (bx * by), zc = br / (bx * by);
            const int x0 = (col % bx) * bw, y0 = (col / bx) * 16;
            const int z0 = zc * zchunk, z1 = min(nz, z0 + zchunk);
            for (int z = z0; z < z1 && !fail; ++z, ++pw) {
                const int tb = (int)(pw & 1u);
                // one lane waits, the warp follows (the TMEM loads below are warp-collective)
                bool ok = lane == 0 ? nn_mbar_wait(&tfull[tb], (pw / 2) & 1u) : true;
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (!ok) {
                    fail = true;
                    break;
                }
                tc_fence_after();
                for (int j = 0; j < A; ++j) {
                    const int gx = x0 + 8 * j + (m & 7), gy = y0 + (m >> 3);
                    const bool vin = gx < nx && gy < ny;
                    const size_t v = ((size_t)z * ny + gy) * nx + gx;
                    for (int c0 = 0; c0 < coutp; c0 += 16) {
                        float acc[16];
                        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(tb * A * coutp + j * coutp + c0), acc);
                        if (!vin) continue;
                        const int cg = co0 + c0; // channel in the full output
                        if (a.bias)
#pragma unroll
                            for (int i = 0; i < 16; ++i) acc[i] += __ldg(a.bias + cg + i);
                        if (a.relu)
#pragma unroll
                            for (int i = 0; i < 16; ++i) acc[i] = fmaxf(acc[i], 0.f);
                        if (a.mask) {
                            const uint4* mp = reinterpret_cast<const uint4*>(a.mask + v * ctot + cg);
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
                            float4* yp = reinterpret_cast<float4*>(static_cast<float*>(a.y) + v * ctot + cg);
#pragma unroll
                            for (int i = 0; i < 4; ++i)
                                yp[i] = make_float4(acc[4 * i], acc[4 * i + 1], acc[4 * i + 2], acc[4 * i + 3]);
                        } else {
                            __align__(16) __nv_bfloat16 o[16];
#pragma unroll
                            for (int i = 0; i < 16; ++i) o[i] = __float2bfloat16(acc[i]);
                            uint4* yp = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.y) + v * ctot + cg);
                            yp[0] = reinterpret_cast<const uint4*>(o)[0];
                            yp[1] = reinterpret_cast<const uint4*>(o)[1];
                        }
                    }
                }
                tc_fence_before();
                nn_mbar_arrive(&tempty[tb]);
            }
        }
        if (fail) atomicExch(s_fail, 1);
    }
    // ---- teardown: every role has stopped issuing; the MMAs still in flight are waited for
    // (one more commit tracks all of them) before the accumulator is released ----
    __syncthreads();
    if (warp == mma_warp && lane == 0) {
        umma_commit(drain);
        if (!nn_mbar_wait(drain, 0u)) atomicExch(s_fail, 1);
    }
    __syncthreads();
    if (*s_fail && tid == 0) atomicExch(a.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == mma_warp) {
        tc_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// ---- weight gradient (CUDA cores, FP32): dW[co][t][ci] = sum_v dY[v][co] X[v + off(t)][ci] ----
// One CTA per (tap, voxel chunk); the CTA's partial goes to part[chunk][co][t][ci] and
// wgrad_reduce_kernel adds the chunks in order (deterministic).  Each thread owns 4 x 4
// (co, ci) outputs; when the layer has fewer than 256 such tiles, G thread groups split the
// staged voxels and their sums are added in shared memory at the end.
constexpr int WG_NT = 256;
constexpr int WG_VOX = 32; // voxels staged per step
__global__ void __launch_bounds__(WG_NT) wgrad_kernel(const __nv_bfloat16* __restrict__ x,
                                                      const __nv_bfloat16* __restrict__ dy, float* __restrict__ part,
                                                      int nx, int ny, int nz, int cin, int cout, int vox_per_chunk) {
    __shared__ __align__(16) float sx[WG_VOX][CONV_MAXC];
    __shared__ __align__(16) float sd[WG_VOX][CONV_MAXC];
    __shared__ __align__(16) float red[WG_NT * 16];
    const int t = blockIdx.x, chunk = blockIdx.y;
    const int dz = t / 9 - 1, dyo = (t / 3) % 3 - 1, dxo = t % 3 - 1;
    const long long V = (long long)nx * ny * nz;
    const long long v0 = (long long)chunk * vox_per_chunk, v1 = min(V, v0 + vox_per_chunk);
    const int tci = cin / 4, ntile = (cout / 4) * tci;
    const int G = ntile >= WG_NT ? 1 : WG_NT / ntile; // thread groups over the voxels
    const int per = (ntile + WG_NT - 1) / WG_NT;      // tiles per thread (G == 1)
    const int tid = threadIdx.x, grp = tid / (WG_NT / G), tin = tid % (WG_NT / G);
    const bool active = tid < G * (WG_NT / G) && (G > 1 ? tin < ntile : true);
    float acc[2][16];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[u][i] = 0.f;
    for (long long vb = v0; vb < v1; vb += WG_VOX) {
        __syncthreads();
        for (int e = tid; e < WG_VOX * (cin / 8); e += WG_NT) {
            const int q = e / (cin / 8), c8 = e % (cin / 8);
            const long long v = vb + q;
            uint4 raw = make_uint4(0u, 0u, 0u, 0u);
            if (v < v1) {
                const int i = (int)(v % nx) + dxo, j = (int)((v / nx) % ny) + dyo, k = (int)(v / ((long long)nx * ny)) + dz;
                if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz)
                    raw = __ldg(reinterpret_cast<const uint4*>(x + ((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)) * cin) + c8);
            }
            const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(&raw);
#pragma unroll
            for (int u = 0; u < 8; ++u) sx[q][c8 * 8 + u] = __bfloat162float(b[u]);
        }
        for (int e = tid; e < WG_VOX * (cout / 8); e += WG_NT) {
            const int q = e / (cout / 8), c8 = e % (cout / 8);
            const long long v = vb + q;
            uint4 raw = make_uint4(0u, 0u, 0u, 0u);
            if (v < v1) raw = __ldg(reinterpret_cast<const uint4*>(dy + (size_t)v * cout) + c8);
            const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(&raw);
#pragma unroll
            for (int u = 0; u < 8; ++u) sd[q][c8 * 8 + u] = __bfloat162float(b[u]);
        }
        __syncthreads();
        if (!active) continue;
        for (int u = 0; u < per && u < 2; ++u) {
            const int tile = G > 1 ? tin : tid + u * WG_NT;
            if (tile >= ntile) break;
            const int co0 = (tile / tci) * 4, ci0 = (tile % tci) * 4;
            for (int q = grp; q < WG_VOX; q += G) {
                const float4 d4 = *reinterpret_cast<const float4*>(&sd[q][co0]);
                const float4 x4 = *reinterpret_cast<const float4*>(&sx[q][ci0]);
                const float dv[4] = {d4.x, d4.y, d4.z, d4.w}, xv[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
                for (int a2 = 0; a2 < 4; ++a2)
#pragma unroll
                    for (int b2 = 0; b2 < 4; ++b2) acc[u][a2 * 4 + b2] += dv[a2] * xv[b2];
            }
        }
    }
    // sum the G groups (index order), then store the tile
    if (G > 1) {
        __syncthreads();
        if (active)
#pragma unroll
            for (int i = 0; i < 16; ++i) red[tid * 16 + i] = acc[0][i];
        __syncthreads();
        if (active && grp == 0) {
            for (int g2 = 1; g2 < G; ++g2)
#pragma unroll
                for (int i = 0; i < 16; ++i) acc[0][i] += red[(g2 * (WG_NT / G) + tin) * 16 + i];
        }
    }
    if (!active || (G > 1 && grp != 0)) return;
    for (int u = 0; u < per && u < 2; ++u) {
        const int tile = G > 1 ? tin : tid + u * WG_NT;
        if (tile >= ntile) break;
        const int co0 = (tile / tci) * 4, ci0 = (tile % tci) * 4;
#pragma unroll
        for (int a2 = 0; a2 < 4; ++a2)
#pragma unroll
            for (int b2 = 0; b2 < 4; ++b2)
                part[((size_t)chunk * cout + co0 + a2) * 27 * cin + (size_t)t * cin + ci0 + b2] = acc[u][a2 * 4 + b2];
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
// cat[v] = (coarse[parent(v)] (Ca channels), skip[v] (Cb channels)); fine grid (nx, ny, nz);
// one thread per 8-channel chunk (Ca, Cb multiples of 8)
__global__ void upcat_kernel(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                             __nv_bfloat16* __restrict__ cat, int nx, int ny, int nz, int Ca, int Cb) {
    const int qa = Ca / 8, qb = Cb / 8, Q = qa + qb, cx = nx / 2, cy = ny / 2;
    const size_t n = (size_t)nx * ny * nz * Q;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e % Q);
        const size_t v = e / Q;
        uint4 val;
        if (q < qa) {
            const int i = (int)(v % nx);
            const size_t r = v / nx;
            const int j = (int)(r % ny), k = (int)(r / ny);
            const size_t P = (size_t)(i >> 1) + (size_t)cx * ((size_t)(j >> 1) + (size_t)cy * (k >> 1));
            val = __ldg(reinterpret_cast<const uint4*>(coarse + P * Ca) + q);
        } else {
            val = __ldg(reinterpret_cast<const uint4*>(skip + v * Cb) + (q - qa));
        }
        reinterpret_cast<uint4*>(cat + v * (Ca + Cb))[q] = val;
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

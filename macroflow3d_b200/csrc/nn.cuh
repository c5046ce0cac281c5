// nn.cuh -- the learned warm start: a 3-D convolutional encoder-decoder with skip
// connections whose output, added to the reference's x-linear head guess, is the PCG initial
// guess (included at the end of solver.cu).  No counterpart in the reference
// (src/physics/flow/solve_head.cu:29-73 is its whole initial guess).
//
// Network (4 resolution levels, 16 -> 32 -> 64 -> 64 channels, 3x3x3 convolutions, ReLU):
//   L0: conv 16->16, conv 16->16 = e0          (input: lnK/2, the x-linear head, 14 zero channels)
//   L1: pool, conv 16->32, conv 32->32 = e1
//   L2: pool, conv 32->64, conv 64->64 = e2
//   L3: pool, conv 64->64, conv 64->64 = e3
//   L2: up(e3) ++ e2 -> conv 128->64 = d2
//   L1: up(d2) ++ e1 -> conv 96->32  = d1
//   L0: up(d1) ++ e0 -> conv 48->16  = d0, conv 16->16 (linear) = out; out[:, 0] predicts
//   (h - h_lin) / 0.1.
// BF16 weights and activations, FP32 accumulation (tensor cores), FP32 master weights and
// Adam moments.  Grid sizes must be multiples of 8 on every axis.
#pragma once
#include "kernels_nn.cuh"

namespace mf3d {
namespace nn {

constexpr double kTargetScale = 0.1; // out[:, 0] = (h - h_lin) / kTargetScale
constexpr size_t kBrickSmemMax = 220 * 1024; // shared memory of the brick convolution, at most

struct LayerSpec {
    int cin, cout, level, relu;
};
static const LayerSpec kLayers[12] = {
    {16, 16, 0, 1}, {16, 16, 0, 1}, {16, 32, 1, 1}, {32, 32, 1, 1}, {32, 64, 2, 1}, {64, 64, 2, 1},
    {64, 64, 3, 1}, {64, 64, 3, 1}, {128, 64, 2, 1}, {96, 32, 1, 1}, {48, 16, 0, 1}, {16, 16, 0, 0},
};
constexpr int kNumLayers = 12;

struct Dims {
    int nx, ny, nz;
    size_t v() const { return (size_t)nx * ny * nz; }
    Dims half() const { return Dims{nx / 2, ny / 2, nz / 2}; }
};

static unsigned ew_grid(size_t n) { return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

class WarmStartNet {
  public:
    explicit WarmStartNet(unsigned long long seed) {
        size_t off = 0;
        for (int l = 0; l < kNumLayers; ++l) {
            woff_[l] = off;
            off += (size_t)kLayers[l].cout * 27 * kLayers[l].cin;
            boff_[l] = off;
            off += kLayers[l].cout;
        }
        nparam_ = off;
        w32_.alloc(nparam_ * 4);
        g32_.alloc(nparam_ * 4);
        m_.alloc(nparam_ * 4);
        v_.alloc(nparam_ * 4);
        wbf_.alloc(nparam_ * 2);
        wflip_.alloc(nparam_ * 2);
        err_.alloc(16);
        MF3D_CK(cudaMemset(m_.p, 0, nparam_ * 4));
        MF3D_CK(cudaMemset(v_.p, 0, nparam_ * 4));
        MF3D_CK(cudaMemset(g32_.p, 0, nparam_ * 4));
        MF3D_CK(cudaMemset(err_.p, 0, 16));
        // He-normal initialisation from a counter-based stream (Box-Muller on Philox draws);
        // the input layer's fan-in counts its two live channels, the output layer starts small
        std::vector<float> h(nparam_, 0.f);
        for (int l = 0; l < kNumLayers; ++l) {
            const LayerSpec& L = kLayers[l];
            const int fan = 27 * (l == 0 ? 2 : L.cin);
            const double sd = std::sqrt(2.0 / fan) * (l == kNumLayers - 1 ? 0.1 : 1.0);
            for (size_t e = 0; e < (size_t)L.cout * 27 * L.cin; ++e) {
                uint32_t o[4];
                Philox::gen(seed, (uint32_t)l + 0x4E4E0000u, (uint32_t)e, o);
                const double u1 = ((double)o[0] + 1.0) / 4294967297.0, u2 = (double)o[1] / 4294967296.0;
                double val = sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                if (l == 0 && (int)(e % L.cin) >= 2) val = 0.0; // zero input channels
                h[woff_[l] + e] = (float)val;
            }
        }
        set_params(h.data());
        step_ = 0;
    }

    size_t num_params() const { return nparam_; }

    void get_params(float* host) const { MF3D_CK(cudaMemcpy(host, w32_.p, nparam_ * 4, cudaMemcpyDeviceToHost)); }
    void get_grads(float* host) const { MF3D_CK(cudaMemcpy(host, g32_.p, nparam_ * 4, cudaMemcpyDeviceToHost)); }

    void set_params(const float* host) {
        MF3D_CK(cudaMemcpy(w32_.p, host, nparam_ * 4, cudaMemcpyHostToDevice));
        refresh_bf16(nullptr);
        MF3D_CK(cudaDeviceSynchronize());
    }

    // x0 = h_lin + scale * net(K)
    void predict(const Dims& d, double hw, double he, const double* K, double* x0, cudaStream_t s) {
        check_dims(d);
        ensure(d);
        nn_input_kernel<double, true><<<ew_grid(d.v()), 256, 0, s>>>(K, bufs_.in, d.nx, d.ny, d.nz, hw, he);
        MF3D_LAUNCH_CK();
        forward(d, s);
        nn_output_kernel<<<ew_grid(d.v()), 256, 0, s>>>(bufs_.out, x0, d.nx, d.ny, d.nz, hw, he, kTargetScale);
        MF3D_LAUNCH_CK();
        check_err(s);
    }

    // One optimisation step on `count` samples (lnK, h: FP32 device arrays of grid d):
    // gradients summed over the samples, Adam with the mean gradient.  lr <= 0: gradients only
    // (left in the gradient buffer, nothing updated).  Returns the mean loss.
    double train_step(const Dims& d, int count, const float* const* lnK, const float* const* h, double hw, double he,
                      float lr, cudaStream_t s) {
        check_dims(d);
        ensure(d);
        MF3D_CK(cudaMemsetAsync(g32_.p, 0, nparam_ * 4, s));
        double loss = 0.0;
        for (int i = 0; i < count; ++i) {
            nn_input_kernel<float, false><<<ew_grid(d.v()), 256, 0, s>>>(lnK[i], bufs_.in, d.nx, d.ny, d.nz, hw, he);
            MF3D_LAUNCH_CK();
            forward(d, s);
            const unsigned nb = std::min<unsigned>(ew_grid(d.v()), 1024);
            nn_loss_kernel<<<nb, 256, 0, s>>>(bufs_.out, h[i], bufs_.dout, bufs_.lpart, d.nx, d.ny, d.nz, hw, he,
                                              1.0 / kTargetScale);
            MF3D_LAUNCH_CK();
            backward(d, s);
            std::vector<float> lp(nb);
            MF3D_CK(cudaMemcpyAsync(lp.data(), bufs_.lpart, nb * 4, cudaMemcpyDeviceToHost, s));
            MF3D_CK(cudaStreamSynchronize(s));
            double sum = 0.0;
            for (float x : lp) sum += x;
            loss += sum / (double)d.v();
        }
        if (lr > 0.f) {
            ++step_;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)step_), c2 = 1.f - std::pow(b2, (float)step_);
            adam_kernel<<<ew_grid(nparam_), 256, 0, s>>>(w32_.as<float>(), nullptr, g32_.as<float>(), m_.as<float>(),
                                                         v_.as<float>(), nparam_, lr, b1, b2, 1e-8f, c1, c2,
                                                         1.f / (float)count);
            MF3D_LAUNCH_CK();
            refresh_bf16(s);
        }
        check_err(s);
        return loss / count;
    }

    // loss of the current weights on samples, no gradient
    double eval(const Dims& d, int count, const float* const* lnK, const float* const* h, double hw, double he,
                cudaStream_t s) {
        check_dims(d);
        ensure(d);
        double loss = 0.0;
        for (int i = 0; i < count; ++i) {
            nn_input_kernel<float, false><<<ew_grid(d.v()), 256, 0, s>>>(lnK[i], bufs_.in, d.nx, d.ny, d.nz, hw, he);
            MF3D_LAUNCH_CK();
            forward(d, s);
            const unsigned nb = std::min<unsigned>(ew_grid(d.v()), 1024);
            nn_loss_kernel<<<nb, 256, 0, s>>>(bufs_.out, h[i], bufs_.dout, bufs_.lpart, d.nx, d.ny, d.nz, hw, he,
                                              1.0 / kTargetScale);
            MF3D_LAUNCH_CK();
            std::vector<float> lp(nb);
            MF3D_CK(cudaMemcpyAsync(lp.data(), bufs_.lpart, nb * 4, cudaMemcpyDeviceToHost, s));
            MF3D_CK(cudaStreamSynchronize(s));
            double sum = 0.0;
            for (float x : lp) sum += x;
            loss += sum / (double)d.v();
        }
        check_err(s);
        return loss / count;
    }

    // ---- single operations (tests) ----
    static void conv(cudaStream_t s, const Dims& d, int cin, int cout, const __nv_bfloat16* x,
                     const __nv_bfloat16* w, const float* bias, int relu, const __nv_bfloat16* mask, int y_f32,
                     void* y, int* err) {
        if (cin % 16 || cout % 16 || cin < 16 || cout < 16 || cin > CONV_MAXC || cout > CONV_MAXC)
            throw Error(MF3D_E_INVALID, "convolution channels must be multiples of 16 in [16, 128]");
        ConvArgs a{};
        a.x = x;
        a.w = w;
        a.bias = bias;
        a.y = y;
        a.mask = mask;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.cin = cin;
        a.cout = cout;
        a.relu = relu;
        a.y_f32 = y_f32;
        a.err = err;
        // brick kernel (halo staged once per plane) when a geometry fits: the output channels
        // in as few launches as possible (1, 2 or 4), then two or one M-tiles per brick, then
        // four or three plane slots
        // More M-tiles per brick (A) give the tensor core more independent accumulators to
        // interleave; no wider than the grid.
        int amax = 1;
        while (amax < 8 && 8 * amax * 2 <= std::max(8, d.nx)) amax *= 2;
        for (int split = 1; split <= 4; split *= 2)
            for (int A = amax; A >= 1; A /= 2)
                for (int NP = 8; NP >= 3; --NP) { // 3 slots read, NP - 3 loading ahead
                    const int coutp = cout / split;
                    if (cout % split || coutp % 16 || cin > 128) continue;
                    if (brick_smem(A, NP, cin, coutp) > kBrickSmemMax || 2 * A * coutp > 512) continue;
                    if (A > 1 && NP < 5 && brick_smem(A / 2, 5, cin, coutp) <= kBrickSmemMax) continue; // keep lookahead
                    auto kern = A == 8 ? conv3d_brick_kernel<8>
                              : A == 4 ? conv3d_brick_kernel<4>
                              : A == 2 ? conv3d_brick_kernel<2> : conv3d_brick_kernel<1>;
                    MF3D_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBrickSmemMax));
                    const int cols = ((d.nx + 8 * A - 1) / (8 * A)) * ((d.ny + 15) / 16);
                    const int nzc = std::max(1, std::min(std::max(1, d.nz / 4), (2 * num_sms() + cols - 1) / cols));
                    BrickArgs g{};
                    g.A = A;
                    g.NP = NP;
                    g.coutp = coutp;
                    g.zchunk = (d.nz + nzc - 1) / nzc;
                    const long long bricks = (long long)cols * ((d.nz + g.zchunk - 1) / g.zchunk);
                    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(bricks, num_sms()));
                    for (int c = 0; c < split; ++c) {
                        g.co0 = c * coutp;
                        kern<<<grid, BR_NT, brick_smem(A, NP, cin, coutp), s>>>(a, g);
                        MF3D_LAUNCH_CK();
                    }
                    return;
                }
        const size_t smem = conv_smem(cin, cout);
        MF3D_CK(cudaFuncSetAttribute(conv3d_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)conv_smem(CONV_MAXC, CONV_MAXC)));
        // all of the unified L1 as shared memory: without it the driver sizes the carveout for
        // the largest allowed allocation and keeps one CTA per SM
        MF3D_CK(cudaFuncSetAttribute(conv3d_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        int occ = 0;
        MF3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, conv3d_tc_kernel, CONV_NT, smem));
        // no more CTAs per SM than their TMEM accumulators fit in (512 columns)
        occ = std::max(1, std::min<int>(occ, (int)(512 / tmem_cols(cout))));
        const long long tiles = ((long long)d.v() + CONV_TM - 1) / CONV_TM;
        const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(tiles, (long long)occ * num_sms()));
        conv3d_tc_kernel<<<grid, CONV_NT, smem, s>>>(a);
        MF3D_LAUNCH_CK();
    }

    // dW (FP32, [cout][27][cin]) and db ([cout]) of a convolution from its input x and the
    // gradient dy of its pre-activation output; accumulate adds to dw / db
    static void wgrad(cudaStream_t s, const Dims& d, int cin, int cout, const __nv_bfloat16* x,
                      const __nv_bfloat16* dy, float* dw, float* db, float* part, size_t part_floats,
                      int accumulate) {
        const long long V = (long long)d.v();
        int vpc = (int)std::max<long long>(WG_VOX, ((V + 63) / 64 + WG_VOX - 1) / WG_VOX * WG_VOX); // <= 64 chunks
        int nch = (int)((V + vpc - 1) / vpc);
        const size_t wn = (size_t)cout * 27 * cin;
        if ((size_t)nch * wn > part_floats) throw Error(MF3D_E_INVALID, "weight-gradient scratch too small");
        if (cout * cin > 2 * 16 * WG_NT) throw Error(MF3D_E_INVALID, "layer too wide for the weight gradient");
        wgrad_kernel<<<dim3(27, nch), WG_NT, 0, s>>>(x, dy, part, d.nx, d.ny, d.nz, cin, cout, vpc);
        MF3D_LAUNCH_CK();
        wgrad_reduce_kernel<<<ew_grid(wn), 256, 0, s>>>(part, nch, wn, dw, accumulate);
        MF3D_LAUNCH_CK();
        bgrad_kernel<<<nch, 256, 0, s>>>(dy, part, V, cout, vpc);
        MF3D_LAUNCH_CK();
        wgrad_reduce_kernel<<<1, 256, 0, s>>>(part, nch, (size_t)cout, db, accumulate);
        MF3D_LAUNCH_CK();
    }

    static void flip(cudaStream_t s, int cin, int cout, const __nv_bfloat16* w, __nv_bfloat16* wt) {
        flip_weights_kernel<<<ew_grid((size_t)cout * 27 * cin), 256, 0, s>>>(w, wt, cin, cout);
        MF3D_LAUNCH_CK();
    }

  private:
    struct Bufs {
        Dims d{0, 0, 0};
        std::vector<std::unique_ptr<DevMem>> mem;
        __nv_bfloat16 *in, *a0, *e0, *p0, *a2, *e1, *p1, *a4, *e2, *p2, *a6, *e3, *c2, *d2, *c1, *d1, *c0, *d0;
        float* out;
        __nv_bfloat16* dout;
        float* lpart;
        // backward: gradient buffers (BF16 for the tensor-core operands, FP32 accumulators)
        __nv_bfloat16 *g0, *g1; // [V0 x 128] ping-pong gradient buffers, sized for the widest level use
        float *acc0, *acc1, *acc2; // FP32 skip-gradient accumulators at L0 (16), L1 (32), L2 (64)
        float* accc;               // FP32 coarse gradient of an upsampling (<= V1 x 64)
        float* part;
        size_t part_floats;
    } bufs_;

    void check_dims(const Dims& d) const {
        if (d.nx % 8 || d.ny % 8 || d.nz % 8 || d.nx < 8 || d.ny < 8 || d.nz < 8)
            throw Error(MF3D_E_INVALID, "the warm-start network needs grid sizes that are multiples of 8");
    }

    void ensure(const Dims& d) {
        if (bufs_.d.nx == d.nx && bufs_.d.ny == d.ny && bufs_.d.nz == d.nz) return;
        bufs_.mem.clear();
        const size_t V0 = d.v(), V1 = V0 / 8, V2 = V1 / 8, V3 = V2 / 8;
        auto bf = [&](size_t n) {
            bufs_.mem.emplace_back(new DevMem(std::max<size_t>(n, 8) * 2));
            return bufs_.mem.back()->as<__nv_bfloat16>();
        };
        auto f32 = [&](size_t n) {
            bufs_.mem.emplace_back(new DevMem(std::max<size_t>(n, 8) * 4));
            return bufs_.mem.back()->as<float>();
        };
        bufs_.in = bf(V0 * 16);
        bufs_.a0 = bf(V0 * 16);
        bufs_.e0 = bf(V0 * 16);
        bufs_.p0 = bf(V1 * 16);
        bufs_.a2 = bf(V1 * 32);
        bufs_.e1 = bf(V1 * 32);
        bufs_.p1 = bf(V2 * 32);
        bufs_.a4 = bf(V2 * 64);
        bufs_.e2 = bf(V2 * 64);
        bufs_.p2 = bf(V3 * 64);
        bufs_.a6 = bf(V3 * 64);
        bufs_.e3 = bf(V3 * 64);
        bufs_.c2 = bf(V2 * 128);
        bufs_.d2 = bf(V2 * 64);
        bufs_.c1 = bf(V1 * 96);
        bufs_.d1 = bf(V1 * 32);
        bufs_.c0 = bf(V0 * 48);
        bufs_.d0 = bf(V0 * 16);
        bufs_.out = f32(V0 * 16);
        bufs_.dout = bf(V0 * 16);
        bufs_.lpart = f32(1024);
        bufs_.g0 = bf(V0 * 48);
        bufs_.g1 = bf(V0 * 48);
        bufs_.acc0 = f32(V0 * 16);
        bufs_.acc1 = f32(V1 * 32);
        bufs_.acc2 = f32(V2 * 64);
        bufs_.accc = f32(V1 * 64);
        bufs_.part_floats = (size_t)64 * 27 * 128 * 64; // 64 chunks of the widest layer
        bufs_.part = f32(bufs_.part_floats);
        bufs_.d = d;
    }

    __nv_bfloat16* W(int l) { return wbf_.as<__nv_bfloat16>() + woff_[l]; }
    __nv_bfloat16* WT(int l) { return wflip_.as<__nv_bfloat16>() + woff_[l]; }
    float* B(int l) { return w32_.as<float>() + boff_[l]; }
    float* GW(int l) { return g32_.as<float>() + woff_[l]; }
    float* GB(int l) { return g32_.as<float>() + boff_[l]; }

    void layer(cudaStream_t s, int l, const Dims& d, const __nv_bfloat16* x, void* y, int y_f32 = 0) {
        conv(s, d, kLayers[l].cin, kLayers[l].cout, x, W(l), B(l), kLayers[l].relu, nullptr, y_f32, y, err_.as<int>());
    }

    void forward(const Dims& d0, cudaStream_t s) {
        Bufs& b = bufs_;
        const Dims d1 = d0.half(), d2 = d1.half(), d3 = d2.half();
        layer(s, 0, d0, b.in, b.a0);
        layer(s, 1, d0, b.a0, b.e0);
        pool_kernel<<<ew_grid(d1.v() * 16), 256, 0, s>>>(b.e0, b.p0, d0.nx, d0.ny, d0.nz, 16);
        MF3D_LAUNCH_CK();
        layer(s, 2, d1, b.p0, b.a2);
        layer(s, 3, d1, b.a2, b.e1);
        pool_kernel<<<ew_grid(d2.v() * 32), 256, 0, s>>>(b.e1, b.p1, d1.nx, d1.ny, d1.nz, 32);
        MF3D_LAUNCH_CK();
        layer(s, 4, d2, b.p1, b.a4);
        layer(s, 5, d2, b.a4, b.e2);
        pool_kernel<<<ew_grid(d3.v() * 64), 256, 0, s>>>(b.e2, b.p2, d2.nx, d2.ny, d2.nz, 64);
        MF3D_LAUNCH_CK();
        layer(s, 6, d3, b.p2, b.a6);
        layer(s, 7, d3, b.a6, b.e3);
        upcat_kernel<<<ew_grid(d2.v() * 16), 256, 0, s>>>(b.e3, b.e2, b.c2, d2.nx, d2.ny, d2.nz, 64, 64);
        MF3D_LAUNCH_CK();
        layer(s, 8, d2, b.c2, b.d2);
        upcat_kernel<<<ew_grid(d1.v() * 12), 256, 0, s>>>(b.d2, b.e1, b.c1, d1.nx, d1.ny, d1.nz, 64, 32);
        MF3D_LAUNCH_CK();
        layer(s, 9, d1, b.c1, b.d1);
        upcat_kernel<<<ew_grid(d0.v() * 6), 256, 0, s>>>(b.d1, b.e0, b.c0, d0.nx, d0.ny, d0.nz, 32, 16);
        MF3D_LAUNCH_CK();
        layer(s, 10, d0, b.c0, b.d0);
        layer(s, 11, d0, b.d0, b.out, 1);
    }

    // gradient of layer l's input from the gradient g of its pre-activation output; mask: the
    // activation whose ReLU derivative multiplies the result (null: none)
    void dgrad(cudaStream_t s, int l, const Dims& d, const __nv_bfloat16* g, const __nv_bfloat16* mask,
               __nv_bfloat16* dx) {
        conv(s, d, kLayers[l].cout, kLayers[l].cin, g, WT(l), nullptr, 0, mask, 0, dx, err_.as<int>());
    }
    void wg(cudaStream_t s, int l, const Dims& d, const __nv_bfloat16* x, const __nv_bfloat16* g) {
        wgrad(s, d, kLayers[l].cin, kLayers[l].cout, x, g, GW(l), GB(l), bufs_.part, bufs_.part_floats, 1);
    }

    void backward(const Dims& d0, cudaStream_t s) {
        Bufs& b = bufs_;
        const Dims d1 = d0.half(), d2 = d1.half(), d3 = d2.half();
        __nv_bfloat16* g = b.g0;  // gradient being consumed
        __nv_bfloat16* gn = b.g1; // gradient being produced
        auto swap = [&] { std::swap(g, gn); };
        MF3D_CK(cudaMemsetAsync(b.acc0, 0, d0.v() * 16 * 4, s));
        MF3D_CK(cudaMemsetAsync(b.acc1, 0, d1.v() * 32 * 4, s));
        MF3D_CK(cudaMemsetAsync(b.acc2, 0, d2.v() * 64 * 4, s));
        // layer 11 (linear output)
        wg(s, 11, d0, b.d0, b.dout);
        dgrad(s, 11, d0, b.dout, b.d0, gn); // d pre-activation of layer 10
        swap();
        // layer 10 on c0 = up(d1) ++ e0
        wg(s, 10, d0, b.c0, g);
        dgrad(s, 10, d0, g, nullptr, gn); // d c0 (48 channels)
        swap();
        upcat_bwd_skip_kernel<<<ew_grid(d0.v() * 16), 256, 0, s>>>(g, b.acc0, d0.v(), 32, 16);
        MF3D_LAUNCH_CK();
        upcat_bwd_coarse_kernel<<<ew_grid(d1.v() * 32), 256, 0, s>>>(g, b.accc, d0.nx, d0.ny, d0.nz, 32, 16);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d1.v() * 32), 256, 0, s>>>(b.accc, b.d1, gn, d1.v() * 32);
        MF3D_LAUNCH_CK();
        swap(); // d pre-activation of layer 9
        // layer 9 on c1 = up(d2) ++ e1
        wg(s, 9, d1, b.c1, g);
        dgrad(s, 9, d1, g, nullptr, gn); // d c1 (96)
        swap();
        upcat_bwd_skip_kernel<<<ew_grid(d1.v() * 32), 256, 0, s>>>(g, b.acc1, d1.v(), 64, 32);
        MF3D_LAUNCH_CK();
        upcat_bwd_coarse_kernel<<<ew_grid(d2.v() * 64), 256, 0, s>>>(g, b.accc, d1.nx, d1.ny, d1.nz, 64, 32);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d2.v() * 64), 256, 0, s>>>(b.accc, b.d2, gn, d2.v() * 64);
        MF3D_LAUNCH_CK();
        swap(); // layer 8 pre-activation
        // layer 8 on c2 = up(e3) ++ e2
        wg(s, 8, d2, b.c2, g);
        dgrad(s, 8, d2, g, nullptr, gn); // d c2 (128)
        swap();
        upcat_bwd_skip_kernel<<<ew_grid(d2.v() * 64), 256, 0, s>>>(g, b.acc2, d2.v(), 64, 64);
        MF3D_LAUNCH_CK();
        upcat_bwd_coarse_kernel<<<ew_grid(d3.v() * 64), 256, 0, s>>>(g, b.accc, d2.nx, d2.ny, d2.nz, 64, 64);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d3.v() * 64), 256, 0, s>>>(b.accc, b.e3, gn, d3.v() * 64);
        MF3D_LAUNCH_CK();
        swap(); // layer 7 pre-activation
        // encoder L3
        wg(s, 7, d3, b.a6, g);
        dgrad(s, 7, d3, g, b.a6, gn);
        swap();
        wg(s, 6, d3, b.p2, g);
        dgrad(s, 6, d3, g, nullptr, gn); // d p2
        swap();
        pool_bwd_kernel<<<ew_grid(d2.v() * 64), 256, 0, s>>>(g, b.acc2, d2.nx, d2.ny, d2.nz, 64);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d2.v() * 64), 256, 0, s>>>(b.acc2, b.e2, gn, d2.v() * 64);
        MF3D_LAUNCH_CK();
        swap(); // layer 5 pre-activation
        // encoder L2
        wg(s, 5, d2, b.a4, g);
        dgrad(s, 5, d2, g, b.a4, gn);
        swap();
        wg(s, 4, d2, b.p1, g);
        dgrad(s, 4, d2, g, nullptr, gn); // d p1
        swap();
        pool_bwd_kernel<<<ew_grid(d1.v() * 32), 256, 0, s>>>(g, b.acc1, d1.nx, d1.ny, d1.nz, 32);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d1.v() * 32), 256, 0, s>>>(b.acc1, b.e1, gn, d1.v() * 32);
        MF3D_LAUNCH_CK();
        swap(); // layer 3 pre-activation
        // encoder L1
        wg(s, 3, d1, b.a2, g);
        dgrad(s, 3, d1, g, b.a2, gn);
        swap();
        wg(s, 2, d1, b.p0, g);
        dgrad(s, 2, d1, g, nullptr, gn); // d p0
        swap();
        pool_bwd_kernel<<<ew_grid(d0.v() * 16), 256, 0, s>>>(g, b.acc0, d0.nx, d0.ny, d0.nz, 16);
        MF3D_LAUNCH_CK();
        mask_to_bf16_kernel<<<ew_grid(d0.v() * 16), 256, 0, s>>>(b.acc0, b.e0, gn, d0.v() * 16);
        MF3D_LAUNCH_CK();
        swap(); // layer 1 pre-activation
        // encoder L0
        wg(s, 1, d0, b.a0, g);
        dgrad(s, 1, d0, g, b.a0, gn);
        swap();
        wg(s, 0, d0, b.in, g);
    }

    // BF16 copies of the weights and their flipped-transposed forms (data gradients)
    void refresh_bf16(cudaStream_t s) {
        convert_kernel<__nv_bfloat16, float>
            <<<ew_grid(nparam_), 256, 0, s>>>(nparam_, w32_.as<float>(), wbf_.as<__nv_bfloat16>());
        // (float -> bf16 conversion rounds to nearest even)
        MF3D_LAUNCH_CK();
        for (int l = 0; l < kNumLayers; ++l) flip(s, kLayers[l].cin, kLayers[l].cout, W(l), WT(l));
    }

    void check_err(cudaStream_t s) {
        int e = 0;
        MF3D_CK(cudaMemcpyAsync(&e, err_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        MF3D_CK(cudaStreamSynchronize(s));
        if (e) {
            MF3D_CK(cudaMemset(err_.p, 0, sizeof(int)));
            throw Error(MF3D_E_CUDA, "a tensor-core pipeline wait timed out in the warm-start network");
        }
    }

    size_t nparam_ = 0;
    size_t woff_[kNumLayers], boff_[kNumLayers];
    DevMem w32_, g32_, m_, v_, wbf_, wflip_, err_;
    long long step_ = 0;
};

} // namespace nn
} // namespace mf3d

// =========================================================================================
// C-ABI of the warm start
// =========================================================================================
struct mf3d_warmstart {
    std::unique_ptr<nn::WarmStartNet> net;
};

namespace {
nn::Dims ws_dims(const mf3d_grid* g) {
    check_grid(g);
    return nn::Dims{g->nx, g->ny, g->nz};
}
// the x-face head values of the x-linear guess (zero on a face that is not Dirichlet)
void ws_faces(const mf3d_bc* bc, double& hw, double& he) {
    need(bc, "bc");
    hw = bc->type[0] == MF3D_BC_DIRICHLET ? bc->value[0] : 0.0;
    he = bc->type[1] == MF3D_BC_DIRICHLET ? bc->value[1] : 0.0;
}
int* ws_err_flag() {
    static std::mutex mu;
    static int* flag = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!flag) {
        MF3D_CK(cudaMalloc(&flag, sizeof(int)));
        MF3D_CK(cudaMemset(flag, 0, sizeof(int)));
    }
    return flag;
}
} // namespace

extern "C" {

int mf3d_ws_create(unsigned long long seed, mf3d_warmstart** out) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        std::unique_ptr<mf3d_warmstart> w(new mf3d_warmstart());
        w->net.reset(new nn::WarmStartNet(seed));
        *out = w.release();
    });
}

int mf3d_ws_destroy(mf3d_warmstart* w) {
    return guard([&] { delete w; });
}

long long mf3d_ws_num_params(const mf3d_warmstart* w) { return w ? (long long)w->net->num_params() : -1; }

int mf3d_ws_get_params(const mf3d_warmstart* w, float* host) {
    return guard([&] {
        need(w, "warmstart");
        need(host, "host");
        w->net->get_params(host);
    });
}

int mf3d_ws_set_params(mf3d_warmstart* w, const float* host) {
    return guard([&] {
        need(w, "warmstart");
        need(host, "host");
        w->net->set_params(host);
    });
}

int mf3d_ws_get_grads(const mf3d_warmstart* w, float* host) {
    return guard([&] {
        need(w, "warmstart");
        need(host, "host");
        w->net->get_grads(host);
    });
}

int mf3d_ws_train_step(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, int count, const float* const* lnK,
                       const float* const* h, float lr, double* loss, void* stream) {
    return guard([&] {
        need(w, "warmstart");
        need(lnK, "lnK");
        need(h, "h");
        if (count < 1) throw Error(MF3D_E_INVALID, "count must be positive");
        double hw, he;
        ws_faces(bc, hw, he);
        const double l = w->net->train_step(ws_dims(g), count, lnK, h, hw, he, lr, (cudaStream_t)stream);
        if (loss) *loss = l;
    });
}

int mf3d_ws_eval(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, int count, const float* const* lnK,
                 const float* const* h, double* loss, void* stream) {
    return guard([&] {
        need(w, "warmstart");
        need(lnK, "lnK");
        need(h, "h");
        need(loss, "loss");
        if (count < 1) throw Error(MF3D_E_INVALID, "count must be positive");
        double hw, he;
        ws_faces(bc, hw, he);
        *loss = w->net->eval(ws_dims(g), count, lnK, h, hw, he, (cudaStream_t)stream);
    });
}

int mf3d_ws_predict(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, const double* K, double* x0,
                    void* stream) {
    return guard([&] {
        need(w, "warmstart");
        need(K, "K");
        need(x0, "x0");
        double hw, he;
        ws_faces(bc, hw, he);
        w->net->predict(ws_dims(g), hw, he, K, x0, (cudaStream_t)stream);
    });
}

int mf3d_nn_conv3d(const mf3d_grid* g, int cin, int cout, const void* x, const void* w, const float* bias, int relu,
                   const void* mask, int y_f32, void* y, void* stream) {
    return guard([&] {
        need(x, "x");
        need(w, "w");
        need(y, "y");
        const nn::Dims d{g ? g->nx : 0, g ? g->ny : 0, g ? g->nz : 0};
        check_grid(g);
        int* err = ws_err_flag();
        nn::WarmStartNet::conv((cudaStream_t)stream, d, cin, cout, (const __nv_bfloat16*)x, (const __nv_bfloat16*)w,
                               bias, relu, (const __nv_bfloat16*)mask, y_f32, y, err);
        int e = 0;
        MF3D_CK(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
        MF3D_CK(cudaStreamSynchronize((cudaStream_t)stream));
        if (e) {
            MF3D_CK(cudaMemset(err, 0, sizeof(int)));
            throw Error(MF3D_E_CUDA, "a tensor-core pipeline wait timed out");
        }
    });
}

int mf3d_nn_flip_weights(int cin, int cout, const void* w, void* wt, void* stream) {
    return guard([&] {
        need(w, "w");
        need(wt, "wt");
        if (cin < 1 || cout < 1) throw Error(MF3D_E_INVALID, "channel counts must be positive");
        nn::WarmStartNet::flip((cudaStream_t)stream, cin, cout, (const __nv_bfloat16*)w, (__nv_bfloat16*)wt);
        MF3D_CK(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

int mf3d_nn_conv3d_wgrad(const mf3d_grid* g, int cin, int cout, const void* x, const void* dy, float* dw, float* db,
                         void* stream) {
    return guard([&] {
        need(x, "x");
        need(dy, "dy");
        need(dw, "dw");
        need(db, "db");
        check_grid(g);
        if (cin % 16 || cout % 16 || cin > nn::CONV_MAXC || cout > nn::CONV_MAXC)
            throw Error(MF3D_E_INVALID, "convolution channels must be multiples of 16 in [16, 128]");
        const size_t part = (size_t)64 * 27 * cin * cout + (size_t)64 * cout;
        DevMem scratch(part * sizeof(float));
        nn::WarmStartNet::wgrad((cudaStream_t)stream, nn::Dims{g->nx, g->ny, g->nz}, cin, cout,
                                (const __nv_bfloat16*)x, (const __nv_bfloat16*)dy, dw, db, scratch.as<float>(), part, 0);
        MF3D_CK(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

} // extern "C"

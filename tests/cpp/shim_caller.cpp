// A C++ caller of include/mf3d.hpp shaped like the reference's own callers of solve_head
// (src/runtime/ensemble/EnsembleRunner.cu:259-317): FlowYamlConfig -> HeadSolveConfig::from_yaml,
// one FlowWorkspace reused across calls, solve_head + compute_velocity_from_head.
//
//   shim_caller config      prints the HeadSolveConfig fields from_yaml produced (no GPU)
//   shim_caller nogpu       expects solve_head to throw std::runtime_error (no GPU present)
//   shim_caller solve       on a GPU: homogeneous K on 32 x 16 x 8 cells, three calls on one
//                           workspace (h_west 1, then 2, then 2 again); prints the west-cell
//                           head of each call and the workspace's solver builds
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mf3d.hpp"

static mf3d::FlowYamlConfig yaml_flow() {
    mf3d::FlowYamlConfig f;
    f.solver = "mg_cg";
    f.mg_levels = 3;
    f.mg_pre_smooth = 1;
    f.mg_post_smooth = 3;
    f.mg_coarse_iters = 40;
    f.mg_max_cycles = 7;
    f.cg_max_iter = 200;
    f.cg_rtol = 1e-11;
    f.cg_check_every = 1;
    f.rtol = 1e-7;
    f.pin = mf3d::PinMode::Off;
    return f;
}

int main(int argc, char** argv) {
    const char* mode = argc > 1 ? argv[1] : "config";
    if (!std::strcmp(mode, "config")) {
        mf3d::HeadSolveConfig c = mf3d::HeadSolveConfig::from_yaml(yaml_flow());
        std::printf("%d %d %d %d %d %d %d %d %.3g %.3g %d\n", c.cfg.solver, c.cfg.mg_levels, c.cfg.mg_pre_smooth,
                    c.cfg.mg_post_smooth, c.cfg.mg_coarse_iters, c.cfg.mg_max_cycles, c.cfg.cg_max_iter,
                    c.cfg.cg_check_every, c.cfg.cg_rtol, c.cfg.rtol, c.cfg.pin_mode);
        mf3d::FlowYamlConfig f;
        f.solver = "cg";
        std::printf("%d", mf3d::HeadSolveConfig::from_yaml(f).cfg.solver);
        f.solver = "mg";
        std::printf(" %d", mf3d::HeadSolveConfig::from_yaml(f).cfg.solver);
        f.solver = "something-else";
        std::printf(" %d\n", mf3d::HeadSolveConfig::from_yaml(f).cfg.solver);
        return 0;
    }
    mf3d::Grid3D g{32, 16, 8, 1.0};
    mf3d::HeadSolveConfig cfg = mf3d::HeadSolveConfig::from_yaml(yaml_flow());
    mf3d::FlowWorkspace ws;
    if (!std::strcmp(mode, "nogpu")) {
        try {
            mf3d::solve_head(nullptr, nullptr, g, mf3d::BCSpec::darcy_x(), cfg, nullptr, ws);
        } catch (const std::runtime_error& e) {
            std::printf("threw: %s\n", e.what());
            return 0;
        }
        std::printf("no exception\n");
        return 1;
    }
    const size_t n = g.num_cells();
    double *K = nullptr, *h = nullptr;
    if (cudaMalloc(&K, n * sizeof(double)) != cudaSuccess || cudaMalloc(&h, n * sizeof(double)) != cudaSuccess) return 2;
    std::vector<double> ones(n, 1.0), hh(n);
    cudaMemcpy(K, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    const double west[3] = {1.0, 2.0, 2.0};
    for (int call = 0; call < 3; ++call) {
        mf3d::HeadSolveResult r = mf3d::solve_head(h, K, g, mf3d::BCSpec::darcy_x(west[call], 0.0), cfg, s, ws);
        cudaMemcpy(hh.data(), h, n * sizeof(double), cudaMemcpyDeviceToHost);
        // exact head for homogeneous K: h_w + (h_e - h_w) (i + 0.5) / nx
        double err = 0.0;
        for (size_t c = 0; c < n; ++c) {
            const int i = (int)(c % g.nx);
            err = std::fmax(err, std::fabs(hh[c] - west[call] * (1.0 - (i + 0.5) / g.nx)));
        }
        std::printf("call %d converged %d iterations %d west %.12f maxerr %.3e builds %d\n", call, (int)r.converged,
                    r.num_iterations, hh[0], err, ws.builds());
    }
    ws.reset();
    cudaStreamDestroy(s);
    cudaFree(K);
    cudaFree(h);
    return 0;
}

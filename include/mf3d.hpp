// mf3d.hpp -- header-only C++ layer over the C-ABI of libmf3d.so, with the shapes of the
// reference's C++ head-solver interface (santi-esquerre/MacroFlow3D):
//
//   mf3d::HeadSolveConfig / HeadSolveResult    src/physics/flow/solve_head.cuh:63-141
//   mf3d::FlowYamlConfig, HeadSolveConfig::from_yaml   src/io/config/Config.hpp:86-114,
//                                                      solve_head.cuh:98-130
//   mf3d::FlowWorkspace                         src/physics/common/workspaces.cuh:111-167
//   mf3d::solve_head(h, K, grid, bc, cfg, ctx, ws)                solve_head.cuh:158-160
//   mf3d::compute_velocity_from_head(U, V, W, layout, h, K, ...)  velocity_from_head.cuh:54-73
//   mf3d::VarCoeffLaplacian::apply / MultigridPreconditioner::apply
//
// Errors throw std::runtime_error, as the reference's MACROFLOW3D_CUDA_CHECK does
// (src/runtime/cuda_check.cuh:12-31); non-convergence is reported in the result.
#pragma once
#include <stdexcept>
#include <string>

#include "mf3d.h"

namespace mf3d {

inline void check(int rc) {
    if (rc != MF3D_OK) throw std::runtime_error(std::string("mf3d: ") + mf3d_last_error());
}

struct Grid3D {
    int nx = 0, ny = 0, nz = 0;
    double dx = 1.0;
    mf3d_grid c() const { return mf3d_grid{nx, ny, nz, dx}; }
    size_t num_cells() const { return (size_t)nx * ny * nz; }
};

struct BCSpec {
    mf3d_bc bc{};
    static BCSpec darcy_x(double h_west = 1.0, double h_east = 0.0) {
        BCSpec s;
        for (int f = 0; f < 6; ++f) s.bc.type[f] = MF3D_BC_NEUMANN;
        s.bc.type[0] = s.bc.type[1] = MF3D_BC_DIRICHLET;
        s.bc.value[0] = h_west;
        s.bc.value[1] = h_east;
        return s;
    }
};

// PinMode (src/numerics/pin_spec.hpp:56-60).
enum class PinMode { Auto = MF3D_PIN_AUTO, On = MF3D_PIN_ON, Off = MF3D_PIN_OFF };

// The `flow:` section of the reference's YAML configuration after parsing
// (src/io/config/Config.hpp:86-114): a caller that parses its YAML with the reference's
// ConfigYaml keeps doing so and copies the fields here, or fills them directly.
struct FlowYamlConfig {
    std::string solver = "mg"; // "mg", "cg", "mg_cg" / "pcg_mg"
    int mg_levels = 4;
    int mg_pre_smooth = 2;
    int mg_post_smooth = 2;
    int mg_coarse_iters = 50;
    int mg_max_cycles = 20;
    int cg_max_iter = 1000;
    double cg_rtol = 1e-8;
    int cg_check_every = 10;
    double rtol = 1e-6;
    BCSpec bc = BCSpec::darcy_x();
    PinMode pin = PinMode::Auto;
};

struct HeadSolveConfig {
    mf3d_solver_config cfg{};
    HeadSolveConfig() { check(mf3d_default_config(&cfg)); }

    // HeadSolveConfig::from_yaml (src/physics/flow/solve_head.cuh:98-130): the solver string
    // maps to the solver type, unknown strings to PCG_MG; every numeric field is copied.
    static HeadSolveConfig from_yaml(const FlowYamlConfig& f) {
        HeadSolveConfig c;
        if (f.solver == "cg") c.cfg.solver = MF3D_SOLVER_CG;
        else if (f.solver == "mg") c.cfg.solver = MF3D_SOLVER_MG;
        else c.cfg.solver = MF3D_SOLVER_PCG_MG;
        c.cfg.mg_levels = f.mg_levels;
        c.cfg.mg_pre_smooth = f.mg_pre_smooth;
        c.cfg.mg_post_smooth = f.mg_post_smooth;
        c.cfg.mg_max_cycles = f.mg_max_cycles;
        c.cfg.mg_coarse_iters = f.mg_coarse_iters;
        c.cfg.cg_max_iter = f.cg_max_iter;
        c.cfg.cg_rtol = f.cg_rtol;
        c.cfg.cg_check_every = f.cg_check_every;
        c.cfg.rtol = f.rtol;
        c.cfg.pin_mode = (int)f.pin;
        return c;
    }
};

struct HeadSolveResult {
    int num_iterations = 0;
    double initial_residual = 0.0;
    double final_residual = 0.0;
    bool converged = false;
    mf3d_solve_result raw{};
};

// Owns the solver of one problem.  The reference rebuilds its hierarchy when the grid changes
// (solve_head.cu:89-94) and takes the BCs and the configuration on every call
// (solve_head.cuh:158-160); the solver here bakes the grid, BCs, configuration and stream into
// its operator and CUDA graph, so it is re-created when any of them differs from the last call.
class FlowWorkspace {
  public:
    FlowWorkspace() = default;
    ~FlowWorkspace() { reset(); }
    FlowWorkspace(const FlowWorkspace&) = delete;
    FlowWorkspace& operator=(const FlowWorkspace&) = delete;
    void reset() {
        if (s_) mf3d_head_solver_destroy(s_);
        s_ = nullptr;
    }
    mf3d_head_solver* ensure(const Grid3D& g, const BCSpec& bc, const HeadSolveConfig& c, void* stream) {
        const bool same = s_ && g.nx == g_.nx && g.ny == g_.ny && g.nz == g_.nz && g.dx == g_.dx &&
                          same_bc(bc.bc, bc_.bc) && same_cfg(c.cfg, cfg_.cfg) && stream == stream_;
        if (!same) {
            reset();
            mf3d_grid gc = g.c();
            check(mf3d_head_solver_create(&gc, &bc.bc, &c.cfg, stream, &s_));
            g_ = g;
            bc_ = bc;
            cfg_ = c;
            stream_ = stream;
            ++builds_;
        }
        return s_;
    }
    mf3d_head_solver* get() const { return s_; }
    // how many times a solver was created (diagnostics)
    int builds() const { return builds_; }

  private:
    static bool same_bc(const mf3d_bc& a, const mf3d_bc& b) {
        for (int f = 0; f < 6; ++f)
            if (a.type[f] != b.type[f] || a.value[f] != b.value[f]) return false;
        return true;
    }
    static bool same_cfg(const mf3d_solver_config& a, const mf3d_solver_config& b) {
        return a.solver == b.solver && a.mg_levels == b.mg_levels && a.mg_pre_smooth == b.mg_pre_smooth &&
               a.mg_post_smooth == b.mg_post_smooth && a.mg_max_cycles == b.mg_max_cycles &&
               a.mg_coarse_iters == b.mg_coarse_iters && a.cg_max_iter == b.cg_max_iter &&
               a.cg_check_every == b.cg_check_every && a.cg_rtol == b.cg_rtol && a.rtol == b.rtol &&
               a.pin_mode == b.pin_mode && a.precision == b.precision && a.flexible == b.flexible &&
               a.conv_norm == b.conv_norm && a.use_graph == b.use_graph;
    }
    mf3d_head_solver* s_ = nullptr;
    Grid3D g_;
    BCSpec bc_;
    HeadSolveConfig cfg_;
    void* stream_ = nullptr;
    int builds_ = 0;
};

// solve_head: h (device, out), K (device), the reference's arguments; `stream` is the
// caller's cudaStream_t (the reference's CudaContext::cuda_stream()).
inline HeadSolveResult solve_head(double* h, const double* K, const Grid3D& g, const BCSpec& bc,
                                  const HeadSolveConfig& cfg, void* stream, FlowWorkspace& ws,
                                  const double* x0 = nullptr) {
    mf3d_head_solver* s = ws.ensure(g, bc, cfg, stream);
    check(mf3d_head_solver_set_K(s, K));
    HeadSolveResult r;
    check(mf3d_head_solve(s, h, x0, &r.raw));
    r.num_iterations = r.raw.num_iterations;
    r.initial_residual = r.raw.initial_residual;
    r.final_residual = r.raw.final_residual;
    r.converged = r.raw.converged != 0;
    return r;
}

inline void compute_velocity_from_head(double* U, double* V, double* W, int layout, const double* h,
                                       const double* K, const Grid3D& g, const BCSpec& bc, void* stream) {
    mf3d_grid gc = g.c();
    check(mf3d_velocity_from_head(&gc, &bc.bc, h, K, layout, U, V, W, stream));
}

// VarCoeffLaplacian (src/numerics/operators/varcoeff_laplacian.cuh:55): y = A x.
class VarCoeffLaplacian {
  public:
    VarCoeffLaplacian(const Grid3D& g, const double* K, const BCSpec& bc, bool pin)
        : g_(g), K_(K), bc_(bc), pin_(pin) {}
    void apply(void* stream, const double* x, double* y) const {
        mf3d_grid gc = g_.c();
        check(mf3d_apply_A(&gc, &bc_.bc, pin_ ? 1 : 0, K_, x, y, stream));
    }

  private:
    Grid3D g_;
    const double* K_;
    BCSpec bc_;
    bool pin_;
};

// MultigridPreconditioner (src/numerics/solvers/mg_preconditioner.cuh): z = V-cycle(r), with
// the hierarchy of a workspace whose K was set by solve_head or set_K.
class MultigridPreconditioner {
  public:
    explicit MultigridPreconditioner(FlowWorkspace& ws) : ws_(&ws) {}
    void apply(const double* r, double* z) const { check(mf3d_head_solver_vcycle(ws_->get(), r, z)); }

  private:
    FlowWorkspace* ws_;
};

} // namespace mf3d

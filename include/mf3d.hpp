// mf3d.hpp -- header-only C++ layer over the C-ABI of libmf3d.so, with the shapes of the
// reference's C++ head-solver interface (santi-esquerre/MacroFlow3D):
//
//   mf3d::HeadSolveConfig / HeadSolveResult    src/physics/flow/solve_head.cuh:63-141
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

struct HeadSolveConfig {
    mf3d_solver_config cfg{};
    HeadSolveConfig() { check(mf3d_default_config(&cfg)); }
};

struct HeadSolveResult {
    int num_iterations = 0;
    double initial_residual = 0.0;
    double final_residual = 0.0;
    bool converged = false;
    mf3d_solve_result raw{};
};

// Owns the solver of one grid; rebuilt when the grid changes (solve_head.cu:89-94).
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
        if (!s_ || g.nx != g_.nx || g.ny != g_.ny || g.nz != g_.nz || g.dx != g_.dx) {
            reset();
            mf3d_grid gc = g.c();
            check(mf3d_head_solver_create(&gc, &bc.bc, &c.cfg, stream, &s_));
            g_ = g;
        }
        return s_;
    }
    mf3d_head_solver* get() const { return s_; }

  private:
    mf3d_head_solver* s_ = nullptr;
    Grid3D g_;
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

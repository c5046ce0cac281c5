/*
 * mf3d.h -- C-ABI of the B200-native Darcy head solve + face velocity (libmf3d.so).
 *
 * Drop-in boundary for MacroFlow3D's head-solver path.  Each entry point names the
 * reference routine it replaces (paths within santi-esquerre/MacroFlow3D).  Conventions:
 *   - plain C types only; device pointers are `double*` (or `void*` where the precision
 *     varies), streams are `void*` holding a cudaStream_t (NULL = the solver's own stream
 *     for solver calls, the legacy default stream otherwise);
 *   - every call returns an int status: 0 ok, < 0 error (see MF3D_E_*); the message of the
 *     last error on the calling thread is returned by mf3d_last_error();
 *   - arrays are cell-centred, x fastest: cell (i,j,k) at i + nx*(j + ny*k)
 *     (src/core/Grid3D.hpp:54);
 *   - no exceptions cross the ABI; non-convergence is reported in the result struct, as in
 *     the reference (src/physics/flow/solve_head.cuh:136-141), not as an error.
 */
#ifndef MF3D_H
#define MF3D_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define MF3D_OK 0
#define MF3D_E_INVALID (-1)   /* bad argument / unsupported configuration */
#define MF3D_E_CUDA (-2)      /* CUDA runtime error */
#define MF3D_E_NOMEM (-3)     /* device allocation failed */
#define MF3D_E_STATE (-4)     /* call out of order (e.g. solve before set_K) */

/* ---- BCType, src/core/BCSpec.hpp:13 ------------------------------------------------------ */
#define MF3D_BC_DIRICHLET 0
#define MF3D_BC_NEUMANN 1
#define MF3D_BC_PERIODIC 2

/* ---- HeadSolverType, src/physics/flow/solve_head.cuh:52-56 -------------------------------- */
#define MF3D_SOLVER_PCG_MG 0
#define MF3D_SOLVER_MG 1
#define MF3D_SOLVER_CG 2

/* ---- PinMode, src/numerics/pin_spec.hpp:56-60 --------------------------------------------- */
#define MF3D_PIN_AUTO 0
#define MF3D_PIN_ON 1
#define MF3D_PIN_OFF 2

/* ---- V-cycle precision (extension: the reference is FP64 only) ---------------------------- */
#define MF3D_PREC_FP64 0 /* FP64 V-cycle, FP64 face coefficients */
#define MF3D_PREC_FP32 1 /* FP32 V-cycle, FP32 face coefficients, FP64 coarse tail */
#define MF3D_PREC_BF16 2 /* FP32 V-cycle, BF16 face coefficients with per-level 2^s scale */

/* ---- stopping-test denominator ------------------------------------------------------------ */
#define MF3D_CONV_R0 0 /* ||r|| / ||r0|| < cg_rtol, as src/numerics/solvers/pcg.cuh:156-164 */
#define MF3D_CONV_B 1  /* ||r|| / ||b||  < cg_rtol */

/* ---- velocity layouts, src/physics/common/fields.cuh:230 ---------------------------------- */
#define MF3D_VEL_COMPACT 0 /* U (nx+1)*ny*nz, V nx*(ny+1)*nz, W nx*ny*(nz+1) */
#define MF3D_VEL_PADDED 1  /* (nx+1)*(ny+1)*(nz+1) per component, padded_layout.cuh:30 */

/* Grid3D (src/core/Grid3D.hpp:32-55); isotropic spacing, as every reference kernel assumes. */
typedef struct mf3d_grid {
    int nx, ny, nz;
    double dx;
} mf3d_grid;

/* BCSpec / BCSpecDevice (src/core/BCSpec.hpp:36-88, BCSpecDevice.cuh:12-51):
 * faces in the order xmin, xmax, ymin, ymax, zmin, zmax. */
typedef struct mf3d_bc {
    int type[6];
    double value[6];
} mf3d_bc;

/* HeadSolveConfig (src/physics/flow/solve_head.cuh:63-96) plus this library's extensions. */
typedef struct mf3d_solver_config {
    int solver;          /* MF3D_SOLVER_* (default PCG_MG) */
    int mg_levels;       /* maximum number of levels (default 4) */
    int mg_pre_smooth;   /* GSRB sweeps before restriction (default 2) */
    int mg_post_smooth;  /* GSRB sweeps after prolongation (default 2) */
    int mg_max_cycles;   /* standalone MG: maximum V-cycles (default 20) */
    int mg_coarse_iters; /* GSRB sweeps on the coarsest level (default 50) */
    int cg_max_iter;     /* default 1000 */
    int cg_check_every;  /* default 10 */
    double cg_rtol;      /* default 1e-8 */
    double rtol;         /* standalone MG tolerance (default 1e-6) */
    int pin_mode;        /* MF3D_PIN_* (default AUTO) */
    /* extensions */
    int precision;       /* MF3D_PREC_* (default FP64) */
    int flexible;        /* -1 auto (Polak-Ribiere beta when precision != FP64), 0 FR, 1 PR */
    int conv_norm;       /* MF3D_CONV_* (default R0, the reference's test) */
    int use_graph;       /* 1 (default): whole PCG loop in one CUDA graph (device while loop) */
} mf3d_solver_config;

/* HeadSolveResult (src/physics/flow/solve_head.cuh:136-141) plus diagnostics. */
typedef struct mf3d_solve_result {
    int num_iterations;
    int converged;
    int status;              /* 0 ok, 1 breakdown (pAp = 0), 2 non-finite, 3 device-time budget exceeded */
    int num_levels;
    double initial_residual; /* ||r0|| */
    double final_residual;   /* ||r|| at the last check (recurrence residual) */
    double true_rel_residual;/* ||b - A h|| / ||b|| recomputed after the loop */
    double b_norm;           /* ||b|| */
    float device_ms;         /* device time of set-up-free solve (CUDA events) */
    int kernel_launches;     /* kernels this library launched for the solve */
} mf3d_solve_result;

/* Per-kernel timing record (diagnostics; no counterpart in the reference). */
typedef struct mf3d_kernel_timing {
    char name[40];
    float ms;              /* mean device time per launch (CUDA events, launch stream) */
    double bytes;          /* algorithmic bytes per launch (each input read once, output written once) */
    int launches_per_iter; /* launches of this kernel per PCG iteration */
} mf3d_kernel_timing;

typedef struct mf3d_head_solver mf3d_head_solver;

/* Library / error handling ------------------------------------------------------------------ */
const char* mf3d_last_error(void);
const char* mf3d_version(void);

/* HeadSolveConfig defaults (solve_head.cuh:63-96; pin auto). */
int mf3d_default_config(mf3d_solver_config* cfg);

/* Head solver: owns the multigrid hierarchy, face coefficients, PCG workspace and CUDA
 * graph.  Replaces FlowWorkspace + the set-up part of solve_head
 * (src/physics/common/workspaces.cuh:111-167, src/physics/flow/solve_head.cu:89-125). */
int mf3d_head_solver_create(const mf3d_grid* grid, const mf3d_bc* bc, const mf3d_solver_config* cfg,
                            void* stream, mf3d_head_solver** out);
int mf3d_head_solver_destroy(mf3d_head_solver* s);
int mf3d_head_solver_num_levels(const mf3d_head_solver* s);
/* The coarse end of a single solve's V-cycle: its first level (*first_level) and the CTAs of
 * the thread-block cluster that runs it (*cluster_ctas; 0 when one CTA runs the levels of at
 * most 4096 cells).  The reference recurses level by level (src/multigrid/cycle/v_cycle.cu:36-74);
 * this reports how the levels below the streamed ones are grouped into one launch. */
int mf3d_head_solver_coarse_info(const mf3d_head_solver* s, int* first_level, int* cluster_ctas);
/* Bytes of device memory the solver holds. */
long long mf3d_head_solver_device_bytes(const mf3d_head_solver* s);

/* Conductivity set-up: copies K (device, FP64, n cells), coarsens it to every level
 * (coarsen_K, src/physics/flow/coarsen_K.cu:55-77), builds every level's face coefficients,
 * the right-hand side (build_rhs_head, rhs_head.cu:121-194) and the initial guess
 * (init_head_guess, solve_head.cu:56-73). */
int mf3d_head_solver_set_K(mf3d_head_solver* s, const double* K_dev);

/* solve_head(h, K, grid, bc, cfg, ctx, ws) (src/physics/flow/solve_head.cuh:158-160).
 * h_dev: output head (device, n).  x0_dev: initial guess (device) or NULL for the
 * reference's x-linear guess.  Blocks until the result is known. */
int mf3d_head_solve(mf3d_head_solver* s, double* h_dev, const double* x0_dev, mf3d_solve_result* res);

/* MultigridPreconditioner::apply (src/numerics/solvers/mg_preconditioner.cu:16-44):
 * z = one V-cycle on r from a zero guess, with the solver's hierarchy (after set_K).
 * r_dev, z_dev: FP64 device arrays of n cells. */
int mf3d_head_solver_vcycle(mf3d_head_solver* s, const double* r_dev, double* z_dev);

/* Diagnostics (no counterpart in the reference): times, with CUDA events on the solver's
 * stream, `reps` launches of each kernel of one PCG iteration on the current state (call after
 * a solve; the solver state is scratch afterwards and is rebuilt by the next solve).  Fills
 * up to `cap` records and sets *count. */
int mf3d_head_solver_profile(mf3d_head_solver* s, int reps, mf3d_kernel_timing* out, int cap, int* count);
/* Device-time limit of one solve of this solver (default 120 s; no counterpart in the
 * reference, whose loop has only its iteration cap).  The loop's first kernel checks
 * %globaltimer once per iteration; past the limit the solve ends with status 3 and
 * converged = 0, and the solver stays usable. */
int mf3d_head_solver_set_time_budget(mf3d_head_solver* s, double seconds);

/* Diagnostics, no counterpart in the reference: runs the bounded mbarrier wait of the staged
 * smoother (which = 0) or of the tensor-core convolution (which = 1) for `tries` polls on a
 * barrier that nothing completes (arrive = 0) or that one arrival completes (arrive = 1), and
 * reports in *gave_up_host whether the wait gave up.  No copy is in flight, so the failure
 * path leaves the context usable. */
int mf3d_diag_bounded_wait(int which, int arrive, int tries, int* gave_up_host);

/* Kernels launched by the last mf3d_head_solver_set_K (diagnostics). */
int mf3d_head_solver_setup_launches(const mf3d_head_solver* s);

/* compute_velocity_from_head (src/physics/flow/velocity_from_head.cuh:54-73): Darcy face
 * velocities, layout MF3D_VEL_*.  Padded entries that are not faces are left untouched. */
int mf3d_velocity_from_head(const mf3d_grid* grid, const mf3d_bc* bc, const double* h_dev,
                            const double* K_dev, int layout, double* U_dev, double* V_dev, double* W_dev,
                            void* stream);

/* Velocity (compact layout) plus discrete mass balance, fused: out_host[0] = max over cells
 * of |sum_f q_f A_f|, out_host[1] = Q_in through x = 0, out_host[2] = Q_out through x = L.
 * (verify_mean_velocity_darcy, velocity_from_head.cu:964, has no caller in the reference.) */
int mf3d_velocity_mass_balance(const mf3d_grid* grid, const mf3d_bc* bc, const double* h_dev,
                               const double* K_dev, double* U_dev, double* V_dev, double* W_dev,
                               double* out_host, void* stream);

/* compute_velocity_diagnostics (src/physics/flow/velocity_diagnostics.cu:22-179): from a face
 * velocity field (layout MF3D_VEL_*; the reference takes the padded one) the cell-centred
 * divergence of every cell, and at the interior cells the magnitude of the curl of the
 * face-averaged cell velocity (centred differences) and the helicity u . curl u, zero at the
 * boundary cells and everywhere when a dimension is below 3.  div / omag / hel (device, n
 * cells each) may be NULL to skip storing that field.  stats_host (9 doubles, may be NULL):
 * min, max and mean of div, |omega| and helicity over all cells, as print_velocity_diagnostics
 * reports them (velocity_diagnostics.cu:181-203). */
int mf3d_velocity_diagnostics(const mf3d_grid* grid, int layout, const double* U_dev, const double* V_dev,
                              const double* W_dev, double* div_dev, double* omag_dev, double* hel_dev,
                              double* stats_host, void* stream);

/* No counterpart in the reference.  Same results as mf3d_velocity_mass_balance, but its
 * reduction scratch is a static device array (64 B + 16 B per block, 262,208 B in all), so it
 * allocates and frees no device memory: for callers whose device memory is fully owned by
 * another allocator, and for callers that cannot afford the implicit device-wide
 * synchronisation of cudaFree.  Limit: at most MF3D_MB_NOALLOC_MAX_BLOCKS reduction blocks,
 * i.e. ceil(nx/32) * ceil(ny/8) <= 16384; larger grids return MF3D_E_INVALID.  The device
 * address of the array is looked up on the first call on each device, so on each device that
 * first call should come before any stream capture.  Calls that overlap on one device share
 * the array and race: serialise them. */
#define MF3D_MB_NOALLOC_MAX_BLOCKS 16384
int mf3d_velocity_mass_balance_noalloc(const mf3d_grid* grid, const mf3d_bc* bc, const double* h_dev,
                                       const double* K_dev, double* U_dev, double* V_dev,
                                       double* W_dev, double* out_host, void* stream);

/* ---- batched ensemble solves -------------------------------------------------------------
 * The realisation loop of run_ensemble (src/runtime/ensemble/EnsembleRunner.cu:259-317) calls
 * solve_head once per realisation.  A batch holds `count` independent head solvers, one grid
 * each (sizes may differ), with one bc and cfg, and solves them together: batched launches over
 * every realisation, the whole PCG loop of all realisations in one CUDA graph, and a
 * per-realisation stopping test (a realisation that has converged does no more work while the
 * others iterate).  Supported: solver = PCG_MG, mg_pre_smooth >= 1, mg_post_smooth >= 1, and a
 * hierarchy with at least one level above the coarse tail (grids of 32 cells per axis or more
 * in practice). */
typedef struct mf3d_batch mf3d_batch;
/* Tuning record of one sweep position of the batched V-cycle (mf3d_batch_autotune). */
typedef struct mf3d_batch_tuning {
    int phase;        /* 0 pre-smoothing (down), 1 post-smoothing (up) */
    int level;        /* level depth */
    int sweep;        /* 2 x the sweep index (1-based); + 1: the residual + restriction after it */
    int mode;         /* fused stages of the sweep (first-sweep zero guess 1, prolongation 2, residual+restriction 4, <r,z> 8) */
    int path;         /* 0 staged quad sweep where the level is 16-byte aligned, 1 L1 sweep for all
                         (2, the batched x-pair sweep, is currently not chosen) */
    int chunks;       /* z chunks per tile: the z depth of a work item is nz / chunks */
    double ms_default;/* device time of the default choice */
    double ms_best;   /* device time of the choice kept */
} mf3d_batch_tuning;
/* EnsembleRunner's per-realisation solver set-up (workspaces.cuh:111-167), for all realisations. */
int mf3d_batch_create(int count, const mf3d_grid* grids, const mf3d_bc* bc, const mf3d_solver_config* cfg,
                      void* stream, mf3d_batch** out);
int mf3d_batch_destroy(mf3d_batch* b);
int mf3d_batch_count(const mf3d_batch* b);
long long mf3d_batch_device_bytes(const mf3d_batch* b);
/* mf3d_head_solver_set_K for every realisation: K_dev[r] is realisation r's K (device). */
int mf3d_batch_set_K(mf3d_batch* b, const double* const* K_dev);
/* solve_head for every realisation (EnsembleRunner.cu:286-289): h_dev[r] receives realisation
 * r's head; x0_dev may be NULL (the reference's guess for all) or hold NULL entries.
 * results[r] as mf3d_head_solve's; device_ms and kernel_launches are the whole batch's. */
int mf3d_batch_solve(mf3d_batch* b, double* const* h_dev, const double* const* x0_dev,
                     mf3d_solve_result* results);
/* Autotuner (no counterpart in the reference): for every sweep position of the batched
 * V-cycle, times the candidate work-item shapes (z chunks per tile 1, 2, 4, 8; staged or L1
 * sweep) on this batch, `reps` launches each, and keeps the fastest.  Fills up to `cap`
 * records and sets *count.  The solver state is scratch afterwards (the next solve rebuilds it). */
int mf3d_batch_autotune(mf3d_batch* b, int reps, mf3d_batch_tuning* out, int cap, int* count);

/* ---- learned warm start (no counterpart in the reference, whose initial guess is the
 * x-linear head, src/physics/flow/solve_head.cu:29-73) ----------------------------------------
 * A 3-D convolutional encoder-decoder (4 levels, 16/32/64/64 channels, 3x3x3 convolutions, skip
 * connections; BF16 weights and activations, FP32 accumulation on the tensor cores) maps lnK
 * and the x-linear head to a correction of that head; x0 = h_lin + correction is passed to
 * mf3d_head_solve as its initial guess, which still iterates to its tolerance.  Trained with
 * this library's forward and backward kernels and Adam on (lnK, head) pairs from the solver.
 * Grid sizes must be multiples of 8 on every axis. */
typedef struct mf3d_warmstart mf3d_warmstart;
int mf3d_ws_create(unsigned long long seed, mf3d_warmstart** out);
int mf3d_ws_destroy(mf3d_warmstart* w);
long long mf3d_ws_num_params(const mf3d_warmstart* w);
/* FP32 master parameters, per layer the weights [cout][27][cin] then the bias [cout] */
int mf3d_ws_get_params(const mf3d_warmstart* w, float* host);
int mf3d_ws_set_params(mf3d_warmstart* w, const float* host);
/* gradient of the last mf3d_ws_train_step, summed over its samples (same layout) */
int mf3d_ws_get_grads(const mf3d_warmstart* w, float* host);
/* One Adam step on `count` samples (lnK_dev[i], h_dev[i]: FP32 device arrays of grid g) with
 * the mean gradient of the mean squared error of the predicted head; lr <= 0 computes the
 * gradients only.  *loss: mean loss before the step. */
int mf3d_ws_train_step(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, int count,
                       const float* const* lnK_dev, const float* const* h_dev, float lr, double* loss,
                       void* stream);
int mf3d_ws_eval(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, int count,
                 const float* const* lnK_dev, const float* const* h_dev, double* loss, void* stream);
/* x0_dev (FP64, n) = x-linear head of bc's x faces + the network's correction, from K_dev (FP64) */
int mf3d_ws_predict(mf3d_warmstart* w, const mf3d_grid* g, const mf3d_bc* bc, const double* K_dev,
                    double* x0_dev, void* stream);
/* The network's operations, for tests: a 3x3x3 convolution on the tensor cores (x: BF16
 * [n][cin], w: BF16 [cout][27][cin], bias FP32 or NULL, relu 0/1, mask BF16 [n][cout] or NULL:
 * y *= (mask > 0), y: BF16 or (y_f32) FP32 [n][cout]; channels multiples of 16 up to 128), the
 * weight flip that turns the data gradient into a convolution, and the weight gradient
 * (dw FP32 [cout][27][cin], db FP32 [cout]). */
int mf3d_nn_conv3d(const mf3d_grid* g, int cin, int cout, const void* x_dev, const void* w_dev,
                   const float* bias_dev, int relu, const void* mask_dev, int y_f32, void* y_dev, void* stream);
int mf3d_nn_flip_weights(int cin, int cout, const void* w_dev, void* wt_dev, void* stream);
int mf3d_nn_conv3d_wgrad(const mf3d_grid* g, int cin, int cout, const void* x_dev, const void* dy_dev,
                         float* dw_dev, float* db_dev, void* stream);

/* ---- operator pieces (device pointers, FP64; in-place where the reference is) ------------- */
/* VarCoeffLaplacian::apply, src/numerics/operators/varcoeff_laplacian.cu:241-277 */
int mf3d_apply_A(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* x,
                 double* y, void* stream);
/* gsrb_smooth_3d, src/multigrid/smoothers/gsrb_3d.cu:368-576 (x updated in place) */
int mf3d_gsrb(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* b,
              double* x, int iters, void* stream);
/* compute_residual_3d, src/multigrid/smoothers/residual_3d.cu:378-502 */
int mf3d_residual(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* x,
                  const double* b, double* r, void* stream);
/* restrict_3d, src/multigrid/transfer/restrict_3d.cu:55-80 (coarse = fine / 2) */
int mf3d_restrict(const mf3d_grid* coarse, const double* r_fine, double* b_coarse, void* stream);
/* prolong_3d_add, src/multigrid/transfer/prolong_3d.cu:520-621 */
int mf3d_prolong_add(const mf3d_grid* coarse, const double* x_coarse, double* x_fine, void* stream);
/* coarsen_K, src/physics/flow/coarsen_K.cu:55-77 */
int mf3d_coarsen_K(const mf3d_grid* coarse, const double* K_fine, double* K_coarse, void* stream);
/* build_rhs_head, src/physics/flow/rhs_head.cu:121-194 */
int mf3d_build_rhs(const mf3d_grid* g, const mf3d_bc* bc, const double* K, double* b, void* stream);
/* init_head_guess, src/physics/flow/solve_head.cu:56-73 */
int mf3d_init_head_guess(const mf3d_grid* g, const mf3d_bc* bc, double* h, void* stream);

/* ---- K-field generator (randomization method; generate_K_field, src/physics/stochastic/
 * stochastic.cu:270-367, with per-axis correlation lengths added) ------------------------- */
#define MF3D_COV_EXPONENTIAL 0
#define MF3D_COV_GAUSSIAN 1
/* Host-side mode sampling (no GPU): modes_host receives 5*n_modes doubles laid out as
 * k1[n], k2[n], k3[n], a[n], b[n]; counter-based (Philox4x32-10) stream from `seed`. */
int mf3d_kfield_modes(unsigned long long seed, int n_modes, int covariance, double lambda_x,
                      double lambda_y, double lambda_z, double* modes_host);
/* K (or lnK when want_exp = 0) at the cell centres of g from device-resident modes. */
int mf3d_kfield_eval(const mf3d_grid* g, int n_modes, const double* modes_dev, double sigma2,
                     double log_kg, int want_exp, double* out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MF3D_H */

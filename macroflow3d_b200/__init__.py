"""macroflow3d_b200 -- B200-native Darcy head solve (CCMG-preconditioned CG) and face velocity.

Python mirror of the reference's head-solver interface (santi-esquerre/MacroFlow3D:
solve_head, init_head_guess, build_rhs_head, coarsen_K, compute_velocity_from_head, the
multigrid free functions and VarCoeffLaplacian::apply) over the C-ABI of libmf3d.so.
Device arrays are torch CUDA tensors (float64, contiguous, numel = nx*ny*nz in the
reference's i + nx*(j + ny*k) layout); torch provides memory and the current stream only.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

from . import _lib
from ._lib import Mf3dError, check, lib
from .config import (BCFace, BCSpec, ConfigError, FlowConfig, load_flow_yaml, parse_flow,  # noqa: F401
                     DIRICHLET, NEUMANN, PERIODIC, PIN_AUTO, PIN_OFF, PIN_ON)

SOLVER_PCG_MG, SOLVER_MG, SOLVER_CG = 0, 1, 2
PREC_FP64, PREC_FP32, PREC_BF16 = 0, 1, 2
CONV_R0, CONV_B = 0, 1
VEL_COMPACT, VEL_PADDED = 0, 1
COV_EXPONENTIAL, COV_GAUSSIAN = 0, 1
MB_NOALLOC_MAX_BLOCKS = 16384


@dataclass
class Grid3D:
    """Grid3D (src/core/Grid3D.hpp:32-55): isotropic spacing dx."""
    nx: int
    ny: int
    nz: int
    dx: float = 1.0

    def num_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def c(self) -> _lib.Grid:
        return _lib.Grid(self.nx, self.ny, self.nz, float(self.dx))


def _bc(bc: BCSpec) -> _lib.BC:
    out = _lib.BC()
    for f in range(6):
        out.type[f] = int(bc.faces[f].type)
        out.value[f] = float(bc.faces[f].value)
    return out


@dataclass
class HeadSolveConfig:
    """HeadSolveConfig (src/physics/flow/solve_head.cuh:63-96) + extensions."""
    solver_type: int = SOLVER_PCG_MG
    mg_levels: int = 4
    mg_pre_smooth: int = 2
    mg_post_smooth: int = 2
    mg_max_cycles: int = 20
    mg_coarse_iters: int = 50
    cg_max_iter: int = 1000
    cg_check_every: int = 10
    cg_rtol: float = 1e-8
    rtol: float = 1e-6
    pin_mode: int = PIN_AUTO
    precision: int = PREC_FP64
    flexible: int = -1
    conv_norm: int = CONV_R0
    use_graph: int = 1

    @staticmethod
    def from_yaml(flow: FlowConfig) -> "HeadSolveConfig":
        """HeadSolveConfig::from_yaml (solve_head.cuh:98-130)."""
        st = {"cg": SOLVER_CG, "mg": SOLVER_MG}.get(flow.solver, SOLVER_PCG_MG)
        flex = {"auto": -1, True: 1, False: 0, "true": 1, "false": 0}.get(flow.flexible, -1)
        return HeadSolveConfig(st, flow.mg_levels, flow.mg_pre_smooth, flow.mg_post_smooth,
                               flow.mg_max_cycles, flow.mg_coarse_iters, flow.cg_max_iter,
                               flow.cg_check_every, flow.cg_rtol, flow.rtol, flow.pin_mode,
                               {"fp64": 0, "fp32": 1, "bf16": 2}[str(flow.precision)], flex,
                               CONV_B if flow.conv_norm == "b" else CONV_R0, int(bool(flow.use_graph)))

    def c(self) -> _lib.SolverConfig:
        return _lib.SolverConfig(self.solver_type, self.mg_levels, self.mg_pre_smooth,
                                 self.mg_post_smooth, self.mg_max_cycles, self.mg_coarse_iters,
                                 self.cg_max_iter, self.cg_check_every, float(self.cg_rtol),
                                 float(self.rtol), self.pin_mode, self.precision, self.flexible,
                                 self.conv_norm, self.use_graph)


@dataclass
class HeadSolveResult:
    """HeadSolveResult (solve_head.cuh:136-141) + diagnostics."""
    num_iterations: int
    initial_residual: float
    final_residual: float
    converged: bool
    status: int
    num_levels: int
    true_rel_residual: float
    b_norm: float
    device_ms: float
    kernel_launches: int = 0


def _ptr(t) -> int:
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def _f64(t, n: int, name: str):
    import torch
    if t.dtype != torch.float64:
        raise TypeError(f"{name} must be float64")
    if t.numel() < n:
        raise ValueError(f"{name} buffer too small")
    return _ptr(t)


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class HeadSolver:
    """Owns the hierarchy, face coefficients, PCG workspace and CUDA graph of one grid
    (the reference's FlowWorkspace, src/physics/common/workspaces.cuh:111-167)."""

    def __init__(self, grid: Grid3D, bc: BCSpec, cfg: Optional[HeadSolveConfig] = None,
                 stream=None):
        self.grid, self.bc = grid, bc
        self.cfg = cfg or HeadSolveConfig()
        h = C.c_void_p()
        s = C.c_void_p(stream) if isinstance(stream, int) else (stream or C.c_void_p())
        check(lib().mf3d_head_solver_create(C.byref(grid.c()), C.byref(_bc(bc)),
                                            C.byref(self.cfg.c()), s, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mf3d_head_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_levels(self) -> int:
        return lib().mf3d_head_solver_num_levels(self._h)

    @property
    def coarse_info(self) -> tuple:
        """(first level of the coarse-end kernel of a single solve, CTAs of its thread-block
        cluster; 0 when one CTA runs the levels of at most 4096 cells)."""
        first, ctas = C.c_int(0), C.c_int(0)
        check(lib().mf3d_head_solver_coarse_info(self._h, C.byref(first), C.byref(ctas)))
        return first.value, ctas.value

    @property
    def device_bytes(self) -> int:
        return lib().mf3d_head_solver_device_bytes(self._h)

    def set_K(self, K) -> None:
        check(lib().mf3d_head_solver_set_K(self._h, _f64(K, self.grid.num_cells(), "K")))

    def solve(self, h, x0=None) -> HeadSolveResult:
        n = self.grid.num_cells()
        r = _lib.SolveResult()
        check(lib().mf3d_head_solve(self._h, _f64(h, n, "h"),
                                    None if x0 is None else _f64(x0, n, "x0"), C.byref(r)))
        return HeadSolveResult(r.num_iterations, r.initial_residual, r.final_residual,
                               bool(r.converged), r.status, r.num_levels, r.true_rel_residual,
                               r.b_norm, r.device_ms, r.kernel_launches)

    @property
    def setup_launches(self) -> int:
        return lib().mf3d_head_solver_setup_launches(self._h)

    def profile(self, reps: int = 20):
        """[(name, ms per launch, algorithmic bytes per launch, launches per iteration)] for
        every kernel of one PCG iteration, timed with CUDA events (diagnostics)."""
        cap = 64
        arr = (_lib.KernelTiming * cap)()
        cnt = C.c_int(0)
        check(lib().mf3d_head_solver_profile(self._h, int(reps), arr, cap, C.byref(cnt)))
        return [(arr[i].name.decode(), float(arr[i].ms), float(arr[i].bytes), int(arr[i].launches_per_iter))
                for i in range(cnt.value)]

    def set_time_budget(self, seconds: float) -> None:
        """Device-time limit of one solve (default 120 s): past it the loop ends with status 3."""
        check(lib().mf3d_head_solver_set_time_budget(self._h, float(seconds)))

    def vcycle(self, r, z) -> None:
        """MultigridPreconditioner::apply (src/numerics/solvers/mg_preconditioner.cu:16-44)."""
        n = self.grid.num_cells()
        check(lib().mf3d_head_solver_vcycle(self._h, _f64(r, n, "r"), _f64(z, n, "z")))


class BatchSolver:
    """Independent head solves of several realisations, each on its own grid, solved together
    (the realisation loop of run_ensemble, src/runtime/ensemble/EnsembleRunner.cu:259-317,
    without the loop): batched launches, one CUDA graph for the whole PCG loop of all
    realisations, and a per-realisation stopping test."""

    def __init__(self, grids: Sequence[Grid3D], bc: BCSpec, cfg: Optional[HeadSolveConfig] = None,
                 stream=None):
        self.grids = list(grids)
        self.bc = bc
        self.cfg = cfg or HeadSolveConfig()
        arr = (_lib.Grid * len(self.grids))(*[g.c() for g in self.grids])
        h = C.c_void_p()
        s = C.c_void_p(stream) if isinstance(stream, int) else (stream or C.c_void_p())
        check(lib().mf3d_batch_create(len(self.grids), arr, C.byref(_bc(bc)), C.byref(self.cfg.c()), s,
                                      C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mf3d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.grids)

    @property
    def device_bytes(self) -> int:
        return lib().mf3d_batch_device_bytes(self._h)

    def _ptrs(self, arrays, what, allow_none=False):
        if len(arrays) != len(self.grids):
            raise ValueError(f"{what}: expected {len(self.grids)} arrays, got {len(arrays)}")
        out = (C.c_void_p * len(arrays))()
        for i, (a, g) in enumerate(zip(arrays, self.grids)):
            out[i] = None if (a is None and allow_none) else _f64(a, g.num_cells(), f"{what}[{i}]")
        return out

    def set_K(self, Ks) -> None:
        check(lib().mf3d_batch_set_K(self._h, self._ptrs(Ks, "K")))

    def solve(self, hs, x0s=None) -> List[HeadSolveResult]:
        res = (_lib.SolveResult * len(self.grids))()
        x0p = None if x0s is None else self._ptrs(x0s, "x0", allow_none=True)
        check(lib().mf3d_batch_solve(self._h, self._ptrs(hs, "h"), x0p, res))
        return [HeadSolveResult(r.num_iterations, r.initial_residual, r.final_residual, bool(r.converged),
                                r.status, r.num_levels, r.true_rel_residual, r.b_norm, r.device_ms,
                                r.kernel_launches) for r in res]

    def autotune(self, reps: int = 3):
        """Times the candidate work-item shapes of every sweep position of the batched V-cycle
        and keeps the fastest; returns one dict per sweep position."""
        cap = 256
        arr = (_lib.BatchTuning * cap)()
        cnt = C.c_int(0)
        check(lib().mf3d_batch_autotune(self._h, int(reps), arr, cap, C.byref(cnt)))
        return [dict(phase=t.phase, level=t.level, sweep=t.sweep, mode=t.mode, path=t.path, chunks=t.chunks,
                     ms_default=t.ms_default, ms_best=t.ms_best) for t in arr[:cnt.value]]


class WarmStart:
    """Learned PCG initial guess (no counterpart in the reference, whose guess is the x-linear
    head, src/physics/flow/solve_head.cu:29-73): a 3-D convolutional encoder-decoder on the
    tensor cores, trained with this library's own forward and backward kernels on lnK -> head
    pairs that the solver generates.  predict() writes x0 = h_lin + net(lnK) for
    HeadSolver.solve(h, x0); PCG still runs to its tolerance, so the network changes only the
    iteration count and the time."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        check(lib().mf3d_ws_create(int(seed), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mf3d_ws_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        return int(lib().mf3d_ws_num_params(self._h))

    def get_params(self):
        import numpy as np
        p = np.empty(self.num_params, dtype=np.float32)
        check(lib().mf3d_ws_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p) -> None:
        import numpy as np
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        check(lib().mf3d_ws_set_params(self._h, p.ctypes.data))

    def get_grads(self):
        import numpy as np
        g = np.empty(self.num_params, dtype=np.float32)
        check(lib().mf3d_ws_get_grads(self._h, g.ctypes.data))
        return g

    def save(self, path: str) -> None:
        import numpy as np
        np.save(path, self.get_params())

    def load(self, path: str) -> None:
        """Parameters from a .npy file: FP32, or BF16 bit patterns stored as uint16."""
        import numpy as np
        p = np.load(path)
        if p.dtype == np.uint16:
            p = (p.astype(np.uint32) << 16).view(np.float32)
        self.set_params(p)

    @classmethod
    def pretrained(cls):
        """The network trained on 2000 solver-generated pairs at 128^3 (lnK variance 0.5-4,
        correlation length 4-12 cells; macroflow3d_b200.warmstart_train), shipped as BF16."""
        import os
        ws = cls(seed=0)
        ws.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_c5_bf16.npy"))
        return ws

    @staticmethod
    def _f32_ptrs(arrays, n, what):
        import torch
        out = (C.c_void_p * len(arrays))()
        for i, a in enumerate(arrays):
            if a.dtype != torch.float32 or not a.is_cuda or not a.is_contiguous() or a.numel() != n:
                raise ValueError(f"{what}[{i}] must be a contiguous float32 CUDA tensor of {n} cells")
            out[i] = a.data_ptr()
        return out

    def train_step(self, grid: Grid3D, bc: BCSpec, lnKs, hs, lr: float) -> float:
        """One Adam step on the mean gradient of the samples (lnK, h: float32 CUDA tensors);
        lr = 0 computes the gradients only (get_grads).  Returns the mean loss."""
        n = grid.num_cells()
        loss = C.c_double(0.0)
        check(lib().mf3d_ws_train_step(self._h, C.byref(grid.c()), C.byref(_bc(bc)), len(lnKs),
                                       self._f32_ptrs(lnKs, n, "lnK"), self._f32_ptrs(hs, n, "h"), float(lr),
                                       C.byref(loss), _stream()))
        return loss.value

    def eval(self, grid: Grid3D, bc: BCSpec, lnKs, hs) -> float:
        n = grid.num_cells()
        loss = C.c_double(0.0)
        check(lib().mf3d_ws_eval(self._h, C.byref(grid.c()), C.byref(_bc(bc)), len(lnKs),
                                 self._f32_ptrs(lnKs, n, "lnK"), self._f32_ptrs(hs, n, "h"), C.byref(loss),
                                 _stream()))
        return loss.value

    def predict(self, grid: Grid3D, bc: BCSpec, K, x0) -> None:
        """x0 (float64 CUDA) = the x-linear head + the network's correction, from K (float64 CUDA)."""
        n = grid.num_cells()
        check(lib().mf3d_ws_predict(self._h, C.byref(grid.c()), C.byref(_bc(bc)), _f64(K, n, "K"),
                                    _f64(x0, n, "x0"), _stream()))


def nn_conv3d(grid: Grid3D, x, w, bias=None, relu=False, mask=None, out_f32=False):
    """One tensor-core 3x3x3 convolution (BF16 x [V, cin], w [cout, 27, cin]; FP32 bias [cout])."""
    import torch
    cin, cout = w.shape[2], w.shape[0]
    y = torch.empty((grid.num_cells(), cout), dtype=torch.float32 if out_f32 else torch.bfloat16, device=x.device)
    check(lib().mf3d_nn_conv3d(C.byref(grid.c()), int(cin), int(cout), x.data_ptr(), w.data_ptr(),
                               None if bias is None else bias.data_ptr(), int(bool(relu)),
                               None if mask is None else mask.data_ptr(), int(bool(out_f32)), y.data_ptr(),
                               _stream()))
    return y


def nn_flip_weights(w):
    """W'[ci, t, co] = W[co, 26 - t, ci] (BF16): the data gradient as a forward convolution."""
    import torch
    cout, _, cin = w.shape
    wt = torch.empty((cin, 27, cout), dtype=torch.bfloat16, device=w.device)
    check(lib().mf3d_nn_flip_weights(int(cin), int(cout), w.data_ptr(), wt.data_ptr(), _stream()))
    return wt


def nn_conv3d_wgrad(grid: Grid3D, x, dy):
    """(dW [cout, 27, cin], db [cout]) in FP32 from BF16 x [V, cin] and dy [V, cout]."""
    import torch
    cin, cout = x.shape[1], dy.shape[1]
    dw = torch.empty((cout, 27, cin), dtype=torch.float32, device=x.device)
    db = torch.empty((cout,), dtype=torch.float32, device=x.device)
    check(lib().mf3d_nn_conv3d_wgrad(C.byref(grid.c()), int(cin), int(cout), x.data_ptr(), dy.data_ptr(),
                                     dw.data_ptr(), db.data_ptr(), _stream()))
    return dw, db


def solve_head(h, K, grid: Grid3D, bc: BCSpec, cfg: HeadSolveConfig,
               workspace: Optional[HeadSolver] = None) -> Tuple[HeadSolveResult, HeadSolver]:
    """solve_head (src/physics/flow/solve_head.cuh:158-160).  Returns (result, workspace);
    pass the workspace back in to reuse the hierarchy and graph, as FlowWorkspace is reused."""
    import torch
    if workspace is None or workspace.grid != grid:
        workspace = HeadSolver(grid, bc, cfg, stream=torch.cuda.current_stream().cuda_stream)
    workspace.set_K(K)
    return workspace.solve(h), workspace


def init_head_guess(h, grid: Grid3D, bc: BCSpec) -> None:
    check(lib().mf3d_init_head_guess(C.byref(grid.c()), C.byref(_bc(bc)),
                                     _f64(h, grid.num_cells(), "h"), _stream()))


def build_rhs_head(rhs, K, grid: Grid3D, bc: BCSpec) -> None:
    n = grid.num_cells()
    check(lib().mf3d_build_rhs(C.byref(grid.c()), C.byref(_bc(bc)), _f64(K, n, "K"),
                               _f64(rhs, n, "rhs"), _stream()))


def coarsen_K(coarse: Grid3D, K_fine, K_coarse) -> None:
    n = coarse.num_cells()
    check(lib().mf3d_coarsen_K(C.byref(coarse.c()), _f64(K_fine, 8 * n, "K_fine"),
                               _f64(K_coarse, n, "K_coarse"), _stream()))


def apply_A(grid: Grid3D, bc: BCSpec, K, x, y, pin: bool = False) -> None:
    """VarCoeffLaplacian::apply (src/numerics/operators/varcoeff_laplacian.cu:241-277)."""
    n = grid.num_cells()
    check(lib().mf3d_apply_A(C.byref(grid.c()), C.byref(_bc(bc)), int(pin), _f64(K, n, "K"),
                             _f64(x, n, "x"), _f64(y, n, "y"), _stream()))


def gsrb_smooth_3d(grid: Grid3D, x, b, K, num_iters: int, bc: BCSpec, pin: bool = False) -> None:
    """gsrb_smooth_3d (src/multigrid/smoothers/gsrb_3d.cu:368-576); x updated in place."""
    n = grid.num_cells()
    check(lib().mf3d_gsrb(C.byref(grid.c()), C.byref(_bc(bc)), int(pin), _f64(K, n, "K"),
                          _f64(b, n, "b"), _f64(x, n, "x"), int(num_iters), _stream()))


def compute_residual_3d(grid: Grid3D, x, b, K, r, bc: BCSpec, pin: bool = False) -> None:
    """compute_residual_3d (src/multigrid/smoothers/residual_3d.cu:378-502)."""
    n = grid.num_cells()
    check(lib().mf3d_residual(C.byref(grid.c()), C.byref(_bc(bc)), int(pin), _f64(K, n, "K"),
                              _f64(x, n, "x"), _f64(b, n, "b"), _f64(r, n, "r"), _stream()))


def restrict_3d(coarse: Grid3D, r_fine, b_coarse) -> None:
    n = coarse.num_cells()
    check(lib().mf3d_restrict(C.byref(coarse.c()), _f64(r_fine, 8 * n, "r_fine"),
                              _f64(b_coarse, n, "b_coarse"), _stream()))


def prolong_3d_add(coarse: Grid3D, x_coarse, x_fine) -> None:
    n = coarse.num_cells()
    check(lib().mf3d_prolong_add(C.byref(coarse.c()), _f64(x_coarse, n, "x_coarse"),
                                 _f64(x_fine, 8 * n, "x_fine"), _stream()))


def velocity_sizes(grid: Grid3D, layout: int = VEL_COMPACT) -> Tuple[int, int, int]:
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    if layout == VEL_PADDED:
        s = (nx + 1) * (ny + 1) * (nz + 1)
        return s, s, s
    return (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)


def compute_velocity_from_head(U, V, W, h, K, grid: Grid3D, bc: BCSpec,
                               layout: int = VEL_COMPACT) -> None:
    """compute_velocity_from_head (src/physics/flow/velocity_from_head.cuh:54-73)."""
    n = grid.num_cells()
    su, sv, sw = velocity_sizes(grid, layout)
    check(lib().mf3d_velocity_from_head(C.byref(grid.c()), C.byref(_bc(bc)), _f64(h, n, "h"),
                                        _f64(K, n, "K"), int(layout), _f64(U, su, "U"),
                                        _f64(V, sv, "V"), _f64(W, sw, "W"), _stream()))


def velocity_mass_balance(U, V, W, h, K, grid: Grid3D, bc: BCSpec) -> Tuple[float, float, float]:
    """Compact velocity + (max_c |div_c|, Q_in, Q_out)."""
    n = grid.num_cells()
    su, sv, sw = velocity_sizes(grid, VEL_COMPACT)
    out = (C.c_double * 3)()
    check(lib().mf3d_velocity_mass_balance(C.byref(grid.c()), C.byref(_bc(bc)), _f64(h, n, "h"),
                                           _f64(K, n, "K"), _f64(U, su, "U"), _f64(V, sv, "V"),
                                           _f64(W, sw, "W"), out, _stream()))
    return out[0], out[1], out[2]


def velocity_mass_balance_noalloc(U, V, W, h, K, grid: Grid3D,
                                  bc: BCSpec) -> Tuple[float, float, float]:
    """velocity_mass_balance without device allocation: the reduction scratch is a static
    device array (at most MB_NOALLOC_MAX_BLOCKS reduction blocks).  Calls that overlap on one
    device race on that array."""
    n = grid.num_cells()
    su, sv, sw = velocity_sizes(grid, VEL_COMPACT)
    out = (C.c_double * 3)()
    check(lib().mf3d_velocity_mass_balance_noalloc(
        C.byref(grid.c()), C.byref(_bc(bc)), _f64(h, n, "h"), _f64(K, n, "K"),
        _f64(U, su, "U"), _f64(V, sv, "V"), _f64(W, sw, "W"), out, _stream()))
    return out[0], out[1], out[2]


def velocity_diagnostics(U, V, W, grid: Grid3D, layout: int = VEL_PADDED, div=None, omag=None, hel=None,
                         stats: bool = True):
    """compute_velocity_diagnostics + the statistics print_velocity_diagnostics reports
    (src/physics/flow/velocity_diagnostics.cu:22-203): the cell-centred divergence, |curl u| and
    helicity are written into div / omag / hel when given (float64 CUDA tensors of n cells);
    returns {"div": (min, max, mean), "vorticity_mag": (...), "helicity": (...)} or None."""
    n = grid.num_cells()
    su, sv, sw = velocity_sizes(grid, layout)
    out = (C.c_double * 9)()
    opt = lambda t, name: None if t is None else _f64(t, n, name)  # noqa: E731
    check(lib().mf3d_velocity_diagnostics(C.byref(grid.c()), int(layout), _f64(U, su, "U"), _f64(V, sv, "V"),
                                          _f64(W, sw, "W"), opt(div, "div"), opt(omag, "omag"), opt(hel, "hel"),
                                          out if stats else None, _stream()))
    if not stats:
        return None
    return {"div": tuple(out[0:3]), "vorticity_mag": tuple(out[3:6]), "helicity": tuple(out[6:9])}


def diag_bounded_wait(which: int, arrive: bool, tries: int) -> bool:
    """Runs one bounded mbarrier wait (0: the staged smoother's, 1: the convolution's) on a
    barrier that nothing completes (arrive False) or that one arrival completes; True when the
    wait gave up."""
    out = C.c_int(-1)
    check(lib().mf3d_diag_bounded_wait(int(which), 1 if arrive else 0, int(tries), C.byref(out)))
    return out.value == 1


def kfield_modes(seed: int, n_modes: int = 1000, covariance: int = COV_EXPONENTIAL,
                 lam=(1.0, 1.0, 1.0)):
    """Randomization-method modes (host, no GPU): numpy array (5, n_modes) = k1,k2,k3,a,b."""
    import numpy as np
    out = np.empty(5 * n_modes, dtype=np.float64)
    check(lib().mf3d_kfield_modes(int(seed), int(n_modes), int(covariance), float(lam[0]),
                                  float(lam[1]), float(lam[2]),
                                  out.ctypes.data_as(C.POINTER(C.c_double))))
    return out.reshape(5, n_modes)


def generate_K_field(grid: Grid3D, sigma2: float, lam=(1.0, 1.0, 1.0), seed: int = 0,
                     n_modes: int = 1000, covariance: int = COV_EXPONENTIAL, K_geo: float = 1.0,
                     log_only: bool = False):
    """generate_K_field (src/physics/stochastic/stochastic.cu:270-367) with per-axis
    correlation lengths: K = K_geo * exp(lnK) as a float64 CUDA tensor (nz, ny, nx)."""
    import math
    import torch
    modes = torch.from_numpy(kfield_modes(seed, n_modes, covariance, lam)).cuda()
    out = torch.empty((grid.nz, grid.ny, grid.nx), dtype=torch.float64, device="cuda")
    check(lib().mf3d_kfield_eval(C.byref(grid.c()), int(n_modes), modes.data_ptr(), float(sigma2),
                                 math.log(K_geo), 0 if log_only else 1, out.data_ptr(), _stream()))
    return out

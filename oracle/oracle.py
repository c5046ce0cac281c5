"""ctypes front-end for the CPU oracle (oracle/liboracle.so) and the reference build
(oracle/_ref/libmf3d_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs as the checker.  The product (macroflow3d_b200) never
imports this module.

All arrays are C-contiguous float64 numpy arrays in the reference layout
(i + nx*(j + ny*k), i.e. numpy shape (nz, ny, nx)).  BC type codes follow
src/core/BCSpec.hpp:13 of the reference: 0 Dirichlet, 1 Neumann, 2 Periodic; face order
xmin, xmax, ymin, ymax, zmin, zmax.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_REF = os.path.join(_HERE, "_ref", "libmf3d_ref.so")

DIRICHLET, NEUMANN, PERIODIC = 0, 1, 2
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class BC(C.Structure):
    _fields_ = [("type", C.c_int * 6), ("value", C.c_double * 6)]


class Result(C.Structure):
    _fields_ = [("iterations", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("converged", C.c_int),
                ("num_levels", C.c_int)]


def make_bc(types, values=(0.0,) * 6) -> BC:
    bc = BC()
    for f in range(6):
        bc.type[f] = int(types[f])
        bc.value[f] = float(values[f])
    return bc


def baseline_bc() -> BC:
    """h = 1 at x = 0, h = 0 at x = L, homogeneous Neumann elsewhere."""
    return make_bc([DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, NEUMANN],
                   [1.0, 0.0, 0.0, 0.0, 0.0, 0.0])


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB) or (
            os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "mf3d_oracle.c"))):
        subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        i, d = C.c_int, C.c_double
        pbc = C.POINTER(BC)
        L.og_apply_A.argtypes = [i, i, i, d, pbc, i, _dp, _dp, _dp]
        L.og_gsrb.argtypes = [i, i, i, d, pbc, i, _dp, _dp, _dp, i]
        L.og_residual.argtypes = [i, i, i, d, pbc, i, _dp, _dp, _dp, _dp]
        L.og_restrict.argtypes = [i, i, i, _dp, _dp]
        L.og_prolong_add.argtypes = [i, i, i, _dp, _dp]
        L.og_coarsen_K.argtypes = [i, i, i, _dp, _dp]
        L.og_build_rhs.argtypes = [i, i, i, d, pbc, _dp, _dp]
        L.og_init_guess.argtypes = [i, i, i, pbc, _dp]
        L.og_vcycle_precond.argtypes = [i, i, i, d, pbc, i, i, i, i, i, _dp, _dp, _dp]
        L.og_vcycle_precond.restype = i
        L.og_solve_head_pcg.argtypes = [i, i, i, d, pbc, i, i, i, i, i, i, i, d, _dp, i, _dp,
                                        C.POINTER(Result)]
        L.og_solve_head_mg.argtypes = [i, i, i, d, pbc, i, i, i, i, i, i, d, _dp, _dp,
                                       C.POINTER(Result)]
        L.og_solve_head_cg.argtypes = [i, i, i, d, pbc, i, i, i, d, _dp, _dp, C.POINTER(Result)]
        L.og_velocity.argtypes = [i, i, i, d, pbc, _dp, _dp, i, _dp, _dp, _dp]
        L.og_mass_balance.argtypes = [i, i, i, d, _dp, _dp, _dp, C.c_void_p, _dp]
        L.og_lnk_eval.argtypes = [i, i, i, d, i, _dp, _dp, _dp, _dp, _dp, d, _dp]
        L.og_velocity_diagnostics.argtypes = [i, i, i, d, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.og_kfield_modes.argtypes = [C.c_uint64, i, i, d, d, d, _dp]
        L.og_kfield_modes.restype = i
        L.og_kfield_eval_runs.argtypes = [i, i, i, d, i, _dp, d, d, i, _dp]
        L.og_num_threads.restype = i
        L.og_set_num_threads.argtypes = [i]
        _lib = L
    return _lib


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dims(a):
    nz, ny, nx = a.shape
    return nx, ny, nz


def set_threads(n: int) -> None:
    lib().og_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().og_num_threads())


def apply_A(K, x, bc, dx=1.0, pin=False):
    K, x = _c(K), _c(x)
    y = np.empty_like(x)
    lib().og_apply_A(*_dims(K), dx, C.byref(bc), int(pin), K.ravel(), x.ravel(), y.ravel())
    return y


def gsrb(K, b, x, bc, iters=1, dx=1.0, pin=False):
    K, b = _c(K), _c(b)
    x = _c(x).copy()
    lib().og_gsrb(*_dims(K), dx, C.byref(bc), int(pin), K.ravel(), b.ravel(), x.ravel(), iters)
    return x


def residual(K, x, b, bc, dx=1.0, pin=False):
    K, x, b = _c(K), _c(x), _c(b)
    r = np.empty_like(x)
    lib().og_residual(*_dims(K), dx, C.byref(bc), int(pin), K.ravel(), x.ravel(), b.ravel(),
                      r.ravel())
    return r


def restrict(rf):
    rf = _c(rf)
    nz, ny, nx = rf.shape
    bc = np.empty((nz // 2, ny // 2, nx // 2))
    lib().og_restrict(nx // 2, ny // 2, nz // 2, rf.ravel(), bc.ravel())
    return bc


def prolong_add(xc, xf):
    xc = _c(xc)
    xf = _c(xf).copy()
    NZ, NY, NX = xc.shape
    lib().og_prolong_add(NX, NY, NZ, xc.ravel(), xf.ravel())
    return xf


def coarsen_K(Kf):
    Kf = _c(Kf)
    nz, ny, nx = Kf.shape
    Kc = np.empty((nz // 2, ny // 2, nx // 2))
    lib().og_coarsen_K(nx // 2, ny // 2, nz // 2, Kf.ravel(), Kc.ravel())
    return Kc


def build_rhs(K, bc, dx=1.0):
    K = _c(K)
    b = np.empty_like(K)
    lib().og_build_rhs(*_dims(K), dx, C.byref(bc), K.ravel(), b.ravel())
    return b


def init_guess(shape, bc):
    h = np.empty(shape)
    nz, ny, nx = shape
    lib().og_init_guess(nx, ny, nz, C.byref(bc), h.ravel())
    return h


def vcycle(K, r, bc, levels, pre=2, post=2, coarse_iters=50, dx=1.0, pin=False):
    K, r = _c(K), _c(r)
    z = np.empty_like(r)
    nl = lib().og_vcycle_precond(*_dims(K), dx, C.byref(bc), int(pin), levels, pre, post,
                                 coarse_iters, K.ravel(), r.ravel(), z.ravel())
    return z, nl


def solve_head_pcg(K, bc, mg_levels, pre=2, post=2, coarse_iters=50, max_iter=1000,
                   check_every=10, rtol=1e-8, dx=1.0, pin_mode=0, h0=None):
    """solve_head(PCG_MG).  Returns (h, Result)."""
    K = _c(K)
    h = np.empty_like(K) if h0 is None else _c(h0).copy()
    res = Result()
    lib().og_solve_head_pcg(*_dims(K), dx, C.byref(bc), pin_mode, mg_levels, pre, post,
                            coarse_iters, max_iter, check_every, rtol, K.ravel(),
                            0 if h0 is None else 1, h.ravel(), C.byref(res))
    return h, res


def solve_head_mg(K, bc, mg_levels, pre=2, post=2, coarse_iters=50, max_cycles=20, rtol=1e-6,
                  dx=1.0, pin_mode=0):
    K = _c(K)
    h = np.empty_like(K)
    res = Result()
    lib().og_solve_head_mg(*_dims(K), dx, C.byref(bc), pin_mode, mg_levels, pre, post,
                           coarse_iters, max_cycles, rtol, K.ravel(), h.ravel(), C.byref(res))
    return h, res


def solve_head_cg(K, bc, max_iter=1000, check_every=10, rtol=1e-8, dx=1.0, pin_mode=0):
    """solve_head(CG): unpreconditioned CG from the x-linear guess.  Returns (h, Result)."""
    K = _c(K)
    h = np.empty_like(K)
    res = Result()
    lib().og_solve_head_cg(*_dims(K), dx, C.byref(bc), pin_mode, max_iter, check_every, rtol,
                           K.ravel(), h.ravel(), C.byref(res))
    return h, res


def velocity(H, K, bc, dx=1.0, layout=0):
    """Face velocities.  layout 0: compact MAC arrays (U (nz,ny,nx+1), V (nz,ny+1,nx),
    W (nz+1,ny,nx)); layout 1: padded (nz+1,ny+1,nx+1) each, zero where not a face."""
    H, K = _c(H), _c(K)
    nz, ny, nx = K.shape
    if layout == 0:
        U, V, W = np.zeros((nz, ny, nx + 1)), np.zeros((nz, ny + 1, nx)), np.zeros((nz + 1, ny, nx))
    else:
        U, V, W = (np.zeros((nz + 1, ny + 1, nx + 1)) for _ in range(3))
    lib().og_velocity(nx, ny, nz, dx, C.byref(bc), H.ravel(), K.ravel(), layout, U.ravel(),
                      V.ravel(), W.ravel())
    return U, V, W


def mass_balance(U, V, W, dx=1.0):
    """Compact layout only.  Returns (div per cell, max|div|, Q_in, Q_out)."""
    U, V, W = _c(U), _c(V), _c(W)
    nz, ny, nxp = U.shape
    nx = nxp - 1
    div = np.empty((nz, ny, nx))
    out = np.zeros(3)
    lib().og_mass_balance(nx, ny, nz, dx, U.ravel(), V.ravel(), W.ravel(),
                          div.ctypes.data_as(C.c_void_p), out)
    return div, out[0], out[1], out[2]


def velocity_diagnostics(U, V, W, shape, dx=1.0, layout=1):
    """Cell-centred divergence, |curl u| and helicity (nz, ny, nx) each, and the statistics
    [min, max, mean] x (div, |omega|, helicity)."""
    U, V, W = _c(U), _c(V), _c(W)
    nz, ny, nx = shape
    div, om, he = np.empty(shape), np.empty(shape), np.empty(shape)
    st = np.empty(9)
    lib().og_velocity_diagnostics(nx, ny, nz, dx, layout, U.ravel(), V.ravel(), W.ravel(), div.ravel(),
                                  om.ravel(), he.ravel(), st)
    return div, om, he, st


def lnk_eval(shape, modes, sigma, dx=1.0):
    """lnK at cell centres from randomization-method modes (k1,k2,k3,a,b)."""
    nz, ny, nx = shape
    k1, k2, k3, a, b = (_c(m) for m in modes)
    out = np.empty(shape)
    lib().og_lnk_eval(nx, ny, nz, dx, len(a), k1, k2, k3, a, b, float(sigma), out.ravel())
    return out


def kfield_modes(seed, n_modes=1000, covariance=0, lam=(1.0, 1.0, 1.0)):
    """Randomization-method modes (5, n_modes) = k1, k2, k3, a, b from the Philox sampler.
    covariance: 0 exponential, 1 Gaussian."""
    out = np.empty(5 * n_modes)
    rc = lib().og_kfield_modes(int(seed) & 0xFFFFFFFFFFFFFFFF, int(n_modes), int(covariance),
                               float(lam[0]), float(lam[1]), float(lam[2]), out)
    if rc != 0:
        raise ValueError("bad K-field parameters")
    return out.reshape(5, n_modes)


def generate_K(shape, sigma2, lam=(1.0, 1.0, 1.0), seed=0, n_modes=1000, covariance=0,
               K_geo=1.0, dx=1.0, log_only=False):
    """K = K_geo exp(lnK) (or lnK) on the host, for a process that must not load the product:
    the same modes and the same run-wise evaluation as the product's generator."""
    nz, ny, nx = shape
    modes = np.ascontiguousarray(kfield_modes(seed, n_modes, covariance, lam)).ravel()
    out = np.empty(shape)
    lib().og_kfield_eval_runs(nx, ny, nz, dx, n_modes, modes, float(np.sqrt(sigma2)),
                              float(np.log(K_geo)), 0 if log_only else 1, out.ravel())
    return out


# ---------------------------------------------------------------------------
# Reference build (GPU).  Present only where oracle/_ref was built.
# ---------------------------------------------------------------------------
_ref = None


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(_REF)
        i, d = C.c_int, C.c_double
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        R.ref_last_error.restype = C.c_char_p
        R.ref_apply_A.argtypes = [i, i, i, d, ip, _dp, i, _dp, _dp, _dp]
        R.ref_gsrb.argtypes = [i, i, i, d, ip, _dp, i, _dp, _dp, _dp, i]
        R.ref_residual.argtypes = [i, i, i, d, ip, _dp, i, _dp, _dp, _dp, _dp]
        R.ref_restrict.argtypes = [i, i, i, _dp, _dp]
        R.ref_prolong_add.argtypes = [i, i, i, _dp, _dp]
        R.ref_coarsen_K.argtypes = [i, i, i, _dp, _dp]
        R.ref_build_rhs.argtypes = [i, i, i, d, ip, _dp, _dp, _dp]
        R.ref_init_guess.argtypes = [i, i, i, d, ip, _dp, _dp]
        R.ref_vcycle.argtypes = [i, i, i, d, ip, _dp, i, i, i, i, i, _dp, _dp, _dp,
                                 C.POINTER(C.c_int)]
        R.ref_solve_head.argtypes = [i, i, i, d, ip, _dp, i, i, i, i, i, i, i, i, d, d, i, _dp,
                                     _dp, ip, _dp]
        R.ref_velocity.argtypes = [i, i, i, d, ip, _dp, i, _dp, _dp, _dp, _dp, _dp]
        R.ref_bench.argtypes = [i, i, i, d, ip, _dp, i, i, i, i, i, i, d, i, i, _dp,
                                C.c_void_p, np.ctypeslib.ndpointer(dtype=np.float32), ip, _dp]
        _ref = R
    return _ref


def _bcarrays(bc: BC):
    return (np.array(list(bc.type), dtype=np.int32), np.array(list(bc.value), dtype=np.float64))


def _chk(rc):
    if rc != 0:
        raise RuntimeError("reference call failed: " + ref().ref_last_error().decode())


def ref_apply_A(K, x, bc, dx=1.0, pin=False):
    K, x = _c(K), _c(x)
    y = np.empty_like(x)
    t, v = _bcarrays(bc)
    _chk(ref().ref_apply_A(*_dims(K), dx, t, v, int(pin), K.ravel(), x.ravel(), y.ravel()))
    return y


def ref_gsrb(K, b, x, bc, iters=1, dx=1.0, pin=False):
    K, b = _c(K), _c(b)
    x = _c(x).copy()
    t, v = _bcarrays(bc)
    _chk(ref().ref_gsrb(*_dims(K), dx, t, v, int(pin), K.ravel(), b.ravel(), x.ravel(), iters))
    return x


def ref_residual(K, x, b, bc, dx=1.0, pin=False):
    K, x, b = _c(K), _c(x), _c(b)
    r = np.empty_like(x)
    t, v = _bcarrays(bc)
    _chk(ref().ref_residual(*_dims(K), dx, t, v, int(pin), K.ravel(), x.ravel(), b.ravel(),
                            r.ravel()))
    return r


def ref_restrict(rf):
    rf = _c(rf)
    nz, ny, nx = rf.shape
    out = np.empty((nz // 2, ny // 2, nx // 2))
    _chk(ref().ref_restrict(nx // 2, ny // 2, nz // 2, rf.ravel(), out.ravel()))
    return out


def ref_prolong_add(xc, xf):
    xc = _c(xc)
    xf = _c(xf).copy()
    NZ, NY, NX = xc.shape
    _chk(ref().ref_prolong_add(NX, NY, NZ, xc.ravel(), xf.ravel()))
    return xf


def ref_coarsen_K(Kf):
    Kf = _c(Kf)
    nz, ny, nx = Kf.shape
    out = np.empty((nz // 2, ny // 2, nx // 2))
    _chk(ref().ref_coarsen_K(nx // 2, ny // 2, nz // 2, Kf.ravel(), out.ravel()))
    return out


def ref_build_rhs(K, bc, dx=1.0):
    K = _c(K)
    b = np.empty_like(K)
    t, v = _bcarrays(bc)
    _chk(ref().ref_build_rhs(*_dims(K), dx, t, v, K.ravel(), b.ravel()))
    return b


def ref_init_guess(shape, bc, dx=1.0):
    h = np.empty(shape)
    nz, ny, nx = shape
    t, v = _bcarrays(bc)
    _chk(ref().ref_init_guess(nx, ny, nz, dx, t, v, h.ravel()))
    return h


def ref_vcycle(K, r, bc, levels, pre=2, post=2, coarse_iters=50, dx=1.0, pin=False):
    K, r = _c(K), _c(r)
    z = np.empty_like(r)
    nl = C.c_int(0)
    t, v = _bcarrays(bc)
    _chk(ref().ref_vcycle(*_dims(K), dx, t, v, int(pin), levels, pre, post, coarse_iters,
                          K.ravel(), r.ravel(), z.ravel(), C.byref(nl)))
    return z, nl.value


def ref_solve_head(K, bc, mg_levels, solver=0, pre=2, post=2, coarse_iters=50, mg_max_cycles=20,
                   max_iter=1000, check_every=10, cg_rtol=1e-8, rtol=1e-6, dx=1.0, pin_mode=0):
    """Reference solve_head.  solver: 0 PCG_MG, 1 MG, 2 CG.
    Returns (h, iterations, converged, initial_residual, final_residual)."""
    K = _c(K)
    h = np.empty_like(K)
    info = np.zeros(4, dtype=np.int32)
    res = np.zeros(2)
    t, v = _bcarrays(bc)
    _chk(ref().ref_solve_head(*_dims(K), dx, t, v, solver, mg_levels, pre, post, coarse_iters,
                              mg_max_cycles, max_iter, check_every, cg_rtol, rtol, pin_mode,
                              K.ravel(), h.ravel(), info, res))
    return h, int(info[0]), bool(info[1]), float(res[0]), float(res[1])


def ref_velocity(H, K, bc, dx=1.0, layout=0):
    H, K = _c(H), _c(K)
    nz, ny, nx = K.shape
    if layout == 0:
        U, V, W = np.zeros((nz, ny, nx + 1)), np.zeros((nz, ny + 1, nx)), np.zeros((nz + 1, ny, nx))
    else:
        U, V, W = (np.zeros((nz + 1, ny + 1, nx + 1)) for _ in range(3))
    t, v = _bcarrays(bc)
    _chk(ref().ref_velocity(nx, ny, nz, dx, t, v, layout, H.ravel(), K.ravel(), U.ravel(),
                            V.ravel(), W.ravel()))
    return U, V, W


def ref_bench(K, bc, mg_levels, max_iter, check_every, cg_rtol, warmup, reps, pre=2, post=2,
              coarse_iters=50, dx=1.0, want_head=False):
    """Times the reference's solve_head(PCG_MG) + compute_velocity_from_head with K resident.
    Returns (ms per repetition, iterations, converged, r0, rfinal, head or None)."""
    K = _c(K)
    ms = np.zeros(max(reps, 1), dtype=np.float32)
    info = np.zeros(4, dtype=np.int32)
    res = np.zeros(2)
    h = np.empty_like(K) if want_head else None
    t, v = _bcarrays(bc)
    _chk(ref().ref_bench(*_dims(K), dx, t, v, mg_levels, pre, post, coarse_iters, max_iter,
                         check_every, cg_rtol, warmup, reps, K.ravel(),
                         h.ctypes.data_as(C.c_void_p) if want_head else None, ms, info, res))
    return ms[:reps], int(info[0]), bool(info[1]), float(res[0]), float(res[1]), h

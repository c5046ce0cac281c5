"""Generates tests/golden/*.npz from the REFERENCE's own CUDA implementation.

The reference (santi-esquerre/MacroFlow3D) has no golden vectors for the head-solve path, so
the fixtures that pin the CPU oracle are produced by running the reference's unmodified
sources, compiled by oracle/Makefile into oracle/_ref/libmf3d_ref.so, on a GPU:

    make -C oracle ref            # where the reference tree is present
    python tests/golden/make_golden.py [--out DIR]   # on a machine with a GPU

Inputs are seeded; each case stores its inputs and the reference outputs.
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
D, N, P = O.DIRICHLET, O.NEUMANN, O.PERIODIC

# (name, shape (nz, ny, nx), bc types, bc values, pin, dx)
OPERATOR_CASES = [
    ("mixed_bc", (8, 10, 6), [D, D, N, D, N, N], [1.0, 0.25, 0.0, 0.5, 0.0, 0.0], False, 1.0),
    ("neumann_pin", (4, 6, 8), [N, N, N, N, N, N], [0.0] * 6, True, 0.5),
    ("periodic_x", (6, 8, 8), [P, P, N, N, D, D], [0.0, 0.0, 0.0, 0.0, 0.3, 0.7], False, 1.0),
    ("baseline16", (16, 16, 16), [D, D, N, N, N, N], [1.0, 0.0, 0.0, 0.0, 0.0, 0.0], False, 1.0),
    ("odd_dirichlet", (5, 7, 3), [D, D, D, D, D, D], [1.0, 0.0, 0.2, 0.4, 0.6, 0.8], False, 2.0),
]


def lognormal(rng, shape, sigma=1.0):
    return np.exp(sigma * rng.standard_normal(shape))


def make_operator_cases():
    for name, shape, types, values, pin, dx in OPERATOR_CASES:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        bc = O.make_bc(types, values)
        K = lognormal(rng, shape)
        x = rng.standard_normal(shape)
        b = rng.standard_normal(shape)
        out = dict(K=K, x=x, b=b, bc_type=np.array(types), bc_value=np.array(values),
                   pin=np.array(int(pin)), dx=np.array(dx))
        out["Ax"] = O.ref_apply_A(K, x, bc, dx, pin)
        out["res"] = O.ref_residual(K, x, b, bc, dx, pin)
        out["gsrb1"] = O.ref_gsrb(K, b, x, bc, 1, dx, pin)
        out["gsrb3"] = O.ref_gsrb(K, b, x, bc, 3, dx, pin)
        out["rhs"] = O.ref_build_rhs(K, bc, dx)
        out["guess"] = O.ref_init_guess(shape, bc, dx)
        for lay in (0, 1):
            U, V, W = O.ref_velocity(x, K, bc, dx, lay)
            out[f"U{lay}"], out[f"V{lay}"], out[f"W{lay}"] = U, V, W
        np.savez_compressed(os.path.join(OUT, f"op_{name}.npz"), **out)
        print("wrote", name)


def make_transfer_cases():
    rng = np.random.default_rng(7)
    fine = rng.standard_normal((4, 6, 8))
    coarse = rng.standard_normal((2, 3, 4))
    Kf = lognormal(rng, (4, 6, 8))
    out = dict(fine=fine, coarse=coarse, Kf=Kf)
    out["restrict"] = O.ref_restrict(fine)
    out["prolong"] = O.ref_prolong_add(coarse, fine)
    out["coarsenK"] = O.ref_coarsen_K(Kf)
    np.savez_compressed(os.path.join(OUT, "transfer.npz"), **out)
    print("wrote transfer")


VCYCLE_CASES = [
    ("vc_baseline16", (16, 16, 16), [D, D, N, N, N, N], [1.0, 0.0, 0, 0, 0, 0], False, 3, 2, 2, 50),
    ("vc_periodic8", (8, 8, 8), [P, P, N, N, D, D], [0, 0, 0, 0, 1.0, 0.0], False, 2, 2, 2, 50),
    ("vc_pin", (8, 8, 16), [N, N, N, N, N, N], [0.0] * 6, True, 3, 1, 3, 20),
]


def make_vcycle_cases():
    for name, shape, types, values, pin, levels, pre, post, coarse in VCYCLE_CASES:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        bc = O.make_bc(types, values)
        K = lognormal(rng, shape)
        r = rng.standard_normal(shape)
        z, nl = O.ref_vcycle(K, r, bc, levels, pre, post, coarse, 1.0, pin)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), K=K, r=r, z=z, bc_type=np.array(types),
                            bc_value=np.array(values), pin=np.array(int(pin)),
                            cfg=np.array([levels, pre, post, coarse, nl]))
        print("wrote", name, nl)


SOLVE_CASES = [
    # name, shape, sigma, levels, rtol, check_every, max_iter
    ("pcg_baseline16", (16, 16, 16), 1.0, 3, 1e-10, 1, 200),
    ("pcg_baseline32", (32, 32, 32), 1.5, 4, 1e-10, 10, 200),
    ("pcg_aniso", (8, 16, 32), 1.0, 3, 1e-9, 1, 200),
]


def make_solve_cases():
    bc = O.baseline_bc()
    for name, shape, sigma, levels, rtol, ce, mi in SOLVE_CASES:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        K = lognormal(rng, shape, sigma)
        h, it, conv, r0, rf = O.ref_solve_head(K, bc, levels, solver=0, max_iter=mi, check_every=ce,
                                               cg_rtol=rtol)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), K=K, h=h,
                            info=np.array([it, int(conv), levels, ce, mi]),
                            res=np.array([r0, rf, rtol]))
        print("wrote", name, it, conv, r0, rf)


OTHER_SOLVERS = [
    # name, shape, sigma, solver (1 MG, 2 CG), levels, tol, check_every, max
    ("mg_baseline16", (16, 16, 16), 1.0, 1, 3, 1e-9, 1, 60),
    ("cg_baseline16", (16, 16, 16), 0.5, 2, 3, 1e-8, 1, 600),
]


def make_other_solver_cases():
    bc = O.baseline_bc()
    for name, shape, sigma, solver, levels, tol, ce, mx in OTHER_SOLVERS:
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        K = lognormal(rng, shape, sigma)
        h, it, conv, r0, rf = O.ref_solve_head(K, bc, levels, solver=solver, mg_max_cycles=mx, max_iter=mx,
                                               check_every=ce, cg_rtol=tol, rtol=tol)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), K=K, h=h,
                            info=np.array([it, int(conv), levels, ce, mx, solver]),
                            res=np.array([r0, rf, tol]))
        print("wrote", name, it, conv, r0, rf)


if __name__ == "__main__":
    if "--out" in sys.argv:
        OUT = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(OUT, exist_ok=True)
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libmf3d_ref.so not built (make -C oracle ref)")
    make_operator_cases()
    make_transfer_cases()
    make_vcycle_cases()
    make_solve_cases()
    make_other_solver_cases()

"""Pins the CPU oracle to the reference: every fixture in tests/golden/ was produced by the
reference's own CUDA code (tests/golden/make_golden.py over oracle/_ref), and the oracle
must reproduce it.  Runs on CPU."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _files(prefix):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_golden_fixtures_present():
    assert _files("op_") and _files("transfer") and _files("vc_") and _files("pcg_"), \
        "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", _files("op_"), ids=os.path.basename)
def test_oracle_operators_match_reference(oracle_mod, path):
    O = oracle_mod
    z = np.load(path)
    bc = O.make_bc(z["bc_type"], z["bc_value"])
    pin, dx = bool(z["pin"]), float(z["dx"])
    K, x, b = z["K"], z["x"], z["b"]
    assert _rel(O.apply_A(K, x, bc, dx, pin), z["Ax"]) < 1e-13
    assert _rel(O.residual(K, x, b, bc, dx, pin), z["res"]) < 1e-13
    assert _rel(O.gsrb(K, b, x, bc, 1, dx, pin), z["gsrb1"]) < 1e-13
    assert _rel(O.gsrb(K, b, x, bc, 3, dx, pin), z["gsrb3"]) < 1e-12
    assert np.array_equal(O.build_rhs(K, bc, dx), z["rhs"])
    assert np.array_equal(O.init_guess(K.shape, bc), z["guess"])
    for lay in (0, 1):
        U, V, W = O.velocity(x, K, bc, dx, lay)
        for a, key in ((U, "U"), (V, "V"), (W, "W")):
            assert _rel(a, z[f"{key}{lay}"]) < 1e-14


def test_oracle_transfer_match_reference(oracle_mod):
    O = oracle_mod
    z = np.load(_files("transfer")[0])
    assert np.array_equal(O.restrict(z["fine"]), z["restrict"])
    assert np.array_equal(O.prolong_add(z["coarse"], z["fine"]), z["prolong"])
    assert _rel(O.coarsen_K(z["Kf"]), z["coarsenK"]) < 1e-15


@pytest.mark.parametrize("path", _files("vc_"), ids=os.path.basename)
def test_oracle_vcycle_matches_reference(oracle_mod, path):
    O = oracle_mod
    z = np.load(path)
    levels, pre, post, coarse, nl = (int(v) for v in z["cfg"])
    bc = O.make_bc(z["bc_type"], z["bc_value"])
    out, nl_o = O.vcycle(z["K"], z["r"], bc, levels, pre, post, coarse, 1.0, bool(z["pin"]))
    assert nl_o == nl
    assert _rel(out, z["z"]) < 1e-11


@pytest.mark.parametrize("path", _files("pcg_"), ids=os.path.basename)
def test_oracle_pcg_matches_reference(oracle_mod, path):
    O = oracle_mod
    z = np.load(path)
    it, conv, levels, ce, mi = (int(v) for v in z["info"])
    r0, rf, rtol = (float(v) for v in z["res"])
    h, res = O.solve_head_pcg(z["K"], O.baseline_bc(), levels, max_iter=mi, check_every=ce, rtol=rtol)
    assert bool(res.converged) == bool(conv)
    assert abs(res.iterations - it) <= (1 if ce == 1 else 0)
    assert abs(res.initial_residual - r0) < 1e-12 * r0
    assert _rel(h, z["h"]) < 1e-9


@pytest.mark.parametrize("path", _files("mg_"), ids=os.path.basename)
def test_oracle_mg_matches_reference(oracle_mod, path):
    O = oracle_mod
    z = np.load(path)
    it, conv, levels, ce, mx, solver = (int(v) for v in z["info"])
    r0, rf, tol = (float(v) for v in z["res"])
    h, res = O.solve_head_mg(z["K"], O.baseline_bc(), levels, max_cycles=mx, rtol=tol)
    assert bool(res.converged) == bool(conv)
    assert abs(res.iterations - it) <= 1
    assert _rel(h, z["h"]) < 1e-8


@pytest.mark.parametrize("path", _files("cg_"), ids=os.path.basename)
def test_reference_cg_defect_is_recorded(oracle_mod, path):
    """The reference's solver=cg path does not converge: cg_solve captures the d_rr / d_rr_new
    spans before its loop (src/numerics/solvers/cg.cuh:29-30) and then swaps the buffers
    (cg.cuh:156), so alpha keeps using ||r0||^2 and the reported residual is ||r0||.  The
    golden run shows exactly that; CG as documented (the oracle, and this library) converges."""
    O = oracle_mod
    z = np.load(path)
    it, conv, levels, ce, mx, solver = (int(v) for v in z["info"])
    r0, rf, tol = (float(v) for v in z["res"])
    assert solver == 2 and not conv and it == mx and rf == r0
    h, res = O.solve_head_cg(z["K"], O.baseline_bc(), max_iter=mx, check_every=ce, rtol=tol)
    assert res.converged and res.iterations < mx
    assert abs(res.initial_residual - r0) < 1e-12 * r0

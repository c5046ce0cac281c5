"""GPU parity against the REFERENCE itself: the committed golden fixtures (produced by the
reference's CUDA code) and, where oracle/_ref/libmf3d_ref.so was built, a live run of the
reference's solve_head on the 64^3 configuration (plain FP64 CCMG-PCG, sigma^2 = 1,
correlation length 4 cells, h = 1 / 0 on the x faces)."""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _files(prefix):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _np(t):
    return t.detach().cpu().numpy()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _bc(M, types, values):
    return M.BCSpec([M.BCFace(int(t), float(v)) for t, v in zip(types, values)])


@pytest.mark.parametrize("path", _files("op_"), ids=os.path.basename)
def test_operators_match_reference_golden(mf3d, path):
    M = mf3d
    z = np.load(path)
    nz, ny, nx = z["K"].shape
    g = M.Grid3D(nx, ny, nz, float(z["dx"]))
    bc, pin = _bc(M, z["bc_type"], z["bc_value"]), bool(z["pin"])
    K, x, b = _t(z["K"]), _t(z["x"]), _t(z["b"])
    y = _t(np.zeros(z["K"].shape))
    M.apply_A(g, bc, K, x, y, pin)
    assert _rel(_np(y), z["Ax"]) < 1e-12
    M.compute_residual_3d(g, x, b, K, y, bc, pin)
    assert _rel(_np(y), z["res"]) < 1e-12
    for it in (1, 3):
        xs = x.clone()
        M.gsrb_smooth_3d(g, xs, b, K, it, bc, pin)
        assert _rel(_np(xs), z[f"gsrb{it}"]) < 1e-11
    for lay in (0, 1):
        su, sv, sw = M.velocity_sizes(g, lay)
        U, V, W = _t(np.zeros(su)), _t(np.zeros(sv)), _t(np.zeros(sw))
        M.compute_velocity_from_head(U, V, W, x, K, g, bc, lay)
        for a, key in ((U, "U"), (V, "V"), (W, "W")):
            assert _rel(_np(a), z[f"{key}{lay}"].ravel()) < 1e-14


@pytest.mark.parametrize("path", _files("vc_"), ids=os.path.basename)
def test_vcycle_matches_reference_golden(mf3d, path):
    M = mf3d
    z = np.load(path)
    levels, pre, post, coarse, nl = (int(v) for v in z["cfg"])
    nz, ny, nx = z["K"].shape
    cfg = M.HeadSolveConfig(mg_levels=levels, mg_pre_smooth=pre, mg_post_smooth=post,
                            mg_coarse_iters=coarse,
                            pin_mode=M.PIN_ON if bool(z["pin"]) else M.PIN_OFF)
    s = M.HeadSolver(M.Grid3D(nx, ny, nz, 1.0), _bc(M, z["bc_type"], z["bc_value"]), cfg)
    s.set_K(_t(z["K"]))
    out = _t(np.zeros(z["K"].shape))
    s.vcycle(_t(z["r"]), out)
    assert s.num_levels == nl
    assert _rel(_np(out), z["z"]) < 1e-10


@pytest.mark.parametrize("path", _files("pcg_"), ids=os.path.basename)
def test_pcg_matches_reference_golden(mf3d, path):
    M = mf3d
    z = np.load(path)
    it, conv, levels, ce, mi = (int(v) for v in z["info"])
    r0, rf, rtol = (float(v) for v in z["res"])
    nz, ny, nx = z["K"].shape
    cfg = M.HeadSolveConfig(mg_levels=levels, cg_rtol=rtol, cg_check_every=ce, cg_max_iter=mi)
    s = M.HeadSolver(M.Grid3D(nx, ny, nz, 1.0), M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(z["K"]))
    h = _t(np.zeros(z["K"].shape))
    res = s.solve(h)
    assert res.converged == bool(conv)
    assert abs(res.num_iterations - it) <= (1 if ce == 1 else 0)
    assert abs(res.initial_residual - r0) < 1e-12 * r0
    assert _rel(_np(h), z["h"]) < 1e-9


def test_live_reference_64cubed(mf3d, oracle_mod):
    O, M = oracle_mod, mf3d
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    g = M.Grid3D(64, 64, 64, 1.0)
    K = M.generate_K_field(g, 1.0, (4.0, 4.0, 4.0), seed=2024)
    Kn = _np(K)
    bc = O.baseline_bc()
    # the reference's test is ||r||/||r0||; ask it for ||r||/||b|| <= 1e-10 via its own rtol
    b = O.build_rhs(Kn, bc)
    r0 = np.linalg.norm(b - O.apply_A(Kn, O.init_guess(Kn.shape, bc), bc))
    rtol = 1e-10 * np.linalg.norm(b) / r0
    href, it_ref, conv_ref, _, _ = O.ref_solve_head(Kn, bc, 5, max_iter=500, check_every=1, cg_rtol=rtol)
    cfg = M.HeadSolveConfig(mg_levels=5, cg_rtol=rtol, cg_check_every=1, cg_max_iter=500)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
    s.set_K(K)
    h = _t(np.zeros(Kn.shape))
    res = s.solve(h)
    assert conv_ref and res.converged
    assert abs(res.num_iterations - it_ref) <= 1
    assert _rel(_np(h), href) < 1e-9
    Ur, Vr, Wr = O.ref_velocity(href, Kn, bc)
    su, sv, sw = M.velocity_sizes(g)
    U, V, W = _t(np.zeros(su)), _t(np.zeros(sv)), _t(np.zeros(sw))
    M.compute_velocity_from_head(U, V, W, h, K, g, M.BCSpec.darcy_x())
    for a, r in ((U, Ur), (V, Vr), (W, Wr)):
        assert _rel(_np(a), r.ravel()) < 1e-9


@pytest.mark.parametrize("path", _files("mg_"), ids=os.path.basename)
def test_mg_solver_matches_reference_golden(mf3d, path):
    M = mf3d
    z = np.load(path)
    it, conv, levels, ce, mx, solver = (int(v) for v in z["info"])
    r0, rf, tol = (float(v) for v in z["res"])
    nz, ny, nx = z["K"].shape
    cfg = M.HeadSolveConfig(solver_type=solver, mg_levels=levels, mg_max_cycles=mx, rtol=tol,
                            cg_max_iter=mx, cg_check_every=ce, cg_rtol=tol)
    s = M.HeadSolver(M.Grid3D(nx, ny, nz, 1.0), M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(z["K"]))
    h = _t(np.zeros(z["K"].shape))
    res = s.solve(h)
    assert res.converged == bool(conv)
    assert abs(res.num_iterations - it) <= (1 if solver == 1 else 2)
    assert _rel(_np(h), z["h"]) < 1e-8

"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle on seeded inputs.

Tolerances: single operator applications are compared element-wise at 1e-12 relative to
the array's max (the arithmetic differs only in rounding: stored vs recomputed harmonic
means, operation order, FMA); solves are compared by head relative max-norm <= 1e-9 and
mass balance <= 1e-10, the targets of the task statement for this path.
"""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

D, N, P = 0, 1, 2
BC_CASES = [
    ("darcy", [D, D, N, N, N, N], [1.0, 0.0, 0, 0, 0, 0], False),
    ("mixed", [D, N, N, D, N, D], [1.0, 0, 0, 0.5, 0, 0.25], False),
    ("neumann_pin", [N, N, N, N, N, N], [0.0] * 6, True),
    ("periodic", [P, P, N, N, D, D], [0, 0, 0, 0, 0.3, 0.7], False),
    ("all_dirichlet", [D] * 6, [1.0, 0.0, 0.2, 0.4, 0.6, 0.8], False),
]
SHAPES = [(8, 10, 6), (6, 8, 12), (12, 34, 40), (16, 16, 16)]


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _np(t):
    return t.detach().cpu().numpy()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _bcs(M, types, values):
    return M.BCSpec([M.BCFace(t, v) for t, v in zip(types, values)])


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("case", BC_CASES, ids=[c[0] for c in BC_CASES])
def test_operators_vs_oracle(mf3d, oracle_mod, shape, case):
    M, O = mf3d, oracle_mod
    name, types, values, pin = case
    rng = np.random.default_rng(zlib.crc32(repr((shape, name)).encode()))
    K = np.exp(rng.normal(size=shape))
    x, b = rng.normal(size=shape), rng.normal(size=shape)
    dx = 0.5
    g = M.Grid3D(shape[2], shape[1], shape[0], dx)
    bc, obc = _bcs(M, types, values), O.make_bc(types, values)
    Kt, xt, bt = _t(K), _t(x), _t(b)
    y = _t(np.zeros(shape))
    M.apply_A(g, bc, Kt, xt, y, pin)
    assert _rel(_np(y), O.apply_A(K, x, obc, dx, pin)) < 1e-12
    M.compute_residual_3d(g, xt, bt, Kt, y, bc, pin)
    assert _rel(_np(y), O.residual(K, x, b, obc, dx, pin)) < 1e-12
    for it in (1, 3):
        xs = xt.clone()
        M.gsrb_smooth_3d(g, xs, bt, Kt, it, bc, pin)
        assert _rel(_np(xs), O.gsrb(K, b, x, obc, it, dx, pin)) < 1e-11, it
    M.build_rhs_head(y, Kt, g, bc)
    assert _rel(_np(y), O.build_rhs(K, obc, dx)) < 1e-14 or np.abs(O.build_rhs(K, obc, dx)).max() == 0
    M.init_head_guess(y, g, bc)
    assert np.abs(_np(y) - O.init_guess(shape, obc)).max() < 1e-15
    for lay in (0, 1):
        su, sv, sw = M.velocity_sizes(g, lay)
        U, V, W = _t(np.zeros(su)), _t(np.zeros(sv)), _t(np.zeros(sw))
        M.compute_velocity_from_head(U, V, W, xt, Kt, g, bc, lay)
        Uo, Vo, Wo = O.velocity(x, K, obc, dx, lay)
        for a, o in ((U, Uo), (V, Vo), (W, Wo)):
            assert np.abs(_np(a) - o.ravel()).max() <= 1e-14 * np.abs(o).max()


# The x-pair sweep (kernels_sweep_pair.cuh) on the shapes that exercise its tile ring: partial
# tiles in x and y, periodic axes of whole tiles (x 32, y 16 cells), odd nz, nx = 2, and grids
# deep enough in z for several z chunks per tile.
PAIR_CASES = [
    ((12, 32, 64), [P, P, P, P, D, D], [0, 0, 0, 0, 0.3, 0.7], False),
    ((10, 16, 32), [P] * 6, [0.0] * 6, True),
    ((7, 20, 50), [D, N, N, D, N, D], [1.0, 0, 0, 0.5, 0, 0.25], False),
    ((40, 18, 34), [D, D, N, N, N, N], [1.0, 0.0, 0, 0, 0, 0], False),
    ((5, 3, 2), [D] * 6, [1.0, 0.0, 0.2, 0.4, 0.6, 0.8], False),
    ((96, 48, 96), [D, D, N, N, N, N], [1.0, 0.0, 0, 0, 0, 0], False),
    # 64 tiles: z chunks of several planes, so that the steady-state staging runs
    ((64, 128, 256), [D, D, N, N, N, N], [1.0, 0.0, 0, 0, 0, 0], False),
    ((48, 128, 128), [D, D, P, P, N, N], [1.0, 0.0, 0, 0, 0, 0], False),
]


@pytest.mark.parametrize("shape,types,values,pin", PAIR_CASES, ids=[str(c[0]) for c in PAIR_CASES])
def test_gsrb_pair_sweep_vs_oracle(mf3d, oracle_mod, shape, types, values, pin):
    M, O = mf3d, oracle_mod
    rng = np.random.default_rng(zlib.crc32(repr(("pair", shape)).encode()))
    K = np.exp(rng.normal(size=shape))
    x, b = rng.normal(size=shape), rng.normal(size=shape)
    g = M.Grid3D(shape[2], shape[1], shape[0], 0.5)
    bc, obc = _bcs(M, types, values), O.make_bc(types, values)
    for it in (1, 2, 3):
        xs = _t(x)
        M.gsrb_smooth_3d(g, xs, _t(b), _t(K), it, bc, pin)
        assert _rel(_np(xs), O.gsrb(K, b, x, obc, it, 0.5, pin)) < 1e-11, it


@pytest.mark.parametrize("shape,levels", [((32, 32, 32), 4), ((24, 16, 52), 3), ((64, 64, 64), 5)])
@pytest.mark.parametrize("case", BC_CASES[:4], ids=[c[0] for c in BC_CASES[:4]])
def test_fp32_vcycle_vs_oracle(mf3d, oracle_mod, shape, levels, case):
    """The FP32 V-cycle (x-pair sweeps in FP32, FP64 coarse tail) against the FP64 oracle: equal
    to FP32 rounding (1e-5 of the correction's max)."""
    M, O = mf3d, oracle_mod
    name, types, values, pin = case
    if types[0] == P and (shape[2] >> (levels - 1)) % 2:
        pytest.skip("periodic x with an odd count on the coarsest level: red-black order is undefined")
    rng = np.random.default_rng(zlib.crc32(repr((shape, name, 32)).encode()))
    K = np.exp(rng.normal(size=shape))
    r = rng.normal(size=shape)
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    cfg = M.HeadSolveConfig(mg_levels=levels, precision=M.PREC_FP32, pin_mode=M.PIN_ON if pin else M.PIN_OFF)
    s = M.HeadSolver(g, _bcs(M, types, values), cfg)
    s.set_K(_t(K))
    z = _t(np.zeros(shape))
    s.vcycle(_t(r), z)
    zo, _ = O.vcycle(K, r, O.make_bc(types, values), levels, 2, 2, 50, 1.0, pin)
    assert _rel(_np(z), zo) < 1e-5


def test_transfer_vs_oracle(mf3d, oracle_mod):
    M, O = mf3d, oracle_mod
    rng = np.random.default_rng(5)
    fine = rng.normal(size=(8, 12, 16))
    coarse = rng.normal(size=(4, 6, 8))
    Kf = np.exp(rng.normal(size=(8, 12, 16)))
    cg = M.Grid3D(8, 6, 4, 2.0)
    out = _t(np.zeros((4, 6, 8)))
    M.restrict_3d(cg, _t(fine), out)
    assert _rel(_np(out), O.restrict(fine)) < 1e-15
    xf = _t(fine)
    M.prolong_3d_add(cg, _t(coarse), xf)
    assert _rel(_np(xf), O.prolong_add(coarse, fine)) < 1e-15
    M.coarsen_K(cg, _t(Kf), out)
    assert _rel(_np(out), O.coarsen_K(Kf)) < 1e-14


@pytest.mark.parametrize("shape,levels,pre,post,coarse", [
    ((16, 16, 16), 3, 2, 2, 50), ((32, 32, 32), 4, 2, 2, 50), ((64, 32, 32), 4, 1, 3, 20),
    ((8, 8, 8), 2, 2, 2, 50), ((64, 64, 64), 5, 2, 2, 50),
    # level 1 is 18 / 26 cells wide: 16-byte rows in FP64 but not whole 4-cell quads
    ((16, 20, 36), 3, 2, 2, 50), ((24, 16, 52), 3, 2, 2, 20)])
@pytest.mark.parametrize("case", BC_CASES[:4], ids=[c[0] for c in BC_CASES[:4]])
def test_vcycle_vs_oracle(mf3d, oracle_mod, shape, levels, pre, post, coarse, case):
    M, O = mf3d, oracle_mod
    name, types, values, pin = case
    if types[0] == P and (shape[2] >> (levels - 1)) % 2:
        pytest.skip("periodic x with an odd count on the coarsest level: red-black order is undefined")
    rng = np.random.default_rng(zlib.crc32(repr((shape, name, 1)).encode()))
    K = np.exp(rng.normal(size=shape))
    r = rng.normal(size=shape)
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    cfg = M.HeadSolveConfig(mg_levels=levels, mg_pre_smooth=pre, mg_post_smooth=post,
                            mg_coarse_iters=coarse, pin_mode=M.PIN_ON if pin else M.PIN_OFF)
    s = M.HeadSolver(g, _bcs(M, types, values), cfg)
    s.set_K(_t(K))
    z = _t(np.zeros(shape))
    s.vcycle(_t(r), z)
    zo, nl = O.vcycle(K, r, O.make_bc(types, values), levels, pre, post, coarse, 1.0, pin)
    assert nl == s.num_levels
    assert _rel(_np(z), zo) < 1e-10


@pytest.mark.parametrize("shape,levels", [((64, 64, 64), 5), ((24, 16, 52), 3), ((32, 32, 32), 4),
                                          ((64, 48, 32), 4)])
@pytest.mark.parametrize("bcname", ["darcy", "periodic_yz"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cluster_coarse_end_matches_one_cta_tail(mf3d, monkeypatch, shape, levels, bcname, prec):
    """The coarse end in one thread-block cluster (levels of up to 32^3 cells in z slabs over
    the cluster's CTAs, FP64) against the same V-cycle with the one-CTA tail and x-pair sweeps
    above it: equal to rounding in FP64 (1e-12), to FP32 rounding of the levels it replaces
    in the FP32 V-cycle (1e-5)."""
    M = mf3d
    rng = np.random.default_rng(zlib.crc32(repr((shape, levels, bcname)).encode()))
    K = np.exp(rng.normal(size=shape))
    r = rng.normal(size=shape)
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    if bcname == "darcy":
        bc = M.BCSpec.darcy_x()
    else:
        bc = _bcs(M, [D, D, P, P, P, P], [1.0, 0.0, 0, 0, 0, 0])
    P_ = {"fp64": M.PREC_FP64, "fp32": M.PREC_FP32}[prec]
    cfg = M.HeadSolveConfig(mg_levels=levels, precision=P_)
    z = {}
    for mode in ("cluster", "tail"):
        if mode == "tail":
            monkeypatch.setenv("MF3D_NO_CLUSTER_TAIL", "1")
        s = M.HeadSolver(g, bc, cfg)
        first, ctas = s.coarse_info
        if mode == "cluster":
            assert ctas >= 2, (first, ctas)
        else:
            assert ctas == 0
        s.set_K(_t(K))
        zz = _t(np.zeros(shape))
        s.vcycle(_t(r), zz)
        z[mode] = _np(zz)
        s.close()
        monkeypatch.delenv("MF3D_NO_CLUSTER_TAIL", raising=False)
    assert _rel(z["cluster"], z["tail"]) < (1e-12 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("shape,levels", [((64, 64, 64), 5), ((32, 48, 64), 4), ((16, 16, 128), 3)])
@pytest.mark.parametrize("bcname", ["darcy", "all_dirichlet"])
def test_bf16_vcycle_staged_matches_unstaged(mf3d, monkeypatch, shape, levels, bcname):
    """The BF16-coefficient V-cycle on the TMA-staged x-pair sweep and the staged residual +
    restriction against the same V-cycle on the unstaged sweep (MF3D_NO_TMA): the same BF16
    coefficients and FP32 arithmetic, so equal to FP32 rounding (1e-5 of the max)."""
    M = mf3d
    rng = np.random.default_rng(zlib.crc32(repr((shape, levels, bcname, "bf16")).encode()))
    K = np.exp(rng.normal(size=shape))
    r = rng.normal(size=shape)
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    case = [c for c in BC_CASES if c[0] == bcname][0]
    bc = _bcs(M, case[1], case[2])
    cfg = M.HeadSolveConfig(mg_levels=levels, precision=M.PREC_BF16)
    z = {}
    for mode in ("staged", "unstaged"):
        if mode == "unstaged":
            monkeypatch.setenv("MF3D_NO_TMA", "1")
        s = M.HeadSolver(g, bc, cfg)
        s.set_K(_t(K))
        zz = _t(np.zeros(shape))
        s.vcycle(_t(r), zz)
        z[mode] = _np(zz)
        s.close()
        monkeypatch.delenv("MF3D_NO_TMA", raising=False)
    assert _rel(z["staged"], z["unstaged"]) < 1e-5


def _lognormal(shape, sigma, seed):
    return np.exp(sigma * np.random.default_rng(seed).normal(size=shape))


@pytest.mark.parametrize("shape,sigma,levels", [((16, 16, 16), 1.0, 3), ((24, 40, 32), 2.0, 4),
                                                ((64, 64, 64), 1.0, 5)])
def test_pcg_reference_semantics_vs_oracle(mf3d, oracle_mod, shape, sigma, levels):
    """Reference stopping rule (||r||/||r0|| < rtol every check_every): same iteration count."""
    M, O = mf3d, oracle_mod
    K = _lognormal(shape, sigma, 11)
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    bc = M.BCSpec.darcy_x()
    cfg = M.HeadSolveConfig(mg_levels=levels, cg_rtol=1e-10, cg_check_every=1)
    s = M.HeadSolver(g, bc, cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h)
    ho, ro = O.solve_head_pcg(K, O.baseline_bc(), levels, rtol=1e-10, check_every=1)
    assert res.converged and ro.converged
    assert abs(res.num_iterations - ro.iterations) <= 1
    assert _rel(_np(h), ho) < 1e-9
    assert res.true_rel_residual < 1e-9


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_mixed_precision_reaches_fp64_tolerance(mf3d, oracle_mod, prec):
    """FP32 / BF16-coefficient V-cycle inside flexible FP64 PCG to ||r||/||b|| <= 1e-10;
    the head agrees with a tightly solved FP64 oracle head."""
    M, O = mf3d, oracle_mod
    shape = (32, 32, 32)
    K = _lognormal(shape, 2.0, 12)
    g = M.Grid3D(32, 32, 32, 1.0)
    cfg = M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B,
                            precision=prec)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h)
    assert res.converged, res
    assert res.true_rel_residual <= 1.5e-10
    ho, _ = O.solve_head_pcg(K, O.baseline_bc(), 4, rtol=1e-15, check_every=1, max_iter=100)
    # measured 3.7e-9 (FP32, BF16) and 5.6e-9 (the FP64 reference algorithm) at 1e-10 on this
    # field of uncorrelated cell values, 1.04e-9 (FP32) at 1e-11: the head bound 1e-9 needs
    # ||r|| / ||b|| <= 1e-12 here (next assertion)
    assert _rel(_np(h), ho) < 1e-8
    s.close()
    cfg.cg_rtol = 1e-12
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(K))
    res = s.solve(h)
    assert res.converged and res.true_rel_residual <= 1.5e-12, res
    assert _rel(_np(h), ho) < 1e-9


def test_solvers_with_different_coarse_tails_coexist(mf3d):
    """A solver created later with a smaller coarse tail must not lower the tail kernel's
    shared-memory limit under an earlier solver's tail."""
    M = mf3d
    g = M.Grid3D(32, 32, 32, 1.0)
    K = _t(_lognormal((32, 32, 32), 1.0, 21))
    cfg = dict(cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B)
    big = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=5, **cfg))
    small = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=2, **cfg))
    for s in (big, small, big):
        s.set_K(K)
        h = _t(np.zeros((32, 32, 32)))
        assert s.solve(h).converged


def test_graph_and_host_loop_identical(mf3d):
    M = mf3d
    shape = (32, 32, 32)
    K = _t(_lognormal(shape, 1.5, 13))
    g = M.Grid3D(32, 32, 32, 1.0)
    out = []
    for ug in (1, 0):
        cfg = M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-10, cg_check_every=1, use_graph=ug)
        s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
        s.set_K(K)
        h = _t(np.zeros(shape))
        r = s.solve(h)
        out.append((r.num_iterations, _np(h)))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])  # deterministic reductions: bitwise equal


def test_repeated_solves_deterministic(mf3d):
    M = mf3d
    shape = (32, 32, 64)
    K = _t(_lognormal(shape, 1.0, 14))
    g = M.Grid3D(64, 32, 32, 1.0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-10))
    s.set_K(K)
    hs = []
    for _ in range(3):
        h = _t(np.zeros(shape))
        s.solve(h)
        hs.append(_np(h))
    assert np.array_equal(hs[0], hs[1]) and np.array_equal(hs[1], hs[2])


def test_velocity_mass_balance_after_solve(mf3d, oracle_mod):
    M, O = mf3d, oracle_mod
    shape = (32, 32, 32)
    K = _lognormal(shape, 1.0, 15)
    g = M.Grid3D(32, 32, 32, 1.0)
    bc = M.BCSpec.darcy_x()
    s = M.HeadSolver(g, bc, M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-12, cg_check_every=1,
                                              conv_norm=M.CONV_B))
    Kt = _t(K)
    s.set_K(Kt)
    h = _t(np.zeros(shape))
    s.solve(h)
    su, sv, sw = M.velocity_sizes(g)
    U, V, W = _t(np.zeros(su)), _t(np.zeros(sv)), _t(np.zeros(sw))
    mx, qin, qout = M.velocity_mass_balance(U, V, W, h, Kt, g, bc)
    assert mx / abs(qin) < 1e-10 and abs(qin - qout) / abs(qin) < 1e-10
    Uo, _, _ = O.velocity(_np(h), K, O.baseline_bc())
    assert _rel(_np(U), Uo.ravel()) < 1e-14


def test_warm_start_and_nonconvergence_reporting(mf3d):
    M = mf3d
    shape = (32, 32, 32)
    K = _t(_lognormal(shape, 1.0, 16))
    g = M.Grid3D(32, 32, 32, 1.0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-10,
                                                              cg_check_every=1, conv_norm=M.CONV_B))
    s.set_K(K)
    h = _t(np.zeros(shape))
    r1 = s.solve(h)
    h2 = _t(np.zeros(shape))
    r2 = s.solve(h2, x0=h)  # warm start from the converged head
    assert r2.num_iterations <= 1 and r2.converged
    s3 = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=4, cg_rtol=1e-14,
                                                               cg_max_iter=3, cg_check_every=1))
    s3.set_K(K)
    r3 = s3.solve(h2)
    assert not r3.converged and r3.num_iterations == 3 and r1.converged


def test_nonfinite_K_reports_status(mf3d):
    M = mf3d
    shape = (16, 16, 16)
    Kn = _lognormal(shape, 1.0, 17)
    Kn[3, 4, 5] = np.nan
    g = M.Grid3D(16, 16, 16, 1.0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=3, cg_rtol=1e-10))
    s.set_K(_t(Kn))
    res = s.solve(_t(np.zeros(shape)))
    assert not res.converged and res.status == 2


def test_kfield_vs_oracle(mf3d, oracle_mod):
    M, O = mf3d, oracle_mod
    g = M.Grid3D(37, 9, 5, 1.0)
    modes = M.kfield_modes(99, 1000, M.COV_EXPONENTIAL, (4.0, 4.0, 2.0))
    lnk = M.generate_K_field(g, 2.0, (4.0, 4.0, 2.0), seed=99, log_only=True)
    ref = O.lnk_eval((5, 9, 37), modes, np.sqrt(2.0))
    assert np.abs(_np(lnk) - ref).max() < 1e-9
    K = M.generate_K_field(g, 2.0, (4.0, 4.0, 2.0), seed=99)
    assert np.allclose(_np(K), np.exp(ref), rtol=1e-9)


def test_host_kfield_equals_device_kfield(mf3d, oracle_mod):
    """The oracle's host generator (the reference arm's K) and the product's device generator
    give the same field at the headline statistics (sigma^2 = 4, lambda = 8, 1000 modes)."""
    M, O = mf3d, oracle_mod
    g = M.Grid3D(64, 48, 40, 1.0)
    K = M.generate_K_field(g, 4.0, (8.0, 8.0, 8.0), seed=20240601, n_modes=1000)
    Ko = O.generate_K((40, 48, 64), 4.0, (8.0, 8.0, 8.0), seed=20240601, n_modes=1000)
    assert _rel(_np(K), Ko) < 1e-12


@pytest.mark.parametrize("prec", [0, 1])
def test_standalone_mg_solver_vs_oracle(mf3d, oracle_mod, prec):
    """solver = mg: V-cycles on the current head until ||r||/||r0|| < rtol
    (mg_solve, src/multigrid/cycle/v_cycle.cu:76-116)."""
    M, O = mf3d, oracle_mod
    shape = (32, 32, 32)
    K = _lognormal(shape, 1.0, 21)
    g = M.Grid3D(32, 32, 32, 1.0)
    cfg = M.HeadSolveConfig(solver_type=M.SOLVER_MG, mg_levels=4, mg_max_cycles=60, rtol=1e-10,
                            precision=prec)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h)
    ho, ro = O.solve_head_mg(K, O.baseline_bc(), 4, max_cycles=60, rtol=1e-10)
    assert res.converged and ro.converged
    if prec == 0:
        assert abs(res.num_iterations - ro.iterations) <= 1
    assert _rel(_np(h), ho) < 1e-8


def test_plain_cg_solver_vs_oracle(mf3d, oracle_mod):
    """solver = cg: unpreconditioned CG (cg_solve, src/numerics/solvers/cg.cuh:14-171)."""
    M, O = mf3d, oracle_mod
    shape = (16, 16, 16)
    K = _lognormal(shape, 0.5, 22)
    g = M.Grid3D(16, 16, 16, 1.0)
    cfg = M.HeadSolveConfig(solver_type=M.SOLVER_CG, cg_max_iter=800, cg_check_every=1, cg_rtol=1e-9)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h)
    ho, ro = O.solve_head_cg(K, O.baseline_bc(), max_iter=800, check_every=1, rtol=1e-9)
    assert res.converged and ro.converged
    assert abs(res.num_iterations - ro.iterations) <= 2
    assert _rel(_np(h), ho) < 1e-7


@pytest.mark.parametrize("case", BC_CASES, ids=[c[0] for c in BC_CASES])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pcg_every_bc_case_vs_oracle(mf3d, oracle_mod, case, prec):
    """PCG (search-direction update fused with the matvec) on every boundary kind: periodic
    wrap, the pinned cell, all-Dirichlet; 40 x 20 x 12 leaves partial column tiles in x and y
    and halves evenly through the three levels (the CUDA hierarchy stops at an odd axis)."""
    M, O = mf3d, oracle_mod
    name, types, values, _ = case
    shape = (12, 20, 40)
    K = _lognormal(shape, 1.0, zlib.crc32(name.encode()))
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    P = {"fp64": M.PREC_FP64, "fp32": M.PREC_FP32}[prec]
    cfg = M.HeadSolveConfig(mg_levels=3, cg_rtol=1e-10, cg_check_every=1, precision=P)
    # a random initial guess: with no Dirichlet face the right-hand side is zero, and the
    # pinned system then iterates from x0 towards h = 0
    x0 = np.random.default_rng(5).normal(size=shape)
    s = M.HeadSolver(g, _bcs(M, types, values), cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h, _t(x0))
    ho, ro = O.solve_head_pcg(K, O.make_bc(types, values), 3, rtol=1e-10, check_every=1, h0=x0)
    assert res.converged and ro.converged and ro.iterations > 3
    if prec == "fp64":
        assert abs(res.num_iterations - ro.iterations) <= 1
    assert np.abs(_np(h) - ho).max() / max(np.abs(ho).max(), np.abs(x0).max()) < 1e-8
    s.close()


@pytest.mark.parametrize("case", BC_CASES, ids=[c[0] for c in BC_CASES])
def test_plain_cg_every_bc_case_vs_oracle(mf3d, oracle_mod, case):
    """Plain CG (z = r, the FP64 form of the fused update) on every boundary kind."""
    M, O = mf3d, oracle_mod
    name, types, values, _ = case
    shape = (10, 18, 36)
    K = _lognormal(shape, 0.5, zlib.crc32(("cg" + name).encode()))
    g = M.Grid3D(shape[2], shape[1], shape[0], 1.0)
    cfg = M.HeadSolveConfig(solver_type=M.SOLVER_CG, cg_max_iter=3000, cg_check_every=1, cg_rtol=1e-10)
    s = M.HeadSolver(g, _bcs(M, types, values), cfg)
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    res = s.solve(h)
    ho, ro = O.solve_head_cg(K, O.make_bc(types, values), max_iter=3000, check_every=1, rtol=1e-10)
    assert res.converged and ro.converged
    assert abs(res.num_iterations - ro.iterations) <= 2
    assert _rel(_np(h), ho) < 1e-7
    s.close()


@pytest.mark.parametrize("shape", [(24, 20, 32), (2, 6, 8), (9, 5, 3)])
@pytest.mark.parametrize("layout", [0, 1])
def test_velocity_diagnostics_vs_oracle(mf3d, oracle_mod, shape, layout):
    """compute_velocity_diagnostics on the velocity of a solved head: divergence, |curl u| and
    helicity per cell and their min / max / mean, against the oracle (1e-12 of each field's
    max); (2, 6, 8) has a dimension below 3 (no curl)."""
    M, O = mf3d, oracle_mod
    K = _lognormal(shape, 1.0, 21)
    g = M.Grid3D(shape[2], shape[1], shape[0], 0.5)
    bc = M.BCSpec.darcy_x()
    s = M.HeadSolver(g, bc, M.HeadSolveConfig(mg_levels=2, cg_rtol=1e-12, cg_check_every=1))
    Kt = _t(K)
    s.set_K(Kt)
    h = _t(np.zeros(shape))
    s.solve(h)
    su, sv, sw = M.velocity_sizes(g, layout)
    U, V, W = _t(np.zeros(su)), _t(np.zeros(sv)), _t(np.zeros(sw))
    M.compute_velocity_from_head(U, V, W, h, Kt, g, bc, layout)
    div, om, he = _t(np.zeros(shape)), _t(np.zeros(shape)), _t(np.zeros(shape))
    st = M.velocity_diagnostics(U, V, W, g, layout, div, om, he)
    Un, Vn, Wn = _np(U), _np(V), _np(W)
    if layout == 0:
        Un = Un.reshape(shape[0], shape[1], shape[2] + 1)
        Vn = Vn.reshape(shape[0], shape[1] + 1, shape[2])
        Wn = Wn.reshape(shape[0] + 1, shape[1], shape[2])
    else:
        Un, Vn, Wn = (a.reshape(shape[0] + 1, shape[1] + 1, shape[2] + 1) for a in (Un, Vn, Wn))
    do, oo, ho, so = O.velocity_diagnostics(Un, Vn, Wn, shape, 0.5, layout)
    scale = max(np.abs(_np(U)).max(), 1e-300)
    for a, o in ((div, do), (om, oo), (he, ho)):
        assert np.abs(_np(a) - o).max() <= 1e-12 * max(np.abs(o).max(), scale)
    got = np.array(st["div"] + st["vorticity_mag"] + st["helicity"])
    assert np.allclose(got, so, rtol=1e-12, atol=1e-12 * scale ** 2)
    if min(shape) < 3:
        assert not _np(om).any() and not _np(he).any()
    # fields may be skipped; the statistics stay the same
    st2 = M.velocity_diagnostics(U, V, W, g, layout)
    assert st2 == st


@pytest.mark.parametrize("use_graph", [1, 0])
def test_time_budget_ends_the_loop_and_the_solver_recovers(mf3d, use_graph):
    """The device-time budget bounds a solve independently of the reductions: with a budget of
    one microsecond the loop's first kernel stops it (status 3, not converged) in the graph
    and in the host-driven loop; with the budget restored the same solver converges."""
    M = mf3d
    shape = (64, 64, 64)
    K = _lognormal(shape, 1.0, 31)
    g = M.Grid3D(64, 64, 64, 1.0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=5, cg_rtol=1e-10, cg_check_every=1,
                                                             use_graph=use_graph))
    s.set_K(_t(K))
    h = _t(np.zeros(shape))
    s.set_time_budget(1e-6)
    res = s.solve(h)
    assert res.status == 3 and not res.converged, res
    assert res.num_iterations <= 2
    s.set_time_budget(120.0)
    res = s.solve(h)
    assert res.status == 0 and res.converged and res.true_rel_residual < 1e-9, res
    with pytest.raises(Exception):
        s.set_time_budget(0.0)


def test_bounded_mbarrier_waits_give_up_and_leave_the_context_usable(mf3d):
    """The bounded waits of the staged smoother and of the tensor-core convolution give up on a
    barrier that nothing completes and succeed on one that an arrival completes; the context
    then still runs a solve."""
    M = mf3d
    for which in (0, 1):
        assert M.diag_bounded_wait(which, False, 64)
        assert not M.diag_bounded_wait(which, True, 64)
    g = M.Grid3D(16, 16, 16, 1.0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), M.HeadSolveConfig(mg_levels=3, cg_rtol=1e-10, cg_check_every=1))
    s.set_K(_t(_lognormal((16, 16, 16), 1.0, 3)))
    res = s.solve(_t(np.zeros((16, 16, 16))))
    assert res.converged

"""Known-answer and structural tests of the CPU oracle (no GPU).

The reference ships no tests for this path; these pin the oracle's discretisation to
closed-form solutions of the discrete problem (cell-centred 7-point stencil with half-cell
Dirichlet ghosts, src/multigrid/common/mg_conventions.cuh:44-110).
"""
import numpy as np
import pytest


def _darcy_bc(O, hw=1.0, he=0.0):
    return O.make_bc([O.DIRICHLET, O.DIRICHLET, O.NEUMANN, O.NEUMANN, O.NEUMANN, O.NEUMANN],
                     [hw, he, 0, 0, 0, 0])


def test_homogeneous_K_linear_head(oracle_mod):
    O = oracle_mod
    shape = (6, 5, 12)
    K = np.full(shape, 3.7)
    bc = _darcy_bc(O, 2.0, -1.0)
    # start from zero, not from the exact linear guess
    h, res = O.solve_head_pcg(K, bc, mg_levels=2, rtol=1e-13, check_every=1,
                              h0=np.zeros(shape))
    x = (np.arange(12) + 0.5) / 12
    exact = 2.0 + (-3.0) * x
    assert res.converged
    assert np.abs(h - exact[None, None, :]).max() < 1e-11
    # the reference's own initial guess is already the exact solution: r0 = 0
    guess = O.init_guess(shape, bc)
    assert np.abs(O.residual(K, guess, O.build_rhs(K, bc), bc)).max() < 1e-13


def test_x_layered_harmonic_mean_flux(oracle_mod):
    O = oracle_mod
    nx, ny, nz = 16, 4, 4
    kx = np.exp(np.random.default_rng(1).normal(size=nx))
    K = np.broadcast_to(kx[None, None, :], (nz, ny, nx)).copy()
    bc = _darcy_bc(O)
    h, res = O.solve_head_pcg(K, bc, mg_levels=3, rtol=1e-13, check_every=1)
    U, V, W = O.velocity(h, K, bc)
    q_expected = 1.0 / (nx * np.mean(1.0 / kx))  # (h_w - h_e) / (L * mean(1/K))
    assert np.abs(U - q_expected).max() < 1e-10 * q_expected
    assert np.abs(V).max() < 1e-10 and np.abs(W).max() < 1e-10


def test_y_layered_arithmetic_mean_flux(oracle_mod):
    O = oracle_mod
    nx, ny, nz = 8, 16, 4
    ky = np.exp(np.random.default_rng(2).normal(size=ny))
    K = np.broadcast_to(ky[None, :, None], (nz, ny, nx)).copy()
    bc = _darcy_bc(O)
    h, _ = O.solve_head_pcg(K, bc, mg_levels=3, rtol=1e-13, check_every=1)
    U, _, _ = O.velocity(h, K, bc)
    Q = U[:, :, 0].sum()  # dx = 1
    assert abs(Q - nz * ky.sum() / nx) < 1e-10 * Q


def test_divergence_equals_residual(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    shape = (6, 7, 9)
    K = np.exp(rng.normal(size=shape))
    bc = _darcy_bc(O, 1.5, 0.5)
    h = rng.normal(size=shape)
    r = O.residual(K, h, O.build_rhs(K, bc), bc)
    U, V, W = O.velocity(h, K, bc)
    div, _, _, _ = O.mass_balance(U, V, W)
    assert np.abs(div - r).max() < 1e-12 * np.abs(r).max()


@pytest.mark.parametrize("types", [
    [0, 0, 1, 1, 1, 1], [1, 1, 1, 1, 0, 0], [2, 2, 1, 1, 0, 0], [0, 0, 0, 0, 0, 0]])
def test_operator_symmetric_negative_definite(oracle_mod, types):
    O = oracle_mod
    rng = np.random.default_rng(4)
    shape = (6, 4, 8)
    K = np.exp(rng.normal(size=shape))
    bc = O.make_bc(types, [0.3] * 6)
    x, y = rng.normal(size=shape), rng.normal(size=shape)
    Ax, Ay = O.apply_A(K, x, bc), O.apply_A(K, y, bc)
    assert abs((Ax * y).sum() - (x * Ay).sum()) < 1e-11 * np.abs(Ax).max() * x.size
    assert (x * Ax).sum() < 0


def test_residual_matches_operator(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(5)
    shape = (5, 6, 7)
    K = np.exp(rng.normal(size=shape))
    bc = O.make_bc([0, 1, 2, 2, 0, 1], [1.0, 0, 0, 0, 0.5, 0])
    x, b = rng.normal(size=shape), rng.normal(size=shape)
    r = O.residual(K, x, b, bc, dx=0.7)
    assert np.abs(r - (b - O.apply_A(K, x, bc, dx=0.7))).max() < 1e-12 * np.abs(r).max()


def test_restriction_prolongation_adjoint(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(6)
    rf = rng.normal(size=(4, 6, 8))
    ec = rng.normal(size=(2, 3, 4))
    lhs = 8.0 * (O.restrict(rf) * ec).sum()
    rhs = (rf * (O.prolong_add(ec, np.zeros_like(rf)))).sum()
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_coarsen_geometric_mean(oracle_mod):
    O = oracle_mod
    Kf = np.exp(np.random.default_rng(7).normal(size=(4, 4, 4)))
    Kc = O.coarsen_K(Kf)
    blk = np.log(Kf).reshape(2, 2, 2, 2, 2, 2).transpose(0, 2, 4, 1, 3, 5).reshape(2, 2, 2, 8)
    assert np.allclose(Kc, np.exp(blk.mean(-1)), rtol=1e-14)


def test_gsrb_converges_to_solution(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(8)
    shape = (4, 4, 6)
    K = np.exp(0.5 * rng.normal(size=shape))
    bc = _darcy_bc(O)
    b = O.build_rhs(K, bc)
    x = O.gsrb(K, b, np.zeros(shape), bc, iters=3000)
    assert np.abs(O.residual(K, x, b, bc)).max() < 1e-10


def test_vcycle_reduces_error(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(9)
    shape = (16, 16, 16)
    K = np.exp(rng.normal(size=shape))
    bc = _darcy_bc(O)
    b = O.build_rhs(K, bc)
    z, nl = O.vcycle(K, b, bc, levels=3)
    assert nl == 3
    assert np.linalg.norm(O.residual(K, z, b, bc)) < 0.3 * np.linalg.norm(b)


def test_pcg_true_residual_and_mass_balance(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(10)
    K = np.exp(1.5 * rng.normal(size=(16, 16, 16)))
    bc = _darcy_bc(O)
    h, res = O.solve_head_pcg(K, bc, mg_levels=3, rtol=1e-11, check_every=1)
    b = O.build_rhs(K, bc)
    assert res.converged
    assert np.linalg.norm(b - O.apply_A(K, h, bc)) / np.linalg.norm(b) < 1e-10
    U, V, W = O.velocity(h, K, bc)
    _, mx, qin, qout = O.mass_balance(U, V, W)
    assert mx / abs(qin) < 1e-10 and abs(qin - qout) / abs(qin) < 1e-10


def test_mg_solver_converges(oracle_mod):
    O = oracle_mod
    K = np.exp(np.random.default_rng(11).normal(size=(16, 16, 16)))
    h, res = O.solve_head_mg(K, _darcy_bc(O), mg_levels=3, max_cycles=50, rtol=1e-9)
    assert res.converged and res.final_residual / res.initial_residual < 1e-9


def test_velocity_diagnostics_known_answers(oracle_mod):
    """Solid-body rotation about z plus a uniform axial velocity c: u = -y, v = x, w = c, so
    div u = 0, curl u = (0, 0, 2) at every interior cell and helicity = 2c; boundary cells and
    grids with a dimension below 3 report zero curl (velocity_diagnostics.cu:82-87)."""
    O = oracle_mod
    nz, ny, nx, dx, c = 5, 6, 7, 0.5, 0.75
    for layout in (0, 1):
        if layout:
            shp = (nz + 1, ny + 1, nx + 1)
            U, V, W = np.zeros(shp), np.zeros(shp), np.zeros(shp)
            kk, jj, ii = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
            U[:] = -(jj + 0.5) * dx
            V[:] = (ii + 0.5) * dx
            W[:] = c
        else:
            kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx + 1), indexing="ij")
            U = -(jj + 0.5) * dx
            kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny + 1), np.arange(nx), indexing="ij")
            V = (ii + 0.5) * dx
            W = np.full((nz + 1, ny, nx), c)
        div, om, he, st = O.velocity_diagnostics(U, V, W, (nz, ny, nx), dx, layout)
        assert np.abs(div).max() < 1e-14
        inner = (slice(1, -1),) * 3
        assert np.allclose(om[inner], 2.0, rtol=1e-14) and np.allclose(he[inner], 2.0 * c, rtol=1e-14)
        mask = np.ones(om.shape, bool)
        mask[inner] = False
        assert not om[mask].any() and not he[mask].any()
        ninner = (nz - 2) * (ny - 2) * (nx - 2)
        assert np.allclose(st[3:6], [0.0, 2.0, 2.0 * ninner / om.size], rtol=1e-14)
    # a dimension below 3: divergence only
    U, V, W = np.ones((2, 4, 5)), np.ones((2, 5, 4)), np.ones((3, 4, 4))
    div, om, he, st = O.velocity_diagnostics(U, V, W, (2, 4, 4), 1.0, 0)
    assert not om.any() and not he.any() and np.abs(div).max() == 0.0

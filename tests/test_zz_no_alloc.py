"""mf3d_velocity_mass_balance_noalloc: the fused velocity + mass-balance kernel with its
reduction scratch in a static device array instead of a per-call allocation.

Checked through the C-ABI against mf3d_velocity_mass_balance on the same inputs, on two calls
in a row whose second call has the smaller divergence (a max or a ticket left over from the
first call would show), and refused with MF3D_E_INVALID past its scratch size.  Kept in a file
of its own so that it runs last, after every other GPU test has used the library.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# both entry points run the same kernel with the same deterministic reduction order
TOL = 1e-12


def _inputs(M, nx, ny, nz, seed):
    """K log-normal; head = the linear x trend plus noise (returned apart)."""
    import torch
    rng = np.random.default_rng(seed)
    K = torch.from_numpy(np.exp(rng.normal(0.0, 1.0, (nz, ny, nx)))).cuda()
    trend = np.ascontiguousarray(np.broadcast_to(1.0 - (np.arange(nx) + 0.5) / nx, (nz, ny, nx)))
    return K, torch.from_numpy(trend).cuda(), torch.from_numpy(rng.standard_normal((nz, ny, nx))).cuda()


def _velocity_buffers(M, g):
    import torch
    return [torch.full((n,), np.nan, dtype=torch.float64, device="cuda") for n in M.velocity_sizes(g)]


@pytest.mark.parametrize("bc_kind", ["darcy_x", "periodic_yz"])
def test_noalloc_matches_allocating_entry_point_twice(mf3d, bc_kind):
    import torch
    M = mf3d
    nx, ny, nz = 48, 40, 24
    g = M.Grid3D(nx, ny, nz, 0.5)
    bc = M.BCSpec.darcy_x()
    if bc_kind == "periodic_yz":
        bc = M.BCSpec(bc.faces[:2] + [M.BCFace(M.PERIODIC) for _ in range(4)])
    K, trend, noise = _inputs(M, nx, ny, nz, 11)
    maxima = []
    for scale in (0.1, 0.01):  # second call: smaller divergence, so stale scratch would show
        hs = (trend + scale * noise).contiguous()
        Ua, Va, Wa = _velocity_buffers(M, g)
        ref = M.velocity_mass_balance(Ua, Va, Wa, hs, K, g, bc)
        Ub, Vb, Wb = _velocity_buffers(M, g)
        got = M.velocity_mass_balance_noalloc(Ub, Vb, Wb, hs, K, g, bc)
        torch.cuda.synchronize()
        for a, b in ((Ua, Ub), (Va, Vb), (Wa, Wb)):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            assert np.all(np.isfinite(b))
            np.testing.assert_allclose(b, a, rtol=TOL, atol=0.0)
        np.testing.assert_allclose(np.array(got), np.array(ref), rtol=TOL, atol=0.0)
        assert got[0] > 0.0
        maxima.append(got[0])
    assert maxima[1] < 0.5 * maxima[0]


def test_noalloc_refuses_grid_past_scratch(mf3d):
    import torch
    from macroflow3d_b200._lib import Mf3dError
    M = mf3d
    # ceil(8192/32) * ceil(1032/8) = 256 * 129 reduction blocks > MB_NOALLOC_MAX_BLOCKS
    nx, ny, nz = 8192, 1032, 1
    assert (nx // 32) * ((ny + 7) // 8) > M.MB_NOALLOC_MAX_BLOCKS
    g = M.Grid3D(nx, ny, nz, 1.0)
    bc = M.BCSpec.darcy_x()
    n = nx * ny * nz
    K = torch.ones(n, dtype=torch.float64, device="cuda")
    h = torch.zeros(n, dtype=torch.float64, device="cuda")
    U, V, W = _velocity_buffers(M, g)
    with pytest.raises(Mf3dError, match="static mass-balance scratch"):
        M.velocity_mass_balance_noalloc(U, V, W, h, K, g, bc)
    # the refusal happens before any launch: the outputs are untouched
    torch.cuda.synchronize()
    assert torch.isnan(U).all()

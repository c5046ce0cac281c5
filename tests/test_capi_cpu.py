"""CPU-side tests of the product: the C-ABI library loads and exports every symbol that
include/mf3d.h declares, host-only entry points work, the YAML `flow:` loader mirrors the
reference's strict parser, and argument errors come back as status codes (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "mf3d.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(mf3d_[A-Za-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(mf3d):
    from macroflow3d_b200 import _lib
    L = _lib.lib()
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_defaults(mf3d):
    from macroflow3d_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.mf3d_version()
    cfg = _lib.SolverConfig()
    assert L.mf3d_default_config(C.byref(cfg)) == 0
    # HeadSolveConfig defaults, src/physics/flow/solve_head.cuh:63-96
    assert (cfg.solver, cfg.mg_levels, cfg.mg_pre_smooth, cfg.mg_post_smooth) == (0, 4, 2, 2)
    assert (cfg.mg_max_cycles, cfg.mg_coarse_iters, cfg.cg_max_iter, cfg.cg_check_every) == (20, 50, 1000, 10)
    assert cfg.cg_rtol == 1e-8 and cfg.rtol == 1e-6 and cfg.use_graph == 1


def test_invalid_arguments_return_status(mf3d):
    from macroflow3d_b200 import _lib
    L = _lib.lib()
    assert L.mf3d_default_config(None) == _lib.MF3D_E_INVALID
    assert b"null" in L.mf3d_last_error()
    h = C.c_void_p()
    g = _lib.Grid(0, 4, 4, 1.0)
    bc = _lib.BC()
    cfg = _lib.SolverConfig()
    L.mf3d_default_config(C.byref(cfg))
    assert L.mf3d_head_solver_create(C.byref(g), C.byref(bc), C.byref(cfg), None, C.byref(h)) == _lib.MF3D_E_INVALID
    assert not h.value
    modes = np.zeros(5, dtype=np.float64)
    assert L.mf3d_kfield_modes(1, 1, 0, -1.0, 1.0, 1.0, modes.ctypes.data_as(C.POINTER(C.c_double))) \
        == _lib.MF3D_E_INVALID


def test_batch_refuses_bad_arguments_before_any_device_call(mf3d):
    from macroflow3d_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    grids = (_lib.Grid * 2)(_lib.Grid(32, 32, 32, 1.0), _lib.Grid(0, 32, 32, 1.0))
    bc = _lib.BC()
    cfg = _lib.SolverConfig()
    L.mf3d_default_config(C.byref(cfg))
    assert L.mf3d_batch_create(0, grids, C.byref(bc), C.byref(cfg), None, C.byref(h)) == _lib.MF3D_E_INVALID
    assert b"count" in L.mf3d_last_error()
    assert L.mf3d_batch_create(2, grids, C.byref(bc), C.byref(cfg), None, C.byref(h)) == _lib.MF3D_E_INVALID
    grids[1] = _lib.Grid(48, 32, 32, 1.0)
    cfg.solver = 2  # plain CG: not batched
    assert L.mf3d_batch_create(2, grids, C.byref(bc), C.byref(cfg), None, C.byref(h)) == _lib.MF3D_E_INVALID
    assert b"PCG_MG" in L.mf3d_last_error()
    cfg.solver = 0
    cfg.mg_post_smooth = 0
    assert L.mf3d_batch_create(2, grids, C.byref(bc), C.byref(cfg), None, C.byref(h)) == _lib.MF3D_E_INVALID
    assert not h.value
    assert L.mf3d_batch_solve(None, None, None, None) == _lib.MF3D_E_INVALID
    assert L.mf3d_batch_device_bytes(None) == -1


def test_kfield_modes_deterministic_and_distributed(mf3d):
    m1 = mf3d.kfield_modes(1234, 4000, mf3d.COV_EXPONENTIAL, (4.0, 4.0, 4.0))
    m2 = mf3d.kfield_modes(1234, 4000, mf3d.COV_EXPONENTIAL, (4.0, 4.0, 4.0))
    m3 = mf3d.kfield_modes(1235, 4000, mf3d.COV_EXPONENTIAL, (4.0, 4.0, 4.0))
    assert np.array_equal(m1, m2) and not np.array_equal(m1, m3)
    k1, k2, k3, a, b = m1
    # Fourier coefficients ~ N(0,1)
    assert abs(a.mean()) < 0.08 and abs(a.std() - 1) < 0.08 and abs(b.std() - 1) < 0.08
    # radial density of the exponential covariance: k^2 / (1+k^2)^2 (in units of 1/lambda),
    # whose CDF is (atan(k) - k/(1+k^2)) * 2/pi; compare at a few quantiles
    kk = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2) * 4.0
    for q in (0.5, 1.0, 2.0, 5.0):
        cdf = (np.arctan(q) - q / (1 + q * q)) * 2 / np.pi
        assert abs((kk < q).mean() - cdf) < 0.03
    # isotropic directions
    assert abs(np.mean(k3 / np.sqrt(k1**2 + k2**2 + k3**2))) < 0.05


def test_kfield_modes_anisotropic_scaling(mf3d):
    iso = mf3d.kfield_modes(7, 100, mf3d.COV_EXPONENTIAL, (1.0, 1.0, 1.0))
    ani = mf3d.kfield_modes(7, 100, mf3d.COV_EXPONENTIAL, (16.0, 16.0, 4.0))
    assert np.allclose(ani[0], iso[0] / 16) and np.allclose(ani[2], iso[2] / 4)
    assert np.array_equal(ani[3], iso[3])


def test_kfield_covariance_statistics(mf3d, oracle_mod):
    """Ensemble covariance of the generated lnK matches sigma^2 exp(-r/lambda) (exponential)
    using the oracle's direct evaluation of the modes at a few separations."""
    O = oracle_mod
    lam, sig2 = 4.0, 2.0
    pts = np.zeros((1, 1, 13))
    acc = np.zeros(13)
    R = 300
    for s in range(R):
        modes = mf3d.kfield_modes(10_000 + s, 400, mf3d.COV_EXPONENTIAL, (lam, lam, lam))
        f = O.lnk_eval(pts.shape, modes, np.sqrt(sig2))[0, 0]
        acc += f[0] * f
    cov = acc / R
    for d in (0, 2, 4, 8):
        assert abs(cov[d] - sig2 * np.exp(-d / lam)) < 0.35 * sig2, (d, cov[d])


YAML = """
grid: {nx: 8}
flow:
  solver: mg_cg
  mg_levels: 5
  cg_rtol: 1.0e-10
  cg_check_every: 1
  pin_first_cell: true
  precision: fp32
  bc:
    west: {type: dirichlet, value: 1.0}
    east: {type: dirichlet, value: 0.0}
    ymin: {type: neumann}
    north: {type: neumann, value: 0}
    bottom: {type: periodic}
    top: {type: periodic}
"""


def test_flow_yaml_parsing(mf3d):
    cfg = mf3d.load_flow_yaml(YAML)
    assert cfg.solver == "mg_cg" and cfg.mg_levels == 5 and cfg.cg_rtol == 1e-10
    assert cfg.pin_mode == mf3d.PIN_ON
    assert cfg.bc.types == (0, 0, 1, 1, 2, 2) and cfg.bc.values[0] == 1.0
    hc = mf3d.HeadSolveConfig.from_yaml(cfg)
    assert hc.solver_type == mf3d.SOLVER_PCG_MG and hc.precision == mf3d.PREC_FP32
    assert hc.cg_check_every == 1


def test_flow_yaml_strict_keys(mf3d):
    with pytest.raises(mf3d.ConfigError, match="flow.bogus"):
        mf3d.load_flow_yaml("flow:\n  bogus: 1\n")
    with pytest.raises(mf3d.ConfigError, match="Periodic"):
        mf3d.load_flow_yaml("flow:\n  bc:\n    west: {type: periodic}\n")
    with pytest.raises(mf3d.ConfigError):
        mf3d.load_flow_yaml("flow:\n  solver: bicgstab\n")
    # defaults of FlowYamlConfig (Config.hpp:86-114)
    d = mf3d.load_flow_yaml("flow: {}\n")
    assert d.solver == "mg" and d.cg_max_iter == 1000 and d.bc.types == (0,) * 6


def test_solve_once_cli_parses_without_a_gpu():
    """The single-solve CLI used for kernel captures parses its options before any device work."""
    import subprocess
    import sys
    out = subprocess.run([sys.executable, "-m", "macroflow3d_b200.solve_once", "--help"], capture_output=True,
                         text=True, timeout=120, cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out.returncode == 0, out.stderr
    assert "--precision" in out.stdout and "--graph" in out.stdout


def test_oracle_kfield_generator_matches_the_product(mf3d, oracle_mod):
    """The oracle's host K generator (used where the product must not be loaded: the
    reference arm of the bench) draws bit-identical modes to the product's Philox sampler,
    and its run-wise evaluation equals the direct per-cell sum to rounding."""
    M, O = mf3d, oracle_mod
    for seed in (0, 20240601, 2 ** 40 + 3):
        for cov in (0, 1):
            for lam in ((4.0, 4.0, 4.0), (16.0, 16.0, 4.0)):
                assert np.array_equal(O.kfield_modes(seed, 300, cov, lam), M.kfield_modes(seed, 300, cov, lam))
    modes = O.kfield_modes(5, 200, 0, (4.0, 4.0, 4.0))
    shape = (12, 10, 37)  # nx = 37: a ragged last run of the 16-cell x runs
    direct = O.lnk_eval(shape, modes, 1.5)
    runs = O.generate_K(shape, 1.5 ** 2, (4.0, 4.0, 4.0), seed=5, n_modes=200, log_only=True)
    assert np.abs(runs - direct).max() / np.abs(direct).max() < 1e-12
    K = O.generate_K(shape, 1.5 ** 2, (4.0, 4.0, 4.0), seed=5, n_modes=200, K_geo=2.0)
    assert np.allclose(K, 2.0 * np.exp(runs), rtol=1e-14, atol=0)

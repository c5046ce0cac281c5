"""The C++ boundary (include/mf3d.hpp) compiled by a C++ caller, as a maintainer integrating
this library into the reference's C++ code would: HeadSolveConfig::from_yaml maps the
reference's FlowYamlConfig (src/physics/flow/solve_head.cuh:98-130), solve_head throws
std::runtime_error on failure, and a FlowWorkspace reused with other boundary conditions
solves the new problem (the reference takes the BCs on every call, solve_head.cuh:158-160)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def caller(mf3d, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "shim_caller")
    lib_dir = os.path.join(ROOT, "macroflow3d_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "shim_caller.cpp"), "-o", exe,
           "-L", lib_dir, "-lmf3d", f"-Wl,-rpath,{lib_dir}", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True)
    return exe


def _run(exe, mode):
    p = subprocess.run([exe, mode], capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout


def test_from_yaml_maps_the_reference_fields(caller):
    rc, out = _run(caller, "config")
    assert rc == 0, out
    first, second = out.strip().splitlines()
    # solver "mg_cg" -> PCG_MG (0); pin Off -> 2
    assert first.split() == ["0", "3", "1", "3", "40", "7", "200", "1", "1e-11", "1e-07", "2"]
    # "cg" -> CG (2), "mg" -> MG (1), unknown -> PCG_MG (0)
    assert second.split() == ["2", "1", "0"]


def test_solve_head_throws_without_a_device(caller):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the no-device error path cannot be reached")
    rc, out = _run(caller, "nogpu")
    assert rc == 0 and out.startswith("threw: mf3d:"), out


@pytest.mark.gpu
def test_workspace_follows_boundary_condition_changes(caller):
    rc, out = _run(caller, "solve")
    assert rc == 0, out
    lines = [ln.split() for ln in out.strip().splitlines()]
    assert len(lines) == 3
    west = [float(ln[7]) for ln in lines]
    err = [float(ln[9]) for ln in lines]
    builds = [int(ln[11]) for ln in lines]
    assert all(ln[3] == "1" for ln in lines), out
    # the exact linear head of each call's boundary values
    assert abs(west[0] - (1.0 - 0.5 / 32)) < 1e-9 and abs(west[1] - 2.0 * (1.0 - 0.5 / 32)) < 1e-9, out
    assert max(err) < 1e-9, out
    # a new solver for the new BCs, none for a repeated call
    assert builds == [1, 2, 2], out

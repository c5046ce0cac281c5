"""Replaying a stored K / h / velocity case on the GPU reproduces the stored head and velocities."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_save_and_replay(mf3d, tmp_path):
    from macroflow3d_b200 import replay as R
    stem = str(tmp_path / "c32")
    assert R.main(["save", stem, "--n", "32", "--sigma2", "1", "--lam", "4", "--seed", "3"]) == 0
    c = R.load_case(stem)
    assert c["meta"]["iterations"] > 0 and c["meta"]["true_rel_residual"] <= 1e-10
    assert c["h"].shape == (32, 32, 32) and c["U"].shape == (32, 32, 33)
    # the solver is deterministic: the replay gives the same bits
    out = R.solve_case(c)
    assert R.compare(c, out) == {"h": 0.0, "U": 0.0, "V": 0.0, "W": 0.0}
    assert R.main(["check", stem]) == 0
    # a stored head that is off by more than the tolerance fails the check
    c["h"][0, 0, 0] += 1.0
    R.save_case(stem, c["grid"], c["bc"], c["K"], c["h"], c["U"], c["V"], c["W"], c["meta"])
    assert R.main(["check", stem]) == 1

"""K / h / velocity case files (macroflow3d_b200.replay): round trip and header checks, no GPU."""
import json

import numpy as np
import pytest

import macroflow3d_b200 as M
from macroflow3d_b200 import replay as R


def _case(tmp_path, with_outputs=True):
    g = M.Grid3D(6, 5, 4, 0.5)
    bc = M.BCSpec([M.BCFace(M.DIRICHLET, 1.0), M.BCFace(M.DIRICHLET, 0.0), M.BCFace(M.PERIODIC, 0.0),
                   M.BCFace(M.PERIODIC, 0.0), M.BCFace(M.NEUMANN, 0.0), M.BCFace(M.NEUMANN, 0.0)])
    rng = np.random.default_rng(3)
    arrs = {"K": np.exp(rng.normal(size=(4, 5, 6)))}
    if with_outputs:
        arrs.update(h=rng.normal(size=4 * 5 * 6), U=rng.normal(size=(4, 5, 7)), V=rng.normal(size=(4, 6, 6)),
                    W=rng.normal(size=(5, 5, 6)))
    stem = str(tmp_path / "case")
    R.save_case(stem, g, bc, meta={"seed": 7}, **arrs)
    return stem, g, bc, arrs


def test_round_trip(tmp_path):
    stem, g, bc, arrs = _case(tmp_path)
    c = R.load_case(stem)
    assert (c["grid"].nx, c["grid"].ny, c["grid"].nz, c["grid"].dx) == (6, 5, 4, 0.5)
    assert c["bc"].types == bc.types and [f.value for f in c["bc"].faces] == [f.value for f in bc.faces]
    assert c["meta"] == {"seed": 7}
    for name, a in arrs.items():
        assert c[name].shape == R._shape(name, 6, 5, 4)
        assert np.array_equal(c[name].reshape(-1), np.asarray(a).reshape(-1))
    # raw little-endian FP64, arrays back to back in header order
    raw = np.fromfile(stem + ".f64", dtype="<f8")
    assert raw.size == sum(np.asarray(a).size for a in arrs.values())
    assert np.array_equal(raw[:120], arrs["K"].reshape(-1))
    assert R.compare(c, {"h": c["h"] * (1 + 1e-12)})["h"] < 2e-12


def test_inputs_only_and_json_suffix(tmp_path):
    stem, _, _, _ = _case(tmp_path, with_outputs=False)
    c = R.load_case(stem + ".json")
    assert set(k for k in c if k not in ("grid", "bc", "meta")) == {"K"}


def test_bad_inputs_are_rejected(tmp_path):
    g = M.Grid3D(4, 4, 4)
    with pytest.raises(R.CaseError):
        R.save_case(str(tmp_path / "x"), g, M.BCSpec.darcy_x(), np.ones(63))
    stem, _, _, _ = _case(tmp_path)
    head = json.load(open(stem + ".json"))
    head["arrays"][1]["shape"] = [4, 5, 7]
    json.dump(head, open(stem + ".json", "w"))
    with pytest.raises(R.CaseError):
        R.load_case(stem)
    stem2, _, _, _ = _case(tmp_path / "b")
    with open(stem2 + ".f64", "r+b") as f:
        f.truncate(100)
    with pytest.raises(R.CaseError):
        R.load_case(stem2)
    head = json.load(open(stem2 + ".json"))
    head["format"] = "other"
    json.dump(head, open(stem2 + ".json", "w"))
    with pytest.raises(R.CaseError):
        R.load_case(stem2)

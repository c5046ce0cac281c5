"""K / h / velocity case files: raw little-endian FP64 arrays plus a small JSON header.

A case holds the inputs of one head solve (grid, boundary conditions, K) and, optionally, its
outputs (head, face velocities) and free-form metadata (seed, statistics, solver settings).
It serves two uses: replaying a solve later, or on another machine, and comparing the head
with the stored one; and storing (K, h) pairs as training data for the learned initial guess.

Files: `<stem>.json` (header) and `<stem>.f64` (the arrays, concatenated in header order).
Header fields: "format" ("mf3d-case"), "version" (1), "grid" {nx, ny, nz, dx}, "bc" {"types":
six face codes 0 Dirichlet / 1 Neumann / 2 periodic in the order xmin, xmax, ymin, ymax, zmin,
zmax, "values": six floats}, "arrays": [{"name", "shape", "offset", "nbytes"}], "meta": {...}.
Cell arrays are stored in the reference's i + nx*(j + ny*k) order (numpy shape (nz, ny, nx));
U, V, W in the compact face layout ((nx+1) x ny x nz, nx x (ny+1) x nz, nx x ny x (nz+1)).

    python -m macroflow3d_b200.replay save STEM --n 64 --sigma2 1 --lam 4 [--seed S] [--precision fp64]
    python -m macroflow3d_b200.replay check STEM [--precision fp64]
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

import numpy as np

FORMAT, VERSION = "mf3d-case", 1
CELL_NAMES = ("K", "h")
FACE_NAMES = ("U", "V", "W")


class CaseError(ValueError):
    pass


def _shape(name: str, nx: int, ny: int, nz: int):
    if name in CELL_NAMES:
        return (nz, ny, nx)
    if name == "U":
        return (nz, ny, nx + 1)
    if name == "V":
        return (nz, ny + 1, nx)
    if name == "W":
        return (nz + 1, ny, nx)
    raise CaseError(f"unknown array {name!r}")


def _host(a) -> np.ndarray:
    if hasattr(a, "detach"):  # torch tensor, on any device
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def save_case(stem: str, grid, bc, K, h=None, U=None, V=None, W=None, meta: Optional[dict] = None) -> str:
    """Writes `<stem>.json` and `<stem>.f64`; returns the header path.  `grid` is a Grid3D,
    `bc` a BCSpec; arrays are numpy arrays or torch tensors of the shapes above (flat arrays of
    the right size are accepted)."""
    nx, ny, nz = int(grid.nx), int(grid.ny), int(grid.nz)
    arrays = []
    blobs = []
    off = 0
    for name, a in (("K", K), ("h", h), ("U", U), ("V", V), ("W", W)):
        if a is None:
            continue
        shp = _shape(name, nx, ny, nz)
        v = _host(a)
        if v.size != int(np.prod(shp)):
            raise CaseError(f"{name}: {v.size} values, expected {int(np.prod(shp))} for shape {shp}")
        b = v.reshape(shp).astype("<f8", copy=False).tobytes()
        arrays.append({"name": name, "shape": list(shp), "offset": off, "nbytes": len(b)})
        blobs.append(b)
        off += len(b)
    if not arrays or arrays[0]["name"] != "K":
        raise CaseError("a case needs K")
    head = {
        "format": FORMAT,
        "version": VERSION,
        "grid": {"nx": nx, "ny": ny, "nz": nz, "dx": float(grid.dx)},
        "bc": {"types": [int(f.type) for f in bc.faces], "values": [float(f.value) for f in bc.faces]},
        "arrays": arrays,
        "meta": meta or {},
    }
    d = os.path.dirname(os.path.abspath(stem))
    os.makedirs(d, exist_ok=True)
    with open(stem + ".f64", "wb") as f:
        for b in blobs:
            f.write(b)
    with open(stem + ".json", "w") as f:
        json.dump(head, f, indent=1)
    return stem + ".json"


def load_case(stem: str) -> Dict:
    """Reads a case: {"grid": Grid3D, "bc": BCSpec, "meta": dict, name: numpy array ...}.
    Raises CaseError on a header that does not describe the data file."""
    from . import BCFace, BCSpec, Grid3D
    if stem.endswith(".json"):
        stem = stem[:-5]
    with open(stem + ".json") as f:
        head = json.load(f)
    if head.get("format") != FORMAT or head.get("version") != VERSION:
        raise CaseError(f"not a {FORMAT} v{VERSION} header")
    g = head["grid"]
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    if min(nx, ny, nz) < 1:
        raise CaseError("grid dimensions must be positive")
    types, values = head["bc"]["types"], head["bc"]["values"]
    if len(types) != 6 or len(values) != 6:
        raise CaseError("six boundary faces expected")
    size = os.path.getsize(stem + ".f64")
    out = {
        "grid": Grid3D(nx, ny, nz, float(g["dx"])),
        "bc": BCSpec([BCFace(int(t), float(v)) for t, v in zip(types, values)]),
        "meta": head.get("meta", {}),
    }
    with open(stem + ".f64", "rb") as f:
        for a in head["arrays"]:
            shp = _shape(a["name"], nx, ny, nz)
            if list(shp) != list(a["shape"]) or a["nbytes"] != 8 * int(np.prod(shp)):
                raise CaseError(f"{a['name']}: header shape {a['shape']} / {a['nbytes']} B do not match the grid")
            if a["offset"] < 0 or a["offset"] + a["nbytes"] > size:
                raise CaseError(f"{a['name']}: bytes {a['offset']}..{a['offset'] + a['nbytes']} beyond the data file")
            f.seek(a["offset"])
            out[a["name"]] = np.frombuffer(f.read(a["nbytes"]), dtype="<f8").reshape(shp).copy()
    if "K" not in out:
        raise CaseError("a case needs K")
    return out


def solve_case(case: Dict, cfg=None, velocity: bool = True) -> Dict:
    """Solves a loaded case on the GPU with this library; returns {"h", "U", "V", "W", "result"}
    as numpy arrays (velocity only when `velocity`)."""
    import torch

    import macroflow3d_b200 as M
    g, bc = case["grid"], case["bc"]
    if cfg is None:
        cfg = M.HeadSolveConfig(mg_levels=8, cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B)
    K = torch.from_numpy(case["K"].reshape(-1)).cuda()
    h = torch.empty_like(K)
    s = M.HeadSolver(g, bc, cfg, stream=torch.cuda.current_stream().cuda_stream)
    try:
        s.set_K(K)
        res = s.solve(h)
    finally:
        s.close()
    out = {"h": h.cpu().numpy().reshape(g.nz, g.ny, g.nx), "result": res}
    if velocity:
        nu, nv, nw = M.velocity_sizes(g)
        U = torch.empty(nu, dtype=torch.float64, device="cuda")
        V = torch.empty(nv, dtype=torch.float64, device="cuda")
        W = torch.empty(nw, dtype=torch.float64, device="cuda")
        M.compute_velocity_from_head(U, V, W, h, K, g, bc)
        torch.cuda.synchronize()
        for name, t in (("U", U), ("V", V), ("W", W)):
            out[name] = t.cpu().numpy().reshape(_shape(name, g.nx, g.ny, g.nz))
    return out


def compare(case: Dict, solved: Dict) -> Dict:
    """Relative max-norm differences between the stored and the new head / velocities."""
    rep = {}
    for name in ("h",) + FACE_NAMES:
        if name in case and name in solved:
            ref = case[name]
            rep[name] = float(np.abs(solved[name] - ref).max() / max(np.abs(ref).max(), 1e-300))
    return rep


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("save", help="generate K, solve, store K / h / U / V / W")
    s.add_argument("stem")
    s.add_argument("--n", type=int, default=64)
    s.add_argument("--sigma2", type=float, default=1.0)
    s.add_argument("--lam", type=float, default=4.0)
    s.add_argument("--seed", type=int, default=0)
    s.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    c = sub.add_parser("check", help="solve a stored case again and compare")
    c.add_argument("stem")
    c.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    c.add_argument("--tol", type=float, default=1e-9)
    args = ap.parse_args(argv)
    import macroflow3d_b200 as M
    prec = {"fp64": M.PREC_FP64, "fp32": M.PREC_FP32}[args.precision]
    cfg = M.HeadSolveConfig(mg_levels=8, cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B, precision=prec)
    if args.cmd == "save":
        g = M.Grid3D(args.n, args.n, args.n, 1.0)
        K = M.generate_K_field(g, args.sigma2, (args.lam,) * 3, seed=args.seed)
        case = {"grid": g, "bc": M.BCSpec.darcy_x(), "K": K.cpu().numpy()}
        out = solve_case(case, cfg)
        r = out["result"]
        meta = {"generator": "randomization method, exponential covariance, 1000 modes", "sigma2": args.sigma2,
                "lambda": args.lam, "seed": args.seed, "precision": args.precision,
                "iterations": r.num_iterations, "true_rel_residual": r.true_rel_residual}
        path = save_case(args.stem, g, case["bc"], case["K"], out["h"], out["U"], out["V"], out["W"], meta)
        print(json.dumps({"saved": path, "iterations": r.num_iterations, "true_rel_residual": r.true_rel_residual}))
        return 0
    case = load_case(args.stem)
    out = solve_case(case, cfg)
    rep = compare(case, out)
    ok = all(v <= args.tol for v in rep.values()) and out["result"].converged
    print(json.dumps({"case": args.stem, "rel_diff": rep, "iterations": out["result"].num_iterations,
                      "converged": bool(out["result"].converged), "ok": ok}))
    return 0 if ok else 1


if __name__ == "__main__":
    raise SystemExit(main())

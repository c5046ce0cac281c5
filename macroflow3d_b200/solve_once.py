"""One head solve on a generated log-normal K field, with plain kernel launches by default
(no CUDA graph), for profiling a single PCG iteration's kernels:

    python -m macroflow3d_b200.solve_once [--n 256] [--sigma2 4] [--lam 8] [--precision fp32] [--graph]

Prints the iteration count, ||b - A h|| / ||b|| and whether the solve converged.
"""
from __future__ import annotations

import argparse


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--sigma2", type=float, default=4.0)
    ap.add_argument("--lam", type=float, default=8.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--graph", action="store_true", help="run the PCG loop as one CUDA graph")
    args = ap.parse_args()
    import torch
    import macroflow3d_b200 as M
    n = args.n
    g = M.Grid3D(n, n, n, 1.0)
    K = M.generate_K_field(g, args.sigma2, (args.lam, args.lam, args.lam), seed=args.seed)
    prec = {"fp64": M.PREC_FP64, "fp32": M.PREC_FP32, "bf16": M.PREC_BF16}[args.precision]
    cfg = M.HeadSolveConfig(mg_levels=8, cg_rtol=1e-10, cg_check_every=1, conv_norm=M.CONV_B,
                            precision=prec, use_graph=1 if args.graph else 0)
    s = M.HeadSolver(g, M.BCSpec.darcy_x(), cfg, stream=torch.cuda.current_stream().cuda_stream)
    s.set_K(K)
    h = torch.empty_like(K)
    r = s.solve(h)
    torch.cuda.synchronize()
    print(r.num_iterations, r.true_rel_residual, r.converged)
    s.close()


if __name__ == "__main__":
    main()

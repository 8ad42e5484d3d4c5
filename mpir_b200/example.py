"""The reference's example driver (examples/example.cpp) on the GPU solver.

    python -m mpir_b200.example <matrix_file_path> [--log]

Reads a Matrix Market file as the reference does (mpir_b200.mmio), solves
A x = b for b = A * ones with GMRES-IR (tolerance 1e-15, at most 200
refinement steps of at most 50 GMRES iterations; residual in double-double)
and prints the same lines: the symmetry, the factorization and solve times,
||x - xref|| / ||xref|| and ||b - Ax|| / ||b||.  With --log (the reference's
VERBOSE build) it writes <matrix>_<timestamp>.json beside the matrix: the
solver log (GmresLDLIR::DumpLog schema) plus matrix, precisions,
relative_error, relative_residual and ilu_k.

Differences from the reference driver: the factor type is float (the
reference's example uses double, which this library does not provide; its
float32 factor with float64 GMRES-IR reaches the same residual), and the
factor is a complete LDL^T instead of FGPILU (ILU_K is accepted and unused,
as in the drop-in GmresLDLIR).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import sys
import time

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("matrix_file_path")
    ap.add_argument("--log", action="store_true",
                    help="write the JSON log beside the matrix (the reference's VERBOSE build)")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    path = args.matrix_file_path
    if not os.path.exists(path):
        print(f"Error: Matrix file does not exist at {path!r}")
        return 1

    import mpir_b200 as mp
    from mpir_b200 import kkt
    from mpir_b200.mmio import read_matrix_market

    n, Ap, Ai, Ax, symmetry = read_matrix_market(path)
    print("symmetric" if symmetry == "symmetric" else "non symmetric")
    ilu_k = 0
    solver = mp.GmresLDLIR(uf="f32", uw="f64", ur="dd", device=args.device)
    solver.SetTolerance(1e-15)
    solver.SetMaxIRIterations(200)
    solver.SetMaxGmresIterations(50)
    t0 = time.perf_counter()
    solver.Compute(Ap, Ai, Ax, ilu_k)
    print(f"{'factorization time':<30}: {int(1e3 * (time.perf_counter() - t0))} ms")

    x_ref = np.ones(n)
    b = kkt.symmetric_matvec(n, Ap, Ai, Ax, x_ref)
    t0 = time.perf_counter()
    x = solver.Solve(b)
    print(f"{'solve time':<30}: {int(1e3 * (time.perf_counter() - t0))} ms")
    relative_error = float(np.max(np.abs(x - x_ref)) / np.max(np.abs(x_ref)))
    relative_residual = float(np.max(np.abs(b - kkt.symmetric_matvec(n, Ap, Ai, Ax, x)))
                              / np.max(np.abs(b)))
    print(f"{'||x - xref|| / ||xref||':<30}: {relative_error}")
    print(f"{'||b - Ax|| / ||b||':<30}: {relative_residual}")

    if args.log:
        log = solver.DumpLog()
        name = os.path.splitext(os.path.basename(path))[0]
        log["matrix"] = name
        log["factorization_precision"] = "single"
        log["working_precision"] = "double"
        log["residual_precision"] = "quadruple"
        log["relative_error"] = relative_error
        log["relative_residual"] = relative_residual
        log["ilu_k"] = ilu_k
        stamp = datetime.datetime.now().strftime("%Y-%m-%d-%H-%M-%S")
        out = os.path.join(os.path.dirname(os.path.abspath(path)), f"{name}_{stamp}.json")
        with open(out, "w") as f:
            f.write(json.dumps(log, indent=2) + "\n")
    solver.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

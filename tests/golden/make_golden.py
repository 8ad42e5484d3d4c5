"""Regenerate the golden fixtures from the reference's own code.

Runs the reference harness (oracle/_ref/libmpir_ref.so, built from the
reference headers by oracle/Makefile) on seeded synthetic systems and stores
its outputs:

  small2d_natural.npz   QDLDL_etree / QDLDL_factor<float> on the n = 1280
                        KKT system in natural order: etree, Lnz, D, Dinv,
                        sha256 of Li and of Lx, a slice of Lx
  small2d_gmres.npz     GmresLDLIR<float,double,double>::Solve preconditioned
                        by the QDLDL factor: x, AD, refinement steps
  small2d_solve.npz     QDLDL_solve<float,double> of b with that factor
  small2d_luir.npz      LUIR_QDLDL<float,double,double,double> (plain
                        iterative refinement, at most 10 steps): x, steps,
                        relative residual

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from mpir_b200 import kkt  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    R = oracle.Reference()
    s = kkt.small2d()
    tot, Lnz, et = R.etree(s.n, s.Ap, s.Ai)
    st, Lp, Li, Lx, D, Dinv = R.factor(s.n, s.Ap, s.Ai, s.Ax, np.float32)
    np.savez_compressed(os.path.join(HERE, "small2d_natural.npz"),
                        sumLnz=tot, Lnz=Lnz, etree=et, npos=st, Lp=Lp, D=D, Dinv=Dinv,
                        Li_sha=sha(Li), Lx_sha=sha(Lx), Lx_head=Lx[:4096])
    x = R.solve(s.n, Lp, Li, Lx, Dinv, s.b)
    np.savez_compressed(os.path.join(HERE, "small2d_solve.npz"), x=x)
    xg, AD, info = R.gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b)
    np.savez_compressed(os.path.join(HERE, "small2d_gmres.npz"), x=xg, AD=AD,
                        ir_steps=info["ir_steps"], npos=info["npos"])
    xl, li = R.luir(s.n, s.Ap, s.Ai, s.Ax, s.b, 10)
    np.savez_compressed(os.path.join(HERE, "small2d_luir.npz"), x=xl, steps=li["steps"],
                        relres=li["relres"])
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()

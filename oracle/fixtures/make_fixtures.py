"""Writes the inputs the reference arm of bench.py needs without the CUDA
library: the fill-reducing permutations of the benchmark systems and the
per-pattern symbolic facts of the serving stream.

The reference (MPIR) has no ordering of its own and factors in natural
order, which at the benchmark sizes does not fit in memory; both arms
therefore run on the permuted matrix P K P^T, with P from this library's
host analysis (mpir_b200 analyze_host).  Running this script needs the built
library; the bench's reference arm only reads its outputs:

  perm_small2d_s0.npy    perm[new] = old, int32, the n = 1,280 system
  perm_grid3d48_s0.npy   the same for the n = 138,240 system
  stream_facts.json      for each pattern of the default serving stream
                         (seed 0, its first 1,000 requests): n, nnz of the
                         upper triangle, nnz(L) and the multiply-subtract
                         count of QDLDL_factor, sum_j Lnz_j (Lnz_j - 1) / 2,
                         all from the etree of P K P^T (equal to
                         QDLDL_etree's, qdldl.hpp:48-105)

    python oracle/fixtures/make_fixtures.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    import mpir_b200 as mp
    from mpir_b200 import kkt, stream
    for name, s in (("small2d_s0", kkt.small2d(seed=0)), ("grid3d48_s0", kkt.grid3d(seed=0))):
        perm = mp.analyze_host(s.Ap, s.Ai, s.Ax)["perm"].astype(np.int32)
        np.save(os.path.join(HERE, f"perm_{name}.npy"), perm)
        print(name, s.n)
    st = stream.Stream(1000, rate=1e3, seed=0)
    facts = []
    for p in st.patterns:
        s = p.system()
        out = mp.analyze_host(s.Ap, s.Ai, s.Ax)
        lnz = out["Lnz"].astype(np.float64)
        facts.append({"pattern": p.pid, "n": int(s.n), "nnz_upper": int(s.nnz),
                      "nnz_L": int(lnz.sum()), "factor_updates": float((lnz * (lnz - 1) / 2).sum())})
        print(p.pid, s.n, facts[-1]["nnz_L"])
    with open(os.path.join(HERE, "stream_facts.json"), "w") as f:
        json.dump({"stream": {"seed": 0, "requests": 1000}, "patterns": facts}, f, indent=0)


if __name__ == "__main__":
    main()

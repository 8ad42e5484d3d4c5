"""Seeded request stream for the serving benchmark and tests.

The workload: requests with Poisson arrivals, each a quasi-definite KKT system
K = [[H, A^T], [A, -delta I]] from the 2-D (5-point Laplacian, 4 entries per
constraint row) or 3-D (7-point Laplacian, 6 entries per row) generator of
:mod:`mpir_b200.kkt`, total size n log-uniform in [1e3, 5e5] and m ~ n1 / 4
constraint rows, and a right-hand side b = K x_true with x_true ~ U(-1, 1).
The kinds, in the proportions 60 / 30 / 10:

* ``rhs``     a new right-hand side on a factor used before (one of the most
  recently used ones);
* ``values``  new values on a pattern used before (one of the most recently
  used patterns): H gets a new diagonal shift and the constraint block new
  N(0,1) values, so the pattern is unchanged and K stays quasi-definite;
* ``pattern`` a new system with a new size.

The first request is always a new pattern.  Every request carries the keys
that name its pattern and its values (equal keys, equal arrays), as the
serving engine expects.  Systems are built lazily and cached, so a stream of
a few hundred requests touches a few dozen systems.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import kkt


@dataclass
class StreamRequest:
    index: int
    kind: str            # "rhs", "values" or "pattern"
    pattern: int         # pattern id
    values: int          # values id on that pattern (0 = the generator's own)
    rhs_seed: int
    t_arrival: float     # seconds from the start of the stream

    @property
    def pattern_key(self) -> int:
        return self.pattern + 1

    @property
    def values_key(self) -> int:
        return (self.pattern + 1) * 1_000_003 + self.values


@dataclass
class Pattern:
    pid: int
    n_target: int
    dim: int
    seed: int
    base: kkt.KKT | None = None
    values: dict = field(default_factory=dict)

    def system(self) -> kkt.KKT:
        if self.base is None:
            n1 = self.n_target / 1.25
            grid = max(4, int(round(n1 ** (1.0 / self.dim))))
            m = max(1, grid ** self.dim // 4)
            per_row = 6 if self.dim == 3 else 4
            self.base = kkt.make(grid, self.dim, m, per_row, 1e-6 if self.dim == 3 else 1e-4,
                                 shift=1e-2, seed=self.seed)
        return self.base

    def Ax(self, v: int) -> np.ndarray:
        """Values set v on the pattern (v = 0: the generator's values)."""
        s = self.system()
        if v == 0:
            return s.Ax
        if v not in self.values:
            rng = np.random.default_rng((self.seed, v))
            Ax = s.Ax.copy()
            cols = np.repeat(np.arange(s.n, dtype=np.int64), np.diff(s.Ap))
            diag_h = (s.Ai == cols) & (cols < s.n1)
            Ax[diag_h] += rng.uniform(0.0, 0.1)             # H + c I, c >= 0
            cons = (cols >= s.n1) & (s.Ai < s.n1)            # A^T block
            Ax[cons] = rng.standard_normal(int(cons.sum()))
            self.values[v] = Ax
        return self.values[v]

    def rhs(self, v: int, seed: int):
        """(b, x_true) for values set v."""
        s = self.system()
        x_true = np.random.default_rng((self.seed, v, seed)).uniform(-1.0, 1.0, size=s.n)
        return kkt.symmetric_matvec(s.n, s.Ap, s.Ai, self.Ax(v), x_true), x_true


class Stream:
    """``nreq`` requests at Poisson rate ``rate`` (requests per second)."""

    def __init__(self, nreq: int, rate: float, seed: int = 0, n_range=(1e3, 5e5),
                 mix=(0.6, 0.3, 0.1), recent: int = 8):
        rng = np.random.default_rng(seed)
        self.patterns: list[Pattern] = []
        self.requests: list[StreamRequest] = []
        factors: list[tuple[int, int]] = []   # (pattern, values) in order of last use
        used_patterns: list[int] = []
        next_values: dict[int, int] = {}
        t = 0.0
        lo, hi = math.log(n_range[0]), math.log(n_range[1])
        for i in range(nreq):
            t += rng.exponential(1.0 / rate)
            u = rng.uniform()
            kind = ("rhs" if u < mix[0] else "values" if u < mix[0] + mix[1] else "pattern")
            if not factors:
                kind = "pattern"
            if kind == "pattern":
                pid = len(self.patterns)
                self.patterns.append(Pattern(pid, int(round(math.exp(rng.uniform(lo, hi)))),
                                             2 if rng.uniform() < 0.5 else 3,
                                             int(rng.integers(1 << 31))))
                vid = 0
                next_values[pid] = 1
            elif kind == "values":
                pool = used_patterns[-recent:]
                pid = pool[int(rng.integers(len(pool)))]
                vid = next_values[pid]
                next_values[pid] += 1
            else:
                pool = factors[-recent:]
                pid, vid = pool[int(rng.integers(len(pool)))]
            self.requests.append(StreamRequest(i, kind, pid, vid, int(rng.integers(1 << 31)), t))
            if (pid, vid) in factors:
                factors.remove((pid, vid))
            factors.append((pid, vid))
            if pid in used_patterns:
                used_patterns.remove(pid)
            used_patterns.append(pid)

    def materialise(self, req: StreamRequest):
        """(system, Ax, b, x_true) of one request."""
        p = self.patterns[req.pattern]
        s = p.system()
        b, x_true = p.rhs(req.values, req.rhs_seed)
        return s, p.Ax(req.values), b, x_true

    def retime(self, rate: float, seed: int = 1):
        """The same requests with new Poisson arrival times at ``rate``."""
        rng = np.random.default_rng(seed)
        t = 0.0
        for r in self.requests:
            t += rng.exponential(1.0 / rate)
            r.t_arrival = t
        return self

"""The serving engine on the GPU (through the C ABI).

* Each result in a mixed stream equals the same request solved alone (a
  fresh GmresLDLIR: analysis, factor and GMRES-IR solve): backward error
  <= 1e-14, forward error within 10x of the solo solve's, and the two
  solutions within 20x of the solo forward error.
* Requests on one factor queued together are solved in lockstep batches.
* Admission: a factor larger than the budget is refused with status -4
  (MPIR_ERR_NOMEM); a budget that holds only a few factors evicts (with
  nothing queued behind a request: the least recently used first) and still
  answers every request correctly."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt, stream

pytestmark = pytest.mark.gpu


def _solo(s, Ax, b):
    g = mp.GmresLDLIR()
    g.Compute(s.Ap, s.Ai, Ax)
    x = g.Solve(b)
    g.close()
    return x


def test_mixed_stream_matches_solo_solves():
    st = stream.Stream(48, rate=1e4, seed=11, n_range=(1e3, 2e4))
    srv = mp.Server(workers=4, max_batch=16)
    ids = []
    for r in st.requests:
        s, Ax, b, xt = st.materialise(r)
        ids.append((r, srv.submit(r.pattern_key, r.values_key, s.Ap, s.Ai, Ax, b)))
    paths = set()
    for r, rid in ids:
        x, res = srv.wait(rid)
        assert res["status"] == 0, res
        paths.add(res["path"])
        s, Ax, b, xt = st.materialise(r)
        be = kkt.backward_error(s.n, s.Ap, s.Ai, Ax, x, b)
        assert be <= 1e-14, (r, be)
        xs = _solo(s, Ax, b)
        fe_s = kkt.forward_error(xs, xt)
        assert kkt.forward_error(x, xt) <= max(10 * fe_s, 1e-12)
        assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) <= max(20 * fe_s, 1e-12)
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == len(st.requests) and stats["failed"] == 0
    assert paths == {0, 1, 2}  # resident factors, refactorizations, new patterns


def test_queued_requests_on_one_factor_are_batched():
    s = kkt.small2d(seed=4)
    srv = mp.Server(workers=1, max_batch=16)
    rng = np.random.default_rng(0)
    xts = rng.uniform(-1, 1, size=(20, s.n))
    ids = [srv.submit(1, 1, s.Ap, s.Ai, s.Ax, kkt.symmetric_matvec(s.n, s.Ap, s.Ai, s.Ax, xt))
           for xt in xts]
    batches = []
    for rid, xt in zip(ids, xts):
        x, res = srv.wait(rid)
        assert res["status"] == 0
        batches.append(res["batch"])
        b = kkt.symmetric_matvec(s.n, s.Ap, s.Ai, s.Ax, xt)
        assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, b) <= 1e-14
    stats = srv.stats()
    srv.close()
    assert max(batches) > 1 and stats["batched_rhs"] >= 2


def test_admission_refuses_and_evicts():
    s = kkt.grid3d(grid=10, seed=2)
    srv = mp.Server(workers=1, budget_bytes=1 << 20)
    x, res = srv.wait(srv.submit(7, 7, s.Ap, s.Ai, s.Ax, s.b))
    assert res["status"] == -4
    assert srv.stats()["refused"] == 1
    srv.close()
    # room for about two factors of this size: the third evicts the oldest
    probe = mp.Server(workers=1)
    probe.wait(probe.submit(1, 1, s.Ap, s.Ai, s.Ax, s.b))
    one = probe.stats()["bytes_in_use"]
    probe.close()
    srv = mp.Server(workers=1, budget_bytes=int(2.5 * one))
    systems = [kkt.grid3d(grid=10, seed=q) for q in range(4)]
    for rounds in range(2):
        for q, sq in enumerate(systems):
            x, res = srv.wait(srv.submit(100 + q, 100 + q, sq.Ap, sq.Ai, sq.Ax, sq.b))
            assert res["status"] == 0, res
            assert kkt.backward_error(sq.n, sq.Ap, sq.Ai, sq.Ax, x, sq.b) <= 1e-14
    stats = srv.stats()
    srv.close()
    assert stats["evictions"] >= 2
    assert stats["peak_bytes"] <= int(2.5 * one)

"""Replay a request stream against the serving engine or the drop-in solver.

``served``  submits every request at its arrival time (a submitter thread
            sleeps until then) to one :class:`mpir_b200.Server` and collects
            each result; latency is submit-to-result on the host clock.
``dropin``  serves the same requests one at a time as the reference's
            usage does (examples/example.cpp: a GmresLDLIR per system,
            Compute then Solve, nothing kept between requests) and measures
            each request's service time; latencies under the same arrivals
            follow from the first-come-first-served queue
            (done_i = max(arrival_i, done_{i-1}) + service_i).

Both return per-request records and the stream's solves/s (requests that
finished with status 0 over the time from the first arrival to the last
completion).
"""
from __future__ import annotations

import threading
import time

import numpy as np

from . import kkt


def materialise(stream):
    """The arrays of every request (built once, outside any timing)."""
    return [stream.materialise(r) for r in stream.requests]


def _summary(records, t_total):
    ok = [r for r in records if r["status"] == 0]
    lat = np.array([r["latency_ms"] for r in ok]) if ok else np.zeros(1)
    return {"solves_per_s": len(ok) / t_total if t_total > 0 else float("nan"),
            "completed": len(ok), "failed": len(records) - len(ok), "seconds": t_total,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "backward_error_max": max((r.get("backward_error", float("nan")) for r in ok),
                                      default=float("nan")),
            "forward_error_max": max((r.get("forward_error", float("nan")) for r in ok),
                                     default=float("nan"))}


def served(stream, arrays, check=True, progress=None, **server_kwargs):
    """(summary, records, server stats).  The errors of each result are
    computed after the last one arrived (outside the timed span);
    ``progress`` (seconds) prints the engine's counters to stderr that
    often while the stream runs."""
    import sys

    import mpir_b200 as mp
    srv = mp.Server(**server_kwargs)
    reqs = stream.requests
    ids = [None] * len(reqs)
    ready = threading.Event()

    def submitter(t0):
        for i, r in enumerate(reqs):
            delay = t0 + r.t_arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            s, Ax, b, _ = arrays[i]
            ids[i] = srv.submit(r.pattern_key, r.values_key, s.Ap, s.Ai, Ax, b)
            if i == 0:
                ready.set()

    finished = threading.Event()

    def reporter(t0):
        while not finished.wait(progress):
            c = srv.stats()
            print(f"[served] {time.perf_counter() - t0:7.1f}s completed {c['completed']}"
                  f"/{len(reqs)} failed {c['failed']} queued {c['queued']} factors "
                  f"{c['resident_factors']} in use {c['bytes_in_use'] / 1e9:.1f} GB "
                  f"evictions {c['evictions']}", file=sys.stderr, flush=True)

    t0 = time.perf_counter()
    th = threading.Thread(target=submitter, args=(t0,), daemon=True)
    th.start()
    if progress:
        threading.Thread(target=reporter, args=(t0,), daemon=True).start()
    results = []
    t_last = t0
    for i in range(len(reqs)):
        while ids[i] is None:
            time.sleep(0.0002)
        results.append(srv.wait(ids[i]))
        t_last = max(t_last, time.perf_counter())
    finished.set()
    th.join()
    stats = srv.stats()
    srv.close()
    records = []
    for i, (r, (x, res)) in enumerate(zip(reqs, results)):
        rec = {"index": i, "kind": r.kind, "status": res["status"], "path": res["path"],
               "batch": res["batch"], "latency_ms": res["latency_ms"],
               "queue_ms": res["queue_ms"], "n": arrays[i][0].n,
               "ir": res["report"]["ir_iterations"], "gmres": res["report"]["gmres_iterations"],
               "message": res["message"]}
        if check and res["status"] == 0:
            s, Ax, b, xt = arrays[i]
            rec["backward_error"] = kkt.backward_error(s.n, s.Ap, s.Ai, Ax, x, b)
            rec["forward_error"] = kkt.forward_error(x, xt)
        records.append(rec)
    t_first = t0 + reqs[0].t_arrival
    return _summary(records, t_last - t_first), records, stats


def dropin(stream, arrays, uf="f32", ir_iter=10, gmres_iter=10, tol=1e-10, check=True,
           progress=None):
    """(summary, records): one request at a time, nothing kept between them;
    ``progress`` (seconds) prints the count done to stderr about that often."""
    import sys

    import mpir_b200 as mp
    records = []
    done_prev = 0.0
    busy = 0.0
    t_print = time.perf_counter()
    for i, r in enumerate(stream.requests):
        if progress and time.perf_counter() - t_print >= progress:
            t_print = time.perf_counter()
            print(f"[drop-in] {i}/{len(stream.requests)} requests, {busy:.1f}s of service",
                  file=sys.stderr, flush=True)
        s, Ax, b, xt = arrays[i]
        t0 = time.perf_counter()
        status = 0
        msg = ""
        try:
            g = mp.GmresLDLIR(uf=uf)
            g.SetMaxIRIterations(ir_iter)
            g.SetMaxGmresIterations(gmres_iter)
            g.SetTolerance(tol)
            g.Compute(s.Ap, s.Ai, Ax)
            x = g.Solve(b)
            rep = g.last_report
            g.close()
        except mp.MpirError as e:
            status, msg, x, rep = e.code, str(e), None, {}
        service = time.perf_counter() - t0
        busy += service
        start = max(r.t_arrival, done_prev)
        done_prev = start + service
        rec = {"index": i, "kind": r.kind, "status": status, "n": s.n,
               "service_ms": 1e3 * service, "latency_ms": 1e3 * (done_prev - r.t_arrival),
               "ir": rep.get("ir_iterations"), "gmres": rep.get("gmres_iterations"),
               "message": msg}
        if check and status == 0:
            rec["backward_error"] = kkt.backward_error(s.n, s.Ap, s.Ai, Ax, x, b)
            rec["forward_error"] = kkt.forward_error(x, xt)
        records.append(rec)
    t_total = done_prev - stream.requests[0].t_arrival
    return _summary(records, t_total), records

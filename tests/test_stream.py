"""The serving workload generator (host only): seeded and reproducible, the
60/30/10 mix, the size range, and keys that name equal arrays."""
import numpy as np

from mpir_b200 import stream


def test_stream_is_seeded_and_mixed():
    a = stream.Stream(400, rate=100.0, seed=3, n_range=(1e3, 2e4))
    b = stream.Stream(400, rate=100.0, seed=3, n_range=(1e3, 2e4))
    assert [(r.kind, r.pattern, r.values, r.rhs_seed) for r in a.requests] == \
           [(r.kind, r.pattern, r.values, r.rhs_seed) for r in b.requests]
    kinds = [r.kind for r in a.requests]
    assert kinds[0] == "pattern"
    frac = {k: kinds.count(k) / len(kinds) for k in ("rhs", "values", "pattern")}
    assert abs(frac["rhs"] - 0.6) < 0.08 and abs(frac["values"] - 0.3) < 0.08
    assert abs(frac["pattern"] - 0.1) < 0.05
    t = np.array([r.t_arrival for r in a.requests])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert 0.7 / 100 < gaps.mean() < 1.3 / 100


def test_stream_keys_and_systems():
    st = stream.Stream(60, rate=50.0, seed=5, n_range=(1e3, 5e3))
    seen = {}
    for r in st.requests[:30]:
        s, Ax, b, xt = st.materialise(r)
        assert 800 <= s.n <= 6500
        key = (r.pattern_key, r.values_key)
        if key in seen:
            np.testing.assert_array_equal(seen[key], Ax)
        seen[key] = Ax
        # b = K x_true for these values
        from mpir_b200 import kkt
        np.testing.assert_allclose(kkt.symmetric_matvec(s.n, s.Ap, s.Ai, Ax, xt), b, rtol=0,
                                   atol=1e-12 * np.abs(b).max())
    # a values request keeps the pattern, changes the values
    for r in st.requests:
        if r.kind == "values":
            p = st.patterns[r.pattern]
            assert not np.array_equal(p.Ax(r.values), p.Ax(0))
            break

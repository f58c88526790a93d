"""The serving workload's request stream (host logic, no GPU)."""
import numpy as np

from hmglib_b200 import serve


def test_poisson_mix_is_seeded_and_shaped():
    sizes = [1000, 2000, 3000]
    a = serve.poisson_requests(400, 2000.0, sizes, seed=4)
    b = serve.poisson_requests(400, 2000.0, sizes, seed=4)
    assert [type(q) for q in a] == [type(q) for q in b]
    assert all(np.array_equal(getattr(p, "x", 0), getattr(q, "x", 0)) for p, q in zip(a, b))
    t = np.array([q.arrival for q in a])
    assert (np.diff(t) > 0).all()
    # mean inter-arrival ~ 1/rate
    assert abs(t[-1] / len(t) - 1 / 2000.0) < 0.15 / 2000.0
    kinds = np.array([0 if isinstance(q, serve.Matvec) else 1 if isinstance(q, serve.Solve) else 2 for q in a])
    frac = np.bincount(kinds, minlength=3) / len(a)
    assert abs(frac[0] - 0.80) < 0.06 and abs(frac[1] - 0.15) < 0.05 and abs(frac[2] - 0.05) < 0.04
    for q in a:
        if isinstance(q, serve.Matvec):
            assert q.x.shape == (sizes[q.mid],) and np.abs(q.x).max() <= 1
        elif isinstance(q, serve.Solve):
            assert q.B.shape == (8, sizes[q.mid]) and q.shift > 0
        else:
            assert q.points.shape[0] == 3 and 2 ** 14 - 1 <= q.points.shape[1] <= 2 ** 18 + 1


def test_admission_against_latency_targets():
    # outstanding work: per H-matrix (queued + running batches) x batch time + solve
    # iterations left x iteration time, summed over the H-matrices sharing the GPU
    w = serve.outstanding_seconds([2, 0], [1, 1], [10.0, 0.0], [0.1, 0.2], [0.01, 0.5])
    assert abs(w[0] - (3 * 0.1 + 10 * 0.01)) < 1e-12 and abs(w[1] - 0.2) < 1e-12
    # own stream in order (A = 0.3 + 0.1); others interleave: at most their work, at
    # most (busy - 1) x A
    assert abs(serve.predict_latency(0.3, 0.1, 5.0, 3) - (0.4 + 0.8)) < 1e-12
    assert abs(serve.predict_latency(0.3, 0.1, 0.2, 3) - (0.4 + 0.2)) < 1e-12
    assert abs(serve.predict_latency(0.0, 0.1, 9.0, 1) - 0.1) < 1e-12
    assert serve.admit(0.9, 1.0) and not serve.admit(1.1, 1.0) and serve.admit(1e9, None)
    assert serve.ewma(0.0, 2.0) == 2.0 and abs(serve.ewma(1.0, 2.0, 0.25) - 1.25) < 1e-12


def test_latency_summary_counts_refused_apart():
    a = serve.Matvec(0, np.zeros(3), arrival=0.0)
    a.done = 0.5
    b = serve.Matvec(0, np.zeros(3), arrival=0.1)
    b.done, b.rejected = 0.1, "predicted 2.00 s > matvec target 1.00 s"
    c = serve.Solve(0, np.zeros((2, 3)), 1.0, arrival=0.0)
    c.done = 2.0
    lat = serve.latency_summary([a, b, c])
    assert lat["matvec"]["count"] == 1 and lat["matvec"]["refused"] == 1
    assert abs(lat["matvec"]["p99_ms"] - 500.0) < 1e-9
    assert lat["all"]["count"] == 2 and lat["all"]["refused"] == 1 and lat["solve"]["refused"] == 0

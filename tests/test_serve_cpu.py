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

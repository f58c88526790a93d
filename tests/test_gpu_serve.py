"""The serving loop (hmglib_b200.serve): every request's result in a mixed stream of
products, solves and constructions equals the same request served alone.  No
reference counterpart.

Tolerances: products 1e-6 relative (a product batched with others runs the
multi-vector kernels, alone the single-vector ones: FP32 sums in another order);
solves 1e-4 relative in X (both runs stop at relative residual 1e-6 on an operator
with condition number ~1e2)."""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _resident(hmg, serve, torch, sizes, precs):
    out = []
    for i, (n, prec) in enumerate(zip(sizes, precs)):
        st = torch.cuda.Stream()
        p = hmg.synth.uniform_points(n, 3, 40 + i)
        H = serve.build_hmatrix(p, hmg.KERNEL_MATERN32, 0.2, 1e-6, prec, stream=st.cuda_stream)
        out.append((H, st))
    return out


def test_mixed_stream_matches_alone(hmg, cuda):
    torch = cuda
    from hmglib_b200 import serve, synth
    hmg.synth = synth
    sizes = [4000, 6000]
    res = _resident(hmg, serve, torch, sizes, [hmg.PREC_FP32, hmg.PREC_MIXED])
    srv = serve.Server(budget_bytes=16e9)
    for H, st in res:
        srv.add(H, st)
    reqs = serve.poisson_requests(60, 2000.0, sizes, seed=4, mix=(0.72, 0.2, 0.08), solve_rhs=3,
                                  build_lo=12.0, build_hi=12.5, eps=1e-5, shift_per_point=1e-2, tol=1e-6)
    done, wall = srv.run(reqs, time_limit=300.0)
    assert all(q.done is not None for q in done)
    lat = serve.latency_summary(done)
    assert lat["all"]["count"] + lat["all"]["refused"] == len(reqs)
    assert lat["all"]["p99_ms"] >= lat["all"]["p50_ms"] > 0
    batched = 0
    for q in done:
        if isinstance(q, serve.Matvec):
            alone = res[q.mid][0].matvec(q.x)
            assert rel_err(q.y, alone) < 1e-6, (q.mid, q.batch, rel_err(q.y, alone))
            batched += q.batch > 1
        elif isinstance(q, serve.Solve):
            solo = serve.Server(budget_bytes=16e9)
            for H, st in res:
                solo.add(H, st)
            q2 = serve.Solve(q.mid, q.B, q.shift, tol=q.tol)
            solo.run([q2])
            assert (q.relres <= q.tol).all() and (q2.relres <= q.tol).all()
            assert rel_err(q.X.ravel(), q2.X.ravel()) < 1e-4
            # the residual against the operator, recomputed column by column
            H = res[q.mid][0]
            for j in range(q.B.shape[0]):
                r = q.B[j] - (H.matvec(q.X[j]) + q.shift * q.X[j])
                assert np.linalg.norm(r) <= 1e-4 * np.linalg.norm(q.B[j])
        else:
            assert q.rejected is None and q.mid is not None
            if q.mid in srv.res:  # still resident: usable
                assert np.isfinite(srv.res[q.mid].H.matvec(np.ones(q.points.shape[1]))).all()
    assert batched > 0  # at 2000 requests/s some products shared a pass
    assert srv.used_bytes() <= srv.budget
    for mid in list(srv.res):
        srv.res.pop(mid).H.close()


def test_latency_targets_refuse_on_arrival(hmg, cuda):
    """With a latency target of a few batch times, products arriving behind a backlog
    are refused at once (no result) while the admitted ones still equal their products
    served alone."""
    torch = cuda
    from hmglib_b200 import serve, synth
    hmg.synth = synth
    sizes = [6000]
    res = _resident(hmg, serve, torch, sizes, [hmg.PREC_FP32])
    # a target of 2.5 batch times (the seed estimate): the first products are admitted,
    # those that arrive behind a batch in flight and a queued one are refused
    target = 2.5 * serve.resident_bytes(res[0][0]) / serve.HBM_BYTES_PER_S
    srv = serve.Server(budget_bytes=16e9, slo_s={"matvec": target})
    for H, st in res:
        srv.add(H, st)
    reqs = serve.poisson_requests(40, 1e5, sizes, seed=6, mix=(1.0, 0.0, 0.0))
    done, _ = srv.run(reqs, time_limit=120.0)
    refused = [q for q in done if q.rejected is not None]
    served = [q for q in done if q.rejected is None]
    assert refused and served and all(q.y is None for q in refused)
    for q in served:
        assert rel_err(q.y, res[0][0].matvec(q.x)) < 1e-6
    for H, _ in res:
        H.close()

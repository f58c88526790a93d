"""Products replayed as CUDA graphs (hmg_set_graphs): bit-identical to direct launches,
captured anew whenever the arguments or the handle change.  No reference counterpart."""
import numpy as np
import pytest

from helpers import engine, make_points

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1, 2], ids=["fp64", "fp32", "mixed"])
def test_graph_replay_matches_direct(hmg, cuda, prec):
    torch = cuda
    n = 20000
    p = make_points("uniform", n, 3, 31)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(64, 1e-8, prec)
    H.precompute_dense(hmg.PREC_FP64 if prec == 0 else hmg.PREC_FP32)
    rng = np.random.default_rng(7)
    xs = [rng.uniform(-1, 1, n) for _ in range(3)]
    direct = [H.matvec(x) for x in xs]
    H.set_graphs(True)
    for _ in range(2):  # capture, then replay
        for x, y in zip(xs, direct):
            np.testing.assert_array_equal(H.matvec(x), y)
    # device tensors (other x / y pointers) and a change of product arithmetic
    X = torch.from_numpy(xs[0]).cuda()
    Y = torch.empty_like(X)
    for _ in range(2):
        H.matvec(X, Y)
        H.synchronize()
        np.testing.assert_array_equal(Y.cpu().numpy(), direct[0])
    if prec != 0:
        H.set_product_precision(hmg.PREC_FP64)
        y64 = H.matvec(xs[1])
        H.set_graphs(False)
        np.testing.assert_array_equal(H.matvec(xs[1]), y64)
        H.set_graphs(True)
        H.set_product_precision(hmg.PREC_FP32)
    # new kernel parameter and storage: the graph follows
    H.set_kernel(hmg.KERNEL_MATERN32, 0.3, 0.0)
    H.precompute_aca(64, 1e-8, prec)
    H.precompute_dense(hmg.PREC_FP64 if prec == 0 else hmg.PREC_FP32)
    yg = H.matvec(xs[2])
    H.set_graphs(False)
    np.testing.assert_array_equal(H.matvec(xs[2]), yg)
    assert not np.array_equal(yg, direct[2])
    H.close()

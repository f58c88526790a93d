"""Tensor-core multi-vector products (hmg_build_bf16_factors + hmg_matvec_multi): the
low-rank part on tcgen05 with BF16 operands agrees with the FP32 CUDA-core product to
the BF16 rounding of the factors and of t_b (relative 5e-3 per vector), is
deterministic, and leaves single-vector products on the FP32 factors unchanged.  No
reference counterpart."""
import numpy as np
import pytest

from helpers import engine, make_points, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [("uniform", 20000, 3, 128, 4, 0.2), ("gmm", 30000, 2, 64, 3, 0.05)],
                         ids=["uniform3d-matern", "gmm2d-gauss"])
def test_tensor_core_products(hmg, cuda, case):
    torch = cuda
    gen, n, dim, leaf, kind, param = case
    p = make_points(gen, n, dim, 13)
    H = engine(hmg, p, p, 1.5, leaf, rule=1)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (12, n))).cuda()
    Y32 = torch.empty_like(X)
    H.matvec_multi(X, Y32)
    y1 = H.matvec(X[0].cpu().numpy())
    H.build_bf16_factors()
    Ytc = torch.full_like(X, float("nan"))
    H.matvec_multi(X, Ytc)
    H.synchronize()
    a, b = Ytc.cpu().numpy(), Y32.cpu().numpy()
    assert np.isfinite(a).all()
    for j in range(X.shape[0]):
        assert rel_err(a[j], b[j]) < 5e-3, (j, rel_err(a[j], b[j]))
    Y2 = torch.empty_like(X)
    H.matvec_multi(X, Y2)
    H.synchronize()
    np.testing.assert_array_equal(Y2.cpu().numpy(), a)
    np.testing.assert_array_equal(H.matvec(X[0].cpu().numpy()), y1)
    H.close()

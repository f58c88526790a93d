"""Tensor-core multi-vector products (hmg_build_bf16_factors + hmg_matvec_multi): every
product (V^T X, U t_b and the near field times X) on tcgen05 with BF16 operands agrees
with the FP32 CUDA-core product to the BF16 rounding of factors, near field, X and t_b
(2^-8 = 3.9e-3 per entry; typically 3e-3 per vector, bound 1e-2 over up to 64 vectors),
is deterministic, writes every row of Y, and leaves
single-vector products on the FP32 storage unchanged.  No reference counterpart."""
import numpy as np
import pytest

from helpers import engine, make_points, rel_err

pytestmark = pytest.mark.gpu

MATERN, GAUSS = 4, 3


@pytest.mark.parametrize("case", [
    ("uniform", 20000, 3, 128, MATERN, 0.2, 64, 1e-6, 12),
    ("gmm", 30000, 2, 64, GAUSS, 0.05, 64, 1e-6, 12),
    # ranks up to 128 (two K chunks per low-rank pair) and tiles of at most 32 rows
    ("uniform", 12000, 3, 32, MATERN, 0.2, 128, 1e-10, 32),
    ("uniform", 9000, 2, 128, GAUSS, 0.1, 64, 1e-6, 2),
    # 33..64 vectors: MMAs of N = 64
    ("uniform", 20000, 3, 128, MATERN, 0.2, 64, 1e-6, 64),
    ("gmm", 30000, 2, 64, GAUSS, 0.05, 64, 1e-6, 41),
], ids=["uniform3d-matern", "gmm2d-gauss", "rank128-leaf32", "two-vectors", "64-vectors", "41-vectors"])
def test_tensor_core_products(hmg, cuda, case):
    torch = cuda
    gen, n, dim, leaf, kind, param, kmax, eps, nrhs = case
    p = make_points(gen, n, dim, 13)
    H = engine(hmg, p, p, 1.5, leaf, rule=1)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(kmax, eps, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (nrhs, n))).cuda()
    Y32 = torch.empty_like(X)
    H.matvec_multi(X, Y32)
    y1 = H.matvec(X[0].cpu().numpy())
    H.build_bf16_factors()
    Ytc = torch.full_like(X, float("nan"))
    H.matvec_multi(X, Ytc)
    H.synchronize()
    a, b = Ytc.cpu().numpy(), Y32.cpu().numpy()
    assert np.isfinite(a).all()
    for j in range(nrhs):
        assert rel_err(a[j], b[j]) < 1e-2, (j, rel_err(a[j], b[j]))
    Y2 = torch.empty_like(X)
    H.matvec_multi(X, Y2)
    H.synchronize()
    np.testing.assert_array_equal(Y2.cpu().numpy(), a)
    np.testing.assert_array_equal(H.matvec(X[0].cpu().numpy()), y1)
    if kmax == 128:
        assert H.info()["max_rank"] > 96  # the two-chunk path ran
    H.close()


def test_fp32_near_field_on_cuda_cores(hmg, cuda):
    """near=PREC_FP32: only the low-rank part on the tensor cores; the near field stays
    FP32 on the CUDA cores and the low-rank sums are added to it.  Closer to the FP32
    product than the all-BF16 variant, within the same 5e-3."""
    torch = cuda
    p = make_points("uniform", 20000, 3, 21)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(MATERN, 0.2, 0.0)
    H.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (16, 20000))).cuda()
    Y32, Ya, Yb = torch.empty_like(X), torch.empty_like(X), torch.full_like(X, float("nan"))
    H.matvec_multi(X, Y32)
    H.build_bf16_factors(near=hmg.PREC_BF16)
    H.matvec_multi(X, Ya)
    H.build_bf16_factors(near=hmg.PREC_FP32)
    H.matvec_multi(X, Yb)
    H.synchronize()
    ref, a, b = Y32.cpu().numpy(), Ya.cpu().numpy(), Yb.cpu().numpy()
    assert np.isfinite(b).all()
    ea = max(rel_err(a[j], ref[j]) for j in range(16))
    eb = max(rel_err(b[j], ref[j]) for j in range(16))
    assert eb < 5e-3 and eb < ea, (ea, eb)
    with pytest.raises(hmg.HmgError):
        H.build_bf16_factors(near=hmg.PREC_MIXED)
    H.close()


def test_copies_follow_the_storage(hmg, cuda):
    """Recomputing the near field drops the BF16 copies (products fall back to the
    FP32 CUDA-core kernels); a handle without an FP32 stored near field is refused."""
    torch = cuda
    p = make_points("uniform", 8000, 3, 5)
    H = engine(hmg, p, p, 1.5, 64, rule=1)
    H.set_kernel(MATERN, 0.2, 0.0)
    H.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    with pytest.raises(hmg.HmgError):
        H.build_bf16_factors()  # near field not stored
    H.precompute_dense(hmg.PREC_FP32)
    H.build_bf16_factors()
    X = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, (4, 8000))).cuda()
    Ytc, Y32 = torch.empty_like(X), torch.empty_like(X)
    H.matvec_multi(X, Ytc)
    H.precompute_dense(hmg.PREC_FP32)  # drops the copies
    H.matvec_multi(X, Y32)
    H.synchronize()
    ref = np.stack([H.matvec(X[j].cpu().numpy()) for j in range(4)])
    assert max(rel_err(Y32.cpu().numpy()[j], ref[j]) for j in range(4)) < 1e-6
    assert 1e-6 < max(rel_err(Ytc.cpu().numpy()[j], ref[j]) for j in range(4)) < 5e-3
    H.close()


def test_leading_dimensions_and_33_vectors(hmg, cuda):
    """Column-major X and Y with leading dimensions past n (X: n + 17, Y: n + 5) and
    33 vectors (MMAs of N = 64 with 31 zero columns): rows past n are never written."""
    torch = cuda
    n = 12000
    p = make_points("uniform", n, 3, 23)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(MATERN, 0.2, 0.0)
    H.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    nrhs = 33
    Xb = torch.from_numpy(np.random.default_rng(8).uniform(-1, 1, (nrhs, n + 17))).cuda()
    X = Xb[:, :n]
    Yref = torch.empty(nrhs, n, dtype=torch.float64, device="cuda")
    H.matvec_multi(X.contiguous(), Yref)
    H.build_bf16_factors()
    Yb = torch.full((nrhs, n + 5), 7.0, dtype=torch.float64, device="cuda")
    Y = Yb[:, :n]
    H.matvec_multi(X, Y)
    H.synchronize()
    a, b = Y.cpu().numpy(), Yref.cpu().numpy()
    for j in range(nrhs):
        assert rel_err(a[j], b[j]) < 1e-2, (j, rel_err(a[j], b[j]))
    assert float((Yb[:, n:] - 7.0).abs().max()) == 0.0
    H.close()


@pytest.mark.parametrize("eta", [0.05, 1e6], ids=["all-dense", "mostly-low-rank"])
def test_extreme_partitions(hmg, cuda, eta):
    """Tensor-core operands of an H-matrix with (almost) no admissible blocks (pass 1
    has no jobs) and of one where nearly everything is low rank."""
    torch = cuda
    n = 5000
    p = make_points("uniform", n, 2, 29)
    H = engine(hmg, p, p, eta, 64, rule=1)
    H.set_kernel(GAUSS, 0.1, 0.0)
    H.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, (4, n))).cuda()
    Yref, Ytc = torch.empty_like(X), torch.full_like(X, float("nan"))
    H.matvec_multi(X, Yref)
    H.build_bf16_factors()
    H.matvec_multi(X, Ytc)
    H.synchronize()
    a, b = Ytc.cpu().numpy(), Yref.cpu().numpy()
    assert np.isfinite(a).all()
    for j in range(4):
        assert rel_err(a[j], b[j]) < 1e-2, (j, rel_err(a[j], b[j]))
    H.close()


@pytest.mark.parametrize("nrhs", [8, 40])
def test_split_operands(hmg, cuda, nrhs):
    """HMG_PREC_BF16X3 (operands as BF16 hi + lo pairs, three MMAs per K step) and
    HMG_PREC_BF16X6 (three BF16 parts, six MMAs): each step's products in their own
    accumulators, summed in FP32 on the CUDA cores.  Against the FP32 products: pairs
    to ~5e-6 (bound 2e-5), triples closer still; both deterministic."""
    torch = cuda
    n = 20000
    p = make_points("uniform", n, 3, 37)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(MATERN, 0.2, 0.0)
    H.precompute_aca(64, 1e-8, hmg.PREC_FP32)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(9).uniform(-1, 1, (nrhs, n))).cuda()
    Y32 = torch.empty_like(X)
    H.matvec_multi(X, Y32)
    ref = Y32.cpu().numpy()
    errs = {}
    for prec in (hmg.PREC_BF16, hmg.PREC_BF16X3, hmg.PREC_BF16X6):
        H.build_bf16_factors(near=prec)
        Ya, Yb = torch.full_like(X, float("nan")), torch.empty_like(X)
        H.matvec_multi(X, Ya)
        H.matvec_multi(X, Yb)
        H.synchronize()
        a = Ya.cpu().numpy()
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(Yb.cpu().numpy(), a)
        errs[prec] = max(rel_err(a[j], ref[j]) for j in range(nrhs))
    print("errors vs FP32 products", errs)
    e1, e2, e3 = errs[hmg.PREC_BF16], errs[hmg.PREC_BF16X3], errs[hmg.PREC_BF16X6]
    assert e2 < 2e-5 and e2 < e1 / 100, errs
    assert e3 < e2 / 2, errs
    H.close()

"""Tensor-core products with operands converted on chip (HMG_PREC_BF16X6_ONCHIP):
the pass kernels read the stored FP32 or mixed FP32/FP16/FP8 factors and the FP32
near field and split every value into three BF16 parts in shared memory.  No
reference counterpart (the reference multiplies one vector per call, hmglib.cu:271-286).

Checked against FP64 directly (hmg_full_matvec / hmg_full_matvec_rows) on every
vector: relative L2 error <= 1e-6 at ACA eps 1e-8 (measured ~3e-7); against the
stored three-part copies (HMG_PREC_BF16X6, same splits, other step boundaries) to
1e-6; deterministic; writes every row; refused without a stored FP32 near field."""
import numpy as np
import pytest

from helpers import engine, fp64_rows, make_points, rel_err

pytestmark = pytest.mark.gpu

MATERN, GAUSS = 4, 3


def _build(hmg, gen, n, dim, leaf, kind, param, kmax, eps, prec, seed=13):
    p = make_points(gen, n, dim, seed)
    H = engine(hmg, p, p, 1.5, leaf, rule=1)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(kmax, eps, prec)
    H.precompute_dense(hmg.PREC_FP32)
    return H


def _errors_vs_fp64(torch, H, X, Y, nrows=2048, seed=0):
    rng = np.random.default_rng(seed)
    Yh = Y.cpu().numpy()
    out = []
    for j in range(X.shape[0]):
        rows = rng.choice(X.shape[1], min(nrows, X.shape[1]), replace=False)
        out.append(rel_err(Yh[j][rows], fp64_rows(torch, H, X[j].contiguous(), rows)))
    return out


@pytest.mark.parametrize("case", [
    ("uniform", 20000, 3, 128, MATERN, 0.2, 96, 1e-8, 64, "mixed"),
    ("uniform", 20000, 3, 128, MATERN, 0.2, 96, 1e-8, 16, "fp32"),
    ("gmm", 30000, 2, 64, GAUSS, 0.05, 64, 1e-8, 41, "mixed"),
    # ranks up to 128 and tiles of at most 32 rows
    ("uniform", 12000, 3, 32, MATERN, 0.2, 128, 1e-10, 32, "mixed"),
    ("uniform", 9000, 2, 128, GAUSS, 0.1, 64, 1e-8, 2, "fp32"),
], ids=["uniform3d-mixed-64", "uniform3d-fp32-16", "gmm2d-mixed-41", "rank128-leaf32", "two-vectors"])
def test_onchip_products_vs_fp64(hmg, cuda, case):
    torch = cuda
    gen, n, dim, leaf, kind, param, kmax, eps, nrhs, storage = case
    prec = hmg.PREC_MIXED if storage == "mixed" else hmg.PREC_FP32
    H = _build(hmg, gen, n, dim, leaf, kind, param, kmax, eps, prec)
    X = torch.from_numpy(np.random.default_rng(nrhs).uniform(-1, 1, (nrhs, n))).cuda()
    Ycc = torch.empty_like(X)
    H.matvec_multi(X, Ycc)  # CUDA cores, before the plan exists
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    H.set_tensor_core_min_vectors(2)  # every multi-vector product on the tensor cores
    info = H.info()
    assert info["tc_onchip"] == 1 and info["tc_parts"] == 3 and info["tc_bytes"] == 0
    Y = torch.full_like(X, float("nan"))
    H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(Y).all())
    errs = _errors_vs_fp64(torch, H, X, Y, seed=nrhs)
    print(f"{storage}, {nrhs} vectors: max error vs FP64 {max(errs):.2e}")
    assert max(errs) <= 1e-6, errs
    # close to the CUDA-core product of the same storage
    a, b = Y.cpu().numpy(), Ycc.cpu().numpy()
    assert max(rel_err(a[j], b[j]) for j in range(nrhs)) < 1e-6
    # deterministic
    Y2 = torch.empty_like(X)
    H.matvec_multi(X, Y2)
    torch.cuda.synchronize()
    assert torch.equal(Y2, Y)
    if kmax == 128:
        assert H.info()["max_rank"] > 96
    H.close()


def test_onchip_equals_stored_parts(hmg, cuda):
    """FP32 storage: the on-chip split and the stored three-part copies are the same
    parts, multiplied with other step boundaries: equal to FP32 rounding of the sums."""
    torch = cuda
    n = 20000
    H = _build(hmg, "uniform", n, 3, 128, MATERN, 0.2, 64, 1e-8, hmg.PREC_FP32, seed=37)
    X = torch.from_numpy(np.random.default_rng(9).uniform(-1, 1, (40, n))).cuda()
    Ys, Yo = torch.empty_like(X), torch.empty_like(X)
    H.build_bf16_factors(near=hmg.PREC_BF16X6)
    H.matvec_multi(X, Ys)
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    H.matvec_multi(X, Yo)
    torch.cuda.synchronize()
    a, b = Yo.cpu().numpy(), Ys.cpu().numpy()
    d = max(rel_err(a[j], b[j]) for j in range(40))
    assert d < 1e-6, d
    H.close()


def test_onchip_leading_dimensions_and_refusals(hmg, cuda):
    torch = cuda
    n = 9000
    H = _build(hmg, "uniform", n, 2, 64, GAUSS, 0.1, 32, 1e-6, hmg.PREC_MIXED, seed=3)
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    H.set_tensor_core_min_vectors(2)
    nrhs, ld = 5, n + 17
    Xb = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, (nrhs, ld))).cuda()
    Yb = torch.zeros(nrhs, ld + 5, dtype=torch.float64, device="cuda")
    H._call("hmg_matvec_multi", nrhs, Xb.data_ptr(), ld, Yb.data_ptr(), ld + 5)
    torch.cuda.synchronize()
    for j in range(nrhs):
        yj = H.matvec(Xb[j, :n].cpu().numpy())
        assert rel_err(Yb[j, :n].cpu().numpy(), yj) < 1e-6
    assert float(Yb[:, n:].abs().max()) == 0.0  # nothing written past n rows
    H.close()
    # an FP64 near field cannot be converted
    p = make_points("uniform", 4000, 2, 4)
    G = engine(hmg, p, p, 1.5, 64, rule=1)
    G.set_kernel(GAUSS, 0.1, 0.0)
    G.precompute_aca(32, 1e-6, hmg.PREC_FP32)
    G.precompute_dense(hmg.PREC_FP64)
    with pytest.raises(hmg.HmgError):
        G.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    G.close()


def test_onchip_group_vs_fp64(hmg, cuda):
    torch = cuda
    rng = np.random.default_rng(23)
    sizes = [2000, 5000, 700, 3000]
    sets = []
    for i, n in enumerate(sizes):
        dim = 2 if i % 2 == 0 else 3
        p = make_points("uniform", n, dim, 23000 + i)
        Hs = engine(hmg, p, p, 1.5, 64 if dim == 2 else 128, rule=1)
        Hs.set_kernel(hmg.KERNEL_GAUSSIAN, float(rng.uniform(0.01, 0.2)), 0.0)
        sets.append(Hs)
    G = hmg.group(sets)
    G.precompute_aca(64, 1e-8, hmg.PREC_MIXED)
    G.precompute_dense(hmg.PREC_FP32)
    G.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    G.set_tensor_core_min_vectors(2)
    off = G.offsets(0)
    X = torch.from_numpy(np.random.default_rng(24).uniform(-1, 1, (8, int(off[-1])))).cuda()
    Y = torch.empty_like(X)
    G.matvec_multi(X, Y)
    torch.cuda.synchronize()
    for i, Hs in enumerate(sets):
        for j in (0, 7):
            xi = X[j, off[i]:off[i + 1]].contiguous()
            yf = torch.empty_like(xi)
            Hs.full_matvec(xi, yf)
            torch.cuda.synchronize()
            e = rel_err(Y[j, off[i]:off[i + 1]].cpu().numpy(), yf.cpu().numpy())
            assert e <= 1e-6, (i, j, e)
    for Hs in sets:
        Hs.close()
    G.close()


def test_onchip_rectangular_and_plan_rebuild(hmg, cuda):
    """Rows and columns from different point clouds (n1 != n2), mixed storage: on-chip
    products within 1e-6 of FP64; the plan, built on several host threads, gives
    bit-identical products when it is built again."""
    torch = cuda
    n1, n2 = 21000, 14000
    p1 = make_points("uniform", n1, 3, 71)
    p2 = make_points("uniform", n2, 3, 72)
    H = engine(hmg, p1, p2, 1.5, 128, rule=1)
    H.set_kernel(MATERN, 0.2, 0.0)
    H.precompute_aca(96, 1e-8, hmg.PREC_MIXED)
    H.precompute_dense(hmg.PREC_FP32)
    X = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (24, n2))).cuda()
    Y = torch.empty(24, n1, dtype=torch.float64, device="cuda")
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    errs = _errors_vs_fp64(torch, H, X, Y, seed=3)
    assert max(errs) <= 1e-6, errs
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    Y2 = torch.empty_like(Y)
    H.matvec_multi(X, Y2)
    torch.cuda.synchronize()
    assert torch.equal(Y2, Y)
    H.close()


def test_onchip_min_vectors_dispatch(hmg, cuda):
    """Below the threshold (default 17 vectors) a handle with on-chip operands
    multiplies on the CUDA cores: the same bits as before the plan existed; at or above
    it, on the tensor cores (other rounding, same accuracy)."""
    torch = cuda
    n = 20000
    H = _build(hmg, "uniform", n, 3, 128, MATERN, 0.2, 96, 1e-8, hmg.PREC_MIXED, seed=51)
    X = torch.from_numpy(np.random.default_rng(52).uniform(-1, 1, (8, n))).cuda()
    Ycc, Y = torch.empty_like(X), torch.empty_like(X)
    H.matvec_multi(X, Ycc)
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    H.matvec_multi(X, Y)  # 8 < 17: CUDA cores
    torch.cuda.synchronize()
    assert torch.equal(Y, Ycc)
    H.set_tensor_core_min_vectors(8)
    H.matvec_multi(X, Y)  # tensor cores
    torch.cuda.synchronize()
    assert not torch.equal(Y, Ycc)
    assert max(_errors_vs_fp64(torch, H, X, Y, nrows=1024, seed=4)) <= 1e-6
    with pytest.raises(hmg.HmgError):
        H.set_tensor_core_min_vectors(1)
    H.close()

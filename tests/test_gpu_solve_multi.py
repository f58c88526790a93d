"""Block-lockstep kernel-ridge solves (hmg_cg_solve_multi and the step API
hmg_cg_multi_*): several right-hand sides, one multi-vector product per iteration,
FP64 vectors and inner products, FP64-product refinement.

No reference counterpart (hmglib has no solver).  Checked against the definition
(the residual recomputed from X with FP64-arithmetic products), against the
single-vector solver hmg_cg_solve column by column, and for determinism: the step
API driven with arbitrary polling gives the blocking solve's X bit for bit."""
import numpy as np
import pytest

from helpers import engine, make_points

pytestmark = pytest.mark.gpu


def _hmatrix(hmg, prec, n=8192):
    p = make_points("gmm", n, 2, 2)
    H = engine(hmg, p, p, 1.5, 64, rule=1)
    H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05, 0.0)
    H.precompute_aca(64, 1e-9, prec)
    H.precompute_dense(hmg.PREC_FP64 if prec == 0 else hmg.PREC_FP32)
    return H, n


def _op_residual(torch, hmg, H, B, X, shift):
    """max_j |b_j - (H + shift I) x_j| / |b_j| with FP64-arithmetic products"""
    H.set_product_precision(hmg.PREC_FP64)
    rel = []
    for j in range(B.shape[0]):
        y = torch.empty_like(X[j])
        H.matvec(X[j].contiguous(), y)
        H.synchronize()
        rel.append(float(torch.linalg.norm(B[j] - (y + shift * X[j])) / torch.linalg.norm(B[j])))
    H.set_product_precision(hmg.PREC_FP32)
    return max(rel)


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "mixed"])
def test_block_cg_with_refinement(hmg, cuda, prec):
    torch = cuda
    H, n = _hmatrix(hmg, prec)
    shift, tol, k = 1e-3, 1e-8, 8
    B = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (k, n))).cuda()
    X = torch.zeros_like(B)
    iters, rel = H.cg_solve_multi(B, X, shift, tol=tol, maxit=5000, refine=True)
    assert 0 < iters < 5000 and (rel <= tol).all(), (iters, rel)
    assert _op_residual(torch, hmg, H, B, X, shift) <= 2 * tol
    # every column against the single-vector solver
    for j in (0, k - 1):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        H.cg_solve(B[j].contiguous(), x, shift, tol=tol, maxit=5000, refine=True)
        torch.cuda.synchronize()
        d = float(torch.linalg.norm(x - X[j]) / torch.linalg.norm(x))
        assert d < 1e-4, (j, d)  # both solve to tol; cond(H + 1e-3 I) ~ 1e4 amplifies it
    # deterministic: the same solve again gives the same X
    X2 = torch.zeros_like(B)
    it2, rel2 = H.cg_solve_multi(B, X2, shift, tol=tol, maxit=5000, refine=True)
    assert it2 == iters
    assert torch.equal(X2, X)
    H.close()


def test_step_api_equals_blocking_solve(hmg, cuda):
    torch = cuda
    H, n = _hmatrix(hmg, 1)
    shift, tol, k = 1e-2, 1e-7, 5
    B = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, (k, n))).cuda()
    X = torch.zeros_like(B)
    it_a, rel_a = H.cg_solve_multi(B, X, shift, tol=tol, maxit=3000, refine=True)
    Y = torch.zeros_like(B)
    s = H.cg_multi(B, Y, shift, tol=tol, maxit=3000, refine=True)
    rng = np.random.default_rng(0)
    spins = 0
    while True:
        s.advance()
        done, it_b, rel_b = s.poll()
        if done:
            break
        if rng.uniform() < 0.3:  # poll at irregular times: decisions must not depend on it
            torch.cuda.synchronize()
        spins += 1
        assert spins < 10 ** 6
    s.close()
    assert it_b == it_a
    np.testing.assert_array_equal(rel_b, rel_a)
    assert torch.equal(Y, X)
    H.close()


def test_block_cg_plain_and_errors(hmg, cuda):
    torch = cuda
    H, n = _hmatrix(hmg, 0, n=4096)
    B = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (3, n))).cuda()
    X = torch.zeros_like(B)
    iters, rel = H.cg_solve_multi(B, X, 1e-3, tol=1e-9, maxit=4000, refine=False)
    assert (rel <= 1e-9).all(), rel
    assert _op_residual(torch, hmg, H, B, X, 1e-3) <= 2e-9
    # a zero right-hand side converges at once with X = 0
    Z, XZ = torch.zeros_like(B), torch.zeros_like(B)
    it0, rel0 = H.cg_solve_multi(Z, XZ, 1e-3, tol=1e-9, maxit=10)
    assert it0 == 0 and float(XZ.abs().max()) == 0.0
    for bad in (0, 65):
        with pytest.raises(hmg.HmgError):
            H._call("hmg_cg_solve_multi", bad, 1e-3, B.data_ptr(), n, X.data_ptr(), n, 1e-8, 10, 1, None, None)
    H.close()

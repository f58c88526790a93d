"""Several right-hand sides per product (hmg_matvec_multi) against one product per
vector.  No reference counterpart: the reference multiplies one vector per
apply_h_matrix_mvp call (hmglib.cu:271-286).

Tolerances (relative L2 per column): FP64 storage 1e-13 (summation order differs);
FP32 and mixed storage 1e-6 (FP32 sums per slice in a different order)."""
import numpy as np
import pytest

from helpers import engine, make_points, rel_err

pytestmark = pytest.mark.gpu


def _build(hmg, prec, n=30000, dim=3, seed=7, c_leaf=128):
    p = make_points("uniform", n, dim, seed)
    H = engine(hmg, p, p, 1.5, c_leaf, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(64, 1e-8, prec)
    H.precompute_dense(prec)
    return H, n


def _columns(torch, H, X):
    out = torch.empty_like(X)
    for j in range(X.shape[0]):
        H.matvec(X[j], out[j])
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("prec,tol", [(0, 1e-13), (1, 1e-6), (2, 1e-6)], ids=["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("nrhs", [2, 5, 16, 32, 45])
def test_multi_matches_single(hmg, cuda, prec, tol, nrhs):
    torch = cuda
    H, n = _build(hmg, prec)
    X = torch.from_numpy(np.random.default_rng(nrhs).uniform(-1, 1, (nrhs, n))).cuda()
    Y = torch.full_like(X, float("nan"))
    H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    ref = _columns(torch, H, X)
    Yh, Rh = Y.cpu().numpy(), ref.cpu().numpy()
    assert np.isfinite(Yh).all()
    for j in range(nrhs):
        if tol == 0.0:
            np.testing.assert_array_equal(Yh[j], Rh[j])
        else:
            assert rel_err(Yh[j], Rh[j]) < tol, (j, rel_err(Yh[j], Rh[j]))
    # deterministic
    Y2 = torch.empty_like(X)
    H.matvec_multi(X, Y2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Y2.cpu().numpy(), Yh)
    H.close()


def test_multi_leading_dimensions_and_errors(hmg, cuda):
    torch = cuda
    H, n = _build(hmg, 1, n=9000, dim=2, seed=3, c_leaf=64)
    nrhs, ld = 3, n + 17
    Xb = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, (nrhs, ld))).cuda()
    X = Xb[:, :n]
    Yb = torch.zeros(nrhs, ld + 5, dtype=torch.float64, device="cuda")
    Y = Yb[:, :n]
    H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    ref = _columns(torch, H, X.contiguous())
    for j in range(nrhs):
        assert rel_err(Y[j].cpu().numpy(), ref[j].cpu().numpy()) < 1e-6
    assert float(Yb[:, n:].abs().max()) == 0.0  # nothing written past n rows
    for bad in (0, 65):
        Xe = torch.zeros(bad if bad else 1, n, dtype=torch.float64, device="cuda")
        with pytest.raises(hmg.HmgError):
            H._call("hmg_matvec_multi", bad, Xe.data_ptr(), n, Xe.data_ptr(), n)
    H.close()

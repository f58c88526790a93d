"""Kernel-ridge solves (H + shift I) x = b with CG on the GPU (hmg_cg_solve).

No reference counterpart (hmglib has no solver); checked against the definition:
the residual recomputed from x with the same operator, and the residual against
the exact kernel matrix from the FP64 direct product."""
import numpy as np
import pytest

from helpers import engine, make_points, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("refine", [False, True], ids=["cg", "cg+refinement"])
@pytest.mark.parametrize("prec", [0, 1, 2], ids=["fp64", "fp32", "mixed"])
def test_kernel_ridge_cg(hmg, cuda, refine, prec):
    torch = cuda
    n = 8192
    if prec == 0 or refine:
        shift, tol = 1e-3, 1e-8
    else:
        # plain CG in FP32 arithmetic stalls near 1e-7 * cond(H + shift I): a better
        # conditioned system and a tolerance above that floor
        shift, tol = 1.0, 1e-3
    p = make_points("gmm", n, 2, 2)
    H = engine(hmg, p, p, 1.5, 64, rule=1)
    H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05, 0.0)
    H.precompute_aca(64, 1e-9, prec)
    H.precompute_dense(prec)
    b = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, n)).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    iters, rel = H.cg_solve(b, x, shift, tol=tol, maxit=5000, refine=refine)
    assert rel <= tol, (iters, rel)
    assert 0 < iters < 5000
    # residual against the operator, recomputed here in the arithmetic the solver
    # reports in (FP64 products when refining)
    if refine:
        H.set_product_precision(hmg.PREC_FP64)
    y = torch.empty_like(x)
    H.matvec(x, y)
    H.synchronize()
    H.set_product_precision(hmg.PREC_FP32)
    r_op = b - (y + shift * x)
    assert float(torch.linalg.norm(r_op) / torch.linalg.norm(b)) <= 2 * tol
    # the H-matrix error on a generic vector
    z = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, n)).cuda()
    hz, kz = torch.empty_like(z), torch.empty_like(z)
    H.matvec(z, hz)
    H.full_matvec(z, kz)
    torch.cuda.synchronize()
    h_err = float(torch.linalg.norm(hz - kz) / torch.linalg.norm(kz))
    assert h_err < (1e-8 if prec == 0 else 1e-6), h_err
    # residual against the exact kernel matrix: the operator residual plus (H - K) x.
    # x leans on the kernel's small eigenvalues (|x| ~ |b| / shift), which amplifies the
    # H-matrix error there (FP32 storage rounding included) far beyond its size on a
    # generic vector.
    yd = torch.empty_like(x)
    H.full_matvec(x, yd)
    torch.cuda.synchronize()
    r_ex = b - (yd + shift * x)
    assert float(torch.linalg.norm(r_ex) / torch.linalg.norm(b)) < (5e-5 if prec == 0 else 2e-2)
    H.close()


def test_cg_rejects_rectangular(hmg, cuda):
    torch = cuda
    p1 = make_points("uniform", 500, 2, 1)
    p2 = make_points("uniform", 400, 2, 2)
    H = engine(hmg, p1, p2, 1.5, 32)
    H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.1, 0.0)
    H.precompute_aca(16, 1e-6)
    b = torch.zeros(500, dtype=torch.float64, device="cuda")
    x = torch.zeros(500, dtype=torch.float64, device="cuda")
    with pytest.raises(hmg.HmgError):
        H.cg_solve(b, x, 1e-3)
    H.close()

"""ACA and H-matvec on the GPU against the oracle, the FP64 direct sum and the
reference's own results (golden fixtures).  Reference: linear_algebra.cu:769-1147,
1429-1591, 2009-2222, 2817-3511, 3684-4012, 4292-4379; hmglib.cu:271-286,351-401.

Tolerances (relative L2 over y):
  * FP64 storage vs the oracle's FP64 H-matvec on the same tree:   1e-9
    (the fixed-rank ACA keeps adding terms down to residual rows of norm 1e-13,
    whose pivots are rounding noise; ranks may differ by one on such rows)
  * FP64 storage vs the reference build's apply_h_matrix_mvp: error vs the FP64
    direct product <= 1.5x the reference's own, difference <= 3x it
    (check_vs_reference_product)
  * direct sum vs the reference's apply_full_mvp / the oracle:     1e-12
  * adaptive ACA (eps) vs FP64 direct sum: 10 eps (FP64 storage), max(10 eps, 3e-6) (FP32)
"""
import numpy as np
import pytest

from helpers import engine, make_points, oracle_setup, rel_err
from conftest import golden
from test_oracle_cpu import check_vs_reference_product

pytestmark = pytest.mark.gpu


def _torch_vec(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _setup_pair(hmg, O, gen, n, dim, seed, eta, c_leaf, kind, param, reg=0.0, n2=None, scale=1.0):
    p1 = make_points(gen, n, dim, seed, scale)
    p2 = p1 if n2 is None else make_points(gen, n2, dim, seed + 100, scale)
    H = engine(hmg, p1, p2, eta, c_leaf)
    H.set_kernel(kind, param, reg)
    ref = oracle_setup(O, p1, p2, eta, c_leaf)
    return H, ref, p1, p2


FIXED = [
    # gen, n, dim, seed, eta, c_leaf, kind, param, k
    ("uniform", 4096, 2, 0, 1.5, 32, 1, 0.0, 16),
    ("uniform", 4096, 3, 1, 1.5, 64, 2, 0.0, 8),
    ("gmm", 6000, 2, 2, 1.0, 32, 3, 0.05, 12),
    ("uniform", 3000, 3, 3, 1.5, 64, 4, 0.2, 20),
]


@pytest.mark.parametrize("case", FIXED, ids=[f"{c[0]}-{c[1]}-d{c[2]}-k{c[6]}" for c in FIXED])
def test_fixed_rank_aca_and_matvec_fp64(hmg, oracle, cuda, case):
    torch = cuda
    gen, n, dim, seed, eta, c_leaf, kind, param, k = case
    H, ref, p1, p2 = _setup_pair(hmg, oracle, gen, n, dim, seed, eta, c_leaf, kind, param, reg=0.25)
    H.precompute_aca(k, 0.0, hmg.PREC_FP64)
    H.precompute_dense(hmg.PREC_FP64)
    b = ref["blocks"]
    aca_mask = b.type == 1
    oparam = oracle.kernel_param(kind, param)
    fac = oracle.aca(kind, oparam, 0.25, ref["z1"], ref["z2"], b.subset(aca_mask), k)
    ranks = H.ranks()[aca_mask]
    assert np.abs(ranks - fac.ranks).max() <= 1
    assert (ranks == fac.ranks).mean() > 0.98
    # factor pairs of blocks whose rank agrees: the products agree to rounding of
    # the leading terms
    idx = np.nonzero(aca_mask)[0]
    same = np.nonzero(ranks == fac.ranks)[0]
    for jj in same[:: max(1, len(same) // 7)][:8]:
        bi = idx[jj]
        m1, m2, r = b.m1[bi], b.m2[bi], fac.ranks[jj]
        U, V = H.factors(int(bi), int(m1), int(m2), int(r))
        Uo = fac.U[fac.uoff[jj]:fac.uoff[jj] + m1 * fac.kb[jj]].reshape(fac.kb[jj], m1)[:r]
        Vo = fac.V[fac.voff[jj]:fac.voff[jj] + m2 * fac.kb[jj]].reshape(fac.kb[jj], m2)[:r]
        A, Ao = U.T @ V, Uo.T @ Vo
        assert np.linalg.norm(A - Ao) <= 1e-9 * max(np.linalg.norm(Ao), 1e-300)
    x = np.random.default_rng(seed).uniform(-1, 1, p2.shape[1])
    y = H.matvec(x)
    xs = x[ref["order2"]]
    ys = oracle.hmatvec(kind, oparam, 0.25, ref["z1"], ref["z2"], b, fac, xs)
    y_or = np.empty_like(ys)
    y_or[ref["order1"]] = ys
    assert rel_err(y, y_or) < 1e-9
    # on-the-fly near field gives the same product (other summation order)
    H.set_near_mode(hmg.NEAR_ONTHEFLY)
    y2 = H.matvec(x)
    assert rel_err(y2, y) < 1e-12
    # deterministic: a second product is bit-identical
    H.set_near_mode(hmg.NEAR_STORED)
    np.testing.assert_array_equal(H.matvec(x), y)
    # direct sum on the GPU vs the oracle's
    dx = _torch_vec(torch, x)
    dy = torch.empty(p1.shape[1], dtype=torch.float64, device="cuda")
    H.full_matvec(dx, dy)
    torch.cuda.synchronize()
    yd = oracle.direct(kind, oparam, 0.25, ref["z1"], ref["z2"], xs)
    yd_or = np.empty_like(yd)
    yd_or[ref["order1"]] = yd
    assert rel_err(dy.cpu().numpy(), yd_or) < 1e-12
    H.close()


ADAPTIVE = [
    # gen, n, dim, seed, eta, c_leaf, kind, param, eps, tol
    ("uniform", 16384, 2, 0, 1.5, 64, 3, 0.1, 1e-6, 2e-6),
    ("uniform", 20000, 3, 1, 1.5, 128, 4, 0.2, 1e-8, 1e-7),
    ("gmm", 20000, 2, 2, 1.5, 64, 3, 0.05, 1e-6, 2e-6),
]


@pytest.mark.parametrize("case", ADAPTIVE, ids=[f"{c[0]}-{c[1]}-d{c[2]}-eps{c[8]}" for c in ADAPTIVE])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_adaptive_aca_error_vs_direct(hmg, oracle, cuda, case, prec):
    torch = cuda
    gen, n, dim, seed, eta, c_leaf, kind, param, eps, tol = case
    p = make_points(gen, n, dim, seed)
    H = engine(hmg, p, p, eta, c_leaf, rule=1)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(96, eps, prec)
    H.precompute_dense(prec)
    x = np.random.default_rng(seed + 1).uniform(-1, 1, n)
    y = H.matvec(x)
    dx = _torch_vec(torch, x)
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    H.full_matvec(dx, dy)
    torch.cuda.synchronize()
    err = rel_err(y, dy.cpu().numpy())
    assert err < (10 * eps if prec == 0 else max(10 * eps, 3e-6)), err
    # the device-pointer path gives the same y as the host path
    dy2 = torch.empty(n, dtype=torch.float64, device="cuda")
    H.matvec(dx, dy2)
    H.synchronize()
    np.testing.assert_array_equal(dy2.cpu().numpy(), y)
    info = H.info()
    assert info["far_entries"] > 0 and info["max_rank"] <= 96
    H.close()


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_streaming_kernels_match_simple_kernels(hmg, cuda, prec):
    """The bulk-copy pipelined product kernels (default) and the plain-load kernels
    compute the same product; each is deterministic run to run."""
    n = 40000
    p = make_points("uniform", n, 3, 8)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(4, 0.2, 0.0)
    H.precompute_aca(96, 1e-7, prec)
    H.precompute_dense(prec)
    x = np.random.default_rng(3).uniform(-1, 1, n)
    H.set_matvec_variant(0)
    y0 = H.matvec(x)
    np.testing.assert_array_equal(H.matvec(x), y0)
    H.set_matvec_variant(1)
    y1 = H.matvec(x)
    np.testing.assert_array_equal(H.matvec(x), y1)
    # FP64 storage: both sum FP64 products (order differs); FP32 storage: the simple
    # kernels sum each slice in FP32 first
    assert rel_err(y0, y1) < (1e-13 if prec == 0 else 2e-7)
    H.close()


@pytest.mark.parametrize("case", [("uniform", 60000, 3, 1, 4, 0.2, 1e-8), ("gmm", 40000, 2, 2, 3, 0.05, 1e-8)],
                         ids=["uniform3d-matern", "gmm2d-gauss"])
def test_mixed_precision_factors(hmg, cuda, case):
    """Mixed storage (leading terms FP32, tail terms FP16 / FP8 by their share of the
    block norm) stays within 3e-7 of the FP64 direct product at eps = 1e-8, stores
    fewer bytes than FP32, and agrees with the FP32 storage to ~1e-7."""
    torch = cuda
    gen, n, dim, seed, kind, param, eps = case
    p = make_points(gen, n, dim, seed)
    x = np.random.default_rng(seed).uniform(-1, 1, n)
    dx = _torch_vec(torch, x)
    ys, nbytes, Hs = {}, {}, {}
    for prec in (hmg.PREC_FP32, hmg.PREC_MIXED):
        H = Hs[prec] = engine(hmg, p, p, 1.5, 128 if dim == 3 else 64, rule=1)
        H.set_kernel(kind, param, 0.0)
        H.precompute_aca(96, eps, prec)
        H.precompute_dense(prec)
        ys[prec] = H.matvec(x)
        nbytes[prec] = H.info()["far_bytes"]
        np.testing.assert_array_equal(H.matvec(x), ys[prec])  # deterministic
        if prec == hmg.PREC_MIXED:
            dy = torch.empty(n, dtype=torch.float64, device="cuda")
            H.full_matvec(dx, dy)
            torch.cuda.synchronize()
            yd = dy.cpu().numpy()
    # decoded factors: the same low-rank terms, within the tail thresholds of the FP32 ones
    ranks = Hs[hmg.PREC_MIXED].ranks()
    np.testing.assert_array_equal(ranks, Hs[hmg.PREC_FP32].ranks())
    s1l, s1u, s2l, s2u, _ = Hs[hmg.PREC_MIXED].blocks()
    far = np.nonzero(ranks > 0)[0]
    for b in far[np.argsort(-ranks[far], kind="stable")[:6]]:
        shape = (int(b), int(s1u[b] - s1l[b] + 1), int(s2u[b] - s2l[b] + 1), int(ranks[b]))
        u32, v32 = Hs[hmg.PREC_FP32].factors(*shape)
        um, vm = Hs[hmg.PREC_MIXED].factors(*shape)
        a, c = u32.T @ v32, um.T @ vm
        assert np.linalg.norm(a - c) <= 1e-6 * np.linalg.norm(a), (b, np.linalg.norm(a - c) / np.linalg.norm(a))
    for H in Hs.values():
        H.close()
    assert rel_err(ys[hmg.PREC_MIXED], yd) < 3e-7, rel_err(ys[hmg.PREC_MIXED], yd)
    assert rel_err(ys[hmg.PREC_MIXED], ys[hmg.PREC_FP32]) < 3e-7
    assert nbytes[hmg.PREC_MIXED] < 0.8 * nbytes[hmg.PREC_FP32]


def test_adaptive_matches_oracle_adaptive(hmg, oracle, cuda):
    """Same pivot rules as the oracle's adaptive ACA: ranks agree within one and the
    products agree to the ACA tolerance."""
    n, dim, eta, c_leaf, kind, param, eps = 6000, 3, 1.5, 64, 4, 0.2, 1e-6
    p = make_points("uniform", n, dim, 4)
    H = engine(hmg, p, p, eta, c_leaf, rule=1)
    H.set_kernel(kind, param, 0.0)
    H.precompute_aca(64, eps, hmg.PREC_FP64)
    ref = oracle_setup(oracle, p, p, eta, c_leaf, rule=1)
    b = ref["blocks"]
    m = b.type == 1
    fac = oracle.aca(kind, oracle.kernel_param(kind, param), 0.0, ref["z1"], ref["z2"], b.subset(m), 64, eps=eps)
    r = H.ranks()[m]
    assert np.abs(r - fac.ranks).max() <= 1
    assert (r == fac.ranks).mean() > 0.97
    H.close()


GOLDEN = ["config1_parity", "uniform3d_matern", "rect2d", "lattice_dups",
          "kat_lattice2d", "kat_lattice3d"]


@pytest.mark.parametrize("name", GOLDEN)
def test_matvec_vs_reference_build(hmg, cuda, name):
    """The legacy-mode product (fixed-rank ACA, FP64) agrees with the reference
    GPU build's apply_h_matrix_mvp and the direct sum with its apply_full_mvp."""
    torch = cuda
    from golden.make_golden import CASES as GC, case_inputs
    g = golden(name)
    c = GC[name]
    p1, p2, x = case_inputs(c)
    H = engine(hmg, p1, p2, c["eta"], c["c_leaf"], rule=0)
    H.set_kernel(c["kernel"], 0.0, 0.0)
    H.precompute_aca(c["k"], 0.0, hmg.PREC_FP64)
    if c["pre_dense"]:
        H.precompute_dense(hmg.PREC_FP64)
    y = H.matvec(x)
    check_vs_reference_product(y, g)
    dx = _torch_vec(torch, x)
    dy = torch.empty(p1.shape[1], dtype=torch.float64, device="cuda")
    H.full_matvec(dx, dy)
    torch.cuda.synchronize()
    assert rel_err(dy.cpu().numpy(), g["y_full"]) < 1e-12
    H.close()


def test_errors_are_statuses_not_crashes(hmg, cuda):
    p = make_points("uniform", 100, 2, 0)
    H = hmg.HMatrix(100, 100, 2)
    with pytest.raises(hmg.HmgError):
        H.setup(1.5, 8)  # points not set
    H.set_points(0, p)
    H.set_points(1, p)
    with pytest.raises(hmg.HmgError):
        H.setup(1.5, 0)  # c_leaf < 1
    with pytest.raises(hmg.HmgError):
        H.setup(1.5, 8, root_levels=(0, 1))
    H.setup(1.5, 8)
    with pytest.raises(hmg.HmgError):
        H.matvec(np.zeros(100))  # no kernel
    H.set_kernel(3, 0.1)
    if H.info()["aca_count"]:
        with pytest.raises(hmg.HmgError):
            H.matvec(np.zeros(100))  # no factors
    with pytest.raises(hmg.HmgError):
        H.precompute_aca(100000, 0.0)
    H.precompute_aca(8, 0.0)
    with pytest.raises(hmg.HmgError):
        H.set_near_mode(hmg.NEAR_STORED)  # nothing stored
    H.matvec(np.zeros(100))
    H.close()


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "mixed"])
def test_fp64_arithmetic_products(hmg, cuda, prec):
    """FP64 arithmetic over FP32 / mixed storage applies the stored operator exactly:
    the product is linear to FP64 rounding (FP32 arithmetic is linear only to ~1e-7)
    and its distance to the FP64 direct product is the storage error alone."""
    torch = cuda
    n = 40000
    p = make_points("uniform", n, 3, 5)
    rng = np.random.default_rng(5)
    x, z = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(64, 1e-8, prec)
    H.precompute_dense(prec)
    y32 = H.matvec(x)
    H.set_product_precision(hmg.PREC_FP64)
    y64 = H.matvec(x)
    np.testing.assert_array_equal(H.matvec(x), y64)
    a, c = 0.75, -1.25
    lin = rel_err(H.matvec(a * x + c * z), a * y64 + c * H.matvec(z))
    assert lin < 1e-13, lin
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    H.full_matvec(_torch_vec(torch, x), dy)
    torch.cuda.synchronize()
    yd = dy.cpu().numpy()
    assert rel_err(y64, yd) < 2.5e-7, rel_err(y64, yd)
    assert rel_err(y64, y32) < 3e-7
    with pytest.raises(hmg.HmgError):
        H.set_product_precision(hmg.PREC_MIXED)
    H.close()


def test_host_buffer_products(hmg, cuda):
    """hmg_matvec_host copies x and y directly between the caller's memory and the
    device: pageable and pinned host vectors give the device product bit for bit, and
    the input vector is left unchanged."""
    torch = cuda
    n = 30000
    p = make_points("uniform", n, 3, 41)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(96, 1e-8, hmg.PREC_MIXED)
    H.precompute_dense(hmg.PREC_FP32)
    x = np.random.default_rng(9).uniform(-1, 1, n)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    H.matvec(dx, dy)
    torch.cuda.synchronize()
    ref = dy.cpu().numpy()
    x_keep = x.copy()
    np.testing.assert_array_equal(H.matvec(x), ref)  # pageable in, pageable out
    np.testing.assert_array_equal(x, x_keep)
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.empty(n, dtype=torch.float64).pin_memory()
    H.matvec(xp.numpy(), yp.numpy())  # pinned in, pinned out
    np.testing.assert_array_equal(yp.numpy(), ref)
    for _ in range(3):  # repeated calls reuse the handle's device vectors
        np.testing.assert_array_equal(H.matvec(x), ref)
    H.close()

"""Many independent H-matrices multiplied as one (hmg_group_create).  No reference
counterpart: the reference runs one h_matrix_data per call (hmglib.cu:119), so the
check is against each set's own handle, bit for bit (a group never mixes sets inside
a tile and keeps every tile's pair order)."""
import numpy as np
import pytest

from helpers import engine, make_points, rel_err

pytestmark = pytest.mark.gpu


def _sets(hmg, sizes, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        dim = 2 if i % 2 == 0 else 3
        p = make_points("uniform", n, dim, seed * 1000 + i)
        H = engine(hmg, p, p, 1.5, 64 if dim == 2 else 128, rule=1)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, float(rng.uniform(0.01, 0.2)), 0.0)
        out.append(H)
    return out


@pytest.mark.parametrize("prec", [1, 0], ids=["fp32", "fp64"])
def test_group_equals_sets(hmg, cuda, prec):
    torch = cuda
    sizes = [1024, 3000, 700, 5000, 64, 2500, 9000, 1500]
    sets = _sets(hmg, sizes)
    G = hmg.group(sets)
    for H in sets:
        H.precompute_aca(64, 1e-5, prec)
        H.precompute_dense(prec)
    G.precompute_aca(64, 1e-5, prec)
    G.precompute_dense(prec)
    off = G.offsets(0)
    assert list(off) == list(np.concatenate([[0], np.cumsum(sizes)]))
    n = int(off[-1])
    x = np.random.default_rng(5).uniform(-1, 1, n)
    y = G.matvec(x)
    parts = [H.matvec(x[off[i]:off[i + 1]]) for i, H in enumerate(sets)]
    np.testing.assert_array_equal(y, np.concatenate(parts))
    # the admissible blocks' ranks: every set's, in set order
    info = G.info()
    r = G.ranks()
    per = [H.ranks()[H.info()["dense_count"]:] for H in sets]
    np.testing.assert_array_equal(r[info["dense_count"]:], np.concatenate(per))
    assert info["group_count"] == len(sizes)
    # several vectors at once
    X = torch.from_numpy(np.random.default_rng(6).uniform(-1, 1, (4, n))).cuda()
    Y = torch.empty_like(X)
    G.matvec_multi(X, Y)
    torch.cuda.synchronize()
    for j in range(4):
        yj = G.matvec(X[j].cpu().numpy())
        assert rel_err(Y[j].cpu().numpy(), yj) < (1e-13 if prec == 0 else 1e-6)
    for H in sets:
        H.close()
    G.close()


def test_group_solve_and_errors(hmg, cuda):
    torch = cuda
    sets = _sets(hmg, [2000, 3000, 1200], seed=4)
    G = hmg.group(sets)
    with pytest.raises(hmg.HmgError):  # the near field must be stored first
        G.precompute_aca(64, 1e-6, 1)
        G.matvec(np.zeros(G.n2))
    G.precompute_dense(1)
    n = G.n1
    b = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, n)).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    it, rel = G.cg_solve(b, x, 0.1, tol=1e-8, maxit=2000, refine=True)
    assert rel <= 1e-8 and it > 0
    # the group's solution solves every set's own system
    off = G.offsets(0)
    for i, H in enumerate(sets):
        H.precompute_aca(64, 1e-6, 1)
        H.precompute_dense(1)
        H.set_product_precision(hmg.PREC_FP64)
        xi = x[off[i]:off[i + 1]].contiguous()
        yi = torch.empty_like(xi)
        H.matvec(xi, yi)
        H.synchronize()
        ri = b[off[i]:off[i + 1]] - (yi + 0.1 * xi)
        assert float(torch.linalg.norm(ri)) <= 2e-8 * float(torch.linalg.norm(b))
    d = torch.empty_like(b)
    for call in (lambda: G.full_matvec(b, d), lambda: G.set_near_mode(hmg.NEAR_ONTHEFLY),
                 lambda: G.set_kernel(hmg.KERNEL_GAUSSIAN, 0.1, 0.0)):
        with pytest.raises(hmg.HmgError):
            call()
    # sets with different kernel kinds do not group
    other = _sets(hmg, [500], seed=9)[0]
    other.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    with pytest.raises(hmg.HmgError):
        hmg.group([sets[0], other])
    for H in sets + [other]:
        H.close()
    G.close()


def _raw_sets(hmg, sizes, seed=3):
    """The sets of _sets (same points and kernel parameters) with points and kernel
    only: no hmg_setup."""
    rng = np.random.default_rng(seed)
    out, leaf = [], []
    for i, n in enumerate(sizes):
        dim = 2 if i % 2 == 0 else 3
        p = make_points("uniform", n, dim, seed * 1000 + i)
        H = hmg.HMatrix(n, n, dim)
        H.set_points(0, p)
        H.set_points(1, p)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, float(rng.uniform(0.01, 0.2)), 0.0)
        out.append(H)
        leaf.append(64 if dim == 2 else 128)
    return out, leaf


@pytest.mark.parametrize("rule", [1, 0], ids=["min", "max"])
def test_group_setup_equals_per_set_setup(hmg, cuda, rule):
    """hmg_group_setup orders and clusters every set in the same launches; the handle
    must equal the one hmg_group_create makes from sets set up one by one: offsets,
    Z-ordered points, permutations, every set's Morton codes, the block list in
    order, the ranks and the products, bit for bit."""
    sizes = [1024, 3000, 700, 5000, 64, 2500, 9000, 1500, 65, 4097]
    ref = []
    rng = np.random.default_rng(3)
    for i, n in enumerate(sizes):
        dim = 2 if i % 2 == 0 else 3
        p = make_points("uniform", n, dim, 3 * 1000 + i)
        H = engine(hmg, p, p, 1.5, 64 if dim == 2 else 128, rule=rule)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, float(rng.uniform(0.01, 0.2)), 0.0)
        ref.append(H)
    G0 = hmg.group(ref)
    raw, leaf = _raw_sets(hmg, sizes)
    G1 = hmg.group_setup(raw, 1.5, leaf, rule=rule)
    off = G1.offsets(0)
    np.testing.assert_array_equal(off, G0.offsets(0))
    np.testing.assert_array_equal(G1.offsets(1), G0.offsets(1))
    i0, i1 = G0.info(), G1.info()
    for k in ("block_count", "dense_count", "aca_count", "tile_count", "group_count", "levels"):
        assert i1[k] == i0[k], k
    for a, b in zip(G1.blocks(), G0.blocks()):
        np.testing.assert_array_equal(a, b)
    for w in (0, 1):
        np.testing.assert_array_equal(G1.order(w), G0.order(w))
        np.testing.assert_array_equal(G1.points(w), G0.points(w))
        c = G1.codes(w)
        for i, H in enumerate(ref):
            np.testing.assert_array_equal(c[off[i]:off[i + 1]], H.codes(w))
    for G in (G0, G1):
        G.precompute_aca(64, 1e-5, 1)
        G.precompute_dense(1)
    np.testing.assert_array_equal(G1.ranks(), G0.ranks())
    x = np.random.default_rng(7).uniform(-1, 1, int(off[-1]))
    np.testing.assert_array_equal(G1.matvec(x), G0.matvec(x))
    # the sets themselves are untouched: still without a tree
    with pytest.raises(hmg.HmgError):
        raw[0].blocks()
    for H in ref + raw:
        H.close()
    G0.close()
    G1.close()


def test_group_setup_many_sets(hmg, cuda):
    """512 sets of 2^8 .. 2^11 points, 2D and 3D: one grouped setup against per-set
    setups, compared on the block list and one product."""
    from hmglib_b200 import synth
    sets = synth.group_sets(512, 5, 8.0, 11.0)
    ref, raw, leaf = [], [], []
    for p, l2 in sets:
        dim, n = p.shape
        c = 64 if dim == 2 else 128
        H = engine(hmg, p, p, 1.5, c, rule=1)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, l2, 0.0)
        ref.append(H)
        R = hmg.HMatrix(n, n, dim)
        R.set_points(0, p)
        R.set_points(1, p)
        R.set_kernel(hmg.KERNEL_GAUSSIAN, l2, 0.0)
        raw.append(R)
        leaf.append(c)
    G0 = hmg.group(ref)
    G1 = hmg.group_setup(raw, 1.5, leaf, rule=1)
    for a, b in zip(G1.blocks(), G0.blocks()):
        np.testing.assert_array_equal(a, b)
    for w in (0, 1):
        np.testing.assert_array_equal(G1.order(w), G0.order(w))
    for G in (G0, G1):
        G.precompute_aca(32, 1e-5, 1)
        G.precompute_dense(1)
    x = np.random.default_rng(8).uniform(-1, 1, G0.n2)
    np.testing.assert_array_equal(G1.matvec(x), G0.matvec(x))
    for H in ref + raw:
        H.close()
    G0.close()
    G1.close()


def test_group_setup_errors(hmg, cuda):
    raw, leaf = _raw_sets(hmg, [500, 800])
    with pytest.raises(ValueError):
        hmg.group_setup(raw, 1.5, [64])
    with pytest.raises(hmg.HmgError):
        hmg.group_setup(raw, 1.5, [64, 0])
    with pytest.raises(hmg.HmgError):
        hmg.group_setup(raw, -1.0, leaf)
    bare = hmg.HMatrix(300, 300, 3)  # no points, no kernel
    with pytest.raises(hmg.HmgError):
        hmg.group_setup(raw + [bare], 1.5, leaf + [128])
    other = hmg.HMatrix(300, 300, 3)
    p = make_points("uniform", 300, 3, 9)
    other.set_points(0, p)
    other.set_points(1, p)
    other.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)  # another kernel kind
    with pytest.raises(hmg.HmgError):
        hmg.group_setup(raw + [other], 1.5, leaf + [128])
    for H in raw + [bare, other]:
        H.close()


def test_group_setup_one_set(hmg, cuda):
    """A group of one set: the same tree as hmg_setup on that set alone."""
    raw, leaf = _raw_sets(hmg, [6000])
    G = hmg.group_setup(raw, 1.5, leaf, rule=1)
    ref = _sets(hmg, [6000])[0]
    for a, b in zip(G.blocks(), ref.blocks()):
        np.testing.assert_array_equal(a, b)
    for w in (0, 1):
        np.testing.assert_array_equal(G.order(w), ref.order(w))
        np.testing.assert_array_equal(G.codes(w), ref.codes(w))
    assert G.info()["levels"] == ref.info()["levels"]
    for H in raw + [ref]:
        H.close()
    G.close()


def test_group_setup_rectangular(hmg, cuda):
    """Sets whose rows and columns are different point clouds (n1 != n2), one of them
    on a line: grouped setup against per-set setup, on the blocks, both orders and one
    product."""
    shapes = [(3000, 1200), (700, 2500), (4096, 4000), (90, 300)]
    rng = np.random.default_rng(11)
    ref, raw, leaf = [], [], []
    for i, (n1, n2) in enumerate(shapes):
        dim = 3 if i % 2 == 0 else 2
        # the last set lies on a line: max == min in every dimension but the first
        gen = "line" if i == len(shapes) - 1 else "uniform"
        p1 = make_points(gen, n1, dim, 500 + i)
        p2 = make_points(gen, n2, dim, 600 + i)
        l2 = float(rng.uniform(0.01, 0.2))
        c = 64 if dim == 2 else 128
        H = engine(hmg, p1, p2, 1.5, c, rule=1)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, l2, 0.0)
        ref.append(H)
        R = hmg.HMatrix(n1, n2, dim)
        R.set_points(0, p1)
        R.set_points(1, p2)
        R.set_kernel(hmg.KERNEL_GAUSSIAN, l2, 0.0)
        raw.append(R)
        leaf.append(c)
    G0 = hmg.group(ref)
    G1 = hmg.group_setup(raw, 1.5, leaf, rule=1)
    np.testing.assert_array_equal(G1.offsets(1), G0.offsets(1))
    for a, b in zip(G1.blocks(), G0.blocks()):
        np.testing.assert_array_equal(a, b)
    for w in (0, 1):
        np.testing.assert_array_equal(G1.order(w), G0.order(w))
    for G in (G0, G1):
        G.precompute_aca(64, 1e-6, 1)
        G.precompute_dense(1)
    x = np.random.default_rng(12).uniform(-1, 1, G0.n2)
    np.testing.assert_array_equal(G1.matvec(x), G0.matvec(x))
    for H in ref + raw:
        H.close()
    G0.close()
    G1.close()


@pytest.mark.parametrize("max_level", [1, 3, 6])
def test_group_setup_max_level(hmg, cuda, max_level):
    """A level cap: the traversal's last level turns every remaining node into a leaf,
    for all sets at once; the trees equal those of per-set setups with the same cap."""
    sizes = [3000, 5000, 800]
    ref = []
    rng = np.random.default_rng(3)
    for i, n in enumerate(sizes):
        dim = 2 if i % 2 == 0 else 3
        p = make_points("uniform", n, dim, 3 * 1000 + i)
        H = engine(hmg, p, p, 1.5, 64 if dim == 2 else 128, rule=1, max_level=max_level)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, float(rng.uniform(0.01, 0.2)), 0.0)
        ref.append(H)
    G0 = hmg.group(ref)
    raw, leaf = _raw_sets(hmg, sizes)
    G1 = hmg.group_setup(raw, 1.5, leaf, max_level=max_level, rule=1)
    for a, b in zip(G1.blocks(), G0.blocks()):
        np.testing.assert_array_equal(a, b)
    assert G1.info()["levels"] == G0.info()["levels"] <= max_level
    for H in ref + raw:
        H.close()
    G0.close()
    G1.close()

"""Setup path on the GPU: Morton codes, Z-order permutation and block-cluster tree must
be bit-exact against the oracle and against the reference's own build (golden
fixtures).  Reference: morton.cu:21-112, helper.cu:108-167,293-328, tree.cu:40-160,
215-447,1429-1557, linear_algebra.cu:63-86."""
import numpy as np
import pytest

from helpers import bits_for, engine, make_points, oracle_setup
from conftest import golden

pytestmark = pytest.mark.gpu

CASES = [
    # gen, n1, n2, dim, seed, eta, c_leaf, rule
    ("uniform", 16384, 16384, 2, 0, 1.5, 64, 0),
    ("uniform", 16384, 16384, 2, 0, 1.5, 64, 1),
    ("uniform", 20000, 20000, 3, 1, 1.5, 128, 1),
    ("gmm", 30000, 30000, 2, 2, 1.0, 32, 0),
    ("uniform", 1000, 777, 2, 7, 0.8, 16, 0),
    ("lattice", 4096, 4096, 2, 0, 1.0, 8, 0),
    ("lattice", 3375, 3375, 3, 0, 1.5, 10, 0),
    ("uniform", 50, 50, 3, 3, 1.5, 64, 0),     # a single dense block
    ("line", 5000, 5000, 3, 5, 1.5, 16, 0),    # degenerate dimensions (max == min)
    ("uniform", 1, 1, 2, 4, 1.5, 1, 0),        # one point
    # the batching workload's tree: N = 2^20 uniform 3D, leaf 128, eta 1.5, min rule
    # (1,661,755 blocks, 15 levels, more than 2^16 radix tiles)
    ("uniform", 1 << 20, 1 << 20, 3, 1, 1.5, 128, 1),
]


def _check_against_oracle(hmg, O, gen, n1, n2, dim, seed, eta, c_leaf, rule):
    p1 = make_points(gen, n1, dim, seed)
    p2 = p1 if n2 == n1 else make_points(gen, n2, dim, seed + 100)
    H = engine(hmg, p1, p2, eta, c_leaf, rule=rule)
    ref = oracle_setup(O, p1, p2, eta, c_leaf, rule=rule)
    np.testing.assert_array_equal(H.codes(0), ref["codes1"])
    np.testing.assert_array_equal(H.codes(1), ref["codes2"])
    np.testing.assert_array_equal(H.order(0), ref["order1"])
    np.testing.assert_array_equal(H.order(1), ref["order2"])
    np.testing.assert_array_equal(H.points(0), ref["z1"])
    s1l, s1u, s2l, s2u, typ = H.blocks()
    b = ref["blocks"]
    assert len(s1l) == len(b)
    np.testing.assert_array_equal(s1l, b.s1l)
    np.testing.assert_array_equal(s1u, b.s1u)
    np.testing.assert_array_equal(s2l, b.s2l)
    np.testing.assert_array_equal(s2u, b.s2u)
    np.testing.assert_array_equal(typ, b.type)
    info = H.info()
    assert info["dense_count"] == int((b.type == 2).sum())
    assert info["levels"] == b.levels
    H.close()


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}x{c[2]}-d{c[3]}-r{c[7]}" for c in CASES])
def test_setup_bit_exact_vs_oracle(hmg, oracle, cuda, case):
    _check_against_oracle(hmg, oracle, *case)


GOLDEN = ["config1_parity", "uniform3d_matern", "rect2d", "lattice_dups",
          "kat_lattice2d", "kat_lattice3d"]


@pytest.mark.parametrize("name", GOLDEN)
def test_setup_bit_exact_vs_reference(hmg, cuda, name):
    """Codes, permutation and work-item list equal the reference GPU build's."""
    from golden.make_golden import CASES as GC, case_inputs
    g = golden(name)
    c = GC[name]
    p1, p2, _ = case_inputs(c)
    H = engine(hmg, p1, p2, c["eta"], c["c_leaf"], rule=0)
    np.testing.assert_array_equal(H.codes(0), g["codes1"])
    np.testing.assert_array_equal(H.codes(1), g["codes2"])
    np.testing.assert_array_equal(H.order(0), g["order1"])
    np.testing.assert_array_equal(H.order(1), g["order2"])
    s1l, s1u, s2l, s2u, typ = H.blocks()
    ours = np.stack([s1l, s1u, s2l, s2u, typ], 1)
    np.testing.assert_array_equal(ours, g["blocks"])
    assert H.info()["dense_count"] == int(g["dense_count"])
    H.close()


@pytest.mark.parametrize("n,key_bits,distinct", [(0, 64, 10), (1, 64, 10), (4095, 64, 7),
                                                 (100000, 64, 1 << 62), (262144, 20, 1000),
                                                 (300001, 35, 50), (65536, 64, 1)])
def test_radix_sort_stable(hmg, cuda, n, key_bits, distinct):
    torch = cuda
    rng = np.random.default_rng(n + key_bits)
    keys = rng.integers(0, min(distinct, 1 << min(key_bits, 62)), size=n, dtype=np.int64).astype(np.uint64)
    if key_bits == 64 and distinct > (1 << 40):
        keys |= rng.integers(0, 2, size=n, dtype=np.int64).astype(np.uint64) << np.uint64(63)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    hmg.radix_sort_u64(dk.data_ptr(), dv.data_ptr(), n, key_bits)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


def test_morton_primitive_matches_oracle(hmg, oracle, cuda):
    torch = cuda
    for dim in (2, 3):
        p = make_points("gmm", 5000, dim, 9)
        d = torch.from_numpy(p).cuda()
        out = torch.empty(p.shape[1], dtype=torch.int64, device="cuda")
        hmg.morton_codes(d.data_ptr(), p.shape[1], dim, bits_for(dim), out.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), oracle.morton(p, bits_for(dim)))

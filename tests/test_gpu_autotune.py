"""hmg_autotune: it times the product's V^T task sizes and grids on the handle and
keeps the fastest; the product is bit-identical whatever it chose (a term's row sum
does not depend on how terms are grouped into tasks or on the grid).  No reference
counterpart."""
import numpy as np
import pytest

from helpers import engine, make_points

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [1, 2], ids=["fp32", "mixed"])
def test_autotune_keeps_the_product(hmg, cuda, prec):
    n = 30000
    p = make_points("uniform", n, 3, 41)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(96, 1e-8, prec)
    H.precompute_dense(hmg.PREC_FP32)
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y0 = H.matvec(x)
    t = H.autotune(reps=2)
    assert t["piece_bytes"] in (32768, 65536, 131072) and t["ctas_per_sm"] in (4, 8, 16) and t["ms"] > 0
    np.testing.assert_array_equal(H.matvec(x), y0)
    with pytest.raises(hmg.HmgError):
        H.autotune(reps=0)
    H.close()

"""H-matrices on disk (hmg_save / hmg_load): a loaded H-matrix has the saved one's
tree, ranks and factors and multiplies bit-identically.  No reference counterpart
(the reference only prints its tree, tree.cu:173-183)."""
import numpy as np
import pytest

from helpers import engine, make_points

pytestmark = pytest.mark.gpu


def _same(H, G, x):
    for w in (0, 1):
        np.testing.assert_array_equal(H.codes(w), G.codes(w))
        np.testing.assert_array_equal(H.order(w), G.order(w))
    for a, b in zip(H.blocks(), G.blocks()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(H.ranks(), G.ranks())
    np.testing.assert_array_equal(H.matvec(x), G.matvec(x))
    hi, gi = H.info(), G.info()
    for k in ("far_bytes", "near_bytes", "far_u_bytes", "far_v_bytes", "matvec_bytes", "max_rank", "tile_count"):
        assert hi[k] == gi[k], k


@pytest.mark.parametrize("prec,dense", [(0, True), (1, True), (2, True), (1, False)],
                         ids=["fp64", "fp32", "mixed", "fp32-onthefly"])
def test_save_load_roundtrip(hmg, cuda, tmp_path, prec, dense):
    p = make_points("uniform", 20000, 3, 11)
    H = engine(hmg, p, p, 1.5, 128, rule=1)
    H.set_kernel(hmg.KERNEL_MATERN32, 0.2, 0.0)
    H.precompute_aca(64, 1e-8, prec)
    if dense:
        H.precompute_dense(hmg.PREC_FP64 if prec == 0 else hmg.PREC_FP32)
    path = tmp_path / "h.hmg"
    H.save(str(path))
    G = hmg.load(str(path))
    x = np.random.default_rng(1).uniform(-1, 1, 20000)
    _same(H, G, x)
    H.close()
    G.close()


def test_group_roundtrip_and_bad_files(hmg, cuda, tmp_path):
    sets = []
    for i, n in enumerate([3000, 5000, 1200]):
        dim = 2 + i % 2
        p = make_points("uniform", n, dim, 20 + i)
        H = engine(hmg, p, p, 1.5, 64, rule=1)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05 * (i + 1), 0.0)
        sets.append(H)
    G = hmg.group(sets)
    G.precompute_aca(64, 1e-6, hmg.PREC_FP32)
    G.precompute_dense(hmg.PREC_FP32)
    path = tmp_path / "g.hmg"
    G.save(str(path))
    L = hmg.load(str(path))
    x = np.random.default_rng(2).uniform(-1, 1, G.n2)
    np.testing.assert_array_equal(G.matvec(x), L.matvec(x))
    assert L.info()["group_count"] == 3
    np.testing.assert_array_equal(L.offsets(0), G.offsets(0))
    # truncated and foreign files are refused, not read past their end
    raw = path.read_bytes()
    (tmp_path / "short.hmg").write_bytes(raw[: len(raw) // 2])
    (tmp_path / "junk.hmg").write_bytes(b"not an h-matrix" * 10)
    for bad in ("short.hmg", "junk.hmg", "missing.hmg"):
        with pytest.raises(hmg.HmgError):
            hmg.load(str(tmp_path / bad))
    for H in sets + [G, L]:
        H.close()

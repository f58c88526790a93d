"""hmg_load refuses files whose metadata would make a product read or write outside
its buffers: block ranges outside the matrix, factor slices outside their
allocation, near-field slices outside the near field, a broken permutation, a
truncated file.  Every refusal happens on the host before anything is copied to the
device, and no product runs on a refused file."""
import struct

import numpy as np
import pytest

from helpers import engine, hmg_file_layout, make_points

pytestmark = pytest.mark.gpu


def _saved(hmg, tmp_path):
    p = make_points("uniform", 6000, 2, 5)
    H = engine(hmg, p, p, 1.5, 32, rule=1)
    H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05, 0.0)
    H.precompute_aca(32, 1e-6, hmg.PREC_MIXED)
    H.precompute_dense(hmg.PREC_FP32)
    path = tmp_path / "h.hmg"
    H.save(str(path))
    ranks = H.ranks()
    H.close()
    return path, path.read_bytes(), ranks


def _refused(hmg, path, buf, words):
    bad = bytearray(buf)
    for off, fmt, val in words:
        struct.pack_into(fmt, bad, off, val)
    q = path.with_name("bad.hmg")
    q.write_bytes(bytes(bad))
    with pytest.raises(hmg.HmgError) as e:
        hmg.load(str(q))
    assert e.value.status == 1, str(e.value)  # HMG_ERR_INVALID
    return str(e.value)


def test_load_refuses_corrupt_files(hmg, cuda, tmp_path):
    path, buf, ranks = _saved(hmg, tmp_path)
    L = hmg_file_layout(buf)
    n1 = L["n"][0]
    nd, nb = L["ndense"], L["nblocks"]
    b = nd + int(np.argmax(ranks[nd:] > 0))  # an admissible block with factors
    # a block range past the last row
    msg = _refused(hmg, path, buf, [(L["blocks"]["m1"] + 4 * b, "<i", n1 + 1)])
    assert "outside" in msg
    # a negative column start
    _refused(hmg, path, buf, [(L["blocks"]["c0"] + 4 * 3, "<i", -1)])
    # a dense block typed as admissible
    _refused(hmg, path, buf, [(L["blocks"]["type"], "<i", 1)])
    # the U slice of block b moved past the end of its allocation
    msg = _refused(hmg, path, buf, [(L["place"] + 24 * b + 8, "<q", 1 << 40)])
    assert "allocation" in msg
    # a factor allocation index that does not exist
    _refused(hmg, path, buf, [(L["place"] + 24 * b, "<q", L["nchunks"])])
    # a rank above the block's size, a tier split that is not the format's
    _refused(hmg, path, buf, [(L["rank"] + 4 * b, "<i", 100000)])
    _refused(hmg, path, buf, [(L["rank"] + 4 * nb + 4 * b, "<i", -3)])
    # a dense block's near-field slice past the end of the near field
    msg = _refused(hmg, path, buf, [(L["near_off"] + 8 * (nd - 1), "<q", 1 << 40)])
    assert "near field" in msg
    # two points mapped to one
    _refused(hmg, path, buf, [(L["perm"][0], "<i", 1), (L["perm"][0] + 4, "<i", 1)])
    # a negative block count in the header
    _refused(hmg, path, buf, [(16 + 40, "<i", -5)])
    # truncated files
    for cut in (len(buf) // 3, len(buf) - 1):
        q = path.with_name("cut.hmg")
        q.write_bytes(buf[:cut])
        with pytest.raises(hmg.HmgError):
            hmg.load(str(q))
    # the unmodified file still loads and multiplies
    G = hmg.load(str(path))
    y = G.matvec(np.ones(n1))
    assert np.isfinite(y).all()
    G.close()

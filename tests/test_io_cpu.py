"""hmg_load checks a file on the host before it touches a device (no GPU needed).

tests/golden/small_mixed.hmg.gz is a real file written by hmg_save
(tests/golden/make_hmg_fixture.py).  Unmodified, it passes every check, so on a
machine without a GPU the load gets as far as creating the device handle and fails
there (HMG_ERR_CUDA); with a GPU it loads.  Each corruption below must instead be
refused as HMG_ERR_INVALID, which proves the refusal came from the host-side checks
that run before any device allocation or copy."""
import gzip
import os
import struct

import pytest

from helpers import hmg_file_layout

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_mixed.hmg.gz")
INVALID, CUDA = 1, 2


@pytest.fixture(scope="module")
def saved(tmp_path_factory):
    buf = gzip.open(FIXTURE, "rb").read()
    return tmp_path_factory.mktemp("hmg"), buf


def _status(hmg, path):
    try:
        H = hmg.load(str(path))
    except hmg.HmgError as e:
        return e.status, str(e)
    H.close()
    return 0, ""


def _corrupt(d, buf, words, name="bad.hmg"):
    bad = bytearray(buf)
    for off, fmt, val in words:
        struct.pack_into(fmt, bad, off, val)
    p = d / name
    p.write_bytes(bytes(bad))
    return p


def test_fixture_passes_host_checks(hmg, saved):
    d, buf = saved
    L = hmg_file_layout(buf)
    assert L["header_bytes"] == 192 and L["far_prec"] == 2 and L["near_prec"] == 1
    p = d / "good.hmg"
    p.write_bytes(buf)
    st, msg = _status(hmg, p)
    assert st in (0, CUDA), msg


def test_corrupt_fields_are_refused_on_the_host(hmg, saved):
    d, buf = saved
    L = hmg_file_layout(buf)
    n1, nb, nd = L["n"][0], L["nblocks"], L["ndense"]
    ranks = struct.unpack_from(f"<{nb}i", buf, L["rank"])
    b = next(i for i in range(nd, nb) if ranks[i] > 0)
    cases = {
        "block rows past the end": [(L["blocks"]["m1"] + 4 * b, "<i", n1 + 1)],
        "negative block start": [(L["blocks"]["r0"] + 4 * 2, "<i", -7)],
        "empty block": [(L["blocks"]["m2"] + 4 * 1, "<i", 0)],
        "dense block typed admissible": [(L["blocks"]["type"], "<i", 1)],
        "U slice outside its allocation": [(L["place"] + 24 * b + 8, "<q", 1 << 40)],
        "V slice outside its allocation": [(L["place"] + 24 * b + 16, "<q", -16)],
        "unaligned U slice": [(L["place"] + 24 * b + 8, "<q", 4)],
        "missing allocation": [(L["place"] + 24 * b, "<q", 99)],
        "rank above block size": [(L["rank"] + 4 * b, "<i", 10 ** 6)],
        "tier split": [(L["rank"] + 4 * nb + 4 * b, "<i", ranks[b] + 1)],
        "near slice outside": [(L["near_off"] + 8 * (nd - 1), "<q", 1 << 40)],
        "broken permutation": [(L["perm"][0], "<i", 1), (L["perm"][0] + 4, "<i", 1)],
        "negative block count": [(16 + 40, "<i", -5)],
        "dense count above block count": [(16 + 44, "<i", nb + 1)],
        "unknown precision": [(16 + 92, "<i", 9)],
    }
    for what, words in cases.items():
        st, msg = _status(hmg, _corrupt(d, buf, words))
        assert st == INVALID, (what, st, msg)
    # truncated anywhere after the header
    for cut in (300, len(buf) // 2, len(buf) - 1):
        p = d / "cut.hmg"
        p.write_bytes(buf[:cut])
        st, msg = _status(hmg, p)
        assert st == INVALID, (cut, st, msg)

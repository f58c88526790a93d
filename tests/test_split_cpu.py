"""The BF16 parts of split tensor-core operands (tc.cu store_parts, k_tc_x and the t_b
epilogue): part 0 is the round-to-nearest BF16 of an FP32 value, part p the BF16 of
what parts 0..p-1 miss.  Each difference is exact in FP32, two parts keep 16
significant bits, and three parts give back every FP32 value exactly.  Checked with
torch's CPU bfloat16, which rounds to nearest-even like __float2bfloat16_rn.  No
reference counterpart."""
import numpy as np
import pytest


def _parts(v, n):
    import torch
    r = torch.from_numpy(v)
    out = []
    for _ in range(n):
        p = r.to(torch.bfloat16).to(torch.float32)
        out.append(p.numpy().astype(np.float64))
        r = r - p  # exact: p is r rounded to 8 significant bits
    return out, r.numpy()


@pytest.fixture(scope="module")
def values():
    rng = np.random.default_rng(5)
    mag = 10.0 ** rng.uniform(-30, 30, 200000)
    v = (mag * rng.choice([-1.0, 1.0], mag.size)).astype(np.float32)
    # values of every significand pattern near 1, and exact powers of two
    v = np.concatenate([v, (1.0 + np.arange(1 << 16, dtype=np.float64) / (1 << 16)).astype(np.float32),
                        np.float32(2.0) ** np.arange(-100, 100).astype(np.float32)])
    return v


def test_three_parts_rebuild_fp32_exactly(values):
    parts, rest = _parts(values, 3)
    np.testing.assert_array_equal(parts[0] + parts[1] + parts[2], values.astype(np.float64))
    assert not rest.any()


def test_differences_are_exact_and_two_parts_keep_16_bits(values):
    v = values.astype(np.float64)
    parts, rest = _parts(values, 2)
    # the FP32 residual equals the exact difference
    np.testing.assert_array_equal(v - parts[0] - parts[1], rest.astype(np.float64))
    rel = np.abs(rest.astype(np.float64)) / np.abs(v)
    assert rel.max() <= 2.0 ** -16
    one, _ = _parts(values, 1)
    assert (np.abs(v - one[0]) / np.abs(v)).max() <= 2.0 ** -8

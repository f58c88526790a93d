"""Writes tests/golden/small_mixed.hmg.gz: a small H-matrix saved by hmg_save
(format version 1), gzip-compressed, the input of the host-side checks of hmg_load
in tests/test_io_cpu.py.

    python tests/golden/make_hmg_fixture.py OUT_PATH.hmg.gz      (needs a GPU)

The H-matrix: 256 points uniform in [0,1]^2 (seed 5), leaf 8, eta 1.5, min rule,
Gaussian kernel length^2 0.05, adaptive ACA eps 1e-4 rank <= 16 in mixed storage,
FP32 near field stored."""
from __future__ import annotations

import gzip
import os
import shutil
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import hmglib_b200 as hmg  # noqa: E402
from hmglib_b200 import synth  # noqa: E402


def main(out: str) -> None:
    p = synth.uniform_points(256, 2, 5)
    H = hmg.HMatrix(256, 256, 2)
    H.set_points(0, p)
    H.set_points(1, p)
    H.setup(1.5, 8, rule=hmg.ADMISSIBLE_MIN)
    H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05, 0.0)
    H.precompute_aca(16, 1e-4, hmg.PREC_MIXED)
    H.precompute_dense(hmg.PREC_FP32)
    raw = out[:-3] if out.endswith(".gz") else out
    H.save(raw)
    if raw != out:
        with open(raw, "rb") as f, gzip.open(out, "wb", compresslevel=9) as g:
            shutil.copyfileobj(f, g)
        os.remove(raw)
    i = H.info()
    print(out, os.path.getsize(out), "bytes:", i["block_count"], "blocks,", i["dense_count"], "dense")
    H.close()


if __name__ == "__main__":
    main(sys.argv[1])

"""The reference's own entry points (include/hmglib.h) driven by a C++ program
written against them, like the reference's hmglib_test.cu: it compiles against the
drop-in headers, links libhmg.so and reproduces the FP64 results."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="module")
def driver(hmg, tmp_path_factory):
    out = tmp_path_factory.mktemp("legacy") / "legacy_driver"
    libdir = os.path.join(ROOT, "hmglib_b200")
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "legacy_driver.cu"), "-o", str(out), "-L", libdir, "-lhmg",
                    "-Xlinker", f"-rpath,{libdir}"], check=True)
    return str(out)


@pytest.mark.parametrize("n,k,leaf,eta,dense,bound", [(16384, 64, 64, 1.5, 1, 1e-4),
                                                      (8192, 16, 32, 1.0, 0, 1e-3),
                                                      (500, 8, 600, 1.5, 1, 1e-14)])
def test_reference_style_driver(cuda, driver, n, k, leaf, eta, dense, bound):
    r = subprocess.run([driver, str(n), str(k), str(leaf), str(eta), str(dense), str(bound)],
                       capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, r.stdout + r.stderr
    d = json.loads(line[-1])
    assert r.returncode == 0, d
    assert d["rel_err"] < bound and d["x_unchanged"] and d["codes_sorted"] and d["order_is_permutation"]
    assert d["dense"] + d["aca"] == d["blocks"]

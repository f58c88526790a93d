"""Golden fixtures from kadircs/hmglib's own GPU build.

Two steps, because the reference only runs on a GPU and its sources only exist
where it was built:

1. here (with the reference checkout):  ``oracle/refbuild/build_ref.sh``
   builds ``oracle/_ref/ref_dump`` (the reference's sources + a MAGMA stand-in +
   a dump driver, sm_100a);
2. on a B200:  ``python tests/golden/make_golden.py run --ref oracle/_ref/ref_dump
   --out RAW_DIR`` writes the inputs of every case below, runs the reference on
   each and keeps its raw outputs in RAW_DIR;
3. with RAW_DIR copied back:  ``python tests/golden/make_golden.py pack --raw
   RAW_DIR`` converts the raw outputs into ``tests/golden/<case>.npz`` (inputs are
   not stored: they are regenerated from the seeds in CASES).

Each fixture holds the reference's sorted Morton codes, its permutation
(``order``), its work-item list after organize_mat_vec_data (bounds inclusive,
work type), ``apply_h_matrix_mvp``'s y and ``apply_full_mvp``'s y.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from hmglib_b200 import synth  # noqa: E402

GOLDEN = os.path.dirname(os.path.abspath(__file__))


def lattice(nx, dim, dup=1):
    g = np.stack(np.meshgrid(*[np.arange(nx, dtype=np.float64)] * dim, indexing="ij"), 0)
    pts = g.reshape(dim, -1)
    return np.ascontiguousarray(np.repeat(pts, dup, axis=1))


# name -> parameters; kernel 1 = the reference's exp(-r^2), 2 = its Bessel-Y "matern"
CASES = {
    # the plain-method workload: N=16384 uniform in [0,1]^2 (seed 0), exp(-r^2/0.1)
    # emulated by scaling coordinates by 1/sqrt(0.1), leaf 64, eta 1.5, rank 64
    "config1_parity": dict(n1=16384, dim=2, gen="uniform", seed=0, scale=0.1 ** -0.5, kernel=1,
                           c_leaf=64, eta=1.5, k=64, pre_dense=1, n_apply=5),
    "uniform3d_matern": dict(n1=8192, dim=3, gen="uniform", seed=5, scale=1.0, kernel=2,
                             c_leaf=64, eta=1.5, k=16, pre_dense=1, n_apply=3),
    # The reference's own build fails on this clustered set: setup_h_matrix exits with
    # "cudaMemcpy12ja: invalid argument" -- single-point clusters (levels 6 and 8 here)
    # collide in its bounding-box lookup keys (tree.cu:1004-1022, 1061-1063).  Kept
    # so the failure can be reproduced; no fixture is packed for it.
    "gmm2d": dict(n1=4096, dim=2, gen="gmm", seed=2, scale=0.05 ** -0.5, kernel=1,
                  c_leaf=32, eta=1.0, k=16, pre_dense=0, n_apply=3, reference_fails=True),
    "rect2d": dict(n1=1000, n2=700, dim=2, gen="uniform", seed=11, seed2=12, scale=3.0, kernel=1,
                   c_leaf=16, eta=0.8, k=8, pre_dense=1, n_apply=3),
    "lattice_dups": dict(n1=2048, dim=2, gen="lattice", nx=32, dup=2, scale=1.0 / 8.0, kernel=1,
                         c_leaf=8, eta=1.0, k=4, pre_dense=1, n_apply=3),
    # the 4x4 and 4x4x4 integer lattices of helper.cu:261-291
    "kat_lattice2d": dict(n1=16, dim=2, gen="lattice", nx=4, dup=1, scale=1.0, kernel=1,
                          c_leaf=2, eta=1.5, k=2, pre_dense=1, n_apply=1),
    "kat_lattice3d": dict(n1=64, dim=3, gen="lattice", nx=4, dup=1, scale=1.0, kernel=1,
                          c_leaf=2, eta=1.5, k=2, pre_dense=1, n_apply=1),
}


def case_inputs(c):
    """(coords1, coords2, x) exactly as fed to the reference (coords already scaled)."""
    dim = c["dim"]
    n1 = c["n1"]
    n2 = c.get("n2", n1)
    if c["gen"] == "uniform":
        p1 = synth.uniform_points(n1, dim, c["seed"])
        p2 = synth.uniform_points(n2, dim, c["seed2"]) if "seed2" in c else p1
    elif c["gen"] == "gmm":
        p1 = synth.gmm_points(n1, dim, c["seed"])
        p2 = p1
    else:
        p1 = lattice(c["nx"], dim, c["dup"])
        p2 = p1
    s = c["scale"]
    p1 = np.ascontiguousarray(p1 * s)
    p2 = np.ascontiguousarray(p2 * s)
    x = synth.rhs_vector(n2, c.get("seed", 0))
    return p1, p2, x


def write_input(c, path):
    p1, p2, x = case_inputs(c)
    dim = c["dim"]
    bits = 32 if dim == 2 else 20
    hdr = np.array([p1.shape[1], p2.shape[1], dim, bits, c["c_leaf"], c["k"], c["kernel"], 50,
                    c["pre_dense"], c["n_apply"]], dtype=np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.array([c["eta"]], dtype=np.float64).tobytes())
        f.write(p1.tobytes())
        f.write(p2.tobytes())
        f.write(x.tobytes())


def read_output(path):
    raw = open(path, "rb").read()
    n1, n2, nd, na = np.frombuffer(raw[:16], dtype=np.int32)
    o = 16
    def take(dt, cnt):
        nonlocal o
        a = np.frombuffer(raw[o:o + cnt * np.dtype(dt).itemsize], dtype=dt).copy()
        o += cnt * np.dtype(dt).itemsize
        return a
    codes1 = take(np.uint64, n1); codes2 = take(np.uint64, n2)
    order1 = take(np.uint64, n1); order2 = take(np.uint64, n2)
    nb = nd + na
    blocks = take(np.int32, nb * 5).reshape(nb, 5)
    yh = take(np.float64, n1); yf = take(np.float64, n1)
    t = take(np.float64, 5)
    d = dict(codes1=codes1, codes2=codes2, order1=order1.astype(np.int64),
             order2=order2.astype(np.int64), blocks=blocks, dense_count=np.int32(nd),
             y_h=yh, y_full=yf, timings_ms=t)
    if len(raw) - o >= 8 * n1:
        d["y_h2"] = take(np.float64, n1)  # a second precompute_aca + product
    return d


def cmd_run(a):
    os.makedirs(a.out, exist_ok=True)
    summary = {}
    for name, c in CASES.items():
        if a.only and name not in a.only:
            continue
        inp = os.path.join(a.out, name + ".in.bin")
        out = os.path.join(a.out, name + ".out.bin")
        write_input(c, inp)
        r = subprocess.run([a.ref, inp, out], capture_output=True, text=True, timeout=900)
        line = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else ""
        summary[name] = {"rc": r.returncode, "stdout_tail": line, "stderr_tail": r.stderr[-400:]}
        os.remove(inp)
        print(name, r.returncode, line, flush=True)
    json.dump(summary, open(os.path.join(a.out, "summary.json"), "w"), indent=1)
    return 0 if all(v["rc"] == 0 for v in summary.values()) else 1


def cmd_pack(a):
    for name in CASES:
        out = os.path.join(a.raw, name + ".out.bin")
        if not os.path.exists(out):
            print("missing", name)
            continue
        d = read_output(out)
        np.savez_compressed(os.path.join(GOLDEN, name + ".npz"), **d)
        print("packed", name, {k: getattr(v, "shape", v) for k, v in d.items()})


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("--ref", default=os.path.join(ROOT, "oracle", "_ref", "ref_dump"))
    r.add_argument("--out", required=True)
    r.add_argument("--only", nargs="*")
    p = sub.add_parser("pack")
    p.add_argument("--raw", required=True)
    a = ap.parse_args(argv)
    return cmd_run(a) if a.cmd == "run" else cmd_pack(a)


if __name__ == "__main__":
    sys.exit(main())

"""Shared helpers of the parity tests: one workload description, built both by the
engine (through the C ABI) and by the CPU oracle."""
from __future__ import annotations

import numpy as np

from hmglib_b200 import synth


def make_points(gen, n, dim, seed, scale=1.0):
    if gen == "uniform":
        p = synth.uniform_points(n, dim, seed)
    elif gen == "gmm":
        p = synth.gmm_points(n, dim, seed)
    elif gen == "line":
        # all points share every coordinate but the first (max == min in those dimensions)
        p = np.full((dim, n), 0.5)
        p[0] = synth.uniform01(seed, n)
    elif gen == "lattice":
        nx = int(round(n ** (1.0 / dim)))
        g = np.stack(np.meshgrid(*[np.arange(nx, dtype=np.float64)] * dim, indexing="ij"), 0)
        p = g.reshape(dim, -1)
        p = np.repeat(p, max(1, n // p.shape[1]), axis=1)[:, :n]
    else:
        raise ValueError(gen)
    return np.ascontiguousarray(p * scale)


def bits_for(dim):
    return 32 if dim == 2 else 20


def engine(hmg, p1, p2, eta, c_leaf, rule=0, max_level=50):
    dim = p1.shape[0]
    H = hmg.HMatrix(p1.shape[1], p2.shape[1], dim)
    H.set_points(0, p1)
    H.set_points(1, p2)
    H.setup(eta, c_leaf, max_level=max_level, rule=rule)
    return H


def oracle_setup(O, p1, p2, eta, c_leaf, rule=0, max_level=50):
    dim = p1.shape[0]
    s1, o1, z1 = O.order_points(p1, bits_for(dim))
    s2, o2, z2 = O.order_points(p2, bits_for(dim))
    blocks = O.tree(z1, s1, z2, s2, eta, c_leaf, max_level=max_level, rule=rule)
    return dict(codes1=s1, order1=o1, z1=z1, codes2=s2, order2=o2, z2=z2, blocks=blocks)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fp64_rows(torch, H, x, rows):
    """FP64 direct sums (K x)[rows] on the GPU (hmg_full_matvec_rows); x a device
    vector in caller order, rows a host int array."""
    r = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int32)).cuda()
    y = torch.empty(len(rows), dtype=torch.float64, device="cuda")
    H.full_matvec_rows(x, r, y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def hmg_file_layout(buf: bytes) -> dict:
    """Byte offsets of the sections of a file written by hmg_save (format version 1,
    csrc/io.cu): magic, u32 version, u32 header bytes, the header struct (fields
    read below at their offsets in it), then per point set pts, zpts, codes, perm,
    iperm; the five int32 block arrays; [group offsets and parameters]; [ranks, two
    tier arrays, allocation sizes, (chunk, U offset, V offset) per block, the
    allocations]; [near-field offsets, near field]."""
    import struct
    hb = struct.unpack_from("<I", buf, 12)[0]
    h = 16
    n1, n2, dim = struct.unpack_from("<3i", buf, h)
    nb, nd = struct.unpack_from("<2i", buf, h + 40)
    gc, far_prec = struct.unpack_from("<2i", buf, h + 88)
    near_prec = struct.unpack_from("<i", buf, h + 112)[0]
    nchunks = struct.unpack_from("<i", buf, h + 172)[0]
    out = dict(header_bytes=hb, n=(n1, n2), dim=dim, nblocks=nb, ndense=nd, far_prec=far_prec,
               near_prec=near_prec, nchunks=nchunks, perm=[], iperm=[])
    o = 16 + hb
    for n in (n1, n2):
        p = o + n * dim * 16 + n * 8
        out["perm"].append(p)
        out["iperm"].append(p + 4 * n)
        o = p + 8 * n
    out["blocks"] = {k: o + i * 4 * nb for i, k in enumerate(("r0", "m1", "c0", "m2", "type"))}
    o += 20 * nb
    if gc:
        o += 8 * (gc + 1) + 8 * nb
    if far_prec >= 0:
        out["rank"] = o
        out["place"] = o + 12 * nb + 8 * nchunks
        cb = struct.unpack_from(f"<{nchunks}q", buf, o + 12 * nb) if nchunks else ()
        o = out["place"] + 24 * nb + sum(cb)
    if near_prec >= 0:
        out["near_off"] = o
    return out

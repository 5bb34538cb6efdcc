"""The reference's binary dataset files: reader, writers and the verification rule.

The reference's test program (main.cpp:62-172) reads three kinds of file, all native-endian
(little-endian here) with 4-byte ints and 8-byte doubles:

* potential file:  int N; x[N], y[N], v[N]; int M; xt[M], yt[M], ref[M]
* velocity file:   the same, followed by ref1[M]; the targets must form 32 x 32-point blocks
                   (M a multiple of 1024), from which the block origins and spacings are taken
                   (main.cpp:148-172), and the reference velocity is (-2 pi ref1, 2 pi ref)
                   (main.cpp:130-141)
* MRAG file:       int N; x[N], y[N], v[N]; int B; x0[B], y0[B], h[B]; the targets are the
                   blocks' points x0 + ix h, y0 + iy h (main.cpp:100-122)

A potential file can also be read as a velocity file when it carries ref1 (main.cpp's
"PV" tests read the same file both ways).  The reference checks every 433rd target from the
8th on against an FP64 direct sum (main.cpp:201-245) with the rule of ``check``
(main.cpp:31-59).
"""
from __future__ import annotations

import math
import struct

import numpy as np

BLOCKSIZE = 32                  # drivers/Makefile:20 of the reference
BS2 = BLOCKSIZE * BLOCKSIZE
SAMPLE_OFFSET, SAMPLE_JUMP = 7, 433   # main.cpp:203-204


class DatasetError(ValueError):
    pass


def _read_int(f):
    b = f.read(4)
    if len(b) != 4:
        raise DatasetError("file ends before a count")
    (n,) = struct.unpack("<i", b)
    if n < 0:
        raise DatasetError(f"negative count {n}")
    return n


def _read_doubles(f, n):
    a = np.fromfile(f, dtype="<f8", count=n)
    if a.size != n:
        raise DatasetError(f"file ends inside an array of {n} doubles")
    return a.astype(np.float64)


def blocks_from_targets(xt, yt):
    """Block origins and spacings of targets laid out as consecutive 32 x 32 blocks
    (main.cpp:148-172): x0 = xt[1024 b], y0 = yt[1024 b], h = xt[1024 b + 1] - xt[1024 b]."""
    m = len(xt)
    if m % BS2:
        raise DatasetError(f"{m} targets are not a whole number of {BLOCKSIZE}x{BLOCKSIZE} blocks")
    first = np.arange(0, m, BS2)
    return xt[first].copy(), yt[first].copy(), xt[first + 1] - xt[first]


def block_targets(x0s, y0s, hs):
    """The targets of MRAG blocks, point (ix, iy) of block b at ix + 32 (iy + 32 b)
    (main.cpp:113-118)."""
    i = np.arange(BLOCKSIZE, dtype=np.float64)
    xt = (x0s[:, None, None] + i[None, None, :] * hs[:, None, None])
    yt = (y0s[:, None, None] + i[None, :, None] * hs[:, None, None])
    shape = (len(x0s), BLOCKSIZE, BLOCKSIZE)
    return np.broadcast_to(xt, shape).reshape(-1).copy(), np.broadcast_to(yt, shape).reshape(-1).copy()


def read(path, kind="potential"):
    """Read a dataset file as main.cpp's test() does.

    kind: 'potential' (the reference potential at every target in ``ref``), 'velocity' (the
    reference velocity in ``uref``, ``vref``; blocks derived from the targets) or 'mrag'
    (blocks read from the file; no reference values).  Returns a dict with xs, ys, vs and,
    as applicable, xt, yt, x0s, y0s, hs, ref, uref, vref."""
    if kind not in ("potential", "velocity", "mrag"):
        raise ValueError(f"unknown dataset kind {kind!r}")
    with open(path, "rb") as f:
        n = _read_int(f)
        out = {"kind": kind, "xs": _read_doubles(f, n), "ys": _read_doubles(f, n),
               "vs": _read_doubles(f, n)}
        m = _read_int(f)
        if kind == "mrag":
            out["x0s"], out["y0s"], out["hs"] = (_read_doubles(f, m) for _ in range(3))
            out["xt"], out["yt"] = block_targets(out["x0s"], out["y0s"], out["hs"])
            return out
        out["xt"], out["yt"] = _read_doubles(f, m), _read_doubles(f, m)
        ref = _read_doubles(f, m)
        if kind == "potential":
            out["ref"] = ref
            return out
        ref1 = _read_doubles(f, m)
        out["uref"], out["vref"] = -ref1 * (2 * math.pi), ref * (2 * math.pi)
        out["x0s"], out["y0s"], out["hs"] = blocks_from_targets(out["xt"], out["yt"])
        return out


def _write(path, ints_and_arrays):
    with open(path, "wb") as f:
        for item in ints_and_arrays:
            if isinstance(item, (int, np.integer)):
                f.write(struct.pack("<i", int(item)))
            else:
                f.write(np.ascontiguousarray(item, dtype="<f8").tobytes())


def write_potential(path, xs, ys, vs, xt, yt, ref, ref1=None):
    """A potential file; with ``ref1`` it also reads as a velocity file."""
    items = [len(xs), xs, ys, vs, len(xt), xt, yt, ref]
    if ref1 is not None:
        items.append(ref1)
    _write(path, items)


def write_mrag(path, xs, ys, vs, x0s, y0s, hs):
    _write(path, [len(xs), xs, ys, vs, len(x0s), x0s, y0s, hs])


def sample_indices(m):
    """The targets main.cpp checks: 7, 7 + 433, ... below m."""
    return np.arange(SAMPLE_OFFSET, m, SAMPLE_JUMP)


def check(ref, res, tol):
    """main.cpp:31-59: element i passes if its relative error err / max(1e-6, max(|res|,
    |ref|)) or its absolute error is below ``tol``.  Returns the error norms the reference
    prints and the failing elements."""
    ref = np.asarray(ref, dtype=np.float64)
    res = np.asarray(res, dtype=np.float64)
    if np.isnan(ref).any() or np.isnan(res).any():
        raise DatasetError("NaN in the values checked")
    err = ref - res
    rel = err / np.maximum(1e-6, np.maximum(np.abs(res), np.abs(ref)))
    bad = np.nonzero((np.abs(rel) >= tol) & (np.abs(err) >= tol))[0]
    return {"ok": bad.size == 0, "linf_abs": float(np.abs(err).max(initial=0.0)),
            "linf_rel": float(np.abs(rel).max(initial=0.0)), "l1_abs": float(np.abs(err).sum()),
            "l1_rel": float(np.abs(rel).sum()), "failures": bad.tolist()}


def direct_potential(xs, ys, vs, xt, yt):
    """main.cpp:205-218 at the given targets: sum_j v_j log sqrt(r^2 + 10 eps) (numpy, for small
    sets)."""
    eps = np.finfo(np.float64).eps * 10
    out = np.empty(len(xt))
    for i, (x, y) in enumerate(zip(xt, yt)):
        xr, yr = x - xs, y - ys
        out[i] = np.sum(np.log(np.sqrt(xr * xr + yr * yr + eps)) * vs)
    return out


def direct_force(xs, ys, vs, xt, yt):
    """main.cpp:221-236 at the given targets: sum_j v_j (xr, yr) / (r^2 + 10 eps)."""
    eps = np.finfo(np.float64).eps * 10
    u = np.empty(len(xt))
    w = np.empty(len(xt))
    for i, (x, y) in enumerate(zip(xt, yt)):
        xr, yr = x - xs, y - ys
        fac = vs / (xr * xr + yr * yr + eps)
        u[i] = np.sum(xr * fac)
        w[i] = np.sum(yr * fac)
    return u, w

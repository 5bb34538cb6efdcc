"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
module, and only as the checker / the timed CPU reference.  It loads the shared objects
that ``oracle/Makefile`` builds into ``oracle/_ref/``:

* ``libref_{potential,force}_{exact64,faithful,big,exact64_big}.so`` -- the reference's own drivers
  (drivers/treecode-potential.cpp, drivers/treecode-force.cpp, drivers/upward.cpp,
  drivers/sort-sources.cpp) compiled verbatim, linked against the restated ISPC kernels
  of ``ispc_kernels.cpp`` and the dump hooks of ``hooks.cpp``;
* ``liboracle_direct.so`` -- the FP64 direct sums of main.cpp:201-245.
"""
from __future__ import annotations

import ctypes
import os
from collections import deque

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

ORDER = {"potential": 12, "force": 24}          # Makefile:13-14 of the reference
LEAF = {"potential": 32 * 16, "force": 192}     # treecode-potential.cpp:99, treecode-force.cpp:216

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_ucp = ctypes.POINTER(ctypes.c_ubyte)
_libs: dict = {}


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"libref_{k}_{m}.so"))
               for k in ("potential", "force") for m in ("exact64", "faithful"))


def lib(kind: str, mode: str = "exact64"):
    """kind: 'potential' | 'force' | 'direct'; mode: 'exact64' | 'faithful' | 'big' (faithful
    kernels, node capacity raised) | 'exact64_big' (EXACT64 kernels, node capacity raised), or
    'exact64_o8' / 'exact64_o16' / 'exact64_o28' (the EXACT64 build at that expansion order),
    'exact64_b16' / 'exact64_b64' (force, the EXACT64 build with that MRAG block side)."""
    key = (kind, mode)
    if key not in _libs:
        name = "liboracle_direct.so" if kind == "direct" else f"libref_{kind}_{mode}.so"
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built (run make -C oracle)")
        L = ctypes.CDLL(path)
        if kind == "potential":
            L.treecode_potential.argtypes = [ctypes.c_double, _dp, _dp, _dp, ctypes.c_int,
                                             _dp, _dp, ctypes.c_int, _dp]
            L.treecode_potential.restype = None
        elif kind == "force":
            L.treecode_force_mrag.argtypes = [ctypes.c_double, _dp, _dp, _dp, ctypes.c_int,
                                              _dp, _dp, _dp, ctypes.c_int, _dp, _dp]
            L.treecode_force_mrag.restype = None
        if kind in ("potential", "force"):
            L.oracle_sort_sources.argtypes = [_dp, _dp, _dp, ctypes.c_int, _ip, _dp, _dp, _dp, _dp]
            L.oracle_sort_sources.restype = None
            L.oracle_tree_build.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            _ip, _ip, _ip, _ucp, _dp, _dp, _dp, _dp, _dp,
                                            _dp, _dp, _dp, _dp]
            L.oracle_tree_build.restype = ctypes.c_int
            L.oracle_order.restype = ctypes.c_int
        if kind == "direct":
            L.oracle_direct_potential.argtypes = [_dp, _dp, _dp, ctypes.c_int, _dp, _dp,
                                                  ctypes.c_int, _dp]
            L.oracle_direct_force.argtypes = [_dp, _dp, _dp, ctypes.c_int, _dp, _dp,
                                              ctypes.c_int, _dp, _dp]
            L.oracle_check.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_double, _dp]
            L.oracle_check.restype = ctypes.c_int
        _libs[key] = L
    return _libs[key]


# --------------------------------------------------------------------------- API calls
def potential(theta, xs, ys, vs, xt, yt, mode="exact64"):
    """drivers/treecode-potential.cpp:93-106 run on the CPU."""
    xs, ys, vs, xt, yt = map(_f64, (xs, ys, vs, xt, yt))
    out = np.zeros(len(xt))
    lib("potential", mode).treecode_potential(float(theta), _ptr(xs), _ptr(ys), _ptr(vs), len(xs),
                                             _ptr(xt), _ptr(yt), len(xt), _ptr(out))
    return out


def force_mrag(theta, xs, ys, vs, x0s, y0s, hs, mode="exact64", blocksize=32):
    """drivers/treecode-force.cpp:203-236 run on the CPU; outputs ix + bs*(iy + bs*ib).  A block
    side other than 32 needs the build of that BLOCKSIZE (mode 'exact64_b16' / 'exact64_b64')."""
    xs, ys, vs, x0s, y0s, hs = map(_f64, (xs, ys, vs, x0s, y0s, hs))
    nb = len(x0s)
    xo = np.zeros(nb * blocksize * blocksize)
    yo = np.zeros(nb * blocksize * blocksize)
    lib("force", mode).treecode_force_mrag(float(theta), _ptr(xs), _ptr(ys), _ptr(vs), len(xs),
                                          _ptr(x0s), _ptr(y0s), _ptr(hs), nb, _ptr(xo), _ptr(yo))
    return xo, yo


def sort_sources(xs, ys, vs, kind="potential", mode="exact64"):
    """drivers/sort-sources.cpp:23-132: (keys, xsorted, ysorted, vsorted, (xmin, ymin, ext))."""
    xs, ys, vs = map(_f64, (xs, ys, vs))
    n = len(xs)
    keys = np.zeros(n, np.int32)
    xo, yo, vo = np.zeros(n), np.zeros(n), np.zeros(n)
    bbox = np.zeros(3)
    lib(kind, mode).oracle_sort_sources(_ptr(xs), _ptr(ys), _ptr(vs), n, _ptr(keys, _ip),
                                        _ptr(xo), _ptr(yo), _ptr(vo), _ptr(bbox))
    return keys, xo, yo, vo, bbox


def tree(xs, ys, vs, kind="potential", mode="exact64", leafcap=None):
    """Tree::build (drivers/upward.cpp:280-314); raw node arrays in the reference's order."""
    xs, ys, vs = map(_f64, (xs, ys, vs))
    n = len(xs)
    p = ORDER[kind]
    leafcap = LEAF[kind] if leafcap is None else leafcap
    # the node bound of the raised-capacity builds (oracle/Makefile), so one build suffices
    cap = max(1024, int(60 * (n / (leafcap + 1.0) + 1) + 1))
    L = lib(kind, mode)
    while True:
        s = np.zeros(cap, np.int32); e = np.zeros(cap, np.int32)
        cb = np.zeros(cap, np.int32); inner = np.zeros(cap, np.uint8)
        mass, xc, yc, r = (np.zeros(cap) for _ in range(4))
        exps = np.zeros(cap * 2 * p)
        xo, yo, vo = np.zeros(n), np.zeros(n), np.zeros(n)
        bbox = np.zeros(3)
        cnt = L.oracle_tree_build(_ptr(xs), _ptr(ys), _ptr(vs), n, leafcap, cap,
                                  _ptr(s, _ip), _ptr(e, _ip), _ptr(cb, _ip), _ptr(inner, _ucp),
                                  _ptr(mass), _ptr(xc), _ptr(yc), _ptr(r), _ptr(exps),
                                  _ptr(xo), _ptr(yo), _ptr(vo), _ptr(bbox))
        if cnt > 0:
            break
        cap = -cnt
    k = cnt
    return dict(n=k, s=s[:k], e=e[:k], childbase=cb[:k], inner=inner[:k] != 0,
                mass=mass[:k], xcom=xc[:k], ycom=yc[:k], r=r[:k],
                exps=exps[:k * 2 * p].reshape(k, 2, p), xs=xo, ys=yo, vs=vo, bbox=bbox, order=p)


def canonical(t):
    """Walk a tree from its root in breadth-first order, children c = 0..3, following only
    nodes flagged inner.  Returns arrays indexed by canonical id plus (level, cx, cy) cell
    coordinates, so that trees with different node numberings compare element-wise.

    ``t`` needs: s, e, inner (bool), child (first child id, any value for leaves), and
    optionally the per-node arrays mass, xcom, ycom, r, exps."""
    child = t["childbase"] if "childbase" in t else t["child"]
    order, level, cx, cy = [], [], [], []
    q = deque([(0, 0, 0, 0)])
    while q:
        nid, l, x, y = q.popleft()
        order.append(nid); level.append(l); cx.append(x); cy.append(y)
        if t["inner"][nid]:
            base = int(child[nid])
            for c in range(4):
                q.append((base + c, l + 1, 2 * x + (c & 1), 2 * y + (c >> 1)))
    order = np.array(order, np.int64)
    out = dict(orig=order, level=np.array(level, np.int32), cx=np.array(cx, np.int32),
               cy=np.array(cy, np.int32), s=np.asarray(t["s"])[order], e=np.asarray(t["e"])[order],
               inner=np.asarray(t["inner"])[order])
    for k in ("mass", "xcom", "ycom", "r", "exps"):
        if k in t:
            out[k] = np.asarray(t[k])[order]
    return out


# --------------------------------------------------------------------------- direct sums
def direct_potential(xs, ys, vs, xt, yt):
    xs, ys, vs, xt, yt = map(_f64, (xs, ys, vs, xt, yt))
    out = np.zeros(len(xt))
    lib("direct").oracle_direct_potential(_ptr(xs), _ptr(ys), _ptr(vs), len(xs),
                                          _ptr(xt), _ptr(yt), len(xt), _ptr(out))
    return out


def direct_force(xs, ys, vs, xt, yt):
    xs, ys, vs, xt, yt = map(_f64, (xs, ys, vs, xt, yt))
    xo, yo = np.zeros(len(xt)), np.zeros(len(xt))
    lib("direct").oracle_direct_force(_ptr(xs), _ptr(ys), _ptr(vs), len(xs),
                                      _ptr(xt), _ptr(yt), len(xt), _ptr(xo), _ptr(yo))
    return xo, yo


def check(ref, res, tol):
    """main.cpp:31-58 pass rule; returns (passed, {linf, l1, linf_rel, l1_rel})."""
    ref, res = _f64(ref), _f64(res)
    st = np.zeros(4)
    ok = lib("direct").oracle_check(_ptr(ref), _ptr(res), len(ref), float(tol), _ptr(st))
    return bool(ok), dict(linf=st[0], l1=st[1], linf_rel=st[2], l1_rel=st[3])


def mrag_targets(x0s, y0s, hs, bs=32):
    """Explicit target coordinates of MRAG blocks in output order ix + bs*(iy + bs*ib)
    (main.cpp:117-123)."""
    x0s, y0s, hs = map(_f64, (x0s, y0s, hs))
    ix = np.arange(bs, dtype=np.float64)
    xt = (x0s[:, None, None] + ix[None, None, :] * hs[:, None, None]) + 0 * ix[None, :, None]
    yt = (y0s[:, None, None] + ix[None, :, None] * hs[:, None, None]) + 0 * ix[None, None, :]
    return xt.reshape(-1), yt.reshape(-1)

"""Python host binding of the B200 treecode library (ctypes over the C ABI).

Mirrors the reference's public interface (drivers/treecode-potential.h:21-29,
drivers/treecode-force.h:21-31): ``treecode_potential`` and ``treecode_force_mrag`` take the
same arguments with the same meaning (theta opening criterion, source coordinates and values,
targets / MRAG blocks) and return what the reference writes into its output arrays.  The
``Context`` class exposes the extended device-pointer API (inputs resident in GPU memory,
e.g. torch CUDA tensors), statistics, tree inspection and GPU direct sums.

There is no CPU fallback: if the shared library is missing or no GPU is visible, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "lib2d-treecodes-b200.so")

ORDER = {"potential": 12, "force": 24}
LEAF = {"potential": 512, "force": 192}
BLOCKSIZE = 32
ORDER_POTENTIAL = 12   # the reference's default orders (its Makefile:13-14)
ORDER_FORCE = 24

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

# Every symbol the header include/treecodes_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "treecode_potential": (None, [_d, _dp, _dp, _dp, _i, _dp, _dp, _i, _dp]),
    "treecode_force_mrag": (None, [_d, _dp, _dp, _dp, _i, _dp, _dp, _dp, _i, _dp, _dp]),
    "treecode_last_status": (_i, []),
    "treecode_last_error": (ctypes.c_char_p, []),
    "tc_context_create": (_i, [ctypes.POINTER(_vp), _i, _vp]),
    "tc_context_destroy": (None, [_vp]),
    "tc_set_precision": (_i, [_vp, _i]),
    "tc_set_host_waits": (_i, [_vp, _i]),
    "tc_set_launch_overlap": (_i, [_vp, _i]),
    "tc_set_wait_test": (_i, [_vp, _i, _i, _i]),
    "tc_release_cached_memory": (_i, [_i]),
    "tc_reserve_cached_memory": (_i, [_i, ctypes.c_size_t]),
    "tc_set_orders": (_i, [_vp, _i, _i]),
    "tc_supported_orders": (_i, [ctypes.POINTER(ctypes.c_int), _i]),
    "tc_set_blocksize": (_i, [_vp, _i]),
    "tc_log_probe_device": (_i, [_vp, _vp, _i, _vp]),
    "tc_set_timing": (_i, [_vp, _i]),
    "tc_get_stats": (_i, [_vp, _vp]),
    "tc_get_stream": (_vp, [_vp]),
    "tc_potential_host": (_i, [_vp, _d, _dp, _dp, _dp, _i, _dp, _dp, _i, _dp]),
    "tc_force_mrag_host": (_i, [_vp, _d, _dp, _dp, _dp, _i, _dp, _dp, _dp, _i, _dp, _dp]),
    "tc_potential_device": (_i, [_vp, _d, _vp, _vp, _vp, _i, _vp, _vp, _i, _vp]),
    "tc_force_mrag_device": (_i, [_vp, _d, _vp, _vp, _vp, _i, _vp, _vp, _vp, _i, _vp, _vp]),
    "tc_tree_build_device": (_i, [_vp, _i, _vp, _vp, _vp, _i]),
    "tc_tree_size": (_i, [_vp, _ip, _ip, _ip]),
    "tc_tree_copy": (_i, [_vp] + [_vp] * 19),
    "tc_direct_potential_device": (_i, [_vp, _vp, _vp, _vp, _i, _vp, _vp, _i, _vp]),
    "tc_direct_force_device": (_i, [_vp, _vp, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp]),
    "tc_sort_sources_noalloc": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "tc_context_device_bytes": (ctypes.c_size_t, [_vp]),
    "tc_context_trim": (_i, [_vp]),
    "tc_server_create": (_i, [ctypes.POINTER(_vp), _i, _i, ctypes.c_size_t]),
    "tc_server_destroy": (None, [_vp]),
    "tc_server_submit": (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_longlong)]),
    "tc_server_wait": (_i, [_vp, ctypes.c_longlong, _vp]),
    "tc_server_wait_any": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong), _vp]),
    "tc_server_release_client": (_i, [_vp, ctypes.c_longlong]),
    "tc_server_get_stats": (_i, [_vp, _vp]),
    "tc_request_footprint": (ctypes.c_size_t, [_i, _i, _i, _i, _i]),
    "tc_measure_fma_peak": (_i, [_i, _dp]),
    "tc_version": (ctypes.c_char_p, []),
}

REQUEST_POTENTIAL, REQUEST_FORCE_MRAG = 0, 1


class Request(ctypes.Structure):
    _fields_ = [("kind", _i), ("precision", _i), ("theta", _d), ("client", ctypes.c_longlong),
                ("nsources", _i), ("xsources", _dp), ("ysources", _dp), ("sourcevalues", _dp),
                ("ntargets", _i), ("xtargets", _dp), ("ytargets", _dp),
                ("nblocks", _i), ("x0s", _dp), ("y0s", _dp), ("hs", _dp),
                ("out0", _dp), ("out1", _dp)]


class RequestResult(ctypes.Structure):
    _fields_ = [("status", _i), ("slot", _i), ("queue_ms", _d), ("service_ms", _d),
                ("latency_ms", _d), ("footprint_bytes", ctypes.c_size_t), ("finished_s", _d)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("evictions", ctypes.c_longlong),
                ("hbm_budget", ctypes.c_size_t), ("hbm_charged", ctypes.c_size_t),
                ("hbm_peak", ctypes.c_size_t), ("slots", _i), ("max_in_service", _i),
                ("resident_clients", _i)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TreecodeError(RuntimeError):
    pass


class Stats(ctypes.Structure):
    _fields_ = [("sort_ms", ctypes.c_float), ("tree_ms", ctypes.c_float),
                ("upward_ms", ctypes.c_float), ("lists_ms", ctypes.c_float),
                ("eval_ms", ctypes.c_float), ("total_ms", ctypes.c_float),
                ("nnodes", ctypes.c_longlong), ("nleaves", ctypes.c_longlong),
                ("ninner", ctypes.c_longlong), ("nlevels", ctypes.c_longlong),
                ("n_e2l", ctypes.c_longlong), ("n_e2p", ctypes.c_longlong),
                ("n_p2p", ctypes.c_longlong), ("p2p_pairs", ctypes.c_longlong),
                ("e2p_pairs", ctypes.c_longlong), ("e2l_pairs", ctypes.c_longlong),
                ("l2p_targets", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("eval_kernel_ms", ctypes.c_float), ("list_walks", ctypes.c_int),
                ("far_kernel_ms", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise TreecodeError(f"{path} is missing: build it with `make -C 2d-treecodes_b200`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_dp)


def last_status():
    return load().treecode_last_status()


def last_error():
    return load().treecode_last_error().decode()


def _check(rc):
    if rc != 0:
        raise TreecodeError(f"status {rc}: {last_error()}")


# ----------------------------------------------------------------- reference-compatible API
def treecode_potential(theta, xsources, ysources, sourcevalues, xtargets, ytargets):
    """drivers/treecode-potential.cpp:93-106: potential at every target (host arrays)."""
    xs, ys, vs, xt, yt = map(_f64, (xsources, ysources, sourcevalues, xtargets, ytargets))
    out = np.empty(len(xt))
    load().treecode_potential(float(theta), _p(xs), _p(ys), _p(vs), len(xs), _p(xt), _p(yt),
                              len(xt), _p(out))
    _check(last_status())
    return out


def treecode_force_mrag(theta, xsources, ysources, sourcevalues, x0s, y0s, hs):
    """drivers/treecode-force.cpp:203-236: (xresults, yresults), each 1024 * nblocks long,
    target (ix, iy) of block ib at ix + 32 * (iy + 32 * ib)."""
    xs, ys, vs, x0, y0, h = map(_f64, (xsources, ysources, sourcevalues, x0s, y0s, hs))
    nb = len(x0)
    xo = np.empty(nb * BLOCKSIZE * BLOCKSIZE)
    yo = np.empty(nb * BLOCKSIZE * BLOCKSIZE)
    load().treecode_force_mrag(float(theta), _p(xs), _p(ys), _p(vs), len(xs), _p(x0), _p(y0),
                               _p(h), nb, _p(xo), _p(yo))
    _check(last_status())
    return xo, yo


def supported_orders():
    """The expansion orders Context.set_orders accepts."""
    n = load().tc_supported_orders(None, 0)
    buf = (ctypes.c_int * n)()
    load().tc_supported_orders(buf, n)
    return list(buf)


def release_cached_memory(device=-1):
    """Hands the device's cached, unused pool memory back to the driver (destroyed and trimmed
    contexts leave their memory cached while another context of the device lives)."""
    _check(load().tc_release_cached_memory(int(device)))


def reserve_cached_memory(nbytes, device=-1):
    """Maps up to `nbytes` of device memory into the device's pool ahead of the solves (at
    most the free memory less 2 GB); a request server does this for its budget."""
    _check(load().tc_reserve_cached_memory(int(device), int(nbytes)))


def measure_fma_peak(fp64=True):
    t = ctypes.c_double()
    _check(load().tc_measure_fma_peak(1 if fp64 else 0, ctypes.byref(t)))
    return t.value


def _ptr(t):
    """Device address of a torch CUDA tensor (or an int address)."""
    if isinstance(t, int):
        return t
    if not t.is_contiguous():
        raise TreecodeError("device arrays must be contiguous")
    return t.data_ptr()


class Context:
    """A solver context: a CUDA stream plus device buffers reused across calls."""

    def __init__(self, device=-1, stream=None, precision=0, timing=False):
        self.lib = load()
        h = _vp()
        _check(self.lib.tc_context_create(ctypes.byref(h), int(device), stream))
        self.h = h
        self.blocksize = BLOCKSIZE
        if precision:
            _check(self.lib.tc_set_precision(self.h, int(precision)))
        if timing:
            self.lib.tc_set_timing(self.h, 1)

    def close(self):
        if getattr(self, "h", None):
            self.lib.tc_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return self.lib.tc_get_stream(self.h)

    def set_precision(self, mode):
        _check(self.lib.tc_set_precision(self.h, int(mode)))

    def set_host_waits(self, sleeping):
        """0: the solving thread spins while the device works (lowest latency); 1: it polls
        and sleeps, leaving the host core to other threads."""
        _check(self.lib.tc_set_host_waits(self.h, int(sleeping)))

    def set_launch_overlap(self, on=True):
        """True (the default): the solve's kernel chains use programmatic dependent launch, each
        kernel scheduled while the one before it drains; False: plain launches."""
        _check(self.lib.tc_set_launch_overlap(self.h, int(bool(on))))

    def set_wait_test(self, stall=0, spin_limit=0, stack_limit=0):
        """Test settings: `stall` 1 (source sort) or 2 (tree build) makes one look-back tile
        publish nothing, so the next one's bounded wait runs out (TC_ERR_TIMEOUT); `spin_limit`
        bounds the device waits (0: the default); `stack_limit` caps the force traversal stack
        per warp (0: all of it; exceeding it gives TC_ERR_CAPACITY).  No argument restores the
        defaults."""
        _check(self.lib.tc_set_wait_test(self.h, int(stall), int(spin_limit), int(stack_limit)))

    def set_orders(self, potential_order=ORDER_POTENTIAL, force_order=ORDER_FORCE):
        """Expansion orders of the next solves (the reference's build-time potential-order and
        force-order); one of supported_orders() each."""
        _check(self.lib.tc_set_orders(self.h, int(potential_order), int(force_order)))

    def set_blocksize(self, blocksize=BLOCKSIZE):
        """MRAG block side of the next force solves (8, 16, 32 or 64; the reference's
        build-time mrag-blocksize): outputs of nblocks * blocksize**2 values."""
        _check(self.lib.tc_set_blocksize(self.h, int(blocksize)))
        self.blocksize = int(blocksize)

    def set_timing(self, on=True):
        """True / 1: phase times in stats(); 2: also the force's near- and far-field kernels
        run one after the other, each alone on the GPU (per-kernel times); False / 0: off."""
        _check(self.lib.tc_set_timing(self.h, int(on)))

    def stats(self):
        s = Stats()
        _check(self.lib.tc_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    # ---- host pointers
    def potential_host(self, theta, xs, ys, vs, xt, yt, out=None):
        xs, ys, vs, xt, yt = map(_f64, (xs, ys, vs, xt, yt))
        out = np.empty(len(xt)) if out is None else out
        _check(self.lib.tc_potential_host(self.h, float(theta), _p(xs), _p(ys), _p(vs), len(xs),
                                          _p(xt), _p(yt), len(xt), _p(out)))
        return out

    def force_mrag_host(self, theta, xs, ys, vs, x0s, y0s, hs, xo=None, yo=None):
        xs, ys, vs, x0, y0, h = map(_f64, (xs, ys, vs, x0s, y0s, hs))
        nt = len(x0) * self.blocksize * self.blocksize
        xo = np.empty(nt) if xo is None else xo
        yo = np.empty(nt) if yo is None else yo
        _check(self.lib.tc_force_mrag_host(self.h, float(theta), _p(xs), _p(ys), _p(vs), len(xs),
                                           _p(x0), _p(y0), _p(h), len(x0), _p(xo), _p(yo)))
        return xo, yo

    # ---- device pointers (torch CUDA tensors of dtype float64)
    def potential_device(self, theta, xs, ys, vs, xt, yt, out):
        _check(self.lib.tc_potential_device(self.h, float(theta), _ptr(xs), _ptr(ys), _ptr(vs),
                                            int(xs.numel()), _ptr(xt), _ptr(yt), int(xt.numel()),
                                            _ptr(out)))
        return out

    def force_mrag_device(self, theta, xs, ys, vs, x0s, y0s, hs, xo, yo):
        _check(self.lib.tc_force_mrag_device(self.h, float(theta), _ptr(xs), _ptr(ys), _ptr(vs),
                                             int(xs.numel()), _ptr(x0s), _ptr(y0s), _ptr(hs),
                                             int(x0s.numel()), _ptr(xo), _ptr(yo)))
        return xo, yo

    def direct_potential_device(self, xs, ys, vs, xt, yt, out):
        _check(self.lib.tc_direct_potential_device(self.h, _ptr(xs), _ptr(ys), _ptr(vs),
                                                   int(xs.numel()), _ptr(xt), _ptr(yt),
                                                   int(xt.numel()), _ptr(out)))
        return out

    def direct_force_device(self, xs, ys, vs, xt, yt, xo, yo):
        _check(self.lib.tc_direct_force_device(self.h, _ptr(xs), _ptr(ys), _ptr(vs),
                                               int(xs.numel()), _ptr(xt), _ptr(yt),
                                               int(xt.numel()), _ptr(xo), _ptr(yo)))
        return xo, yo

    def log_probe_device(self, x, out):
        """out[2i] = the potential kernels' log of x[i], out[2i + 1] = the library log."""
        _check(self.lib.tc_log_probe_device(self.h, _ptr(x), int(x.numel()), _ptr(out)))
        return out

    # ---- tree inspection
    def tree(self, kind, xs, ys, vs):
        """Build the tree of `kind` ('potential' | 'force') and copy it to the host."""
        k = 0 if kind == "potential" else 1
        _check(self.lib.tc_tree_build_device(self.h, k, _ptr(xs), _ptr(ys), _ptr(vs),
                                             int(xs.numel())))
        nn, order, n = _i(), _i(), _i()
        _check(self.lib.tc_tree_size(self.h, ctypes.byref(nn), ctypes.byref(order),
                                     ctypes.byref(n)))
        nn, order, n = nn.value, order.value, n.value
        out = dict(keys=np.empty(n, np.int32), perm=np.empty(n, np.int32), xs=np.empty(n),
                   ys=np.empty(n), vs=np.empty(n), frame=np.empty(3))
        for name in ("s", "e", "child", "count", "level", "cx", "cy", "parent"):
            out[name] = np.empty(nn, np.int32)
        for name in ("mass", "xcom", "ycom", "r"):
            out[name] = np.empty(nn)
        out["exps"] = np.empty(nn * 2 * order)
        order_names = ("keys", "perm", "xs", "ys", "vs", "frame", "s", "e", "child", "count",
                       "level", "cx", "cy", "parent", "mass", "xcom", "ycom", "r", "exps")
        args = [out[k].ctypes.data_as(_vp) for k in order_names]
        _check(self.lib.tc_tree_copy(self.h, *args))
        out["exps"] = out["exps"].reshape(nn, 2, order)
        out["inner"] = out["child"] >= 0
        out["n"] = nn
        out["order"] = order
        return out


    def device_bytes(self):
        return int(self.lib.tc_context_device_bytes(self.h))

    def trim(self):
        _check(self.lib.tc_context_trim(self.h))


def request_footprint(kind, nsources, ntargets=0, nblocks=0, precision=0):
    """Device-memory estimate (bytes) the server charges for a request of these sizes."""
    return int(load().tc_request_footprint(int(kind), int(nsources), int(ntargets), int(nblocks),
                                           int(precision)))


class Server:
    """The serving loop: concurrent solves on `slots` streams under a device-memory budget.

    ``submit_*`` return a ticket at once; ``wait(ticket)`` returns the outputs with the
    request's queue / service / latency times.  Host arrays are kept alive here until waited.
    """

    def __init__(self, slots=4, hbm_budget_bytes=32 << 30, device=-1, host_alloc=None):
        """host_alloc(n) -> float64 array for the outputs (e.g. page-locked memory, so that the
        results come back by direct DMA); numpy's allocator by default."""
        self.lib = load()
        h = _vp()
        _check(self.lib.tc_server_create(ctypes.byref(h), int(device), int(slots),
                                         int(hbm_budget_bytes)))
        self.h = h
        self._live = {}
        self._alloc = host_alloc or np.empty

    def _submit(self, req, keep, outs):
        t = ctypes.c_longlong()
        _check(self.lib.tc_server_submit(self.h, ctypes.byref(req), ctypes.byref(t)))
        self._live[t.value] = (req, keep, outs)
        return t.value

    def submit_potential(self, theta, xs, ys, vs, xt, yt, precision=0, client=0):
        xs, ys, vs, xt, yt = map(_f64, (xs, ys, vs, xt, yt))
        out = self._alloc(len(xt))
        req = Request(kind=REQUEST_POTENTIAL, precision=int(precision), theta=float(theta),
                      client=int(client), nsources=len(xs), xsources=_p(xs), ysources=_p(ys),
                      sourcevalues=_p(vs), ntargets=len(xt), xtargets=_p(xt), ytargets=_p(yt),
                      out0=_p(out))
        return self._submit(req, (xs, ys, vs, xt, yt), (out,))

    def submit_force(self, theta, xs, ys, vs, x0s, y0s, hs, precision=0, client=0):
        xs, ys, vs, x0, y0, h = map(_f64, (xs, ys, vs, x0s, y0s, hs))
        nt = len(x0) * BLOCKSIZE * BLOCKSIZE
        xo, yo = self._alloc(nt), self._alloc(nt)
        req = Request(kind=REQUEST_FORCE_MRAG, precision=int(precision), theta=float(theta),
                      client=int(client), nsources=len(xs), xsources=_p(xs), ysources=_p(ys),
                      sourcevalues=_p(vs), nblocks=len(x0), x0s=_p(x0), y0s=_p(y0), hs=_p(h),
                      out0=_p(xo), out1=_p(yo))
        return self._submit(req, (xs, ys, vs, x0, y0, h), (xo, yo))

    def wait(self, ticket):
        """(outputs tuple, result dict); raises if the solve failed."""
        res = RequestResult()
        rc = self.lib.tc_server_wait(self.h, ctypes.c_longlong(ticket), ctypes.byref(res))
        _, _, outs = self._live.pop(ticket)
        if rc != 0:
            raise TreecodeError(f"request {ticket} failed with status {rc}")
        return outs, res.as_dict()

    def wait_any(self):
        """(ticket, outputs tuple, result dict) of the earliest completed request not yet
        collected; raises if that solve failed (the exception carries the ticket) or if no
        request is outstanding."""
        res = RequestResult()
        t = ctypes.c_longlong()
        rc = self.lib.tc_server_wait_any(self.h, ctypes.byref(t), ctypes.byref(res))
        if t.value == 0:
            raise TreecodeError(f"no request outstanding (status {rc})")
        _, _, outs = self._live.pop(t.value)
        if rc != 0:
            err = TreecodeError(f"request {t.value} failed with status {rc}")
            err.ticket = t.value
            raise err
        return t.value, outs, res.as_dict()

    def release_client(self, client):
        _check(self.lib.tc_server_release_client(self.h, ctypes.c_longlong(client)))

    def stats(self):
        s = ServerStats()
        _check(self.lib.tc_server_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.tc_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

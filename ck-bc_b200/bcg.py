"""ctypes binding of libbcg.so, the C ABI declared in include/bcg.h.

This is the Python face of the engine used by the tests and bench.py.  It
loads only the in-tree ``libbcg.so`` (built by ``make -C ck-bc_b200`` or
``__graft_entry__.build()``) and raises when it is missing: there is no
Python or CPU fallback for any device entry point.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbcg.so")

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_OVERFLOW = -4
ERR_TIMEOUT = -5
ERR_IO = -6
ERR_DEPTH = -7
ERR_RANGE = -8
ERR_NOGPU = -9

PRUNE_DEGREE1 = 0x1
DIRECTED = 0x2
PRUNE_TREES = 0x4

SIGMA_AUTO = 0
SIGMA_EXACT = 1
SIGMA_EXTENDED = 2

NOALLOC_MAX_VERTICES = 65536
NOALLOC_MAX_ADJ = 1048576
NOALLOC_MAX_SOURCES = 65536

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class HostCSR(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("nnz", ctypes.c_uint64),
                ("offsets", _u32p), ("adj", _u32p)]


class Stats(ctypes.Structure):
    _fields_ = [("sources", ctypes.c_uint64), ("skipped", ctypes.c_uint64),
                ("roots", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("teps_edges", ctypes.c_uint64), ("visited", ctypes.c_uint64),
                ("comp_vertices", ctypes.c_uint64),
                ("max_depth", ctypes.c_uint32), ("batch_width", ctypes.c_uint32),
                ("kernel_ms", ctypes.c_double), ("extended_sigma", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("search_edges", ctypes.c_uint64), ("launches", ctypes.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BcgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bcg error {code}: {msg}")
        self.code = code


# Every symbol of include/bcg.h with (restype, argtypes).
SIGNATURES = {
    "bcg_csr_read_edgelist": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int,
                                             ctypes.c_int, ctypes.POINTER(HostCSR)]),
    "bcg_csr_from_pairs": (ctypes.c_int, [_u64p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                          ctypes.POINTER(HostCSR)]),
    "bcg_csr_generate": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(HostCSR)]),
    "bcg_csr_write_edgelist": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(HostCSR)]),
    "bcg_csr_free": (None, [ctypes.POINTER(HostCSR)]),
    "bcg_csr_write_binary": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(HostCSR)]),
    "bcg_csr_read_binary": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(HostCSR)]),
    "bcg_sample_sources": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u32p]),
    "bcg_device_count": (ctypes.c_int, []),
    "bcg_graph_create": (ctypes.c_int, [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "bcg_graph_create_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                               ctypes.c_uint64, ctypes.c_uint32,
                                               ctypes.POINTER(ctypes.c_void_p)]),
    "bcg_graph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "bcg_reset_bc": (ctypes.c_int, [ctypes.c_void_p]),
    "bcg_run": (ctypes.c_int, [ctypes.c_void_p, _u32p, ctypes.c_uint64, ctypes.POINTER(Stats)]),
    "bcg_run_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.POINTER(Stats)]),
    "bcg_get_bc": (ctypes.c_int, [ctypes.c_void_p, _f64p]),
    "bcg_bc_device_ptr": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "bcg_bc_csr": (ctypes.c_int, [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64, _u32p, ctypes.c_uint64,
                                  ctypes.c_uint32, _f64p, ctypes.POINTER(Stats)]),
    "bcg_single_source": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _i32p, _u64p, _f64p]),
    "bcg_debug_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _i32p, _u64p,
                                       _f64p]),
    "bcg_graph_pruning": (ctypes.c_int, [ctypes.c_void_p, _u32p, _u32p]),
    "bcg_graph_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint32)]),
    "bcg_graph_set_reach": (ctypes.c_int, [ctypes.c_void_p, _u32p]),
    "bcg_run_weighted": (ctypes.c_int, [ctypes.c_void_p, _u32p, _f64p, _u32p, ctypes.c_uint64,
                                        ctypes.POINTER(Stats)]),
    "bcg_run_root_levels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_double, ctypes.c_uint32,
                                           _i32p, ctypes.POINTER(Stats)]),
    "bcg_run_slots": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "bcg_add_scaled": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, _u32p,
                                      ctypes.POINTER(ctypes.c_double), _u32p, ctypes.POINTER(ctypes.c_double)]),
    "bcg_set_batch_width": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "bcg_set_sigma_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "bcg_single_source_ext": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _i32p, _u64p, _f64p]),
    "bcg_batch_create": (ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(_u32p), ctypes.POINTER(_u32p), _u32p,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "bcg_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "bcg_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Stats)]),
    "bcg_batch_reset_bc": (ctypes.c_int, [ctypes.c_void_p]),
    "bcg_batch_get_bc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _f64p]),
    "bcg_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _u32p, _u32p, _u32p]),
    "bcg_batch_info": (ctypes.c_int, [ctypes.c_void_p, _u32p, _u32p, _u32p, _u32p,
                                      ctypes.POINTER(ctypes.c_int)]),
    "bcg_server_create": (ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(_u32p), ctypes.POINTER(_u32p), _u32p,
                                         ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    "bcg_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "bcg_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, _u32p, ctypes.c_uint64, _u64p]),
    "bcg_server_step": (ctypes.c_int, [ctypes.c_void_p, _u64p, ctypes.c_uint32, _u32p]),
    "bcg_server_wait": (ctypes.c_int, [ctypes.c_void_p, _u64p, ctypes.c_uint32, _u32p]),
    "bcg_server_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _f64p]),
    "bcg_server_info": (ctypes.c_int, [ctypes.c_void_p, _u64p, _u64p, _u32p, _u32p, _u64p]),
    "bcg_bc_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                      ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p]),
    "bcg_last_error": (ctypes.c_char_p, []),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """Loads the in-tree libbcg.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `make -C ck-bc_b200` "
                               "or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _check(rc: int):
    if rc != OK:
        msg = lib().bcg_last_error()
        raise BcgError(rc, msg.decode() if msg else "")


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def _take_csr(h: HostCSR):
    n, nnz = h.n, h.nnz
    offs = np.empty(n + 1, dtype=np.uint32)
    adj = np.empty(nnz, dtype=np.uint32)
    ctypes.memmove(offs.ctypes.data, h.offsets, 4 * (n + 1))
    if nnz:
        ctypes.memmove(adj.ctypes.data, h.adj, 4 * nnz)
    lib().bcg_csr_free(ctypes.byref(h))
    return offs, adj


def generate(spec: str):
    """Seeded synthetic graph -> (offsets uint32[n+1], adj uint32[nnz])."""
    h = HostCSR()
    _check(lib().bcg_csr_generate(spec.encode(), ctypes.byref(h)))
    return _take_csr(h)


def read_edgelist(path: str, n: int, undirected: bool = True, echo_header: bool = False):
    h = HostCSR()
    _check(lib().bcg_csr_read_edgelist(os.fsencode(path), n, int(undirected), int(echo_header),
                                       ctypes.byref(h)))
    return _take_csr(h)


def from_pairs(pairs, n: int, undirected: bool = True):
    p = np.ascontiguousarray(np.asarray(pairs, dtype=np.uint64).reshape(-1))
    h = HostCSR()
    _check(lib().bcg_csr_from_pairs(p.ctypes.data_as(_u64p), p.size // 2, n, int(undirected),
                                    ctypes.byref(h)))
    return _take_csr(h)


def write_edgelist(path: str, offsets: np.ndarray, adj: np.ndarray):
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    h = HostCSR(len(offsets) - 1, len(adj), _p32(offsets), _p32(adj))
    _check(lib().bcg_csr_write_edgelist(os.fsencode(path), ctypes.byref(h)))


def write_binary(path: str, offsets: np.ndarray, adj: np.ndarray):
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    h = HostCSR(len(offsets) - 1, len(adj), _p32(offsets), _p32(adj) if len(adj) else None)
    _check(lib().bcg_csr_write_binary(os.fsencode(path), ctypes.byref(h)))


def read_binary(path: str):
    h = HostCSR()
    _check(lib().bcg_csr_read_binary(os.fsencode(path), ctypes.byref(h)))
    return _take_csr(h)


def ext_log2(raw: np.ndarray) -> np.ndarray:
    """log2 of extended-encoding values ((2^48 + f) * 2^(E - 32816)); -inf for 0."""
    raw = np.asarray(raw, dtype=np.uint64)
    e = (raw >> np.uint64(48)).astype(np.int64)
    f = (raw & np.uint64((1 << 48) - 1)).astype(np.float64)
    out = np.log2(1.0 + f / 2.0**48) + (e - 32816 + 48).astype(np.float64)
    out[raw == 0] = -np.inf
    return out


def sample_sources(n: int, k: int, seed: int) -> np.ndarray:
    out = np.zeros(k, dtype=np.uint32)
    _check(lib().bcg_sample_sources(n, k, seed, _p32(out)))
    return out


def device_count() -> int:
    return lib().bcg_device_count()


class Graph:
    """One graph resident on the current CUDA device (bcg_graph handle)."""

    def __init__(self, offsets: np.ndarray, adj: np.ndarray, flags: int = 0):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.adj = np.ascontiguousarray(adj, dtype=np.uint32)
        self.n = len(self.offsets) - 1
        self.nnz = len(self.adj)
        h = ctypes.c_void_p()
        _check(lib().bcg_graph_create(_p32(self.offsets), _p32(self.adj) if self.nnz else None,
                                      self.n, self.nnz, flags, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().bcg_graph_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def reset(self):
        _check(lib().bcg_reset_bc(self.h))

    def run(self, sources) -> Stats:
        s = np.ascontiguousarray(sources, dtype=np.uint32)
        st = Stats()
        _check(lib().bcg_run(self.h, _p32(s), len(s), ctypes.byref(st)))
        return st

    def run_device(self, d_sources_ptr: int, nsrc: int, stream: int = 0, stats: bool = False):
        st = Stats() if stats else None
        _check(lib().bcg_run_device(self.h, ctypes.c_void_p(d_sources_ptr), nsrc, ctypes.c_void_p(stream),
                                    ctypes.byref(st) if st is not None else None))
        return st

    def bc(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        _check(lib().bcg_get_bc(self.h, out.ctypes.data_as(_f64p)))
        return out

    def bc_device_ptr(self) -> int:
        p = ctypes.c_void_p()
        _check(lib().bcg_bc_device_ptr(self.h, ctypes.byref(p)))
        return p.value

    def single_source(self, src: int):
        lvl = np.zeros(self.n, dtype=np.int32)
        sig = np.zeros(self.n, dtype=np.uint64)
        dl = np.zeros(self.n, dtype=np.float64)
        _check(lib().bcg_single_source(self.h, src, lvl.ctypes.data_as(_i32p), sig.ctypes.data_as(_u64p),
                                       dl.ctypes.data_as(_f64p)))
        return lvl, sig, dl

    def debug_batch(self, roots, width: int):
        """One real batch of `width` slots with roots[k] in slot k -> (level,
        sigma, delta), each of shape (len(roots), n) in the caller's ids."""
        r = np.ascontiguousarray(roots, dtype=np.uint32)
        k = len(r)
        lvl = np.zeros((k, self.n), dtype=np.int32)
        sig = np.zeros((k, self.n), dtype=np.uint64)
        dl = np.zeros((k, self.n), dtype=np.float64)
        _check(lib().bcg_debug_batch(self.h, width, _p32(r), k, lvl.ctypes.data_as(_i32p), sig.ctypes.data_as(_u64p),
                                     dl.ctypes.data_as(_f64p)))
        return lvl, sig, dl

    def pruning(self):
        anc = np.zeros(self.n, dtype=np.uint32)
        rch = np.zeros(self.n, dtype=np.uint32)
        _check(lib().bcg_graph_pruning(self.h, _p32(anc), _p32(rch)))
        return anc, rch

    def info(self):
        n = ctypes.c_uint32()
        nnz = ctypes.c_uint64()
        nnzp = ctypes.c_uint64()
        npr = ctypes.c_uint32()
        _check(lib().bcg_graph_info(self.h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(nnzp),
                                    ctypes.byref(npr)))
        return {"n": n.value, "nnz": nnz.value, "nnz_pruned": nnzp.value, "pruned": npr.value}

    def set_batch_width(self, w: int):
        _check(lib().bcg_set_batch_width(self.h, w))

    def set_sigma_mode(self, mode: int):
        _check(lib().bcg_set_sigma_mode(self.h, mode))

    def single_source_ext(self, src: int):
        """-> (level, sigma as float log2 values (-inf for 0), delta); sigma
        is decoded from the extended encoding."""
        lvl = np.zeros(self.n, dtype=np.int32)
        raw = np.zeros(self.n, dtype=np.uint64)
        dl = np.zeros(self.n, dtype=np.float64)
        _check(lib().bcg_single_source_ext(self.h, src, lvl.ctypes.data_as(_i32p), raw.ctypes.data_as(_u64p),
                                           dl.ctypes.data_as(_f64p)))
        return lvl, ext_log2(raw), dl


class Batch:
    """Many independent graphs resident as one disjoint union; run() adds every
    graph's exact all-sources BC in one packed persistent launch."""

    def __init__(self, graphs):
        self._keep = [(np.ascontiguousarray(o, dtype=np.uint32), np.ascontiguousarray(a, dtype=np.uint32))
                      for o, a in graphs]
        k = len(self._keep)
        self.sizes = [len(o) - 1 for o, _ in self._keep]
        offs = (_u32p * k)(*[_p32(o) for o, _ in self._keep])
        adjs = (_u32p * k)(*[_p32(a) if len(a) else None for _, a in self._keep])
        n = np.array(self.sizes, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(lib().bcg_batch_create(k, offs, adjs, _p32(n), ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().bcg_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self) -> Stats:
        st = Stats()
        _check(lib().bcg_batch_run(self.h, ctypes.byref(st)))
        return st

    def reset(self):
        _check(lib().bcg_batch_reset_bc(self.h))

    def bc(self, i: int) -> np.ndarray:
        out = np.zeros(self.sizes[i], dtype=np.float64)
        _check(lib().bcg_batch_get_bc(self.h, i, out.ctypes.data_as(_f64p)))
        return out

    def autotune(self, sample_batches: int = 0):
        w, tv, te = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().bcg_batch_autotune(self.h, sample_batches, ctypes.byref(w), ctypes.byref(tv),
                                        ctypes.byref(te)))
        return w.value, tv.value, te.value

    def info(self):
        nb, w, tv, te = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        cap = ctypes.c_int()
        _check(lib().bcg_batch_info(self.h, ctypes.byref(nb), ctypes.byref(w), ctypes.byref(tv), ctypes.byref(te),
                                    ctypes.byref(cap)))
        return {"nbatch": nb.value, "width": w.value, "tile_vertices": tv.value, "tile_entries": te.value,
                "captured": bool(cap.value)}


class Server:
    """Resident pool of graphs serving BC requests with continuous batching:
    submit() queues (from any thread), step() retires finished waves, admits
    what fits and keeps the next waves queued without waiting for the GPU,
    wait() does the same after the oldest wave in flight has finished,
    result() returns a finished request's bc."""

    def __init__(self, graphs, budget_bytes: int, wave_batches: int = 64):
        self._keep = [(np.ascontiguousarray(o, dtype=np.uint32), np.ascontiguousarray(a, dtype=np.uint32))
                      for o, a in graphs]
        k = len(self._keep)
        self.sizes = [len(o) - 1 for o, _ in self._keep]
        offs = (_u32p * k)(*[_p32(o) for o, _ in self._keep])
        adjs = (_u32p * k)(*[_p32(a) if len(a) else None for _, a in self._keep])
        n = np.array(self.sizes, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(lib().bcg_server_create(k, offs, adjs, _p32(n), int(budget_bytes), wave_batches, ctypes.byref(h)))
        self.h = h
        self._graph_of = {}

    def close(self):
        if self.h:
            lib().bcg_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, graph: int, sources=None) -> int:
        """sources=None: exact BC (every vertex)."""
        rid = ctypes.c_uint64()
        if sources is None:
            _check(lib().bcg_server_submit(self.h, graph, None, 0, ctypes.byref(rid)))
        else:
            s = np.ascontiguousarray(sources, dtype=np.uint32)
            if len(s) == 0:
                raise ValueError("a k-source request needs at least one source")
            _check(lib().bcg_server_submit(self.h, graph, _p32(s), len(s), ctypes.byref(rid)))
        self._graph_of[rid.value] = graph
        return rid.value

    def step(self, cap: int = 4096):
        ids = (ctypes.c_uint64 * cap)()
        nd = ctypes.c_uint32()
        _check(lib().bcg_server_step(self.h, ids, cap, ctypes.byref(nd)))
        return [ids[i] for i in range(nd.value)]

    def wait(self, cap: int = 4096):
        ids = (ctypes.c_uint64 * cap)()
        nd = ctypes.c_uint32()
        _check(lib().bcg_server_wait(self.h, ids, cap, ctypes.byref(nd)))
        return [ids[i] for i in range(nd.value)]

    def result(self, rid: int) -> np.ndarray:
        out = np.zeros(self.sizes[self._graph_of.pop(rid)], dtype=np.float64)
        _check(lib().bcg_server_result(self.h, rid, out.ctypes.data_as(_f64p)))
        return out

    def info(self):
        rb, ab, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        pend, run = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().bcg_server_info(self.h, ctypes.byref(rb), ctypes.byref(ab), ctypes.byref(pend),
                                     ctypes.byref(run), ctypes.byref(w)))
        return {"resident_bytes": rb.value, "admitted_bytes": ab.value, "pending": pend.value,
                "running": run.value, "waves": w.value}


def bc_noalloc(d_offsets: int, d_adj: int, n: int, nnz: int, d_sources: int, nsrc: int, d_bc: int,
               accumulate: bool = False, stream: int = 0):
    """bcg_bc_noalloc on raw device pointers (ints): exact BC of a device CSR
    into the caller's device buffer d_bc[n], allocating no device memory."""
    _check(lib().bcg_bc_noalloc(ctypes.c_void_p(d_offsets), ctypes.c_void_p(d_adj), n, nnz,
                                ctypes.c_void_p(d_sources), nsrc, ctypes.c_void_p(d_bc), int(bool(accumulate)),
                                ctypes.c_void_p(stream)))


def bc_csr(offsets, adj, sources, flags: int = 0):
    """One-shot drop-in call on host buffers -> (bc float64[n], Stats)."""
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    s = np.ascontiguousarray(sources, dtype=np.uint32)
    n = len(offsets) - 1
    out = np.zeros(n, dtype=np.float64)
    st = Stats()
    _check(lib().bcg_bc_csr(_p32(offsets), _p32(adj) if len(adj) else None, n, len(adj), _p32(s), len(s),
                            flags, out.ctypes.data_as(_f64p), ctypes.byref(st)))
    return out, st


@dataclass
class DeviceArray:
    """Exposes a raw device pointer through __cuda_array_interface__ so that
    torch.as_tensor(..., device='cuda') wraps it without a copy."""
    ptr: int
    n: int
    typestr: str = "<f8"

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.n,), "typestr": self.typestr, "data": (self.ptr, False), "version": 3,
                "strides": None}

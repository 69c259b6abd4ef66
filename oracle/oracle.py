"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/liboracle.so (brandes.c), the CPU restatement of the
reference's Brandes path.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm may import this module, and only as the checker
or the timed CPU baseline; the product (ck-bc_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class OracleStats(ctypes.Structure):
    _fields_ = [("skipped", ctypes.c_uint64), ("ran", ctypes.c_uint64), ("visited", ctypes.c_uint64),
                ("teps_edges", ctypes.c_uint64), ("max_depth", ctypes.c_uint32), ("overflow", ctypes.c_int)]


_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_single_source.restype = ctypes.c_int
        L.oracle_single_source.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _i32p, _u64p,
                                           _f64p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_bc.restype = ctypes.c_int
        L.oracle_bc.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _f64p,
                                ctypes.POINTER(OracleStats)]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_single_source_q.restype = ctypes.c_int
        L.oracle_single_source_q.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _i32p, _f64p, _f64p]
        L.oracle_bc_q.restype = ctypes.c_int
        L.oracle_bc_q.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _f64p,
                                  ctypes.POINTER(OracleStats)]
        L.oracle_path_length_sum.restype = ctypes.c_int
        L.oracle_path_length_sum.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint64, ctypes.c_int,
                                             _u64p]
        _LIB = L
    return _LIB


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def single_source(offsets, adj, src: int):
    """-> (level int32[n] (-1 unreachable), sigma uint64[n], delta float64[n], overflow flag)."""
    offsets, adj = _u32(offsets), _u32(adj)
    n = len(offsets) - 1
    lvl = np.zeros(n, np.int32)
    sig = np.zeros(n, np.uint64)
    dl = np.zeros(n, np.float64)
    ov = ctypes.c_int(0)
    rc = lib().oracle_single_source(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p), src,
                                    lvl.ctypes.data_as(_i32p), sig.ctypes.data_as(_u64p),
                                    dl.ctypes.data_as(_f64p), ctypes.byref(ov))
    if rc:
        raise RuntimeError(f"oracle_single_source failed ({rc})")
    return lvl, sig, dl, bool(ov.value)


def bc(offsets, adj, sources, nthreads: int = 1):
    """Ordered-pair BC sums over the given sources -> (bc float64[n], stats dict)."""
    offsets, adj = _u32(offsets), _u32(adj)
    s = _u32(sources)
    n = len(offsets) - 1
    out = np.zeros(n, np.float64)
    st = OracleStats()
    rc = lib().oracle_bc(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p), s.ctypes.data_as(_u32p),
                         len(s), nthreads, out.ctypes.data_as(_f64p), ctypes.byref(st))
    if rc:
        raise RuntimeError(f"oracle_bc failed ({rc})")
    return out, {f: getattr(st, f) for f, _ in st._fields_}


def path_length_sum(offsets, adj, sources, nthreads: int = 1) -> int:
    """Sum over sources (degree 0 skipped) and reachable t != s of d(s,t) - 1,
    which equals the sum of bc[] over that source set (exact integer)."""
    offsets, adj = _u32(offsets), _u32(adj)
    s = _u32(sources)
    n = len(offsets) - 1
    tot = ctypes.c_uint64(0)
    rc = lib().oracle_path_length_sum(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p),
                                      s.ctypes.data_as(_u32p), len(s), nthreads, ctypes.byref(tot))
    if rc:
        raise RuntimeError(f"oracle_path_length_sum failed ({rc})")
    return int(tot.value)


def single_source_q(offsets, adj, src: int):
    """__float128 restatement -> (level int32[n], log2 sigma float64[n] (-inf: 0), delta float64[n])."""
    offsets, adj = _u32(offsets), _u32(adj)
    n = len(offsets) - 1
    lvl = np.zeros(n, np.int32)
    sl = np.zeros(n, np.float64)
    dl = np.zeros(n, np.float64)
    rc = lib().oracle_single_source_q(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p), src,
                                      lvl.ctypes.data_as(_i32p), sl.ctypes.data_as(_f64p), dl.ctypes.data_as(_f64p))
    if rc:
        raise RuntimeError(f"oracle_single_source_q failed ({rc})")
    return lvl, sl, dl


def bc_q(offsets, adj, sources, nthreads: int = 1):
    """__float128 restatement of bc() for graphs whose path counts overflow uint64."""
    offsets, adj = _u32(offsets), _u32(adj)
    s = _u32(sources)
    n = len(offsets) - 1
    out = np.zeros(n, np.float64)
    st = OracleStats()
    rc = lib().oracle_bc_q(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p), s.ctypes.data_as(_u32p),
                           len(s), nthreads, out.ctypes.data_as(_f64p), ctypes.byref(st))
    if rc:
        raise RuntimeError(f"oracle_bc_q failed ({rc})")
    return out, {f: getattr(st, f) for f, _ in st._fields_}


_TREES = None


class TreeStats(ctypes.Structure):
    _fields_ = [("skipped", ctypes.c_uint64), ("roots", ctypes.c_uint64), ("teps_edges", ctypes.c_uint64),
                ("peel_seconds", ctypes.c_double), ("overflow", ctypes.c_int)]


def _trees_lib():
    global _TREES
    if _TREES is None:
        path = os.path.join(HERE, "libtrees_ref.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "libtrees_ref.so"], check=True)
        L = ctypes.CDLL(path)
        L.oracle_peel_trees.restype = ctypes.c_int
        L.oracle_peel_trees.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p, _u64p]
        L.oracle_bc_trees.restype = ctypes.c_int
        L.oracle_bc_trees.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _f64p,
                                      ctypes.POINTER(TreeStats)]
        _TREES = L
    return _TREES


def bc_trees(offsets, adj, sources, nthreads: int = 1):
    """The same ordered-pair BC sums as bc(), computed with pendant trees
    folded (trees_ref.cpp: peel, reach-weighted searches of the kept graph
    from the sources' anchors, closed-form tree terms) -> (bc float64[n],
    stats dict: skipped, roots, teps_edges, peel_seconds, overflow)."""
    offsets, adj = _u32(offsets), _u32(adj)
    s = _u32(sources)
    n = len(offsets) - 1
    out = np.zeros(n, np.float64)
    st = TreeStats()
    rc = _trees_lib().oracle_bc_trees(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p),
                                      s.ctypes.data_as(_u32p), len(s), nthreads, out.ctypes.data_as(_f64p),
                                      ctypes.byref(st))
    if rc:
        raise RuntimeError(f"oracle_bc_trees failed ({rc})")
    return out, {f: getattr(st, f) for f, _ in st._fields_}


def peel_trees(offsets, adj):
    """Host restatement of pendant-tree peeling (trees_ref.cpp) ->
    (anchor uint32[n], subtree size uint32[n], peeled vertex count)."""
    _trees_lib()
    offsets, adj = _u32(offsets), _u32(adj)
    n = len(offsets) - 1
    anc = np.zeros(n, np.uint32)
    sz = np.zeros(n, np.uint32)
    npl = ctypes.c_uint64(0)
    _TREES.oracle_peel_trees(n, offsets.ctypes.data_as(_u32p), adj.ctypes.data_as(_u32p), anc.ctypes.data_as(_u32p),
                             sz.ctypes.data_as(_u32p), ctypes.byref(npl))
    return anc, sz, int(npl.value)


def max_threads() -> int:
    return lib().oracle_max_threads()

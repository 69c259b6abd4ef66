"""The C-ABI libraries load without a GPU and export every symbol that
include/*.h declares (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import bcg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ck-bc_b200")


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bcg_\w+|\w+)\s*\(", txt, flags=re.M)
    return sorted({n for n in names if not n.startswith(("if", "defined"))})


def _exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(PKG, lib)], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_bcg_header_symbols_exported():
    decl = _declared("bcg.h")
    assert "bcg_run" in decl and "bcg_graph_create" in decl and len(decl) >= 20
    exp = _exported("libbcg.so")
    missing = [d for d in decl if d not in exp]
    assert not missing, missing


def test_compat_header_symbols_exported():
    decl = _declared("bc2d_compat.h")
    for must in ("initcuda", "setcuda", "set_mlp_cuda", "scan_col_csc_cuda_mono", "scan_frt_csc_cuda_mono",
                 "pre_update_bc_cuda", "update_bc_cuda", "get_bc", "fincuda"):
        assert must in decl
    exp = _exported("libbc2d_compat.so")
    missing = [d for d in decl if d not in exp]
    assert not missing, missing


def test_python_binding_covers_header():
    decl = _declared("bcg.h")
    assert sorted(decl) == sorted(bcg.SIGNATURES), set(decl) ^ set(bcg.SIGNATURES)


def test_library_loads_without_gpu():
    L = bcg.lib()
    assert isinstance(L, ctypes.CDLL)
    n = bcg.device_count()  # never fails; 0 on a CPU-only host
    assert n >= 0


def test_device_entry_fails_loudly_without_gpu():
    if bcg.device_count() > 0:
        return
    import numpy as np
    try:
        bcg.Graph(np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32))
    except bcg.BcgError as e:
        assert e.code in (bcg.ERR_NOGPU, bcg.ERR_CUDA)
    else:
        raise AssertionError("graph creation must fail without a GPU")

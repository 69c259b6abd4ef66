"""The oracle pinned to the reference program's own output (CPU only).

tests/golden/ref_rmat12_s1_N4096.txt is the result file written by the
reference (ck-bc program/bc-cuda, unmodified sources built as compute_60 PTX)
running on a B200 on the R-MAT scale-12 graph (scale 12, ef 16, seed 1, all 4096
sources); tests/golden/make_ref_fixture.py made it.  The reference keeps delta
and bc in float32 with atomic adds (cuda_kernels.cu:65,69,595) and prints
"%.2f" of bc/2 (bc2d.c:1065), so the bar is half a unit of the last printed
digit plus a float32 accumulation error of 5e-6 relative."""
import os

import numpy as np

import bcg
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "ref_rmat12_s1_N4096.txt")


def _read(path):
    lines = open(path).read().splitlines()
    assert lines[0] == "BC RESULTS" and lines[1] == "ROWPP 4096" and lines[2] == "NodeId\tBC_VAL"
    ids = np.array([int(l.split("\t")[0]) for l in lines[3:]])
    vals = np.array([float(l.split("\t")[1]) for l in lines[3:]])
    return ids, vals


def test_oracle_matches_reference_program_on_rmat12():
    ids, ref = _read(FIXTURE)
    assert ids.tolist() == list(range(4096))
    offs, adj = bcg.generate("rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1")
    bc, st = oracle.bc(offs, adj, np.arange(4096, dtype=np.uint32), nthreads=oracle.max_threads())
    half = bc / 2
    tol = 0.005 + 1e-9 + 5e-6 * np.abs(half)
    bad = np.nonzero(np.abs(ref - half) > tol)[0]
    assert bad.size == 0, (bad[:10], ref[bad[:10]], half[bad[:10]])
    # the reference's uint32 sigma cannot have wrapped on this graph
    assert not st["overflow"]

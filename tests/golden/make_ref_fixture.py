"""Runs the reference program (ck-bc program/bc-cuda, built from its own
sources by `make -C oracle ref` into oracle/_ref/bc2d_ref) on the R-MAT
scale-12 graph and stores its result file as a fixture:

  tests/golden/ref_rmat12_s1_N4096.txt   reference output, "%d\\t%.2f" of bc/2
  tests/golden/rmat12_s1.txt             (not kept) edge list it was run on

Graph: R-MAT scale 12, edge factor 16, (a,b,c,d) = (0.57,0.19,0.19,0.05),
seed 1, undirected, duplicates and self-loops removed; all 4096 sources
(bc2d -p 1x1 -f <file> -n 4096 -r 0 -N 4096, no pruning).

The reference keeps sigma in uint32 and delta/bc in float32; the fixture pins
the CPU oracle to the reference's own numbers within float32 accuracy
(tests/test_ref_fixture.py).  The reference binary needs a GPU, so this runs on
a GPU machine: python tests/golden/make_ref_fixture.py <path/to/bc2d_ref>
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ck-bc_b200"))

import bcg  # noqa: E402

SPEC = "rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1"
OUT = os.path.join(HERE, "ref_rmat12_s1_N4096.txt")


def main():
    ref_bin = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "oracle", "_ref", "bc2d_ref")
    offs, adj = bcg.generate(SPEC)
    n = len(offs) - 1
    with tempfile.TemporaryDirectory() as td:
        gfile = os.path.join(td, "rmat12_s1.txt")
        bcg.write_edgelist(gfile, offs, adj)
        prefix = os.path.join(td, "res")
        r = subprocess.run([ref_bin, "-p", "1x1", "-f", gfile, "-n", str(n), "-r", "0", "-N", str(n),
                            "-o", prefix], capture_output=True, text=True, timeout=1800)
        sys.stdout.write(r.stdout[-3000:])
        sys.stderr.write(r.stderr[-3000:])
        if r.returncode != 0:
            raise SystemExit(f"reference program failed with {r.returncode}")
        with open(prefix + "_1X1_0.log") as f, open(OUT, "w") as g:
            g.write(f.read())
    print("wrote", OUT)


if __name__ == "__main__":
    main()

"""The drop-in command line (ck-bc_b200/bc2d) and the reference's own host
driver linked over the compat library, checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import bcg
import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BC2D = os.path.join(ROOT, "ck-bc_b200", "bc2d")
REF_ON_BCG = os.path.join(ROOT, "oracle", "_ref", "bc2d_on_bcg")


def _read_result(path):
    with open(path) as f:
        lines = f.read().splitlines()
    assert lines[0] == "BC RESULTS"
    assert lines[1].startswith("ROWPP ")
    assert lines[2] == "NodeId\tBC_VAL"
    ids, vals = [], []
    for ln in lines[3:]:
        a, b = ln.split("\t")
        ids.append(int(a))
        vals.append(float(b))
    return int(lines[1].split()[1]), np.array(ids), np.array(vals)


@pytest.fixture(scope="module")
def graph_file(tmp_path_factory):
    offs, adj = bcg.generate("rmat:scale=10,ef=8,seed=21,pendant_frac=0.1,pendant_mean=4")
    d = tmp_path_factory.mktemp("cli")
    p = str(d / "g.txt")
    bcg.write_edgelist(p, offs, adj)
    return p, offs, adj


@pytest.mark.parametrize("heur", ["0", "1", "1T"])
def test_cli_range_full_precision(graph_file, tmp_path, heur):
    path, offs, adj = graph_file
    n = len(offs) - 1
    out = str(tmp_path / "res")
    extra = ["-T"] if heur.endswith("T") else []
    r = subprocess.run([BC2D, "-p", "1x1", "-f", path, "-n", str(n), "-r", "5", "-N", "300", "-H", heur[0],
                        "-o", out, "-F"] + extra, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "BC rounds" in r.stdout and "RESULTS" in r.stdout
    rowpp, ids, vals = _read_result(out + "_1X1_0.log")
    assert rowpp == n and ids.tolist() == list(range(n))
    ref, st = oracle.bc(offs, adj, np.arange(5, 305, dtype=np.uint32))
    np.testing.assert_allclose(vals, ref / 2, rtol=1e-9, atol=1e-9)
    assert f"task 0 BC skipped: {st['skipped']} " in r.stdout


def test_cli_two_decimals_and_source_file(graph_file, tmp_path):
    path, offs, adj = graph_file
    n = len(offs) - 1
    src = bcg.sample_sources(n, 50, 9)
    sf = tmp_path / "src.txt"
    sf.write_text("\n".join(str(s) for s in src) + "\n")
    out = str(tmp_path / "res2")
    r = subprocess.run([BC2D, "-p", "1x1", "-f", path, "-n", str(n), "-s", str(sf), "-o", out],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    _, _, vals = _read_result(out + "_1X1_0.log")
    ref, _ = oracle.bc(offs, adj, src)
    # "%.2f" of bc/2 (bc2d.c:1065): within half a unit of the last digit
    assert np.all(np.abs(vals - ref / 2) <= 0.005 + 1e-9)


def test_cli_errors(graph_file, tmp_path):
    path, offs, _ = graph_file
    n = len(offs) - 1
    r = subprocess.run([BC2D, "-p", "1x1", "-f", path, "-n", "3"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "invalid edge" in r.stderr
    r = subprocess.run([BC2D, "-p", "2x1", "-f", path, "-n", str(n)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    r = subprocess.run([BC2D, "-p", "1x1", "-f", path, "-n", str(n), "-r", str(n)], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode != 0 and "Invalid start vertex" in r.stderr
    r = subprocess.run([BC2D], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Usage" in r.stderr


def test_cli_generated_rmat(tmp_path):
    out = str(tmp_path / "gen")
    r = subprocess.run([BC2D, "-p", "1x1", "-S", "9", "-E", "8", "-N", "64", "-o", out, "-F"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    offs, adj = bcg.generate("rmat:scale=9,ef=8,a=0.57,b=0.19,c=0.19,seed=1")
    _, _, vals = _read_result(out + "_1X1_0.log")
    ref, _ = oracle.bc(offs, adj, np.arange(64, dtype=np.uint32))
    np.testing.assert_allclose(vals, ref / 2, rtol=1e-9, atol=1e-9)


@pytest.mark.skipif(not os.path.exists(REF_ON_BCG), reason="reference host driver not linked (needs the "
                                                            "reference sources at build time)")
@pytest.mark.parametrize("start,count", [(0, 200), (37, 53)])
def test_reference_host_driver_over_compat(graph_file, tmp_path, start, count):
    """The reference's unmodified bc2d.c linked against libbc2d_compat.so.  The
    shim searches sources six at a time ahead of the driver; a range that
    ends inside such a batch must leave the candidates past its end out."""
    path, offs, adj = graph_file
    n = len(offs) - 1
    out = str(tmp_path / "refres")
    r = subprocess.run([REF_ON_BCG, "-p", "1x1", "-f", path, "-n", str(n), "-r", str(start), "-N", str(count),
                        "-o", out], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    _, ids, vals = _read_result(out + "_1X1_0.log")
    ref, _ = oracle.bc(offs, adj, np.arange(start, start + count, dtype=np.uint32))
    # float32 get_bc and "%.2f" output (cuda_kernels.cu:1039-1041, bc2d.c:1065)
    assert np.all(np.abs(vals - ref / 2) <= 0.005 + 2e-7 * np.abs(ref))


def test_cli_binary_cache(graph_file, tmp_path):
    """-B writes the binary CSR cache on the first run and reads it on the
    second (the text file is then not needed); both runs give the same file."""
    path, offs, adj = graph_file
    n = len(offs) - 1
    cache = str(tmp_path / "g.bcsr")
    outs = []
    for i, f in enumerate([path, str(tmp_path / "absent.txt")]):
        out = str(tmp_path / f"res{i}")
        r = subprocess.run([BC2D, "-p", "1x1", "-f", f, "-n", str(n), "-N", "64", "-B", cache, "-o", out, "-F"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert os.path.exists(cache)
        outs.append(_read_result(out + "_1X1_0.log")[2])
    np.testing.assert_array_equal(outs[0], outs[1])
    ref, _ = oracle.bc(offs, adj, np.arange(64, dtype=np.uint32))
    np.testing.assert_allclose(outs[1], ref / 2, rtol=1e-9, atol=1e-9)

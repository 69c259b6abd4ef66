"""bcg_bc_noalloc, the entry point that allocates no device memory.

Collected last (file name) so that it runs both after every other test and,
on its own, in a fresh process (pytest tests/test_zz_no_alloc.py).  The GPU
tests compare it with the handle path (bcg_graph_create + bcg_run) on calls
made back to back with different graphs, check that further calls leave the
device's free memory unchanged, and check the accumulate flag and the
device-side input checks.  Device buffers of the inputs are the test's own
(torch); the entry point itself only uses its static scratch."""
import numpy as np
import pytest

import bcg
import oracle
from test_gpu_parity import assert_bc_close

SPECS = {
    "rmat12": "rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1",  # has >256-entry hubs
    "grid40": "grid:w=40,h=30,drop=0.05,seed=3",                   # deep, no hubs
    "er11": "er:scale=11,ef=8,seed=4",
}


def _expected(offs, adj, src):
    with bcg.Graph(offs, adj) as G:
        G.run(src)
        return G.bc()


class _DevGraph:
    """The inputs of one call as device tensors (uint32 data viewed as int32)."""

    def __init__(self, torch, offs, adj, src):
        self.n = len(offs) - 1
        self.nnz = len(adj)
        self.nsrc = len(src)
        self.offs = torch.from_numpy(np.ascontiguousarray(offs, np.uint32).view(np.int32)).cuda()
        self.adj = torch.from_numpy(np.ascontiguousarray(adj, np.uint32).view(np.int32)).cuda()
        self.src = torch.from_numpy(np.ascontiguousarray(src, np.uint32).view(np.int32)).cuda()
        self.bc = torch.full((self.n,), -1.0, dtype=torch.float64, device="cuda")

    def call(self, accumulate=False, src=None, nsrc=None):
        s = self.src if src is None else src
        bcg.bc_noalloc(self.offs.data_ptr(), self.adj.data_ptr(), self.n, self.nnz, s.data_ptr(),
                       self.nsrc if nsrc is None else nsrc, self.bc.data_ptr(), accumulate)
        return self.bc.cpu().numpy()


def test_size_limits_rejected():
    """Sizes beyond the static scratch are refused before any device work
    (no GPU needed: the null pointers are never touched)."""
    cases = [(bcg.NOALLOC_MAX_VERTICES + 1, 0, 0, "vertices"),
             (16, bcg.NOALLOC_MAX_ADJ + 1, 0, "adjacency entries"),
             (16, 0, bcg.NOALLOC_MAX_SOURCES + 1, "sources")]
    for n, nnz, nsrc, word in cases:
        with pytest.raises(bcg.BcgError) as ei:
            bcg.bc_noalloc(0, 0, n, nnz, 0, nsrc, 0)
        assert ei.value.code == bcg.ERR_RANGE
        assert "no-allocation limit" in str(ei.value) and word in str(ei.value)


@pytest.mark.gpu
def test_calls_in_a_row_match_handle_path():
    torch = pytest.importorskip("torch")
    inputs = {}
    for name, spec in SPECS.items():
        offs, adj = bcg.generate(spec)
        n = len(offs) - 1
        src = bcg.sample_sources(n, min(n, 300), 5) if name != "grid40" else np.arange(n, dtype=np.uint32)
        inputs[name] = (offs, adj, src, _expected(offs, adj, src), _DevGraph(torch, offs, adj, src))
    torch.cuda.synchronize()
    order = ["rmat12", "grid40", "rmat12", "er11", "grid40"]
    free_after_first = None
    got = {}
    for i, name in enumerate(order):
        offs, adj, src, ref, dg = inputs[name]
        bc = dg.call()
        assert_bc_close(bc, ref, f"call {i} ({name})")
        if i < 3:  # and against the oracle itself
            assert_bc_close(bc, oracle.bc(offs, adj, src, nthreads=oracle.max_threads())[0], f"oracle {name}")
        if name in got:  # the same input again after other graphs used the scratch
            assert_bc_close(bc, got[name], f"repeat of {name}")
        got[name] = bc
        if i == 0:
            torch.cuda.synchronize()
            free_after_first = torch.cuda.mem_get_info()[0]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_after_first, "device free memory changed across calls"


@pytest.mark.gpu
def test_accumulate_and_skip():
    torch = pytest.importorskip("torch")
    offs, adj = bcg.generate(SPECS["rmat12"])
    n = len(offs) - 1
    src = np.arange(n, dtype=np.uint32)  # includes degree-0 vertices (skipped)
    ref = _expected(offs, adj, src)
    dg = _DevGraph(torch, offs, adj, src)
    half = n // 2
    dg.call(accumulate=False, nsrc=half)
    second = dg.src[half:].contiguous()
    bc = dg.call(accumulate=True, src=second, nsrc=n - half)
    assert_bc_close(bc, ref, "two accumulated halves")
    bc = dg.call(accumulate=False)
    assert_bc_close(bc, ref, "overwrite")


@pytest.mark.gpu
def test_invalid_input_found_on_device():
    torch = pytest.importorskip("torch")
    offs, adj = bcg.generate(SPECS["er11"])
    n = len(offs) - 1
    src = np.arange(0, n, 7, dtype=np.uint32)
    ref = _expected(offs, adj, src)
    bad_adj = adj.copy()
    bad_adj[len(adj) // 2] = n + 5
    dg = _DevGraph(torch, offs, bad_adj, src)
    with pytest.raises(bcg.BcgError) as ei:
        dg.call()
    assert ei.value.code == bcg.ERR_ARG and "adjacency id >= n" in str(ei.value)
    bad_src = src.copy()
    bad_src[3] = n
    dg = _DevGraph(torch, offs, adj, bad_src)
    with pytest.raises(bcg.BcgError) as ei:
        dg.call()
    assert ei.value.code == bcg.ERR_ARG and "source id >= n at position 3" in str(ei.value)
    bad_offs = offs.copy()
    bad_offs[-1] += 1
    dg = _DevGraph(torch, bad_offs, adj, src)
    with pytest.raises(bcg.BcgError) as ei:
        dg.call()
    assert ei.value.code == bcg.ERR_ARG and "offsets" in str(ei.value)
    # the scratch is usable again right after a rejected call
    dg = _DevGraph(torch, offs, adj, src)
    assert_bc_close(dg.call(), ref, "after rejected calls")


@pytest.mark.gpu
def test_overflowing_counts_switch_to_extended():
    """A 256 x 256 grid (65,536 vertices, at the vertex limit): path counts
    reach about 2^505, past uint64.  The call must redo the sweep with
    extended-range counts from the accumulators it saved, so an accumulating
    call adds exactly one run's worth on top of what d_bc held."""
    torch = pytest.importorskip("torch")
    offs, adj = bcg.generate("grid:w=256,h=256,drop=0.0,seed=1")
    n = len(offs) - 1
    assert n == bcg.NOALLOC_MAX_VERTICES
    src = np.array([0, 255, 32768, 40000, 65535, 12345], dtype=np.uint32)
    ref, _ = oracle.bc_q(offs, adj, src, nthreads=oracle.max_threads())
    dg = _DevGraph(torch, offs, adj, src)
    dg.bc.fill_(1.0)
    bc = dg.call(accumulate=True)
    assert_bc_close(bc, ref + 1.0, "grid 256x256, accumulate on 1.0")
    bc = dg.call(accumulate=False)
    assert_bc_close(bc, ref, "grid 256x256, overwrite")

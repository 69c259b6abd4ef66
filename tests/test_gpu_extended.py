"""GPU parity of extended-range path counts (bcg_set_sigma_mode,
bcg_single_source_ext) against the oracle's __float128 restatement.

Grids have path counts far beyond uint64 (2^350 on a 300 x 300 grid; the
full-size 2048 x 2048 grid, tested in test_gpu_fullsize.py, passes 2^2000,
beyond double's range).  Levels must be exact, log2 sigma within 1e-9, delta and
bc within 1e-9 relative; the automatic mode must switch to extended counts
only when a count overflows, and the exact mode must refuse."""
import numpy as np
import pytest

import bcg
import oracle
from test_gpu_parity import assert_bc_close

pytestmark = pytest.mark.gpu

GRID40 = "grid:w=40,h=40,drop=0.03,seed=5"
GRID300 = "grid:w=300,h=300,drop=0.05,seed=3"


def _check_single(G, offs, adj, s):
    lvl, slog, dl = G.single_source_ext(s)
    ol, oslog, odl = oracle.single_source_q(offs, adj, s)
    assert np.array_equal(lvl, ol), s
    fin = np.isfinite(oslog)
    assert np.array_equal(np.isfinite(slog), fin), s
    assert np.max(np.abs(slog[fin] - oslog[fin])) < 1e-9, s
    assert_bc_close(dl, odl, f"delta s={s}")
    return oslog[fin].max()


def test_auto_switches_to_extended_on_grid():
    offs, adj = bcg.generate(GRID40)
    n = len(offs) - 1
    src = np.arange(0, n, 7, dtype=np.uint32)
    ref, _ = oracle.bc_q(offs, adj, src, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj) as G:
        st = G.run(src)
        assert st.extended_sigma == 1
        assert_bc_close(G.bc(), ref, "grid40 auto")
        G.set_sigma_mode(bcg.SIGMA_EXACT)
        G.reset()
        with pytest.raises(bcg.BcgError) as ei:
            G.run(src)
        assert ei.value.code == bcg.ERR_OVERFLOW
        with pytest.raises(bcg.BcgError):
            G.single_source(0)  # uint64 counts requested
        assert _check_single(G, offs, adj, 0) > 64


def test_auto_stays_exact_when_counts_fit():
    offs, adj = bcg.generate("rmat:scale=11,ef=8,seed=9")
    with bcg.Graph(offs, adj) as G:
        st = G.run(np.arange(200, dtype=np.uint32))
        assert st.extended_sigma == 0


@pytest.mark.parametrize("width", [1, 3, 6])
def test_extended_mode_on_rmat_with_hubs(width):
    offs, adj = bcg.generate("rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1")
    src = bcg.sample_sources(len(offs) - 1, 120, 4)
    ref, _ = oracle.bc(offs, adj, src)
    with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G:
        G.set_sigma_mode(bcg.SIGMA_EXTENDED)
        G.set_batch_width(width)
        st = G.run(src)
        assert st.extended_sigma == 1
        assert_bc_close(G.bc(), ref, f"rmat12 extended w={width}")


def test_grid_beyond_double_range():
    offs, adj = bcg.generate(GRID300)
    n = len(offs) - 1
    src = bcg.sample_sources(n, 6, 3)
    ref, _ = oracle.bc_q(offs, adj, src, nthreads=oracle.max_threads())
    with bcg.Graph(offs, adj, bcg.PRUNE_DEGREE1) as G:
        st = G.run(src)
        assert st.extended_sigma == 1 and st.max_depth > 300
        assert_bc_close(G.bc(), ref, "grid300 pruned")
    with bcg.Graph(offs, adj) as G:
        assert _check_single(G, offs, adj, int(src[0])) > 300

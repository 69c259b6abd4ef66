"""GPU parity of the serving form (bcg_server_*).

Every request's result must equal the oracle's BC of its graph over its
sources, and the same request served alone, within 1e-9 relative; requests
that do not fit the HBM budget wait for admission and still finish."""
import numpy as np
import pytest

import bcg
import oracle
from test_gpu_parity import assert_bc_close

pytestmark = pytest.mark.gpu

SPECS = ["rmat:scale=9,ef=16,a=0.57,b=0.19,c=0.19,seed=21",
         "er:scale=8,ef=4,seed=22",
         "rmat:scale=10,ef=8,a=0.57,b=0.19,c=0.19,seed=23",
         "grid:w=20,h=15,drop=0.05,seed=24",
         "rmat:scale=7,ef=4,seed=25"]
BUDGET = 8 << 30


@pytest.fixture(scope="module")
def pool():
    return [bcg.generate(s) for s in SPECS]


def _requests(pool, seed=3, count=18):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        g = int(rng.integers(0, len(pool)))
        n = len(pool[g][0]) - 1
        if i % 3 == 0:
            reqs.append((g, None))
        else:
            k = int(rng.integers(1, min(n, 300)))
            reqs.append((g, np.sort(rng.choice(n, size=k, replace=False)).astype(np.uint32)))
    return reqs


def _serve(pool, reqs, budget=BUDGET, wave_batches=8):
    out = {}
    with bcg.Server(pool, budget, wave_batches) as S:
        ids = [S.submit(g, src) for g, src in reqs]
        pending_seen = S.info()["pending"]
        left = set(ids)
        for _ in range(100000):
            for rid in S.step():
                out[rid] = S.result(rid)
                left.discard(rid)
            if not left:
                break
        assert not left, "requests did not finish"
        waves = S.info()["waves"]
    return [out[i] for i in ids], pending_seen, waves


def _oracle(pool, g, src):
    offs, adj = pool[g]
    n = len(offs) - 1
    s = np.arange(n, dtype=np.uint32) if src is None else src
    return oracle.bc(offs, adj, s)[0]


def test_mix_matches_oracle_and_alone(pool):
    reqs = _requests(pool)
    mixed, _, waves = _serve(pool, reqs)
    assert waves >= 2
    for i, (g, src) in enumerate(reqs):
        assert_bc_close(mixed[i], _oracle(pool, g, src), f"request {i} vs oracle")
    for i in (0, 1, 5, 11):
        alone, _, _ = _serve(pool, [reqs[i]])
        assert_bc_close(mixed[i], alone[0], f"request {i} mix vs alone")


def test_budget_defers_admission(pool):
    reqs = _requests(pool, seed=4, count=8)
    with bcg.Server(pool, BUDGET) as S:
        resident = S.info()["resident_bytes"]
    n_max = max(len(o) - 1 for o, _ in pool)
    budget = resident + 2 * 8 * n_max  # room for about two result buffers
    served, pending_seen, _ = _serve(pool, reqs, budget=budget)
    assert pending_seen > 0
    for i, (g, src) in enumerate(reqs):
        assert_bc_close(served[i], _oracle(pool, g, src), f"request {i} under a tight budget")


def test_errors(pool):
    with bcg.Server(pool, BUDGET) as S:
        with pytest.raises(bcg.BcgError):
            S.submit(len(pool), None)
        with pytest.raises(bcg.BcgError):
            S.submit(0, np.array([len(pool[0][0])], dtype=np.uint32))
    with pytest.raises(bcg.BcgError) as ei:
        bcg.Server(pool, 1 << 10)
    assert ei.value.code == bcg.ERR_OOM

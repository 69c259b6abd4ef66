"""GPU parity of the serving form (bcg_server_*).

Every request's result must equal the oracle's BC of its graph over its
sources within 1e-9 relative, and the same request served alone bit for bit
(each source's dependencies reach the request's buffer in source order,
however the wave packs them); requests that do not fit the HBM budget wait
for admission and still finish; requests submitted from another thread
while waves are on the GPU are admitted and served."""
import threading
import time

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
            for rid in S.wait():
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
        assert np.array_equal(mixed[i].view(np.uint64), alone[0].view(np.uint64)), f"request {i} bits"


def test_same_graph_requests_share_waves(pool):
    """Six k-source requests on one graph fit one wave together: they share
    its batches (and adjacency passes) instead of taking a wave each."""
    rng = np.random.default_rng(9)
    n = len(pool[2][0]) - 1
    reqs = [(2, np.sort(rng.choice(n, size=40, replace=False)).astype(np.uint32)) for _ in range(6)]
    served, _, waves = _serve(pool, reqs, wave_batches=64)
    assert waves == 1
    for i, (g, src) in enumerate(reqs):
        assert_bc_close(served[i], _oracle(pool, g, src), f"shared request {i}")
        alone, _, _ = _serve(pool, [reqs[i]], wave_batches=64)
        assert np.array_equal(served[i].view(np.uint64), alone[0].view(np.uint64))


def test_submit_while_waves_run(pool):
    """A second thread submits requests while the first keeps stepping: each
    late request is admitted during a wave in flight and finishes with the
    oracle's result."""
    reqs = _requests(pool, seed=6, count=16)
    early, late = reqs[:6], reqs[6:]
    out, ids_late, seen_running = {}, [], []
    with bcg.Server(pool, BUDGET, 2) as S:
        ids_early = [S.submit(g, src) for g, src in early]
        stop = threading.Event()

        def submitter():
            for g, src in late:
                while not stop.is_set() and S.info()["waves"] == 0:
                    time.sleep(0.0005)
                seen_running.append(S.info()["running"])
                ids_late.append(S.submit(g, src))
                time.sleep(0.002)

        th = threading.Thread(target=submitter)
        th.start()
        left = None
        for _ in range(200000):
            for rid in S.step():
                out[rid] = S.result(rid)
            if not th.is_alive():
                left = set(ids_early + ids_late) - set(out)
                if not left:
                    break
            time.sleep(0.0002)
        stop.set()
        th.join()
        assert not left
    assert max(seen_running) > 0  # some late request arrived while admitted work was on the GPU
    for rid, (g, src) in zip(ids_early + ids_late, early + late):
        assert_bc_close(out[rid], _oracle(pool, g, src), f"request {rid}")


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

"""Seeded synthetic workloads of the batched and serving forms.

Graph specs are strings for bcg.generate (generator in csrc/graph.cpp).  All
draws come from numpy's PCG64 seeded with the workload seed, so a workload is
the same list on every machine.

Batched set: `count` graphs (2000), seed 4.  Scale is log-uniform in [8, 16]:
a continuous draw exp(U(ln 8, ln 16)) rounded to the nearest integer scale.
The edge factor is an integer drawn uniformly from 8..32 (the generator
takes integer edge factors).  Graphs alternate R-MAT (a, b, c, d) =
(0.57, 0.19, 0.19, 0.05) and Erdos-Renyi G(n, M) with the same number of edge
draws M = ef * 2^scale, i.e. the same mean degree.  Each graph gets its own
generator seed.
"""
from __future__ import annotations

import math

import numpy as np

RMAT_ABC = "a=0.57,b=0.19,c=0.19"


def batched_specs(count: int = 2000, seed: int = 4, smin: float = 8.0, smax: float = 16.0,
                  efmin: int = 8, efmax: int = 32) -> list[str]:
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for i in range(count):
        scale = int(round(math.exp(rng.uniform(math.log(smin), math.log(smax)))))
        ef = int(rng.integers(efmin, efmax + 1))
        gseed = int(rng.integers(1, 2**62))
        if i % 2 == 0:
            specs.append(f"rmat:scale={scale},ef={ef},{RMAT_ABC},seed={gseed}")
        else:
            specs.append(f"er:scale={scale},ef={ef},seed={gseed}")
    return specs


def spec_scale_ef(spec: str) -> tuple[int, int]:
    kv = dict(p.split("=") for p in spec.split(":", 1)[1].split(","))
    return int(kv["scale"]), int(kv["ef"])


# Serving form: a pool of 64 resident R-MAT graphs (scale uniform in 10..22,
# edge factor 16, seed 5) and a Poisson stream of BC requests (seed 5): each
# request names a graph uniformly at random and is exact BC (every vertex)
# or k-source BC with k log-uniform in [64, 1024] (rounded, at most the
# graph's vertex count) and the sources drawn uniformly without replacement.
def serving_pool(count: int = 64, seed: int = 5, smin: int = 10, smax: int = 22, ef: int = 16) -> list[str]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        scale = int(rng.integers(smin, smax + 1))
        out.append(f"rmat:scale={scale},ef={ef},{RMAT_ABC},seed={int(rng.integers(1, 2**62))}")
    return out


def serving_stream(sizes: list[int], count: int = 20000, seed: int = 5, rate: float = 100.0,
                   kmin: int = 64, kmax: int = 1024):
    """-> list of (arrival_s, graph, sources or None for exact); `rate` is the
    Poisson arrival rate in requests per second."""
    rng = np.random.Generator(np.random.PCG64(seed + 1000003))
    t = 0.0
    reqs = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        g = int(rng.integers(0, len(sizes)))
        if rng.random() < 0.5:
            reqs.append((t, g, None))
        else:
            k = int(round(math.exp(rng.uniform(math.log(kmin), math.log(kmax)))))
            k = min(k, sizes[g])
            reqs.append((t, g, np.sort(rng.choice(sizes[g], size=k, replace=False)).astype(np.uint32)))
    return reqs

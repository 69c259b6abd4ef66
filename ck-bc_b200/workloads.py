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

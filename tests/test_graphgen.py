"""The numpy restatement of the seeded generators (oracle/graphgen.py, used
by bench.py's CPU reference arm so that it never loads the product library)
gives the library's graphs and source lists bit for bit."""
import numpy as np
import pytest

import bcg
import graphgen

SPECS = [
    "rmat:scale=10,ef=16,seed=7,pendant_frac=0.1,pendant_mean=4",
    "rmat:scale=12,ef=16,a=0.57,b=0.19,c=0.19,seed=1",
    "rmat:scale=11,ef=4,seed=3,pendant_frac=0.3,pendant_mean=12",
    "er:scale=10,ef=8,seed=4",
]


@pytest.mark.parametrize("spec", SPECS)
def test_graph_bit_identical(spec):
    o1, a1 = bcg.generate(spec)
    o2, a2 = graphgen.generate(spec)
    assert np.array_equal(o1, o2)
    assert np.array_equal(a1, a2)


def test_sources_bit_identical():
    for n, k, seed in [(100000, 4096, 2), (1469267, 4096, 2), (300, 300, 5)]:
        assert np.array_equal(bcg.sample_sources(n, k, seed), graphgen.sample_sources(n, k, seed))


def test_other_generators_refused():
    with pytest.raises(ValueError):
        graphgen.generate("grid:w=4,h=4,drop=0.0,seed=1")

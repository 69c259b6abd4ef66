"""Extended-range path counts (CPU only).

1. The arithmetic of ck-bc_b200/csrc/ext64.cuh, compiled for the host into a
   small harness, against exact rational arithmetic: every add, multiply,
   conversion and division must be the exact result rounded to nearest, ties
   to even, on a 49-bit significand.
2. The oracle's __float128 restatement (oracle/brandes.c brandes_one_q)
   against exact big-integer path counts on a grid whose counts overflow
   uint64, and against the uint64 oracle where they fit."""
import math
import os
import random
import subprocess
from fractions import Fraction

import numpy as np
import pytest

import bcg
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIAS = 32768 + 48

HARNESS = r"""
#define __host__
#define __device__
#define __forceinline__ inline
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "ext64.cuh"
using namespace bcg;
int main() {
    char op[8];
    unsigned long long a, b;
    double x;
    int k;
    while (scanf("%7s", op) == 1) {
        if (!strcmp(op, "add") && scanf("%llx %llx", &a, &b) == 2) printf("%llx\n", ext_add(a, b));
        else if (!strcmp(op, "mul") && scanf("%llx %llx", &a, &b) == 2) printf("%llx\n", ext_mul(a, b));
        else if (!strcmp(op, "fd") && scanf("%la %d", &x, &k) == 2) printf("%llx\n", ext_from_double(x, k));
        else if (!strcmp(op, "td") && scanf("%llx", &a) == 1) printf("%a\n", ext_to_double(a));
        else if (!strcmp(op, "div") && scanf("%la %llx", &x, &a) == 2) printf("%llx\n", ext_div(x, a));
    }
}
"""


def decode(e):
    if e == 0:
        return Fraction(0)
    E, f = e >> 48, e & ((1 << 48) - 1)
    return Fraction((1 << 48) + f) * Fraction(2) ** (E - BIAS)


def round_ext(q: Fraction) -> int:
    """Exact value -> encoding, round to nearest even on 49 bits."""
    if q == 0:
        return 0
    e2 = math.floor(math.log2(q.numerator) - math.log2(q.denominator))
    while Fraction(2) ** e2 > q:
        e2 -= 1
    while Fraction(2) ** (e2 + 1) <= q:
        e2 += 1
    scaled = q / Fraction(2) ** (e2 - 48)  # in [2^48, 2^49)
    m = scaled.numerator // scaled.denominator
    rem = scaled - m
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and m % 2 == 1):
        m += 1
    if m == 1 << 49:
        m >>= 1
        e2 += 1
    E = e2 + BIAS - 48  # value = m * 2^(E - BIAS) with q ~ m * 2^(e2 - 48)
    return (E << 48) | (m - (1 << 48))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("ext64")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "ck-bc_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)

    def run(lines):
        r = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
        return r.stdout.split()

    return run


def _rand_ext(rng):
    E = rng.randint(32768 - 3000, 32768 + 3000)
    return (E << 48) | rng.getrandbits(48)


def test_add_mul_round_to_nearest_even(harness):
    rng = random.Random(7)
    pairs = [(_rand_ext(rng), _rand_ext(rng)) for _ in range(300)]
    # close exponents and exact ties, where rounding decides
    for _ in range(200):
        a = _rand_ext(rng)
        b = ((a >> 48) - rng.randint(0, 60) << 48) | rng.getrandbits(48)
        pairs.append((a, b))
    pairs += [(0, 0x8000000000000000), (0x8000000000000000, 0), (0x8000000000000000, 0x8000000000000000),
              (0x8000000000000001, 0x7FCF000000000000)]
    out = harness([f"add {a:x} {b:x}" for a, b in pairs] + [f"mul {a:x} {b:x}" for a, b in pairs])
    for i, (a, b) in enumerate(pairs):
        assert int(out[i], 16) == round_ext(decode(a) + decode(b)), (hex(a), hex(b))
        if a and b:
            assert int(out[len(pairs) + i], 16) == round_ext(decode(a) * decode(b)), (hex(a), hex(b))


def test_conversions_and_division(harness):
    rng = random.Random(11)
    xs = [rng.uniform(0.1, 1e6) * 2.0 ** rng.randint(-300, 300) for _ in range(200)] + [1.0, 0.5, 3.0, 2.0**-1074]
    ks = [rng.randint(-4000, 4000) for _ in xs]
    exts = [_rand_ext(rng) for _ in range(200)]
    lines = [f"fd {x.hex()} {k}" for x, k in zip(xs, ks)]
    lines += [f"td {e:x}" for e in exts]
    lines += [f"div {x.hex()} {e:x}" for x, e in zip(xs, exts)]
    out = harness(lines)
    for i, (x, k) in enumerate(zip(xs, ks)):
        assert int(out[i], 16) == round_ext(Fraction(x) * Fraction(2) ** k), (x, k)
    off = len(xs)
    for j, e in enumerate(exts):
        v = float.fromhex(out[off + j])
        want = decode(e)
        if want > Fraction(2) ** 1023 or want < Fraction(2) ** -1000:
            continue  # outside the double range (the engine never converts these)
        assert v == float(want), hex(e)  # 49 bits fit a double exactly
    off += len(exts)
    for j, (x, e) in enumerate(zip(xs, exts)):
        got = decode(int(out[off + j], 16))
        want = Fraction(x) / decode(e)
        assert abs(got - want) <= want * Fraction(1, 2**47), (x, hex(e))  # one double division, then rounding


def _exact_sigma(offs, adj, s):
    n = len(offs) - 1
    lvl = [-1] * n
    sig = [0] * n
    lvl[s], sig[s] = 0, 1
    frontier = [s]
    while frontier:
        nxt = []
        for c in frontier:
            for r in adj[offs[c]:offs[c + 1]]:
                if lvl[r] == -1:
                    lvl[r] = lvl[c] + 1
                    nxt.append(r)
                if lvl[r] == lvl[c] + 1:
                    sig[r] += sig[c]
        frontier = nxt
    return lvl, sig


def test_oracle_q_exact_counts_beyond_uint64():
    offs, adj = bcg.generate("grid:w=40,h=40,drop=0.03,seed=5")
    lvl, sig = _exact_sigma(offs, adj.tolist(), 0)
    assert max(sig).bit_length() > 64
    ql, qs, _ = oracle.single_source_q(offs, adj, 0)
    assert ql.tolist() == lvl
    for v in range(len(sig)):
        if sig[v]:
            assert abs(qs[v] - math.log2(sig[v])) < 1e-12


def test_oracle_q_matches_uint64_oracle_where_it_fits(golden):
    for name, g in list(golden["graphs"].items())[:8]:
        offs, adj = bcg.from_pairs(np.array(g["edges"], dtype=np.uint64).reshape(-1, 2), g["n"])
        src = g["sources"] if g["sources"] is not None else list(range(g["n"]))
        b1, _ = oracle.bc(offs, adj, src)
        b2, _ = oracle.bc_q(offs, adj, src)
        np.testing.assert_allclose(b2, b1, rtol=1e-12, atol=1e-12, err_msg=name)
        np.testing.assert_allclose(b2 / 2, np.array(g["bc_half"]), rtol=1e-12, atol=1e-12, err_msg=name)

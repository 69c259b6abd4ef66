"""ORACLE — test infrastructure only.

A numpy restatement of the engine's seeded synthetic graph generators (R-MAT,
Erdős–Rényi, pendant trees) and of its source sampler, so that the CPU
reference arm of bench.py can build the benchmark graph without loading the
product library.  Output is bit-identical to bcg_csr_generate /
bcg_sample_sources (tests/test_graphgen.py checks it): the same splitmix64
streams, the same draws in the same order, the same CSR normalisation
(mirror, drop self-loops and duplicates, sorted lists; the reference's
mirror + norm_graph, bc2d.c:152-170, 430-453).

splitmix64 (Steele, Lea, Flood 2014) advances its state by a constant, so
draw k of a stream that starts at state s is mix(s + (k + 1) * GAMMA): the
R-MAT draws are computed for whole blocks of edges at once.
"""
from __future__ import annotations

import math

import numpy as np

GAMMA = 0x9E3779B97F4A7C15
M64 = (1 << 64) - 1
CHUNK = 1 << 16


def _mix(z):
    """splitmix64 output function on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _mix_int(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


class _Stream:
    """Sequential splitmix64 stream (scalar draws)."""

    def __init__(self, state: int):
        self.s = state & M64

    def next(self) -> int:
        self.s = (self.s + GAMMA) & M64
        return _mix_int(self.s)

    def u01(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def below(self, r: int) -> int:
        return (self.next() * r) >> 64


def stream_seed(seed: int, idx: int) -> int:
    s = (seed ^ ((0xD1B54A32D192ED03 * (idx + 1)) & M64)) & M64
    return _mix_int((s + GAMMA) & M64)


def _draws(st0, k):
    """Draw number k (uint64 array) of the streams starting at states st0."""
    with np.errstate(over="ignore"):
        return _mix(st0 + (k + np.uint64(1)) * np.uint64(GAMMA))


def _below_vec(z, r: int):
    """(z * r) >> 64 for r < 2^32, exact."""
    zh = z >> np.uint64(32)
    zl = z & np.uint64(0xFFFFFFFF)
    r = np.uint64(r)
    with np.errstate(over="ignore"):
        return (zh * r + ((zl * r) >> np.uint64(32))) >> np.uint64(32)


def rmat_pairs(scale: int, ef: int, a: float, b: float, c: float, seed: int):
    m = ef << scale
    ab, abc = a + b, a + b + c
    u = np.zeros(m, np.uint64)
    v = np.zeros(m, np.uint64)
    nch = (m + CHUNK - 1) // CHUNK
    seeds = np.array([stream_seed(seed, ch) for ch in range(nch)], dtype=np.uint64)
    per = 16  # chunks per block
    for c0 in range(0, nch, per):
        c1 = min(nch, c0 + per)
        lo, hi = c0 * CHUNK, min(m, c1 * CHUNK)
        idx = np.arange(lo, hi, dtype=np.uint64)
        ch = (idx // np.uint64(CHUNK)).astype(np.int64)
        local = idx - ch.astype(np.uint64) * np.uint64(CHUNK)
        st0 = seeds[ch]
        uu = np.zeros(hi - lo, np.uint64)
        vv = np.zeros(hi - lo, np.uint64)
        for t in range(scale):
            bit = np.uint64(1) << np.uint64(scale - 1 - t)
            z = _draws(st0, local * np.uint64(scale) + np.uint64(t))
            r = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            vb = (r >= a) & (r < ab)
            ub = (r >= ab) & (r < abc)
            both = r >= abc
            vv |= np.where(vb | both, bit, np.uint64(0))
            uu |= np.where(ub | both, bit, np.uint64(0))
        u[lo:hi] = uu
        v[lo:hi] = vv
    return u, v


def er_pairs(scale: int, ef: int, seed: int):
    n, m = 1 << scale, ef << scale
    u = np.zeros(m, np.uint64)
    v = np.zeros(m, np.uint64)
    nch = (m + CHUNK - 1) // CHUNK
    for ch in range(nch):
        lo, hi = ch * CHUNK, min(m, (ch + 1) * CHUNK)
        st0 = np.uint64(stream_seed(seed, ch))
        k = np.arange(2 * (hi - lo), dtype=np.uint64)
        z = _below_vec(_draws(st0, k), n)
        u[lo:hi] = z[0::2]
        v[lo:hi] = z[1::2]
    return u, v


def sample_distinct(n: int, k: int, seed: int) -> np.ndarray:
    """k distinct values of [0, n), partial Fisher-Yates, in draw order."""
    perm = np.arange(n, dtype=np.uint32)
    st = _Stream(stream_seed(seed, 0x5A4D50))
    out = np.empty(k, np.uint32)
    for i in range(k):
        j = i + st.below(n - i)
        perm[i], perm[j] = perm[j], perm[i]
        out[i] = perm[i]
    return out


def pendant_pairs(n0: int, frac: float, mean: float, seed: int):
    na = int(math.floor(frac * float(n0)))
    if na == 0 or mean < 1.0:
        return n0, np.zeros(0, np.uint64), np.zeros(0, np.uint64)
    anchors = np.sort(sample_distinct(n0, na, seed))
    st = _Stream(stream_seed(seed, 0x7EE))
    p = 1.0 / mean
    lq = math.log1p(-p)
    nxt = n0
    pu, pv = [], []
    for anc in anchors.tolist():
        k = 1
        if p < 1.0:
            r = st.u01()
            k = 1 + int(math.floor(math.log1p(-r) / lq))
        tree = [anc]
        for _ in range(k):
            parent = tree[st.below(len(tree))]
            pu.append(parent)
            pv.append(nxt)
            tree.append(nxt)
            nxt += 1
    return nxt, np.array(pu, np.uint64), np.array(pv, np.uint64)


def build_csr(u, v, n: int):
    """Undirected CSR: mirrored, self-loops and duplicates dropped, lists sorted."""
    keep = u != v
    u, v = u[keep], v[keep]
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    keys = np.unique(src * np.uint64(n) + dst)
    s = (keys // np.uint64(n)).astype(np.int64)
    adj = (keys % np.uint64(n)).astype(np.uint32)
    offs = np.zeros(n + 1, np.uint32)
    np.cumsum(np.bincount(s, minlength=n), out=offs[1:])
    return offs, adj


def _parse(spec: str):
    kind, _, rest = spec.partition(":")
    kv = {}
    for item in rest.split(","):
        if item:
            k, _, val = item.partition("=")
            kv[k.strip()] = float(val)
    return kind.strip(), kv


def generate(spec: str):
    """(offsets uint32[n+1], adj uint32[nnz]) for an rmat/er spec, as bcg.generate."""
    kind, kv = _parse(spec)
    if kind not in ("rmat", "er"):
        raise ValueError(f"graphgen restates the rmat and er generators only, not '{kind}'")
    scale = int(kv.get("scale", 12))
    ef = int(kv.get("ef", 16))
    seed = int(kv.get("seed", 1))
    if kind == "rmat":
        u, v = rmat_pairs(scale, ef, kv.get("a", 0.57), kv.get("b", 0.19), kv.get("c", 0.19), seed)
    else:
        u, v = er_pairs(scale, ef, seed)
    n = 1 << scale
    pfrac = kv.get("pendant_frac", 0.0)
    if pfrac > 0:
        pseed = kv.get("pendant_seed", -1)
        ps = (seed ^ 0x50454E44414E54) if pseed < 0 else int(pseed)
        n, pu, pv = pendant_pairs(n, pfrac, kv.get("pendant_mean", 4.0), ps)
        u = np.concatenate([u, pu])
        v = np.concatenate([v, pv])
    return build_csr(u, v, n)


def sample_sources(n: int, k: int, seed: int) -> np.ndarray:
    return sample_distinct(n, k, seed)

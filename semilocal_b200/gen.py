"""Seeded synthetic inputs for the semi-local LCS workloads (splitmix64 streams, numpy-vectorised).

Every generator is a pure function of its arguments, so the GPU run, the CPU oracle and the reference's
CPU code see byte-identical inputs.  Symbols are uint8 in [0, alphabet); permutations are int32 row->col.

Workload shapes (the reference publishes no dataset for this path; these stand in for it):
  * plain pair: a, b uniform over 4 letters, 8192 each;
  * steady-ant: two independent uniform permutations of size n;
  * hybrid pair: a uniform 2^20, b = a with 5 % substitutions, 0.5 % insertions, 0.5 % deletions;
  * batch: 4096 pairs, |a| log-uniform in [256, 65536], b = a with 10 % substitutions + 1 % indels;
  * serving: Poisson arrivals, lengths log-uniform in [1e3, 1e6], 5 % substitutions + 1 % indels.
"""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """`count` outputs of splitmix64 started at state seed ^ (stream * golden ratio)."""
    with np.errstate(over="ignore"):
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) ^ (np.uint64(stream & 0xFFFFFFFFFFFFFFFF) * _GAMMA)
        z = base + (np.arange(1, count + 1, dtype=np.uint64) * _GAMMA)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int, stream: int = 0) -> np.ndarray:
    return (splitmix64(seed, count, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def uniform_string(n: int, alphabet: int = 4, seed: int = 0, stream: int = 0) -> np.ndarray:
    """n i.i.d. uniform symbols over [0, alphabet) as uint8."""
    if n == 0:
        return np.zeros(0, dtype=np.uint8)
    return ((splitmix64(seed, n, stream) >> np.uint64(32)) % np.uint64(alphabet)).astype(np.uint8)


def mutate(a: np.ndarray, subst: float, ins: float, dele: float, alphabet: int = 4, seed: int = 0) -> np.ndarray:
    """b from a: each position independently is deleted w.p. `dele`; otherwise an extra uniform letter is
    inserted before it w.p. `ins`, and it is replaced by a different letter w.p. `subst`."""
    n = len(a)
    if n == 0:
        return a.copy()
    u_del = uniform01(seed, n, 101)
    u_ins = uniform01(seed, n, 102)
    u_sub = uniform01(seed, n, 103)
    r_sub = (splitmix64(seed, n, 104) >> np.uint64(33)) % np.uint64(max(alphabet - 1, 1))
    r_ins = (splitmix64(seed, n, 105) >> np.uint64(33)) % np.uint64(alphabet)
    keep = u_del >= dele
    sym = a.astype(np.int64)
    sub = u_sub < subst
    sym = np.where(sub, (sym + 1 + r_sub.astype(np.int64)) % alphabet, sym)
    do_ins = (u_ins < ins) & keep
    # output layout: for each kept position, optionally an inserted letter, then the (possibly substituted) letter
    cnt = keep.astype(np.int64) + do_ins.astype(np.int64)
    total = int(cnt.sum())
    out = np.empty(total, dtype=np.uint8)
    ends = np.cumsum(cnt)
    pos_sym = ends[keep] - 1
    out[pos_sym] = sym[keep].astype(np.uint8)
    pos_ins = ends[do_ins] - 2
    out[pos_ins] = r_ins[do_ins].astype(np.uint8)
    return out


def permutation(n: int, seed: int = 0, stream: int = 0) -> np.ndarray:
    """A uniform random permutation of [0, n) (argsort of 64-bit keys), int32 row->col."""
    if n == 0:
        return np.zeros(0, dtype=np.int32)
    keys = splitmix64(seed, n, stream)
    return np.argsort(keys, kind="stable").astype(np.int32)


def loguniform_lengths(count: int, lo: int, hi: int, seed: int = 0, stream: int = 7) -> np.ndarray:
    u = uniform01(seed, count, stream)
    lens = np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)
    return np.clip(lens, lo, hi)


# ---------------------------------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------------------------------

def plain_pair(n: int = 8192, seed: int = 1):
    """Plain pair: a, b i.i.d. uniform over 4 letters (8192 each by default)."""
    return uniform_string(n, 4, seed, 1), uniform_string(n, 4, seed, 2)


def steady_ant_pair(n: int = 1 << 22, seed_p: int = 2, seed_q: int = 3):
    """Two independent uniform permutations of size n."""
    return permutation(n, seed_p), permutation(n, seed_q)


def hybrid_pair(n: int = 1 << 20, seed: int = 4):
    """a uniform over 4 letters; b = a with 5 % substitutions, 0.5 % insertions, 0.5 % deletions."""
    a = uniform_string(n, 4, seed, 1)
    b = mutate(a, 0.05, 0.005, 0.005, 4, seed + 1000)
    return a, b


def batch_pairs(count: int = 4096, lo: int = 256, hi: int = 65536, seed: int = 5):
    """count pairs, |a| log-uniform in [lo, hi], b = a with 10 % substitutions and 1 % indels."""
    lens = loguniform_lengths(count, lo, hi, seed)
    pairs = []
    for i, L in enumerate(lens):
        a = uniform_string(int(L), 4, seed * 1000003 + i, 1)
        b = mutate(a, 0.10, 0.005, 0.005, 4, seed * 1000003 + i + 77)
        pairs.append((a, b))
    return pairs


def planted_text(m: int, n: int, copies: int, alphabet: int = 4, seed: int = 0, subst: float = 0.1,
                 indel: float = 0.02):
    """Approximate pattern search input: a pattern of m uniform symbols and a text of n uniform symbols overwritten
    at `copies` seeded positions by mutated copies of the pattern (substitutions, half insertions, half deletions)."""
    p = uniform_string(m, alphabet, seed, 1)
    t = uniform_string(n, alphabet, seed, 2).copy()
    pos = (uniform01(seed, copies, 3) * max(1, n - m)).astype(np.int64)
    for c, at in enumerate(pos):
        seg = mutate(p, subst, indel / 2, indel / 2, alphabet, seed * 1000 + c)[:max(0, n - int(at))]
        t[int(at):int(at) + len(seg)] = seg
    return p, t


def serving_requests(count: int, rate_hz: float, lo: int = 1000, hi: int = 1_000_000, seed: int = 6):
    """Poisson arrivals at `rate_hz`; each request a pair with log-uniform length and a query kind
    uniform over {global, string-substring, prefix-suffix}.  Returns a list of dicts."""
    gaps = -np.log(1.0 - uniform01(seed, count, 11)) / rate_hz
    t = np.cumsum(gaps)
    lens = loguniform_lengths(count, lo, hi, seed, 12)
    kinds = (splitmix64(seed, count, 13) >> np.uint64(40)) % np.uint64(3)
    qa = uniform01(seed, count, 14)
    qb = uniform01(seed, count, 15)
    reqs = []
    for i in range(count):
        L = int(lens[i])
        a = uniform_string(L, 4, seed * 7919 + i, 1)
        b = mutate(a, 0.05, 0.005, 0.005, 4, seed * 7919 + i + 31)
        kind = ("global", "string_substring", "prefix_suffix")[int(kinds[i])]
        reqs.append({"t": float(t[i]), "a": a, "b": b, "kind": kind, "u": float(qa[i]), "v": float(qb[i])})
    return reqs

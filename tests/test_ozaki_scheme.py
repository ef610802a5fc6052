"""The Ozaki split of the tensor-core Gram (csrc/ptt_ozaki.cuh) restated in
numpy, on the CPU.

* digits: N = rint(x 2^(56 - e_j)), M = N + 128 (1 + 256 + ... + 256^5),
  d_0 = M >> 48, d_s = byte (6 - s) of M minus 128: N = sum_s d_s 256^(6-s)
  exactly, d_0 in [-256, 256], d_s in [-128, 127], every digit exact in BF16;
* the tensor-memory schedule: for s = 0, 2, 4, 6 the product of slices
  (s, s + 1) (M = 128) with slices t0 .. t0 + nb - 1 lands in column blocks
  s + t0 ..; block c holds, in lanes 0-63, sum_{s even} D_s^T D_{c-s} and in
  lanes 64-127 sum_{s even} D_{s+1}^T D_{c-s}: every digit pair with s + t <=
  6 is counted exactly once with weight 256^-(s+t), and every block's sums
  stay below 2^24 (exact FP32 accumulation) for 112 rows of worst-case
  digits;
* the recombined partial Gram matrix matches the exact one (Python
  fractions) to 2^-52 max|x_i| max|x_j| per row."""
from fractions import Fraction

import numpy as np
import pytest

KMAX = 112
C_OFF = 0x0000808080808080
PIECES = [(0, 0, 4), (0, 4, 3), (2, 0, 4), (2, 4, 1), (4, 0, 3), (6, 0, 1)]


def exponents(x):
    e = np.zeros(x.shape[1], dtype=np.int64)
    for j in range(x.shape[1]):
        a = np.max(np.abs(x[:, j])) if x.shape[0] else 0.0
        if a > 0:
            e[j] = np.frexp(a)[1]
    return e


def digits(x, e):
    """(7, h, c) integer digits of x (column exponents e)."""
    h, c = x.shape
    d = np.zeros((7, h, c), dtype=np.int64)
    for j in range(c):
        sh = 56 - int(e[j])
        for k in range(h):
            n = int(np.rint(np.ldexp(x[k, j], sh)))
            m = n + C_OFF
            d[0, k, j] = m >> 48
            for s in range(1, 7):
                d[s, k, j] = ((m >> (8 * (6 - s))) & 0xFF) - 128
    return d


def bf16_exact(v):
    f = np.float32(v)
    return float(f) == v and (np.frombuffer(f.tobytes(), dtype=np.uint32)[0] & 0xFFFF) == 0


def blocks(d):
    """Tensor-memory column blocks (lanes 0-63, lanes 64-127) of the schedule."""
    c = d.shape[2]
    zero = np.zeros_like(d[0])
    sl = list(d) + [zero]  # the eighth slice stays zero
    lo = [np.zeros((c, c), dtype=np.int64) for _ in range(7)]
    hi = [np.zeros((c, c), dtype=np.int64) for _ in range(7)]
    count = {}
    for s, t0, nb in PIECES:
        for t in range(t0, t0 + nb):
            blk = s + t
            lo[blk] += sl[s].T @ sl[t]
            hi[blk] += sl[s + 1].T @ sl[t]
            count[(s, t)] = count.get((s, t), 0) + 1
            count[(s + 1, t)] = count.get((s + 1, t), 0) + 1
    return lo, hi, count


def test_schedule_counts_every_pair_once():
    d = np.zeros((7, 1, 1), dtype=np.int64)
    _, _, count = blocks(d)
    want = {(s, t) for s in range(7) for t in range(7) if s + t <= 6}
    got_used = {p for p in count if p[0] + p[1] <= 6 and p[0] <= 6}
    assert got_used == want
    assert all(count[p] == 1 for p in want)
    # tensor-memory columns of every piece inside 448 of the 512 held
    for s, t0, nb in PIECES:
        assert 64 * (s + t0 + nb) <= 448 and 64 * nb <= 256


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_digits_exact_and_bounded(seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((KMAX, 8)) * np.ldexp(1.0, rng.integers(-200, 200, size=8))[None, :]
    x[3, 2] = 0.0
    x[5, :] = -np.max(np.abs(x), axis=0)  # the column maxima themselves
    e = exponents(x)
    d = digits(x, e)
    assert d[0].min() >= -256 and d[0].max() <= 256
    assert d[1:].min() >= -128 and d[1:].max() <= 127
    for v in np.unique(d):
        assert bf16_exact(float(v))
    for j in range(x.shape[1]):
        for k in range(x.shape[0]):
            n = sum(int(d[s, k, j]) * 256 ** (6 - s) for s in range(7))
            assert n == int(np.rint(np.ldexp(x[k, j], 56 - int(e[j]))))


def test_block_sums_below_2_24_worst_case():
    # worst case: every row at the digit bounds, same signs
    d = np.empty((7, KMAX, 2), dtype=np.int64)
    d[0] = 256
    d[1:] = -128
    lo, hi, _ = blocks(d)
    for b in range(7):
        assert np.abs(lo[b]).max() < 2 ** 24
        if b <= 5:
            assert np.abs(hi[b]).max() < 2 ** 24


@pytest.mark.parametrize("seed", [0, 1])
def test_recombined_gram_vs_exact(seed):
    rng = np.random.default_rng(seed)
    h, c = 40, 6
    x = rng.standard_normal((h, c)) * np.ldexp(1.0, rng.integers(-30, 30, size=c))[None, :]
    e = exponents(x)
    lo, hi, _ = blocks(digits(x, e))
    cmax = np.max(np.abs(x), axis=0)
    for i in range(c):
        for j in range(c):
            a = Fraction(0)
            for b in range(7):
                a += Fraction(int(lo[b][i, j]), 256 ** b)
                if b <= 5:
                    a += Fraction(int(hi[b][i, j]), 256 ** (b + 1))
            got = a * Fraction(2) ** (int(e[i]) + int(e[j]) - 16)
            exact = sum(Fraction(float(x[k, i])) * Fraction(float(x[k, j])) for k in range(h))
            assert abs(float(got - exact)) <= h * 2.0 ** -52 * cmax[i] * cmax[j]

"""The stationary-ring pair order of the register Jacobi SVD (k_svd_ring and
the rotation replay, csrc/ptt_round.cu: stat_cols) restated in Python.

For G pairs (a power of two) the order has 2G - 1 rounds; in every round
each column is in exactly one pair, every pair of columns meets exactly once
per sweep, and between rounds of one level only the second column of each
pair changes (one column moves per round).  The physical moves of the kernel
(the second columns shift one pair along rings of hb pairs; between levels a
block swaps pair i's second column with pair i + hb/2's first) reproduce the
same schedule, and a sweep ends with pair g holding columns 2g and 2g + 1."""
import pytest


def stat_cols(i, rd, G):
    x = 2 * G - 1 - rd
    hb = 1 << (x.bit_length() - 1)
    s = rd - (2 * G - 2 * hb)
    b, ii = divmod(i, hb)
    return 2 * hb * b + ii, 2 * hb * b + hb + (ii + s) % hb


@pytest.mark.parametrize("G", [1, 2, 4, 8, 16, 32])
def test_every_pair_meets_once(G):
    seen = set()
    for rd in range(2 * G - 1):
        cols = set()
        for i in range(G):
            a, b = stat_cols(i, rd, G)
            assert a not in cols and b not in cols
            cols |= {a, b}
            pair = (min(a, b), max(a, b))
            assert pair not in seen
            seen.add(pair)
        assert cols == set(range(2 * G))
    assert len(seen) == G * (2 * G - 1)


@pytest.mark.parametrize("G", [2, 4, 8, 16, 32])
def test_physical_moves_follow_the_schedule(G):
    top = list(range(G))
    bot = [G + g for g in range(G)]
    rd = 0
    hb = G
    while hb >= 1:
        for _ in range(hb):
            for g in range(G):
                assert (top[g], bot[g]) == stat_cols(g, rd, G)
            rd += 1
            if hb > 1:  # second columns one pair back along the ring
                bot = [bot[g - (g % hb) + ((g % hb) + 1) % hb] for g in range(G)]
        if hb >= 2:  # split: swap pair i's second with pair i + h's first
            h = hb // 2
            t2, b2 = top[:], bot[:]
            for g in range(G):
                if g % hb < h:
                    b2[g] = top[g ^ h]
                else:
                    t2[g] = bot[g ^ h]
            top, bot = t2, b2
        hb //= 2
    assert rd == 2 * G - 1
    assert top == [2 * g for g in range(G)] and bot == [2 * g + 1 for g in range(G)]


@pytest.mark.parametrize("G", [2, 4, 8, 16, 32])
def test_one_column_moves_per_round_within_a_level(G):
    for rd in range(2 * G - 2):
        x0 = 2 * G - 1 - rd
        x1 = 2 * G - 2 - rd
        if x0.bit_length() != x1.bit_length():
            continue  # a level boundary (the split)
        for i in range(G):
            assert stat_cols(i, rd, G)[0] == stat_cols(i, rd + 1, G)[0]

"""The row sort's comparator network (flip_bitonic_sort in
photons-on-mt3000_b200/csrc/p2p_pass_kernels.cuh) restated in numpy with the
kernel's shift-and-mask indices: for every length, including lengths that are
not powers of two (the padding to the next power of two is implicit: a
comparator whose upper index is at or past the length is skipped), it sorts,
and the rows of the walked lists it sorts come out ascending."""
import numpy as np
import pytest


def flip_bitonic(v):
    v = np.array(v)
    n = len(v)
    lg = 0
    while (1 << lg) < n:
        lg += 1
    i = np.arange((1 << lg) >> 1)
    for lgs in range(1, lg + 1):
        lgh = lgs - 1
        base, off = (i >> lgh) << lgs, i & ((1 << lgh) - 1)
        rounds = [(base + off, base + (1 << lgs) - 1 - off)]
        rounds += [(((i >> s) << (s + 1)) + (i & ((1 << s) - 1)), ((i >> s) << (s + 1)) + (i & ((1 << s) - 1)) + (1 << s))
                   for s in range(lgh - 1, -1, -1)]
        for lo, hi in rounds:
            keep = hi < n
            lo, hi = lo[keep], hi[keep]
            a, b = v[lo], v[hi]
            swap = a > b
            v[lo[swap]], v[hi[swap]] = b[swap], a[swap]
    return v


@pytest.mark.parametrize("n", list(range(0, 70)) + [127, 128, 129, 500, 1023, 1024, 1025, 3000, 8192, 8193])
def test_sorts_every_length(n):
    g = np.random.default_rng(n)
    for v in (g.integers(0, 50, n), g.integers(0, 1 << 30, n), np.arange(n)[::-1], np.zeros(n, int)):
        assert np.array_equal(flip_bitonic(v), np.sort(v))

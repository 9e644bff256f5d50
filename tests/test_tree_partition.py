"""The parallel form of the reference's mean-split partition that the device
kd-tree uses (csrc/p2p_tree_kernels.cuh), against a transcription of the
reference's swap loop (bksort_inplace, src/fmm.c:69-122, non-INTXYZ) on
random arrays with ties and with means inside and outside their range."""
import numpy as np


def reference_partition(p, mean):
    """bksort_inplace's loop (src/fmm.c:100-118): returns the permuted values
    and the left child's size (`but` at exit)."""
    p = list(p)
    but, n = len(p) - 1, 0
    while n < but:
        if p[n] > mean:
            temp = p[n]
            while p[but] > mean and but > n:
                but -= 1
            p[n] = p[but]
            p[but] = temp
        n += 1
    return p, but


def parallel_partition(p, mean):
    """With nS the values not above the mean: the k-th value above it among
    the first nS slots swaps with the k-th value not above it counted from
    the right among the rest; the left child holds nS values, or len - 1
    when none is above the mean."""
    p = list(p)
    big = [x > mean for x in p]
    n_small = len(p) - sum(big)
    lefts = [i for i in range(n_small) if big[i]]
    rights = [i for i in range(len(p) - 1, n_small - 1, -1) if not big[i]]
    assert len(lefts) == len(rights)
    q = list(p)
    for a, b in zip(lefts, rights):
        q[a], q[b] = p[b], p[a]
    return q, (len(p) - 1 if n_small == len(p) else n_small)


def test_parallel_form_equals_the_reference_loop():
    g = np.random.default_rng(20261203)
    for _ in range(20000):
        n = int(g.integers(3, 40))
        p = list(g.integers(0, 6, n).astype(float))
        mean = float(g.choice([np.mean(p), g.uniform(-1.0, 7.0), p[0], p[-1]]))
        assert reference_partition(p, mean) == parallel_partition(p, mean), (p, mean)


def test_all_above_and_all_below():
    assert parallel_partition([3.0, 4.0, 5.0], 1.0) == reference_partition([3.0, 4.0, 5.0], 1.0) == ([3.0, 4.0, 5.0], 0)
    assert parallel_partition([1.0, 1.0, 1.0], 1.0) == reference_partition([1.0, 1.0, 1.0], 1.0) == ([1.0, 1.0, 1.0], 2)

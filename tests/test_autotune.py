"""The launch-shape autotuner's host logic (no GPU): the cache key built from
the leaf-size histogram, the strided row sample it times candidates on, and
the JSON cache round trip."""
import numpy as np

from photons_p2p import abi, autotune


def lists(seed=0, nleaf=400, ntask=20000, cap=32):
    g = np.random.default_rng(seed)
    leaf_npart = g.integers(1, cap + 1, nleaf).astype(np.int32)
    task_t = np.sort(g.integers(0, nleaf, ntask)).astype(np.int32)
    task_s = g.integers(0, nleaf, ntask).astype(np.int32)
    return leaf_npart, task_t, task_s


def test_histogram_key_fields():
    n, t, s = lists()
    key = autotune.histogram_key(n, t, abi.FORM_SPLIT, abi.SOFT_PLUMMER)
    q = np.percentile(n[np.unique(t)], [25, 50, 75]).round().astype(int)
    rows = len(t) / np.unique(t).size
    assert key.startswith(f"cap{n.max()}_q{q[0]}-{q[1]}-{q[2]}_rows")
    assert f"_rows{int(2 ** round(np.log2(rows)))}_" in key
    assert key.endswith("split_fp32_fp64_soft1")


def test_histogram_key_separates_forms_and_histograms():
    n, t, s = lists()
    k1 = autotune.histogram_key(n, t, abi.FORM_SPLIT, abi.SOFT_PLUMMER)
    assert k1 == autotune.histogram_key(n.copy(), t.copy(), abi.FORM_SPLIT, abi.SOFT_PLUMMER)
    assert k1 != autotune.histogram_key(n, t, abi.FORM_KAHAN_FP32, abi.SOFT_PLUMMER)
    assert k1 != autotune.histogram_key(n, t, abi.FORM_SPLIT, abi.SOFT_CLAMP)
    n8 = np.minimum(n, 8)
    assert k1 != autotune.histogram_key(n8, t, abi.FORM_SPLIT, abi.SOFT_PLUMMER)


def test_sample_rows_takes_whole_rows_of_every_kth_sink():
    n, t, s = lists()
    total = int(np.dot(n[t].astype(np.int64), n[s]))
    st, ss, pairs = autotune.sample_rows(n, t, s, total / 10)
    k = int(total // (total / 10))
    assert np.all(st % k == 0)
    keep = (t % k) == 0
    assert np.array_equal(st, t[keep]) and np.array_equal(ss, s[keep])  # rows whole, list order kept
    assert pairs == int(np.dot(n[st].astype(np.int64), n[ss]))
    assert 0.02 * total < pairs < 0.3 * total


def test_sample_rows_whole_list_when_small():
    n, t, s = lists()
    st, ss, pairs = autotune.sample_rows(n, t, s, 1e18)
    assert st is not None and len(st) == len(t) and pairs == int(np.dot(n[t].astype(np.int64), n[s]))


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    assert autotune.load_cache(path) == {}
    rec = {"variant": abi.VARIANT_SINK_REGS, "stage": 256, "warps": 4, "kernel_ms": 1.5}
    autotune.save_cache(path, {"k1": rec})
    assert autotune.load_cache(path) == {"k1": rec}
    with open(path, "w") as f:
        f.write("{not json")
    assert autotune.load_cache(path) == {}


def test_candidates_cover_the_configured_axes():
    """Every packed mapping is a candidate, with several stage sizes and
    block shapes each; the sink-register kernel with 32- and 64-sink tiles
    and 1, 2 and 4 warps per sink leaf."""
    assert all(len(c) == 4 for c in autotune.CANDIDATES)
    variants = {c[0] for c in autotune.CANDIDATES}
    assert {abi.VARIANT_SOURCE_LANES_X2, abi.VARIANT_SOURCE_LANES_X2_S16, abi.VARIANT_SINK_LANES_X2,
            abi.VARIANT_SINK_REGS, abi.VARIANT_SINK_REGS8} <= variants
    for v in variants:
        shapes = {(st, w) for vv, st, w, _ in autotune.CANDIDATES if vv == v}
        assert len({st for st, _ in shapes}) >= 2 and len({w for _, w in shapes}) >= 2
    assert {lw for v, _, _, lw in autotune.CANDIDATES if v == abi.VARIANT_SINK_REGS} == {1, 2, 4}


def test_choose_prefers_repeatable_shapes_within_the_margin():
    """A row spread over several warps sums with atomics (results vary
    between runs): such a shape is kept only when it is more than the margin
    faster than the fastest one-warp shape."""
    one = {"variant": abi.VARIANT_SINK_REGS, "leaf_warps": 1, "pairs_per_s": 1.00e12}
    one_slow = {"variant": abi.VARIANT_SINK_REGS8, "leaf_warps": 1, "pairs_per_s": 0.90e12}
    four_close = {"variant": abi.VARIANT_SINK_REGS, "leaf_warps": 4, "pairs_per_s": 1.02e12}
    four_far = {"variant": abi.VARIANT_SINK_REGS, "leaf_warps": 4, "pairs_per_s": 1.10e12}
    assert autotune.choose([one_slow, four_close, one]) is one
    assert autotune.choose([one, four_far, one_slow]) is four_far
    assert autotune.choose([four_close, one], repeatable_margin=0.0) is four_close
    assert autotune.choose([four_close]) is four_close  # no one-warp candidate timed
    assert autotune.choose([one_slow, one]) is one


def test_sample_rows_keeps_enough_rows():
    """min_rows lowers the stride so the sample holds at least that many
    sink leaves (the pair target alone would take every 10th)."""
    n, t, s = lists()
    total = int(np.dot(n[t].astype(np.int64), n[s]))
    nsink = np.unique(t).size
    st, ss, pairs = autotune.sample_rows(n, t, s, total / 10, min_rows=nsink // 4)
    assert np.unique(st).size >= nsink // 4 - 1
    k = int(nsink // (nsink // 4))
    assert np.array_equal(st, t[(t % k) == 0]) and np.array_equal(ss, s[(t % k) == 0])
    st2, _, _ = autotune.sample_rows(n, t, s, total / 10, min_rows=1)
    assert np.unique(st2).size < np.unique(st).size  # the pair target rules when min_rows is small

"""Launch-shape autotuner of the pair kernel, keyed on the leaf-size histogram.

The shape of a pass is (mapping and sink tile, sources staged per warp,
warps per block, warps per sink leaf): the sink-register kernel keeps four
sinks per lane in registers over 32-sink slices (SINK_REGS) or eight over
64-sink slices (SINK_REGS8, so leaves of up to 64 particles stage their
sources once), and spreads one sink leaf's row over 1, 2 or 4 warps
(warps_per_leaf, partial forces added with atomics); the packed source-lane kernel holds a slice of a sink leaf
in registers against one staged source per lane (32 sinks, SOURCE_LANES_X2,
or 16 sinks with half the partial registers and more resident warps,
SOURCE_LANES_X2_S16); the packed sink-lane kernel keeps one sink pair per
lane and spreads the staged sources over the lanes (SINK_LANES_X2),
stage_sources is the source chunk a warp stages in shared memory before it
computes, and every sink leaf is one warp's work item (the persistent
kernel's work-stealing unit). Which shape wins depends on how many particles
the leaves hold and how long the rows are, so tuned shapes are cached under
a key built from the leaf-size histogram (quartiles of particles per leaf,
mean list entries per sink leaf, leaf cap) plus the form and softening.

tune() times every candidate on a sample of the pass (the rows of every
k-th sink leaf, about `sample_pairs` pair interactions) with CUDA events and
keeps the fastest. The sample holds about `sample_pairs` pairs (1e10) and
at least 64 sink leaves per resident warp: with a few per warp the tail of
uneven rows dominates and spreading a row over several warps wins on the
sample but not on the pass.
A shape that spreads rows over several warps adds their partial forces with
FP64 atomics, so its results do not repeat bit for bit between runs; it is
kept only when it beats the fastest one-warp shape by more than
`repeatable_margin` (choose()).
"""
import json
import os

import numpy as np

from . import abi
from .p2p import Session, params_for

# Shapes of the packed kernels, the mappings that re-decide pairs in the
# cutoff band from FP64 positions (the scalar sink-lane and source-lane
# mappings keep an FP32 cutoff decision and are not candidates for the
# FP32/FP64-split form's accuracy bar).
CANDIDATES = [
    (v, st, w) for v in (abi.VARIANT_SOURCE_LANES_X2, abi.VARIANT_SOURCE_LANES_X2_S16)
    for st in (128, 256, 512) for w in (2, 4)
] + [(abi.VARIANT_SINK_LANES_X2, st, w) for st in (128, 256, 512) for w in (2, 4)
] + [(abi.VARIANT_SINK_REGS, st, w, lw) for st in (256, 384) for w in (2, 4) for lw in (1, 2, 4)
] + [(abi.VARIANT_SINK_REGS8, st, w, lw) for st in (256, 384) for w in (2, 4) for lw in (1, 2)]
# every candidate as (variant, stage, warps per block, warps per leaf)
CANDIDATES = [c if len(c) == 4 else c + (1,) for c in CANDIDATES]


def histogram_key(leaf_npart, task_t, form, soft_mode):
    """Cache key of a pass from its leaf-size histogram."""
    n = np.asarray(leaf_npart)
    active = np.unique(np.asarray(task_t))
    q = np.percentile(n[active], [25, 50, 75]).round().astype(int) if active.size else [0, 0, 0]
    rows = len(task_t) / max(1, active.size)
    rows_bin = int(2 ** round(np.log2(max(rows, 1.0))))   # rows per sink leaf, to a power of 2
    return (f"cap{int(n.max()) if n.size else 0}_q{q[0]}-{q[1]}-{q[2]}_rows{rows_bin}"
            f"_{abi.FORM_NAMES[form]}_soft{soft_mode}")


def sample_rows(leaf_npart, task_t, task_s, sample_pairs, min_rows=0):
    """The rows of every k-th sink leaf, k chosen so the sample holds about
    sample_pairs pair interactions (the whole list if it is smaller) and at
    least min_rows sink leaves (rows) where the list has them."""
    n = np.asarray(leaf_npart, np.int64)
    tt, ts = np.asarray(task_t), np.asarray(task_s)
    total = float(np.dot(n[tt], n[ts]))
    k = max(1, int(total // max(sample_pairs, 1.0)))
    if min_rows > 0 and k > 1:
        nsink = int(np.count_nonzero(np.bincount(tt, minlength=n.size)))
        k = max(1, min(k, nsink // min_rows))
    if k == 1:
        return tt, ts, int(total)
    keep = (tt % k) == 0
    st, ss = tt[keep], ts[keep]
    return st, ss, int(np.dot(n[st], n[ss]))


def load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(path, cache):
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def choose(results, repeatable_margin=0.03):
    """The record to keep among timed candidates: the fastest, unless it
    spreads rows over several warps (leaf_warps > 1) and is not faster than
    the fastest one-warp candidate by more than repeatable_margin, in which
    case that one (its results repeat bit for bit)."""
    best = max(results, key=lambda r: r["pairs_per_s"])
    one = [r for r in results if r.get("leaf_warps", 1) == 1]
    if best.get("leaf_warps", 1) > 1 and one:
        b1 = max(one, key=lambda r: r["pairs_per_s"])
        if best["pairs_per_s"] <= b1["pairs_per_s"] * (1.0 + repeatable_margin):
            return b1
    return best


# Sample size by rows: every resident warp of the persistent pair kernel
# (4 blocks of 4 warps per SM) should take this many sink leaves' rows from
# the sample, so the tail of uneven rows weighs about as little as in a whole
# pass (a few rows per warp favour spreading rows over several warps).
ROWS_PER_WARP = 64
RESIDENT_WARPS_PER_SM = 16


def tune(cfg, lists, form, mass, device=0, sample_pairs=1e10, cache_path=None, repeats=2,
         candidates=CANDIDATES, log=None, repeatable_margin=0.03, min_rows=None):
    """Best launch shape for this pass; returns (params, record). With
    cache_path, a cached record under the same key is reused and new results
    are stored."""
    import torch

    key = histogram_key(lists.leaf_npart, lists.task_t, form, cfg.soft_mode)
    cache = load_cache(cache_path) if cache_path else {}

    def apply(rec):
        p = params_for(cfg, form, mass)
        p.kernel_variant, p.stage_sources, p.warps_per_block = rec["variant"], rec["stage"], rec["warps"]
        p.warps_per_leaf = rec.get("leaf_warps", 1)
        return p

    if key in cache:
        return apply(cache[key]), dict(cache[key], key=key, cached=True)
    dev = torch.device("cuda", device)
    if min_rows is None:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        min_rows = ROWS_PER_WARP * RESIDENT_WARPS_PER_SM * sms
    st, ss, pairs = sample_rows(lists.leaf_npart, lists.task_t, lists.task_s, sample_pairs, min_rows)
    d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (lists.pos, lists.leaf_ipart, lists.leaf_npart, st, ss)]
    args = (lists.npart, d[0].data_ptr(), lists.nleaf, d[1].data_ptr(), d[2].data_ptr(), len(st),
            d[3].data_ptr(), d[4].data_ptr())
    results = []
    cands = candidates if form != abi.FORM_PLAIN_FP64 else [(0, st_, w, 1) for st_ in (64, 128, 256)
                                                              for w in (2, 4, 8)]
    with Session(device) as s:
        for cand in cands:
            variant, stage, warps, lw = cand if len(cand) == 4 else tuple(cand) + (1,)
            p = params_for(cfg, form, mass)
            p.kernel_variant, p.stage_sources, p.warps_per_block = variant, stage, warps
            p.warps_per_leaf = lw
            try:
                s.set_params(p)
                ms = []
                for _ in range(repeats + 1):
                    s.run_device(*args)
                    s.end()
                    ms.append(s.last_kernel_ms())
            except Exception as e:  # a shape that does not fit is skipped
                if log:
                    log(f"[tune] {variant}/{stage}/{warps}/{lw}: {e}")
                continue
            t = min(ms[1:])
            results.append({"variant": variant, "stage": stage, "warps": warps, "leaf_warps": lw,
                            "kernel_ms": t, "pairs_per_s": pairs / (t * 1e-3)})
            if log:
                log(f"[tune] variant {variant} stage {stage} warps {warps} warps/leaf {lw}: {t:.3f} ms "
                    f"{pairs / (t * 1e-3):.3e} pairs/s")
    best = choose(results, repeatable_margin)
    rec = dict(best, sample_pairs=pairs, candidates=len(results))
    if cache_path:
        cache = load_cache(cache_path)
        cache[key] = rec
        save_cache(cache_path, cache)
    return apply(rec), dict(rec, key=key, cached=False, all=results)

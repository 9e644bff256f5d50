"""The caller-side tree build and walk (libphotons_lists.so) against the
reference's own src/fmm.c: identical particle order, leaves and lists."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from photons_p2p import lists as L, workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
need_walk = pytest.mark.skipif(not O.ref_available("libref_walk.so"),
                               reason="oracle/_ref (reference walk) not built")


def assert_same(tl, r):
    assert np.array_equal(tl.perm, r["perm"])
    assert np.array_equal(tl.leaf_ipart, r["leaf_ipart"])
    assert np.array_equal(tl.leaf_npart, r["leaf_npart"])
    assert np.array_equal(tl.leaf_active, r["leaf_active"])
    assert np.array_equal(tl.leaf_center, r["leaf_center"])
    assert np.array_equal(tl.leaf_width, r["leaf_width"])
    assert np.array_equal(tl.task_t, r["task_t"])
    assert np.array_equal(tl.task_s, r["task_s"])


def test_golden_dropin12_walk():
    g = np.load(os.path.join(GOLDEN, "dropin12.npz"))
    tl = L.build_tree_lists(g["input_pos"], g["input_tag"], int(g["maxleaf"]), float(g["box"]),
                            float(g["cutoff_radius"]), float(g["open_angle"]))
    assert_same(tl, g)
    assert tl.pair_count() == int(g["pairs"])


@need_walk
@pytest.mark.parametrize("case", ["dropin16", "c1", "clustered32_theta0", "maxleaf256_sampled"])
def test_walk_matches_reference_live(case):
    if case == "dropin16":
        cfg = W.ref_dropin_config(16, 32, 32)
        pos = W.lattice_gaussian(16, 0.2, W.rng(1))
    elif case == "c1":
        cfg, pos = W.c1_config(), W.c1_positions()
    elif case == "clustered32_theta0":
        cfg = W.scaled(W.c2_config(), n_side=32, mesh=32, eps=1 / (40 * 32))
        pos = W.c2_positions(32)
    else:  # > 1e5 particles: the reference samples the split mean
        cfg = W.ref_dropin_config(48, 96, 256)
        pos = W.lattice_gaussian(48, 0.3, W.rng(9))
    allpos, tag = W.with_ghosts(pos, cfg)
    tl = L.build_tree_lists(allpos, tag, cfg.maxleaf, cfg.box, cfg.cutoff_radius, cfg.open_angle)
    r = O.RefWalk("libref_walk.so").run(allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius,
                                        cfg.cutoff_radius, cfg.eps, 1.0, cfg.open_angle, 1 << 30)
    assert_same(tl, r)


def test_ghosts_cover_shell():
    g = W.rng(8)
    pos = g.random((3, 2000))
    w = 0.1
    gp, src = L.make_ghosts(pos, 0.0, 1.0, w)
    assert gp.shape[1] == src.shape[0] > 0
    assert np.all((gp > -w) & (gp < 1 + w))
    assert np.all(np.any((gp < 0) | (gp >= 1), axis=0))  # every ghost is an image outside the box
    shift = gp - pos[:, src]
    assert np.allclose(shift, np.round(shift), atol=1e-12)  # integer box shifts
    # brute force count
    n = 0
    for s in np.array(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1])).reshape(3, -1).T:
        if not s.any():
            continue
        q = pos + s[:, None]
        n += int(np.sum(np.all((q > -w) & (q < 1 + w), axis=0)))
    assert n == gp.shape[1]


def test_lists_partition_and_symmetry():
    cfg = W.c1_config()
    tl = W.prepare(W.c1_positions(), cfg)
    # leaves partition the particles in order
    assert tl.leaf_ipart[0] == 0
    assert np.array_equal(tl.leaf_ipart[1:], np.cumsum(tl.leaf_npart)[:-1])
    assert tl.leaf_npart.sum() == tl.npart and tl.leaf_npart.max() <= cfg.maxleaf
    # one-sided lists: (A, B) listed => (B, A) listed when B is active
    pairs = set(zip(tl.task_t.tolist(), tl.task_s.tolist()))
    for t, s in list(pairs)[:5000]:
        if tl.leaf_active[s] >= 0:
            assert (s, t) in pairs
    # every active leaf lists itself
    act = np.nonzero(tl.leaf_active >= 0)[0]
    assert all((int(a), int(a)) in pairs for a in act)


@pytest.mark.parametrize("nsink", [1, 50, 3000])
def test_masked_walk_equals_filtered_walk(nsink):
    """The walk restricted to the leaves of sampled sinks emits exactly the
    full walk's rows of those leaves, in the same order (with ghosts and a
    shifted origin, as the precision study uses it)."""
    cfg = W.scaled(W.c5_config(), n_side=40, mesh=40, eps=1 / (200 * 40))
    pos = W.c5_positions(40 ** 3)
    allpos, tag = W.with_ghosts(pos, cfg)
    full = L.build_tree_lists(allpos, tag, cfg.maxleaf, cfg.box, cfg.cutoff_radius,
                              cfg.open_angle)
    sinks = np.random.default_rng(nsink).choice(pos.shape[1], nsink, replace=False)
    part = L.build_tree_lists(allpos, tag, cfg.maxleaf, cfg.box, cfg.cutoff_radius,
                              cfg.open_angle, sink_particles=sinks)
    assert np.array_equal(part.perm, full.perm)
    slot = np.empty(full.npart, np.int64)
    slot[full.perm] = np.arange(full.npart)
    leaf_of = np.repeat(np.arange(full.nleaf), full.leaf_npart)
    keep = np.zeros(full.nleaf, bool)
    keep[leaf_of[slot[sinks]]] = True
    sel = keep[full.task_t]
    assert sel.any()
    assert np.array_equal(part.task_t, full.task_t[sel])
    assert np.array_equal(part.task_s, full.task_s[sel])


def _acceptance(wi, wj, ci, cj, cutoff, open_angle):
    """acceptance (src/fmm.c:409-479, LONGSHORT) in Python doubles."""
    dist = [ci[d] - cj[d] for d in range(3)]
    w = [(wi[d] + wj[d]) * 0.5 for d in range(3)]
    dd2 = dist[0] * dist[0] + dist[1] * dist[1] + dist[2] * dist[2]
    mn = [max(abs(dist[d]) - w[d], 0.0) for d in range(3)]
    if mn[0] + mn[1] + mn[2] < 1e-15:
        return 0
    if mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2] > cutoff * cutoff:
        return -1
    wmax = abs(max(w)) * 2
    return 1 if wmax * wmax < open_angle * open_angle * dd2 else 0


def per_sink_rows(tree, cutoff, open_angle, batch=32):
    """The device walk's algorithm (csrc/p2p_walk_kernels.cuh) restated: for
    each sink leaf, the part of the serial dual-tree walk whose sink side
    holds it, expanded `batch` pending pairs at a time from a stack (one warp's
    lanes), the row sorted ascending at the end."""
    son, first, nc, nw = (a.tolist() for a in tree.nodes())
    lc, lw, act = tree.leaf_center.tolist(), tree.leaf_width.tolist(), tree.leaf_active.tolist()
    ctr = lambda c: nc[c >> 1] if c & 1 else lc[c >> 1]  # noqa: E731
    wid = lambda c: nw[c >> 1] if c & 1 else lw[c >> 1]  # noqa: E731

    def toward(a, leaf):
        s0, s1 = son[a >> 1]
        return s0 if leaf < (first[s1 >> 1] if s1 & 1 else s1 >> 1) else s1

    rows = []
    for leaf in range(tree.nleaf):
        out, stack = [], ([(1, 1)] if act[leaf] >= 0 else [])
        while stack:
            take = min(batch, len(stack))
            pending, stack = stack[len(stack) - take:], stack[:len(stack) - take]
            for a, b in pending:
                if a == b and not a & 1 or not (a & 1 or b & 1):
                    out.append(b >> 1)
                elif a == b:
                    c = toward(a, leaf)
                    stack += [(c, son[a >> 1][0]), (c, son[a >> 1][1])]
                elif _acceptance(wid(a), wid(b), ctr(a), ctr(b), cutoff, open_angle) == 0:
                    if (a & 1) and (not b & 1 or sum(wid(a)) > sum(wid(b))):
                        stack.append((toward(a, leaf), b))
                    else:
                        stack += [(a, son[b >> 1][0]), (a, son[b >> 1][1])]
        rows.append(sorted(out))
    return rows


@pytest.mark.parametrize("config", ["c1", "ref_dropin"])
def test_per_sink_walk_equals_sorted_serial_walk(config):
    """Expanding the walk per sink leaf gives every sink's row of the serial
    walk, entry for entry in the serial order (the rows a stable sort of the
    serial list by sink builds; the serial order of a row is increasing source
    leaf id): open angle 0 (cutoff-only lists) and the reference's 0.4."""
    cfg = W.c1_config() if config == "c1" else W.ref_dropin_config()
    allpos, tag = W.with_ghosts(W.c1_positions(), cfg)
    with L.Tree(allpos, tag, cfg.maxleaf, cfg.box) as tree:
        tt, ts = tree.walk(cfg.cutoff_radius, cfg.open_angle)
        rows = per_sink_rows(tree, cfg.cutoff_radius, cfg.open_angle)
        son, first, _, _ = tree.nodes()
    order = np.argsort(tt, kind="stable")
    got_s = np.concatenate([np.asarray(r, np.int32) for r in rows])
    got_t = np.repeat(np.arange(len(rows)), [len(r) for r in rows])
    assert np.array_equal(got_t, tt[order]) and np.array_equal(got_s, ts[order])
    # pre-order leaf numbering: son[0]'s leaves precede son[1]'s
    s1 = son[:, 1]
    f1 = s1 >> 1
    f1[(s1 & 1) == 1] = first[f1[(s1 & 1) == 1]]
    assert np.all(first < f1)

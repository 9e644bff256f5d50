"""The reference's own far field of the short-range force (p2m, m2m, the M2L
walk and m2l, l2l, l2p: src/operator.c, src/fmm.c:812-957 and :1188-1217),
compiled from its sources by oracle/build_ref.sh and driven by
oracle/ref_walk_harness.c (ref_harness_fmm): the oracle of the GPU far field.

Known answers about the reference itself, checked here on the CPU:
  * every leaf's monopole is its particles' mass;
  * its m2l tests `abs(r2) <= 1e-15` with the integer abs() of <stdlib.h>
    (src/operator.c:340-344), so in a unit box, where every M2L distance is
    below 1, the M2L tasks are made but the far field is exactly zero; in a
    box of 1000 the same particles give a non-zero far field;
  * with the drop-in settings on a lattice (r_s = 1.25 cells, cutoff 4.5
    r_s, open angle 0.4) no pair of boxes within the cutoff is well
    separated: no M2L task at all.
The GPU's breadth-first M2L walk is restated in numpy here and makes the
reference recursion's task count, with and without its pruning of children
that cannot lead to a task."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from photons_p2p import workloads as W

pytestmark = pytest.mark.skipif(not O.ref_available("libref_walk.so"),
                                reason="oracle/_ref walk harness not built")


def quiet(fn):
    """Runs fn with the process's stdout closed (the reference's m2l prints a
    line for every task it skips)."""
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return fn()
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)


def clustered(side, box):
    cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=box / (40 * side), open_angle=0.4, box=box)
    pos = W.c2_positions(side) * box
    allpos, tag = W.with_ghosts(pos, cfg)
    return cfg, allpos, tag, 1.0 / pos.shape[1]


def ref_fmm(cfg, allpos, tag, mass):
    return quiet(lambda: O.RefWalk("libref_walk.so").fmm(allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius,
                                                         cfg.cutoff_radius, cfg.eps, mass, cfg.open_angle))


def test_unit_box_far_field_is_zero_in_the_reference():
    cfg, allpos, tag, mass = clustered(64, 1.0)
    r = ref_fmm(cfg, allpos, tag, mass)
    assert np.allclose(r["leaf_M"][:, 0], r["leaf_npart"] * mass, rtol=1e-14, atol=0)
    big = clustered(64, 1000.0)
    rb = ref_fmm(*big)
    assert rb["n_m2l"] > 0 and np.abs(rb["acc"]).max() > 0
    assert r["n_m2l"] == rb["n_m2l"]
    assert not np.any(r["acc"])


def test_lattice_drop_in_settings_make_no_m2l():
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    r = ref_fmm(cfg, allpos, tag, 1.0 / pos.shape[1])
    assert r["n_m2l"] == 0 and not np.any(r["acc"])


def _acceptance(ca, cb, wa, wb, cutoff, theta):
    """walk_acceptance (src/fmm.c:409-479) on arrays of box pairs, the same
    operations in the same order: 1 accept (M2L), 0 open, -1 drop."""
    dist = ca - cb
    w = (wa + wb) * 0.5
    dd2 = (dist[:, 0] * dist[:, 0] + dist[:, 1] * dist[:, 1]) + dist[:, 2] * dist[:, 2]
    mn = np.maximum(np.abs(dist) - w, 0.0)
    touch = (mn[:, 0] + mn[:, 1]) + mn[:, 2] < 1e-15
    dm2 = (mn[:, 0] * mn[:, 0] + mn[:, 1] * mn[:, 1]) + mn[:, 2] * mn[:, 2]
    wmax = np.abs(w.max(axis=1)) * 2.0
    flag = np.where(wmax * wmax < (theta * theta) * dd2, 1, 0)
    flag = np.where(dm2 > cutoff * cutoff, -1, flag)
    return np.where(touch, 0, flag)


def m2l_tasks_breadth_first(son, ncen, nwid, lcen, lwid, cutoff, theta, prune=True):
    """The GPU M2L walk (csrc/p2p_fmm.cu: fmm_walk_kernel) restated level by
    level in numpy: (sink code, source code) tasks, codes leaf l -> 2l, node
    k -> 2k + 1, and the number of pairs visited. prune keeps only children
    that can lead to a task, as the kernel does; without it every child is
    visited, as walk_task_m2l's recursion does."""
    def boxes(c, node_arr, leaf_arr):
        out = np.empty((len(c), 3))
        isn = (c & 1) == 1
        out[isn] = node_arr[c[isn] >> 1]
        out[~isn] = leaf_arr[c[~isn] >> 1]
        return out

    def live(A, B):
        keep = (A >= 0) & (B >= 0)
        same = A == B
        keep &= np.where(same, (A & 1) == 1, ((A & 1) == 1) | ((B & 1) == 1))
        idx = np.nonzero(keep & ~same)[0]
        if idx.size:
            f = _acceptance(boxes(A[idx], ncen, lcen), boxes(B[idx], ncen, lcen), boxes(A[idx], nwid, lwid),
                            boxes(B[idx], nwid, lwid), cutoff, theta)
            keep[idx[f == -1]] = False
        return keep

    front = np.array([[1, 1]], np.int64)
    tasks, visited = [], 0
    while len(front):
        visited += len(front)
        A, B = front[:, 0], front[:, 1]
        ok = (A >= 0) & (B >= 0)
        A, B = A[ok], B[ok]
        kids = []
        sn = (A == B) & ((A & 1) == 1)
        s0, s1 = son[A[sn] >> 1, 0], son[A[sn] >> 1, 1]
        kids += [np.stack(p, 1) for p in ((s0, s0), (s0, s1), (s1, s0), (s1, s1))]
        d = (A != B) & (((A & 1) == 1) | ((B & 1) == 1))
        A2, B2 = A[d], B[d]
        wa, wb = boxes(A2, nwid, lwid), boxes(B2, nwid, lwid)
        flag = _acceptance(boxes(A2, ncen, lcen), boxes(B2, ncen, lcen), wa, wb, cutoff, theta)
        tasks.append(np.stack([A2[flag == 1], B2[flag == 1]], 1))
        op = flag == 0
        A3, B3, sa, sb = A2[op], B2[op], wa[op], wb[op]
        isa, isb = (A3 & 1) == 1, (B3 & 1) == 1
        open_a = np.where(~isa, False, np.where(~isb, True,
                          (sa[:, 0] + sa[:, 1]) + sa[:, 2] > (sb[:, 0] + sb[:, 1]) + sb[:, 2]))
        Ao, Bo, Ab, Bb = A3[open_a], B3[open_a], A3[~open_a], B3[~open_a]
        kids += [np.stack([son[Ao >> 1, 0], Bo], 1), np.stack([son[Ao >> 1, 1], Bo], 1),
                 np.stack([Ab, son[Bb >> 1, 0]], 1), np.stack([Ab, son[Bb >> 1, 1]], 1)]
        front = np.concatenate(kids).astype(np.int64)
        if prune and len(front):
            front = front[live(front[:, 0], front[:, 1])]
    return np.concatenate(tasks), visited


def test_breadth_first_walk_makes_the_reference_tasks():
    """The breadth-first M2L walk, restated in numpy on the caller-side tree
    (equal to the reference's node for node), makes as many tasks as the
    reference's own recursion (idxM2L) on the clustered 64^3 particles; with
    and without the pruning of children that cannot lead to a task the task
    sets are the same, and pruning visits far fewer pairs."""
    from photons_p2p import lists as Lists

    cfg, allpos, tag, mass = clustered(64, 1000.0)
    ref = ref_fmm(cfg, allpos, tag, mass)
    with Lists.Tree(allpos, tag, cfg.maxleaf, cfg.box) as t:
        son, _, ncen, nwid = t.nodes()
        lcen, lwid = t.leaf_center.copy(), t.leaf_width.copy()
        assert np.array_equal(t.perm, ref["perm"])
    pruned, v1 = m2l_tasks_breadth_first(son, ncen, nwid, lcen, lwid, cfg.cutoff_radius, cfg.open_angle)
    full, v2 = m2l_tasks_breadth_first(son, ncen, nwid, lcen, lwid, cfg.cutoff_radius, cfg.open_angle,
                                       prune=False)
    assert len(pruned) == ref["n_m2l"] > 0
    key = lambda t: np.sort(t[:, 0].astype(np.int64) << 32 | t[:, 1])  # noqa: E731
    assert np.array_equal(key(pruned), key(full))
    assert v1 < v2

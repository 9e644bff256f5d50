"""Caller-side inputs of the P2P pass: periodic ghosts, the kd-tree and the
interaction lists, produced by the host library libphotons_lists.so (a
restatement of the reference's src/fmm.c tree build and walk, see
host/p2p_lists.cpp). This is what PhotoNs hands to task_compute_p2p_gpu.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def make_ghosts(pos, origin, box, width):
    """Periodic ghost images of the particles within `width` of the domain
    [origin, origin+box)^3 (the single-domain case of src/boundary.c:592-680).
    pos: (3, n) float64. Returns (ghost_pos (3, g), src_index (g,))."""
    lib = _native.lists()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = pos.shape[1]
    g = lib.p2p_make_ghosts(n, _ptr(pos, _f64p), origin, box, width, None, 0, None)
    out = np.empty((3, g), dtype=np.float64)
    src = np.empty(g, dtype=np.int32)
    r = lib.p2p_make_ghosts(n, _ptr(pos, _f64p), origin, box, width, _ptr(out, _f64p), g,
                            _ptr(src, _i32p))
    if r != g:
        raise RuntimeError("ghost generation failed")
    return out, src


@dataclass
class TreeLists:
    """One force pass's caller state, in tree order.

    pos      (3, npart) float64 SoA positions, locals and ghosts, tree order
    perm     (npart,) original index of each tree slot
    tag      (npart,) 1 local, 0 ghost (tree order)
    leaf_ipart, leaf_npart, leaf_active  (nleaf,) int32
    leaf_center, leaf_width              (nleaf, 3) float64
    task_t, task_s   (ntask,) int32 sink / source leaf ids (0-based), walk order
    """
    pos: np.ndarray
    perm: np.ndarray
    tag: np.ndarray
    leaf_ipart: np.ndarray
    leaf_npart: np.ndarray
    leaf_active: np.ndarray
    leaf_center: np.ndarray
    leaf_width: np.ndarray
    task_t: np.ndarray
    task_s: np.ndarray

    @property
    def npart(self):
        return self.pos.shape[1]

    @property
    def nleaf(self):
        return self.leaf_npart.shape[0]

    @property
    def ntask(self):
        return self.task_t.shape[0]

    def pair_count(self):
        """sum over list entries of n_sink * n_source (src/gpu_entry.cu:53-58)."""
        n = self.leaf_npart.astype(np.int64)
        return int(np.dot(n[self.task_t], n[self.task_s]))


class Tree:
    """A kd-tree (src/fmm.c:231-327) kept for several walks, e.g. the walk of
    one group of sink leaves at a time when the whole list would not fit in
    host memory. pos (3, n) float64, tag (n,) int: 1 local, 0 ghost."""

    def __init__(self, pos, tag, maxleaf, boxsize):
        self.lib = _native.lists()
        self.pos = np.array(pos, dtype=np.float64, order="C", copy=True)
        tag = np.ascontiguousarray(tag, dtype=np.int32)
        n = self.pos.shape[1]
        self.perm = np.empty(n, dtype=np.int32)
        self.h = self.lib.p2p_tree_build(n, _ptr(self.pos, _f64p), _ptr(tag, _i32p), maxleaf, boxsize,
                                         _ptr(self.perm, _i32p))
        if not self.h:
            raise RuntimeError("tree build failed")
        self.tag = tag[self.perm]
        nleaf = self.lib.p2p_tree_nleaf(self.h)
        self.leaf_ipart = np.empty(nleaf, np.int32)
        self.leaf_npart = np.empty(nleaf, np.int32)
        self.leaf_active = np.empty(nleaf, np.int32)
        self.leaf_center = np.empty((nleaf, 3), np.float64)
        self.leaf_width = np.empty((nleaf, 3), np.float64)
        self.lib.p2p_tree_leaves(self.h, _ptr(self.leaf_ipart, _i32p), _ptr(self.leaf_npart, _i32p),
                                 _ptr(self.leaf_active, _i32p), _ptr(self.leaf_center, _f64p),
                                 _ptr(self.leaf_width, _f64p))

    @property
    def nleaf(self):
        return self.leaf_npart.shape[0]

    def nodes(self):
        """Node table for the device walk: (son (nnode, 2) child codes,
        first leaf id per subtree, centres (nnode, 3), widths (nnode, 3))."""
        nn = self.lib.p2p_tree_nnode(self.h)
        son = np.empty((nn, 2), np.int32)
        first = np.empty(nn, np.int32)
        center = np.empty((nn, 3), np.float64)
        width = np.empty((nn, 3), np.float64)
        self.lib.p2p_tree_nodes(self.h, _ptr(son, _i32p), _ptr(first, _i32p), _ptr(center, _f64p),
                                _ptr(width, _f64p))
        return son, first, center, width

    def walk(self, cutoff, open_angle, leaf_mask=None):
        """(task_t, task_s) of the P2P walk (src/fmm.c:656-792); with
        leaf_mask (nleaf bools) only the rows of the masked sink leaves, in
        the full walk's order."""
        if leaf_mask is None:
            nt = self.lib.p2p_tree_walk(self.h, cutoff, open_angle)
        else:
            m = np.ascontiguousarray(leaf_mask, dtype=np.uint8)
            nt = self.lib.p2p_tree_walk_masked(self.h, cutoff, open_angle, m.ctypes.data_as(ctypes.c_void_p))
        tt = np.empty(nt, np.int32)
        ts = np.empty(nt, np.int32)
        self.lib.p2p_tree_tasks(self.h, _ptr(tt, _i32p), _ptr(ts, _i32p))
        return tt, ts

    def lists(self, task_t, task_s):
        return TreeLists(pos=self.pos, perm=self.perm, tag=self.tag, leaf_ipart=self.leaf_ipart,
                         leaf_npart=self.leaf_npart, leaf_active=self.leaf_active,
                         leaf_center=self.leaf_center, leaf_width=self.leaf_width, task_t=task_t,
                         task_s=task_s)

    def close(self):
        if self.h:
            self.lib.p2p_tree_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def num_threads():
    """Host threads the tree build and walk use (OpenMP)."""
    return _native.lists().p2p_lists_num_threads()


def build_tree_lists(pos, tag, maxleaf, boxsize, cutoff, open_angle, sink_particles=None):
    """kd-tree (src/fmm.c:231-327) + P2P walk (src/fmm.c:656-792) over the
    given particles (pos (3, n) float64, tag (n,) int: 1 local, 0 ghost).
    sink_particles (original indices, optional) keeps only the list rows of
    the leaves holding them (the same entries, in the same order)."""
    with Tree(pos, tag, maxleaf, boxsize) as t:
        mask = None
        if sink_particles is not None:
            n = t.pos.shape[1]
            slot = np.empty(n, np.int64)
            slot[t.perm] = np.arange(n)
            leaf_of_slot = np.repeat(np.arange(t.nleaf), t.leaf_npart)
            mask = np.zeros(t.nleaf, np.uint8)
            mask[leaf_of_slot[slot[np.asarray(sink_particles)]]] = 1
        tt, ts = t.walk(cutoff, open_angle, mask)
        return t.lists(tt, ts)

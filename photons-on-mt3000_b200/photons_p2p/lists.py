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


def build_tree_lists(pos, tag, maxleaf, boxsize, cutoff, open_angle, sink_particles=None):
    """kd-tree (src/fmm.c:231-327) + P2P walk (src/fmm.c:656-792) over the
    given particles (pos (3, n) float64, tag (n,) int: 1 local, 0 ghost).
    sink_particles (original indices, optional) keeps only the list rows of
    the leaves holding them (the same entries, in the same order)."""
    lib = _native.lists()
    pos = np.array(pos, dtype=np.float64, order="C", copy=True)
    tag = np.ascontiguousarray(tag, dtype=np.int32)
    n = pos.shape[1]
    perm = np.empty(n, dtype=np.int32)
    h = lib.p2p_tree_build(n, _ptr(pos, _f64p), _ptr(tag, _i32p), maxleaf, boxsize,
                           _ptr(perm, _i32p))
    if not h:
        raise RuntimeError("tree build failed")
    try:
        nleaf = lib.p2p_tree_nleaf(h)
        ip = np.empty(nleaf, np.int32)
        npt = np.empty(nleaf, np.int32)
        act = np.empty(nleaf, np.int32)
        ctr = np.empty((nleaf, 3), np.float64)
        wid = np.empty((nleaf, 3), np.float64)
        lib.p2p_tree_leaves(h, _ptr(ip, _i32p), _ptr(npt, _i32p), _ptr(act, _i32p),
                            _ptr(ctr, _f64p), _ptr(wid, _f64p))
        if sink_particles is None:
            nt = lib.p2p_tree_walk(h, cutoff, open_angle)
        else:
            slot = np.empty(n, np.int64)
            slot[perm] = np.arange(n)
            leaf_of_slot = np.repeat(np.arange(nleaf), npt)
            mask = np.zeros(nleaf, np.uint8)
            mask[leaf_of_slot[slot[np.asarray(sink_particles)]]] = 1
            nt = lib.p2p_tree_walk_masked(h, cutoff, open_angle, mask.ctypes.data_as(ctypes.c_void_p))
        tt = np.empty(nt, np.int32)
        ts = np.empty(nt, np.int32)
        lib.p2p_tree_tasks(h, _ptr(tt, _i32p), _ptr(ts, _i32p))
    finally:
        lib.p2p_tree_free(h)
    return TreeLists(pos=pos, perm=perm, tag=tag[perm], leaf_ipart=ip, leaf_npart=npt,
                     leaf_active=act, leaf_center=ctr, leaf_width=wid, task_t=tt, task_s=ts)

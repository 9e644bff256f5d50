"""Session: the P2P force pass through the C ABI of libphotons_p2p.so.

Mirrors the reference's gpu_entry protocol (src/gpu_entry.cu:32-209,
src/gravity.c:440-449): begin (particles + leaves) -> submit list chunks
(async) -> end (completion barrier, GPU seconds) -> accumulate (acc += result).
Errors raise P2PError carrying the library's status code and message; there is
no CPU fallback.
"""
import ctypes

import numpy as np

from . import _native, abi
from .abi import (FORM_PLAIN_FP64, P2P_OK, SOFT_CLAMP, Params)


class P2PError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"p2p status {status}: {message}")
        self.status = status


def _check(lib, status):
    if status != P2P_OK:
        raise P2PError(status, lib.p2p_last_error().decode())


def _host(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(ctypes.c_void_p)


def make_params(form=FORM_PLAIN_FP64, soft_mode=SOFT_CLAMP, soften=1.0, split_radius=1.0,
                x_cut=2.8125, mass=1.0, warps_per_block=0, stage_sources=0, blocks_per_sm=0,
                kernel_variant=0, poly_tol=0.0):
    return Params(form, soft_mode, soften, split_radius, x_cut, mass, warps_per_block,
                  stage_sources, blocks_per_sm, kernel_variant, poly_tol)


def params_for(cfg, form, mass):
    """Pass parameters of a workloads.PassConfig."""
    return make_params(form=form, soft_mode=cfg.soft_mode, soften=cfg.eps,
                       split_radius=cfg.split_radius, x_cut=cfg.x_cut, mass=mass)


class Session:
    def __init__(self, device=0, params=None):
        self.lib = _native.core()
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_session_create(device, ctypes.byref(h)))
        self.h = h
        self.npart = 0
        self._keep = []
        if params is not None:
            self.set_params(params)

    def close(self):
        if self.h:
            self.lib.p2p_session_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        _check(self.lib, self.lib.p2p_session_set_params(self.h, ctypes.byref(params)))

    @property
    def stream(self):
        return self.lib.p2p_session_stream(self.h)

    @property
    def poly_degree(self):
        return self.lib.p2p_session_poly_degree(self.h)

    @property
    def poly_error(self):
        return self.lib.p2p_session_poly_error(self.h)

    # -- pass protocol on host buffers --------------------------------------
    def begin(self, pos, leaf_ipart, leaf_npart, masses=None):
        pos, pp = _host(pos, np.float64)
        ip, ipp = _host(leaf_ipart, np.int32)
        npt, npp = _host(leaf_npart, np.int32)
        mp = None
        if masses is not None:
            masses, mp = _host(masses, np.float64)
        self._keep = [pos, ip, npt, masses]
        self.npart = pos.shape[-1]
        self._nleaf = ip.shape[0]
        _check(self.lib, self.lib.p2p_pass_begin(self.h, self.npart, pp, mp, ip.shape[0], ipp, npp))

    def submit(self, task_t, task_s):
        tt, tp = _host(task_t, np.int32)
        ts, sp = _host(task_s, np.int32)
        self._keep.extend([tt, ts])
        _check(self.lib, self.lib.p2p_pass_submit(self.h, tt.shape[0], tp, sp))

    def end(self):
        sec = ctypes.c_double()
        _check(self.lib, self.lib.p2p_pass_end(self.h, ctypes.byref(sec)))
        self._keep = []
        return sec.value

    def accumulate(self, acc):
        assert acc.dtype == np.float64 and acc.flags.c_contiguous and acc.size == 3 * self.npart
        _check(self.lib, self.lib.p2p_pass_accumulate(self.h, acc.ctypes.data_as(ctypes.c_void_p)))
        return acc

    def pair_count(self):
        v = ctypes.c_int64()
        _check(self.lib, self.lib.p2p_pass_pair_count(self.h, ctypes.byref(v)))
        return v.value

    def evaluated_pairs(self):
        """Pair interactions the kernels evaluated in the current pass (the
        listed ones minus those of entries skipped as wholly beyond the cutoff)."""
        v = ctypes.c_int64()
        _check(self.lib, self.lib.p2p_pass_evaluated_pairs(self.h, ctypes.byref(v)))
        return v.value

    def last_kernel_ms(self):
        v = ctypes.c_float()
        _check(self.lib, self.lib.p2p_session_last_kernel_ms(self.h, ctypes.byref(v)))
        return v.value

    def force_pass(self, pos, leaf_ipart, leaf_npart, task_t, task_s, masses=None, chunk=0):
        """One complete pass on host arrays; returns (acc (3, npart), gpu_seconds)."""
        self.begin(pos, leaf_ipart, leaf_npart, masses)
        n = len(task_t)
        step = chunk if chunk and chunk > 0 else max(n, 1)
        for c0 in range(0, n, step):
            self.submit(task_t[c0:c0 + step], task_s[c0:c0 + step])
        sec = self.end()
        acc = np.zeros((3, self.npart), dtype=np.float64)
        self.accumulate(acc)
        return acc, sec

    # -- device list walk ----------------------------------------------------
    def submit_walk(self, tree_dev, cutoff, open_angle):
        """Walks the P2P lists on the GPU into the open pass and launches the
        pair kernel on them; tree_dev from device_walk_tree. Returns the
        number of list entries."""
        n = ctypes.c_int64()
        _check(self.lib, self.lib.p2p_pass_submit_walk(self.h, ctypes.byref(tree_dev.struct), cutoff,
                                                       open_angle, ctypes.byref(n)))
        return n.value

    def rows(self):
        """(row_off, row_src) of the last submitted chunk or walk (host copies)."""
        nleaf = self._nleaf
        off = np.empty(nleaf + 1, np.int64)
        _check(self.lib, self.lib.p2p_pass_rows(self.h, off.ctypes.data_as(ctypes.c_void_p), None))
        src = np.empty(int(off[-1]), np.int32)
        _check(self.lib, self.lib.p2p_pass_rows(self.h, off.ctypes.data_as(ctypes.c_void_p),
                                                src.ctypes.data_as(ctypes.c_void_p)))
        return off, src

    def force_pass_walk(self, tree, tree_dev, cutoff, open_angle, masses=None):
        """One pass on a lists.Tree's particles and leaves with the lists
        walked on the GPU; returns (acc (3, npart) in tree order, gpu_seconds,
        list entries)."""
        self.begin(tree.pos, tree.leaf_ipart, tree.leaf_npart, masses)
        ntask = self.submit_walk(tree_dev, cutoff, open_angle)
        sec = self.end()
        acc = np.zeros((3, self.npart), dtype=np.float64)
        self.accumulate(acc)
        return acc, sec, ntask

    # -- device-resident pass (pointers into HBM, e.g. torch tensors) --------
    def run_device(self, npart, d_pos, nleaf, d_ip, d_np, ntask, d_t, d_s, d_mass=None):
        self.npart = npart
        self._nleaf = nleaf
        _check(self.lib, self.lib.p2p_pass_run_device(self.h, npart, d_pos, d_mass, nleaf, d_ip, d_np,
                                                      ntask, d_t, d_s))

    def result_device(self):
        p = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_pass_result_device(self.h, ctypes.byref(p)))
        return p.value

    def measure_fp32_peak(self):
        v = ctypes.c_double()
        _check(self.lib, self.lib.p2p_measure_fp32_peak(self.h, ctypes.byref(v)))
        return v.value

    def measure_fp64_peak(self):
        v = ctypes.c_double()
        _check(self.lib, self.lib.p2p_measure_fp64_peak(self.h, ctypes.byref(v)))
        return v.value


def kernel_launch_count():
    return _native.core().p2p_kernel_launch_count()


class DeviceWalkTree:
    """A lists.Tree's node and leaf tables in device memory (torch tensors)
    as the p2p_walk_tree the device walk reads."""

    def __init__(self, tree, device):
        import torch

        son, first, center, width = tree.nodes()
        to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self._t = [to(son), to(first), to(center), to(width), to(tree.leaf_center), to(tree.leaf_width),
                   to(tree.leaf_active)]
        t = self._t
        self.struct = abi.WalkTree(son.shape[0], tree.nleaf, t[0].data_ptr(), t[1].data_ptr(),
                                   t[2].data_ptr(), t[3].data_ptr(), t[4].data_ptr(), t[5].data_ptr(),
                                   t[6].data_ptr())


class FarField:
    """The far field of the short-range force within the cutoff (p2p_fmm_*):
    PhotoNs' P2M, M2M, M2L walk and M2L, L2L and L2P (src/operator.c,
    src/fmm.c:812-957, :1188-1217) on the GPU, on the kd-tree of the pass."""

    def __init__(self, session):
        self.lib = session.lib
        self.session = session
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_fmm_create(session.h, ctypes.byref(h)))
        self.h = h
        self.nleaf = 0

    def far(self, tree, d_pos, d_leaf_ipart, d_leaf_npart, npart, mass, split_radius, cutoff, open_angle,
            min_r2, d_acc):
        """tree: an abi.WalkTree of device arrays (DeviceTree.struct); the
        other arrays are device pointers (ints); d_acc receives (3, npart)
        far-field accelerations in tree order."""
        self.nleaf = tree.nleaf
        _check(self.lib, self.lib.p2p_fmm_far(self.h, ctypes.byref(tree), npart, d_pos, d_leaf_ipart, d_leaf_npart,
                                              float(mass), float(split_radius), float(cutoff), float(open_angle),
                                              float(min_r2), d_acc))

    def stats(self):
        """M2L tasks, tasks applied, walk levels and device ms (upward, walk,
        m2l, downward, total) of the last far()."""
        n, a, lv = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        ms = (ctypes.c_float * 5)()
        _check(self.lib, self.lib.p2p_fmm_stats(self.h, ctypes.byref(n), ctypes.byref(a), ctypes.byref(lv), ms))
        return dict(n_m2l=n.value, n_applied=a.value, levels=lv.value,
                    ms=dict(zip(["upward", "walk", "m2l", "downward", "total"], list(ms))))

    def download(self):
        """(leaf multipoles, leaf locals), each (nleaf, 20)."""
        m, l = np.empty((self.nleaf, 20)), np.empty((self.nleaf, 20))
        _check(self.lib, self.lib.p2p_fmm_download(self.h, m.ctypes.data_as(ctypes.c_void_p),
                                                   l.ctypes.data_as(ctypes.c_void_p)))
        return m, l

    def close(self):
        if self.h:
            self.lib.p2p_fmm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ParticleMesh:
    """The PM long-range force (p2p_pm_*): PhotoNs' partmesh_kick force part
    (src/partmesh.c:12-1470, src/conv.f90:239-330) for one periodic domain on
    the session's device and stream."""

    def __init__(self, session, nmesh, boxsize, split_radius):
        self.lib = session.lib
        self.session = session
        self.nmesh = int(nmesh)
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_pm_create(session.h, self.nmesh, float(boxsize), float(split_radius),
                                                ctypes.byref(h)))
        self.h = h

    def forces(self, pos_dev, tag_dev, mass, acc_dev):
        """Queues the long-range accelerations of the particles with tag 1 into
        acc_dev: torch float64 (3, n) tensors on the device (SoA rows), tag_dev
        int32 (n,) or None (all tag 1)."""
        n = int(pos_dev.shape[-1])
        _check(self.lib, self.lib.p2p_pm_forces(self.h, n, pos_dev.data_ptr(),
                                                tag_dev.data_ptr() if tag_dev is not None else None,
                                                float(mass), acc_dev.data_ptr()))

    def timings(self):
        """Device ms of the last forces(): deposit, fft_green_fft, gradient,
        interp, total."""
        ms = (ctypes.c_float * 5)()
        _check(self.lib, self.lib.p2p_pm_timings(self.h, ms))
        return dict(zip(["deposit", "fft_green_fft", "gradient", "interp", "total"], list(ms)))

    def download(self):
        """Host copies (mass per cell, potential), each (n, n, n) indexed [x, y, z]."""
        n = self.nmesh
        mass, phi = np.empty((n, n, n)), np.empty((n, n, n))
        _check(self.lib, self.lib.p2p_pm_download(self.h, mass.ctypes.data_as(ctypes.c_void_p),
                                                  phi.ctypes.data_as(ctypes.c_void_p)))
        return mass, phi

    def close(self):
        if self.h:
            self.lib.p2p_pm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceTree:
    """The kd-tree built on the GPU (p2p_dtree_build): the tree PhotoNs builds
    on the host before its walk (src/fmm.c:69-327), equal node for node.
    pos_dev: torch float64 tensor (3, n) on the session's device (SoA rows);
    tag_dev: torch int32 (n,) or None (all local)."""

    def __init__(self, session, pos_dev, tag_dev, maxleaf, boxsize):
        self.lib = session.lib
        self.session = session
        n = int(pos_dev.shape[-1])
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_dtree_build(session.h, n, pos_dev.data_ptr(),
                                                  tag_dev.data_ptr() if tag_dev is not None else None,
                                                  maxleaf, boxsize, ctypes.byref(h)))
        self.h = h
        self._refresh()

    def rebuild(self, pos_dev, tag_dev, maxleaf, boxsize):
        """Rebuilds this tree from new positions (p2p_dtree_rebuild), in its
        device arrays where they are large enough."""
        n = int(pos_dev.shape[-1])
        _check(self.lib, self.lib.p2p_dtree_rebuild(self.session.h, self.h, n, pos_dev.data_ptr(),
                                                    tag_dev.data_ptr() if tag_dev is not None else None,
                                                    maxleaf, boxsize))
        self._refresh()

    def _refresh(self):
        a, b, c, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        _check(self.lib, self.lib.p2p_dtree_counts(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                   ctypes.byref(ms)))
        self.npart, self.nleaf, self.nnode, self.build_ms = a.value, b.value, c.value, ms.value
        self.struct = abi.WalkTree()
        _check(self.lib, self.lib.p2p_dtree_walk_tree(self.h, ctypes.byref(self.struct)))

    def device_arrays(self):
        """(d_pos, d_perm, d_leaf_ipart, d_leaf_npart) device pointers (ints)."""
        p = [ctypes.c_void_p() for _ in range(4)]
        _check(self.lib, self.lib.p2p_dtree_device_arrays(self.h, *[ctypes.byref(x) for x in p]))
        return tuple(x.value for x in p)

    def unpermute(self, d_in, d_out):
        """d_out (input order) from d_in (tree order): device pointers of
        3*npart doubles, queued on the session's stream."""
        _check(self.lib, self.lib.p2p_dtree_unpermute(self.h, self.session.h, d_in, d_out))

    def download(self):
        """Host copies: dict of pos (3, n), perm, leaf_ipart, leaf_npart,
        leaf_active, leaf_center (nleaf, 3), leaf_width, son (nnode, 2),
        node_first, node_center (nnode, 3), node_width."""
        n, nl, nn = self.npart, self.nleaf, self.nnode
        out = dict(pos=np.empty((3, n)), perm=np.empty(n, np.int32), leaf_ipart=np.empty(nl, np.int32),
                   leaf_npart=np.empty(nl, np.int32), leaf_active=np.empty(nl, np.int32),
                   leaf_center=np.empty((nl, 3)), leaf_width=np.empty((nl, 3)), son=np.empty((nn, 2), np.int32),
                   node_first=np.empty(nn, np.int32), node_center=np.empty((nn, 3)), node_width=np.empty((nn, 3)))
        keys = ["pos", "perm", "leaf_ipart", "leaf_npart", "leaf_active", "leaf_center", "leaf_width", "son",
                "node_first", "node_center", "node_width"]
        _check(self.lib, self.lib.p2p_dtree_download(self.h, *[out[k].ctypes.data_as(ctypes.c_void_p)
                                                               for k in keys]))
        return out

    def close(self):
        if self.h:
            self.lib.p2p_dtree_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

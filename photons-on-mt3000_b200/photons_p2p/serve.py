"""Serving force passes for an ensemble of independent boxes.

Server wraps the C ABI's p2p_server (include/photons_p2p.h): boxes are
registered once, made resident on the device when first requested (or
preloaded), and requests that are pending together are packed into shared
persistent launches while up to `slots` launches run at once. run_poisson()
drives it with Poisson arrivals and reports latency percentiles and
throughput.

Units: every box of a server shares one kernel shape (form, softening mode,
x_cut and the softening in units of the split radius). A box with split
radius r_s is registered with length_scale = 0.5 / r_s, so the shape's split
radius is 0.5 and its softening 0.5 * eps / r_s.
"""
import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _native
from .abi import ServerConfig, ServerStats, SOFT_PLUMMER
from .p2p import P2PError, _check, make_params


def serving_shape(form, eps_over_rs, soft_mode=SOFT_PLUMMER, x_cut=2.25, **kw):
    """Kernel shape of boxes whose softening is eps_over_rs split radii."""
    return make_params(form=form, soft_mode=soft_mode, soften=0.5 * eps_over_rs, split_radius=0.5,
                       x_cut=x_cut, mass=1.0, **kw)


class PinnedArray:
    """Page-locked, device-mapped host doubles (p2p_host_alloc)."""

    def __init__(self, n):
        self.lib = _native.core()
        p = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_host_alloc(8 * max(n, 1), ctypes.byref(p)))
        self.ptr = p.value
        self.n = n
        self.array = np.ctypeslib.as_array((ctypes.c_double * max(n, 1)).from_address(self.ptr))[:n]

    def free(self):
        if self.ptr:
            self.lib.p2p_host_free(self.ptr)
            self.ptr = None


@dataclass
class BoxEntry:
    box_id: int
    npart: int           # particles a request returns
    pairs: int
    keep: tuple          # host arrays the server reads on (re)admission
    free_out: list       # idle result buffers


class Server:
    def __init__(self, shape, device=0, slots=1, max_pack=32, full_grid=True, hbm_bytes=0,
                 rows_per_particle=0.0, particles_per_leaf=0.0, batch_window_ms=0.0, min_pack_pairs=0.0):
        self.lib = _native.core()
        cfg = ServerConfig()
        self.lib.p2p_server_config_default(ctypes.byref(cfg))
        cfg.slots = slots
        cfg.max_pack = max_pack
        cfg.full_grid = 1 if full_grid else 0
        cfg.hbm_bytes = int(hbm_bytes)
        if rows_per_particle:
            cfg.rows_per_particle = rows_per_particle
        if particles_per_leaf:
            cfg.particles_per_leaf = particles_per_leaf
        cfg.batch_window_ms = batch_window_ms
        cfg.min_pack_pairs = min_pack_pairs
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.p2p_server_create(device, ctypes.byref(shape), ctypes.byref(cfg),
                                                    ctypes.byref(h)))
        self.h = h
        self.boxes = []
        self.inflight = {}   # ticket -> (box index, PinnedArray)

    def set_batching(self, batch_window_ms, min_pack_pairs=0.0):
        """Batching window: pending requests wait up to batch_window_ms for
        others to share their launch unless the pack already holds max_pack
        boxes or min_pack_pairs pair interactions (0 ms: launch at once)."""
        _check(self.lib, self.lib.p2p_server_set_batching(self.h, float(batch_window_ms), float(min_pack_pairs)))

    def close(self):
        if self.h:
            self.lib.p2p_server_destroy(self.h)
            self.h = None
            for b in self.boxes:
                for buf in b.free_out:
                    buf.free()
            for _, buf in self.inflight.values():
                buf.free()
            self.inflight = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_box(self, lists, length_scale, mass, locals_only=True):
        """Registers a box from its TreeLists (tree-order positions, leaves
        and the walk's list); returns its index. locals_only: requests return
        the local particles' accelerations in their original order (shape
        (3, n_local)); otherwise every particle in tree order."""
        pos = np.ascontiguousarray(lists.pos, np.float64)
        ip = np.ascontiguousarray(lists.leaf_ipart, np.int32)
        npt = np.ascontiguousarray(lists.leaf_npart, np.int32)
        tt = np.ascontiguousarray(lists.task_t, np.int32)
        ts = np.ascontiguousarray(lists.task_s, np.int32)
        if locals_only:
            slot = np.empty(pos.shape[1], np.int32)
            slot[lists.perm] = np.arange(pos.shape[1], dtype=np.int32)
            res = np.ascontiguousarray(slot[:int(lists.tag.sum())])  # locals come first in perm ids
        else:
            res = None
        nres = pos.shape[1] if res is None else res.shape[0]
        bid = ctypes.c_int()
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        _check(self.lib, self.lib.p2p_server_add_box(
            self.h, float(length_scale), float(mass), pos.shape[1], vp(pos), ip.shape[0], vp(ip),
            vp(npt), tt.shape[0], vp(tt), vp(ts), nres, None if res is None else vp(res),
            ctypes.byref(bid)))
        n64 = npt.astype(np.int64)
        pairs = int(np.dot(n64[tt], n64[ts])) if tt.size else 0
        self.boxes.append(BoxEntry(bid.value, nres, pairs, (pos, ip, npt, tt, ts, res), []))
        return len(self.boxes) - 1

    def preload(self, k, release_host=True):
        """Resident and pinned now; the host arrays may then be dropped."""
        _check(self.lib, self.lib.p2p_server_preload(self.h, self.boxes[k].box_id))
        if release_host:
            self.boxes[k].keep = ()

    def box_bytes(self, k):
        v = ctypes.c_size_t()
        _check(self.lib, self.lib.p2p_server_box_bytes(self.h, self.boxes[k].box_id, ctypes.byref(v)))
        return v.value

    def reserve_outputs(self, per_box):
        """Allocates result buffers ahead of time (page-locking is slow and
        would otherwise fall inside submit)."""
        for b in self.boxes:
            while len(b.free_out) < per_box:
                b.free_out.append(PinnedArray(3 * b.npart))

    def submit(self, k):
        b = self.boxes[k]
        buf = b.free_out.pop() if b.free_out else PinnedArray(3 * b.npart)
        t = ctypes.c_int64()
        st = self.lib.p2p_server_submit(self.h, b.box_id, ctypes.c_void_p(buf.ptr), ctypes.byref(t))
        if st:
            b.free_out.append(buf)
            _check(self.lib, st)
        self.inflight[t.value] = (k, buf)
        return t.value

    def wait(self, ticket, copy=True):
        """(acc (3, npart) or None, latency seconds); the result buffer is
        recycled, so copy=True returns a copy."""
        lat = ctypes.c_double()
        st = self.lib.p2p_server_wait(self.h, ticket, ctypes.byref(lat))
        k, buf = self.inflight.pop(ticket)
        out = buf.array.reshape(3, -1).copy() if (copy and st == 0) else None
        self.boxes[k].free_out.append(buf)
        _check(self.lib, st)
        return out, lat.value

    def drain(self):
        _check(self.lib, self.lib.p2p_server_drain(self.h))

    def stats(self):
        s = ServerStats()
        _check(self.lib, self.lib.p2p_server_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()


def box_lists(box):
    """Ghosts + tree + walk of one workloads.ServingBox."""
    from .workloads import prepare
    return prepare(box.pos, box.cfg)


def run_poisson(server, rate_hz, n_requests, seed=0, boxes=None, keep_results=False, reserve=1):
    """Submits n_requests force passes with exponential inter-arrival times
    (rate rate_hz, boxes drawn uniformly from `boxes` or all) while a second
    thread collects the results as they finish (recycling the page-locked
    result buffers). Returns latency percentiles and throughput; latency is
    the server's own submit-to-result time."""
    import queue
    import threading

    g = np.random.default_rng(seed)
    idx = np.arange(len(server.boxes)) if boxes is None else np.asarray(boxes)
    pick = g.choice(idx, size=n_requests)
    gaps = g.exponential(1.0 / rate_hz, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    server.reserve_outputs(reserve)
    lat = np.empty(n_requests)
    results = []
    todo = queue.Queue()
    failure = []

    def collect():
        while True:
            item = todo.get()
            if item is None:
                return
            i, t, k = item
            try:
                out, lat[i] = server.wait(t, copy=keep_results)
            except Exception as e:  # reported after the run
                failure.append(e)
                lat[i] = np.nan
                continue
            if keep_results:
                results.append((k, out))

    s0 = server.stats()
    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i, (a, k) in enumerate(zip(arrivals, pick)):
        delay = t0 + a - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        todo.put((i, server.submit(int(k)), int(k)))
    todo.put(None)
    th.join()
    span = time.perf_counter() - t0
    if failure:
        raise failure[0]
    s1 = server.stats()
    pairs = sum(server.boxes[int(k)].pairs for k in pick)
    res = {
        "rate_hz": rate_hz, "requests": n_requests,
        "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3),
        "makespan_s": span, "requests_per_s": n_requests / span, "pairs_per_s": pairs / span,
        "launches": s1["launches"] - s0["launches"],
        "boxes_per_launch": (s1["boxes_launched"] - s0["boxes_launched"]) /
                            max(1, s1["launches"] - s0["launches"]),
        "kernel_busy_frac": (s1["kernel_ms"] - s0["kernel_ms"]) / 1e3 / span,
        "builds": s1["builds"] - s0["builds"], "evictions": s1["evictions"] - s0["evictions"],
    }
    if keep_results:
        res["results"] = results
    return res


__all__ = ["Server", "PinnedArray", "serving_shape", "box_lists", "run_poisson", "P2PError"]

"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

  liboracle.so      oracle/p2p_oracle.c, the plain-C restatement (built here
                    with gcc on first use when missing)
  _ref/libref_*.so  the reference's own code compiled for the host by
                    oracle/build_ref.sh (present when the reference sources
                    were available at build time)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(HERE, "liboracle.so")

SOFT_CLAMP = 0
SOFT_PLUMMER = 1

_vp = ctypes.c_void_p


class OracleParams(ctypes.Structure):
    _fields_ = [("soft_mode", ctypes.c_int), ("soften", ctypes.c_double),
                ("split_radius", ctypes.c_double), ("x_cut", ctypes.c_double),
                ("mass", ctypes.c_double)]


def build(force=False):
    src = os.path.join(HERE, "p2p_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", LIB, src, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.oracle_pair.argtypes = [ctypes.POINTER(OracleParams), _vp, _vp, _vp]
        L.oracle_p2p_lists.restype = ctypes.c_int64
        L.oracle_p2p_lists.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int, _vp, _vp,
                                       ctypes.c_int, _vp, _vp, ctypes.c_int64, _vp, _vp,
                                       ctypes.c_int64, _vp]
        L.oracle_pair_count.restype = ctypes.c_int64
        L.oracle_pair_count.argtypes = [_vp, ctypes.c_int64, _vp, _vp]
        L.oracle_direct.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int, _vp, _vp,
                                    ctypes.c_double, ctypes.c_int, _vp, _vp]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def params(soft_mode, soften, split_radius, x_cut, mass):
    return OracleParams(soft_mode, soften, split_radius, x_cut, mass)


def pair(prm, ii, jj):
    ii = np.ascontiguousarray(ii, np.float64)
    jj = np.ascontiguousarray(jj, np.float64)
    out = np.zeros(3)
    lib().oracle_pair(ctypes.byref(prm), _p(ii), _p(jj), _p(out))
    return out


def p2p_lists(prm, pos, leaf_ipart, leaf_npart, task_t, task_s, masses=None, chunk=0):
    """Reference-order P2P over the lists; returns (acc (3, n), pair count)."""
    pos = np.ascontiguousarray(pos, np.float64)
    n = pos.shape[1]
    ip = np.ascontiguousarray(leaf_ipart, np.int32)
    npt = np.ascontiguousarray(leaf_npart, np.int32)
    tt = np.ascontiguousarray(task_t, np.int32)
    ts = np.ascontiguousarray(task_s, np.int32)
    m = np.ascontiguousarray(masses, np.float64) if masses is not None else None
    acc = np.zeros((3, n))
    pairs = lib().oracle_p2p_lists(ctypes.byref(prm), n, _p(pos), _p(m), ip.shape[0], _p(ip),
                                   _p(npt), tt.shape[0], _p(tt), _p(ts), chunk, _p(acc))
    return acc, pairs


def pair_count(leaf_npart, task_t, task_s):
    npt = np.ascontiguousarray(leaf_npart, np.int32)
    tt = np.ascontiguousarray(task_t, np.int32)
    ts = np.ascontiguousarray(task_s, np.int32)
    return lib().oracle_pair_count(_p(npt), tt.shape[0], _p(tt), _p(ts))


def direct(prm, pos, box, sinks, masses=None):
    """FP64 direct minimum-image sum for the given sink indices; (3, nsink)."""
    pos = np.ascontiguousarray(pos, np.float64)
    sinks = np.ascontiguousarray(sinks, np.int32)
    m = np.ascontiguousarray(masses, np.float64) if masses is not None else None
    out = np.zeros((3, sinks.shape[0]))
    lib().oracle_direct(ctypes.byref(prm), pos.shape[1], _p(pos), _p(m), box, sinks.shape[0],
                        _p(sinks), _p(out))
    return out


def num_threads():
    return lib().oracle_num_threads()


# ---------------------------------------------------------- reference libs --

def ref_available(name="libref_pair.so"):
    return os.path.exists(os.path.join(REF_DIR, name))


_ref_pair = None


def ref_pair_lib():
    global _ref_pair
    if _ref_pair is None:
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref_pair.so"))
        for v in ("dp", "dp_cut", "sp_spi"):
            f = getattr(L, f"ref_p2p_lists_{v}")
            f.restype = ctypes.c_int64
            f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                          ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, _vp, _vp,
                          ctypes.c_int64, _vp]
            g = getattr(L, f"ref_pair_{v}")
            g.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp]
        _ref_pair = L
    return _ref_pair


def ref_p2p_lists(variant, soft_mode, soften, split_radius, mass, pos, leaf_ipart, leaf_npart,
                  task_t, task_s, chunk=0):
    """The reference's pair functions (host-compiled) over the lists.
    variant: 'dp' (FP64), 'dp_cut' (FP64 + GPUCUTOFF), 'sp_spi' (FP32 SPI + GPUCUTOFF)."""
    L = ref_pair_lib()
    pos = np.ascontiguousarray(pos, np.float64)
    n = pos.shape[1]
    ip = np.ascontiguousarray(leaf_ipart, np.int32)
    npt = np.ascontiguousarray(leaf_npart, np.int32)
    tt = np.ascontiguousarray(task_t, np.int32)
    ts = np.ascontiguousarray(task_s, np.int32)
    acc = np.zeros((3, n))
    f = getattr(L, f"ref_p2p_lists_{variant}")
    pairs = f(soft_mode, soften, split_radius, mass, n, _p(pos), ip.shape[0], _p(ip), _p(npt),
              tt.shape[0], _p(tt), _p(ts), chunk, _p(acc))
    return acc, pairs


def ref_pair(variant, soft_mode, soften, split_radius, ii, jj):
    L = ref_pair_lib()
    ii = np.ascontiguousarray(ii, np.float64)
    jj = np.ascontiguousarray(jj, np.float64)
    out = np.zeros(3)
    getattr(L, f"ref_pair_{variant}")(soft_mode, soften, split_radius, _p(ii), _p(jj), _p(out))
    return out


class RefWalk:
    """The reference's own fmm_prepare / fmm_task (src/fmm.c) driven by
    oracle/ref_walk_harness.c; records the interaction lists (libref_walk.so)
    or runs the B200 drop-in behind them (libref_dropin_{dp,sp}.so)."""

    def __init__(self, libname="libref_walk.so"):
        L = ctypes.CDLL(os.path.join(REF_DIR, libname), mode=ctypes.RTLD_LOCAL)
        f = L.ref_harness_run
        f.restype = ctypes.c_int
        f.argtypes = ([ctypes.c_int, _vp, _vp, ctypes.c_int] + [ctypes.c_double] * 6 +
                      [ctypes.c_int, ctypes.c_int] + [_vp] * 8)
        self.L = L
        self.recording = hasattr(L, "ref_record_count")
        if self.recording:
            L.ref_record_count.restype = ctypes.c_longlong
            L.ref_record_nchunk.restype = ctypes.c_int

    def fmm(self, pos, tag, maxleaf, boxsize, split_radius, cutoff_radius, soften, mass, open_angle):
        """The reference's far field (ref_harness_fmm): tree order and leaf
        table as run() gives them, the leaves' multipoles M and locals L
        (nleaf, 20), the far-field accelerations of l2p (3, n) in tree order,
        the counts of M2L tasks, m2l calls and nodes, and the seconds of
        the reference's task_compute_m2l (its own timer) and of the l2p."""
        f = self.L.ref_harness_fmm
        f.restype = ctypes.c_int
        f.argtypes = ([ctypes.c_int, _vp, _vp, ctypes.c_int] + [ctypes.c_double] * 6 + [_vp] * 11)
        pos = np.ascontiguousarray(pos, np.float64)
        tag = np.ascontiguousarray(tag, np.int32)
        n = pos.shape[1]
        perm = np.empty(n, np.int32)
        ip = np.empty(n + 1, np.int32)
        npt = np.empty(n + 1, np.int32)
        act = np.empty(n + 1, np.int32)
        ctr = np.empty((n + 1, 3))
        wid = np.empty((n + 1, 3))
        lm = np.empty((n + 1, 20))
        ll = np.empty((n + 1, 20))
        acc = np.empty((3, n))
        counts = np.zeros(3, np.int64)
        times = np.zeros(2)
        nl = f(n, _p(pos), _p(tag), maxleaf, boxsize, split_radius, cutoff_radius, soften, mass, open_angle,
               _p(perm), _p(ip), _p(npt), _p(ctr), _p(wid), _p(act), _p(lm), _p(ll), _p(acc), _p(counts), _p(times))
        if nl < 0:
            raise RuntimeError("reference harness failed")
        return dict(perm=perm, leaf_ipart=ip[:nl].copy(), leaf_npart=npt[:nl].copy(),
                    leaf_active=act[:nl].copy(), leaf_center=ctr[:nl].copy(), leaf_width=wid[:nl].copy(),
                    leaf_M=lm[:nl].copy(), leaf_L=ll[:nl].copy(), acc=acc, n_m2l=int(counts[0]),
                    n_m2l_calls=int(counts[1]), n_node=int(counts[2]), m2l_s=float(times[0]),
                    l2p_s=float(times[1]))

    def run(self, pos, tag, maxleaf, boxsize, split_radius, cutoff_radius, soften, mass,
            open_angle, len_task, collect_acc=False):
        pos = np.ascontiguousarray(pos, np.float64)
        tag = np.ascontiguousarray(tag, np.int32)
        n = pos.shape[1]
        perm = np.empty(n, np.int32)
        ip = np.empty(n + 1, np.int32)
        npt = np.empty(n + 1, np.int32)
        act = np.empty(n + 1, np.int32)
        ctr = np.empty((n + 1, 3))
        wid = np.empty((n + 1, 3))
        acc = np.zeros((3, n)) if collect_acc else None
        ksec = ctypes.c_double(0.0)
        if self.recording:
            self.L.ref_record_reset()
        nl = self.L.ref_harness_run(n, _p(pos), _p(tag), maxleaf, boxsize, split_radius,
                                    cutoff_radius, soften, mass, open_angle, len_task,
                                    1 if collect_acc else 0, _p(perm), _p(ip), _p(npt), _p(ctr),
                                    _p(wid), _p(act), _p(acc), ctypes.addressof(ksec))
        if nl < 0:
            raise RuntimeError("reference harness failed")
        out = dict(perm=perm, leaf_ipart=ip[:nl].copy(), leaf_npart=npt[:nl].copy(),
                   leaf_active=act[:nl].copy(), leaf_center=ctr[:nl].copy(),
                   leaf_width=wid[:nl].copy(), acc=acc, kernel_seconds=ksec.value)
        if self.recording:
            nt = self.L.ref_record_count()
            nc = self.L.ref_record_nchunk()
            tt = np.empty(nt, np.int32)
            ts = np.empty(nt, np.int32)
            ce = np.empty(nc, np.int64)
            self.L.ref_record_copy(_p(tt), _p(ts), _p(ce))
            out.update(task_t=tt, task_s=ts, chunk_end=ce)
        return out


def ref_pack_run(libname, pos, leaf_ipart, leaf_npart, leaf_base, split_radius, soften, mass, packs):
    """The drop-in's multi-pack entry p2ppack_compute_gpu driven as the
    reference's load-balanced walk calls it (oracle/ref_pack_harness.c).
    packs: list of dicts with task_t, task_s (absolute leaf ids, i.e. 0-based
    id + leaf_base), ileaf, nleaf, ipart, npart. Returns (acc (3, npart),
    kernel seconds)."""
    L = ctypes.CDLL(os.path.join(REF_DIR, libname), mode=ctypes.RTLD_LOCAL)
    f = L.ref_pack_run
    f.restype = ctypes.c_int
    pos = np.ascontiguousarray(pos, np.float64)
    n = pos.shape[1]
    ip = np.ascontiguousarray(leaf_ipart, np.int32)
    npt = np.ascontiguousarray(leaf_npart, np.int32)
    col = lambda k: np.ascontiguousarray([p[k] for p in packs], np.int32)  # noqa: E731
    ntask = np.ascontiguousarray([len(p["task_t"]) for p in packs], np.int32)
    tt = np.ascontiguousarray(np.concatenate([p["task_t"] for p in packs]), np.int32)
    ts = np.ascontiguousarray(np.concatenate([p["task_s"] for p in packs]), np.int32)
    cols = [col(k) for k in ("ileaf", "nleaf", "ipart", "npart")]
    acc = np.zeros((3, n))
    ksec = ctypes.c_double(0.0)
    f.argtypes = ([ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int] + [ctypes.c_double] * 3 +
                  [ctypes.c_int] + [_vp] * 9)
    st = f(n, _p(pos), ip.shape[0], _p(ip), _p(npt), leaf_base, split_radius, soften, mass, len(packs),
           _p(ntask), *[_p(c) for c in cols], _p(tt), _p(ts), _p(acc), ctypes.addressof(ksec))
    if st != 0:
        raise RuntimeError("pack harness failed")
    return acc, ksec.value


def ref_act_run(libname, pos, leaf_ipart, leaf_npart, leaf_base, split_radius, soften, mass, packs, act,
                active_level, mode, chunk=0, acc0=None):
    """The drop-in's active-level entries driven through the reference's
    globals (oracle/ref_pack_harness.c, ref_act_run): mode "pack" calls
    p2ppack_compute_act_gpu with the packs, mode "task" calls
    task_compute_p2p_act_gpu over the packs' concatenated entries in chunks
    of `chunk`. act: the particles' levels (part[i].act). Returns acc0 (3,
    npart; zeros if None) plus what the call added."""
    L = ctypes.CDLL(os.path.join(REF_DIR, libname), mode=ctypes.RTLD_LOCAL)
    f = L.ref_act_run
    f.restype = ctypes.c_int
    pos = np.ascontiguousarray(pos, np.float64)
    n = pos.shape[1]
    ip = np.ascontiguousarray(leaf_ipart, np.int32)
    npt = np.ascontiguousarray(leaf_npart, np.int32)
    col = lambda k: np.ascontiguousarray([p[k] for p in packs], np.int32)  # noqa: E731
    ntask = np.ascontiguousarray([len(p["task_t"]) for p in packs], np.int32)
    tt = np.ascontiguousarray(np.concatenate([p["task_t"] for p in packs]), np.int32)
    ts = np.ascontiguousarray(np.concatenate([p["task_s"] for p in packs]), np.int32)
    cols = [col(k) for k in ("ileaf", "nleaf", "ipart", "npart")]
    acc = np.zeros((3, n)) if acc0 is None else np.array(acc0, np.float64, order="C", copy=True)
    act = np.ascontiguousarray(act, np.int32)
    assert act.shape == (n,) and acc.shape == (3, n)
    f.argtypes = ([ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int] + [ctypes.c_double] * 3 +
                  [ctypes.c_int] + [_vp] * 9 + [ctypes.c_int] * 3)
    st = f(n, _p(pos), ip.shape[0], _p(ip), _p(npt), leaf_base, split_radius, soften, mass, len(packs),
           _p(ntask), *[_p(c) for c in cols], _p(tt), _p(ts), _p(acc), _p(act), {"pack": 1, "task": 2}[mode],
           active_level, chunk)
    if st != 0:
        raise RuntimeError("active-level harness failed")
    return acc

"""The drop-in's host logic on the CPU. photons-on-mt3000_b200/csrc/
gpu_entry_b200.cpp is linked with the reference's globals and walk
(src/global.c, src/fmm.c) over a host stand-in for the pass protocol
(oracle/host_session_stub.c) that adds a counting result per submitted entry
(npart of the source leaf, source id + 1, 1) instead of forces. Sums of small
integers are exact, so every check is exact: the chunked protocol as the
reference's own fmm_task drives it, the multi-pack protocol
(rebasing of absolute leaf ids, an inter-subtree pack overlapping the others),
the result update over the packs' particles, and the active-level entries'
row selection and update rule, without and with ACT_OPT. The same entry
points run on the GPU in test_dropin_gpu.py."""
import ctypes
import os

import numpy as np
import pytest

from dropin_cases import act_levels, act_updates, lb_packs
from oracle import oracle as O
from photons_p2p import workloads as W

pytestmark = pytest.mark.skipif(not (O.ref_available("libref_dropin_host.so") and
                                     O.ref_available("libref_dropin_hostact.so")),
                                reason="oracle/_ref host drop-in harness not built")

LEAF_BASE = 5  # a biased leaf pointer, as PhotoNs' first_leaf


@pytest.fixture(scope="module")
def tl():
    cfg = W.ref_dropin_config(32, 64, 32)
    return W.prepare(W.lattice_gaussian(32, 0.2, W.rng(1)), cfg), cfg


def stub(lib):
    L = ctypes.CDLL(os.path.join(O.REF_DIR, f"libref_dropin_{lib}.so"), mode=ctypes.RTLD_LOCAL)
    L.stub_submitted_entries.restype = ctypes.c_longlong
    L.stub_passes.restype = ctypes.c_longlong
    return L


def counting(tl):
    """The stand-in's result for the whole list, per particle (3, n)."""
    n = tl.pos.shape[1]
    per_leaf = np.zeros((3, tl.nleaf))
    np.add.at(per_leaf[0], tl.task_t, tl.leaf_npart[tl.task_s])
    np.add.at(per_leaf[1], tl.task_t, tl.task_s + 1)
    np.add.at(per_leaf[2], tl.task_t, 1)
    out = np.zeros((3, n))
    for l in range(tl.nleaf):
        out[:, tl.leaf_ipart[l]:tl.leaf_ipart[l] + tl.leaf_npart[l]] = per_leaf[:, l:l + 1]
    return out


def leaf_of(tl):
    f = np.full(tl.pos.shape[1], -1)
    for l in range(tl.nleaf):
        f[tl.leaf_ipart[l]:tl.leaf_ipart[l] + tl.leaf_npart[l]] = l
    return f


def test_multi_pack_protocol(tl):
    """p2ppack_compute_gpu + get_last_kntime + devMemcpyDH_updateAcc(-1):
    four subtree packs and the overlapping inter-subtree pack; every entry
    submitted once with 0-based ids, every particle updated once."""
    tl, cfg = tl
    packs = lb_packs(tl, 4, LEAF_BASE)
    L = stub("host")
    L.stub_reset()
    got, ksec = O.ref_pack_run("libref_dropin_host.so", tl.pos, tl.leaf_ipart, tl.leaf_npart, LEAF_BASE,
                               cfg.split_radius, cfg.eps, 1.0, packs)
    assert L.stub_submitted_entries() == tl.ntask and L.stub_passes() == 1
    assert ksec > 0
    assert np.array_equal(got, counting(tl))


def test_update_covers_only_the_packs_particles(tl):
    """One subtree's pack alone: its entries are submitted, and the update
    adds over that pack's particle range only (updateAcc_fromHostBuff,
    src/gpu_func.impl.h:644-653)."""
    tl, cfg = tl
    p = lb_packs(tl, 4, LEAF_BASE)[1]
    got, _ = O.ref_pack_run("libref_dropin_host.so", tl.pos, tl.leaf_ipart, tl.leaf_npart, LEAF_BASE,
                            cfg.split_radius, cfg.eps, 1.0, [p])
    lo, hi = p["ipart"], p["ipart"] + p["npart"]
    t, s = p["task_t"] - LEAF_BASE, p["task_s"] - LEAF_BASE
    want = np.zeros_like(got)
    f = leaf_of(tl)
    for d, val in enumerate((tl.leaf_npart[s], s + 1, np.ones_like(s))):
        per_leaf = np.bincount(t, weights=val, minlength=tl.nleaf)
        want[d, lo:hi] = per_leaf[f[lo:hi]]
    assert np.array_equal(got, want)
    assert not got[:, :lo].any() and not got[:, hi:].any()


@pytest.mark.parametrize("lib,mode,level,chunk", [
    ("host", "pack", 2, 0), ("host", "pack", 0, 0), ("host", "pack", -1, 0), ("host", "task", 1, 3000),
    ("host", "task", 3, 1), ("host", "task", -1, 7919), ("hostact", "task", 2, 3000),
    ("hostact", "task", -1, 5000), ("hostact", "task", 255, 100000)])
def test_active_level_protocol(tl, lib, mode, level, chunk):
    """task_compute_p2p_act_gpu / p2ppack_compute_act_gpu: the particles the
    reference's pass would change get the whole list's result, all others
    keep their acc bit for bit, and exactly the rows of sink leaves holding
    such a particle are submitted."""
    tl, cfg = tl
    g = np.random.default_rng(11)
    act = act_levels(tl, g)
    packs = lb_packs(tl, 4, LEAF_BASE)
    full = counting(tl)
    acc0 = g.normal(size=full.shape)
    L = stub(lib)
    L.stub_reset()
    got = O.ref_act_run(f"libref_dropin_{lib}.so", tl.pos, tl.leaf_ipart, tl.leaf_npart, LEAF_BASE,
                        cfg.split_radius, cfg.eps, 1.0, packs, act, level, mode, chunk, acc0)
    upd = act_updates(act, level, lib == "hostact")
    assert np.array_equal(got[:, ~upd], acc0[:, ~upd])
    assert np.array_equal(got[:, upd], acc0[:, upd] + full[:, upd])
    live = np.zeros(tl.nleaf, bool)
    live[leaf_of(tl)[upd]] = True
    assert L.stub_submitted_entries() == int(live[tl.task_t].sum())
    assert L.stub_passes() == 1
    if level not in (0, -1) or lib == "hostact":
        assert 0 < L.stub_submitted_entries() < tl.ntask  # rows were dropped


@pytest.mark.skipif(not O.ref_available("libref_walk.so"), reason="oracle/_ref reference walk not built")
def test_reference_fmm_task_chunks_through_the_dropin():
    """The reference's own fmm_prepare / fmm_task (src/fmm.c) calls
    task_compute_p2p_gpu in LEN_TASK chunks and collects the result as
    gravity.c does: every entry of its list is submitted once, rebased to
    0-based leaf ids, across several chunks, and every particle receives its
    rows' result."""
    cfg = W.ref_dropin_config(16, 32, 32)
    allpos, tag = W.with_ghosts(W.lattice_gaussian(16, 0.2, W.rng(3)), cfg)
    args = (allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius, cfg.cutoff_radius, cfg.eps, 1.0,
            cfg.open_angle, 3000)
    walk = O.RefWalk("libref_walk.so").run(*args)
    assert len(walk["chunk_end"]) > 1
    L = stub("host")
    L.stub_reset()
    out = O.RefWalk("libref_dropin_host.so").run(*args, collect_acc=True)
    assert np.array_equal(out["perm"], walk["perm"])
    nt = len(walk["task_t"])
    assert L.stub_submitted_entries() == nt and L.stub_passes() == 1
    ip, npt = walk["leaf_ipart"], walk["leaf_npart"]
    per_leaf = np.zeros((3, ip.size))
    np.add.at(per_leaf[0], walk["task_t"], npt[walk["task_s"]])
    np.add.at(per_leaf[1], walk["task_t"], walk["task_s"] + 1)
    np.add.at(per_leaf[2], walk["task_t"], 1)
    want = np.zeros_like(out["acc"])
    for l in range(ip.size):
        want[:, ip[l]:ip[l] + npt[l]] = per_leaf[:, l:l + 1]
    assert np.array_equal(out["acc"], want)

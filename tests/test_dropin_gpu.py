"""Drop-in check: the reference's own fmm_prepare / fmm_task (src/fmm.c,
compiled unchanged) calls the B200 library through the legacy gpu_entry
symbols (task_compute_p2p_gpu, get_last_kntime, devMemcpyDH_updateAcc ...),
in LEN_TASK chunks, and the accelerations it receives match the oracle run on
the lists the same walk produces.

The harness libraries are built from the reference sources by
oracle/build_ref.sh (oracle/_ref); the test is skipped where they are absent.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O
from photons_p2p import workloads as W
from dropin_cases import act_levels, act_updates, lb_packs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (O.ref_available("libref_dropin_dp.so") and
                                      O.ref_available("libref_walk.so")),
                                 reason="oracle/_ref drop-in harness not built")]

LEN_TASK = 20000


@pytest.fixture(scope="module")
def case():
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    mass = 1.0 / pos.shape[1]
    args = (allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius, cfg.cutoff_radius, cfg.eps, mass,
            cfg.open_angle, LEN_TASK)
    walk = O.RefWalk("libref_walk.so").run(*args)
    assert len(walk["chunk_end"]) > 1  # the walk really streamed several chunks
    tree_pos = allpos[:, walk["perm"]]
    ref, _ = O.p2p_lists(O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass),
                         tree_pos, walk["leaf_ipart"], walk["leaf_npart"], walk["task_t"],
                         walk["task_s"], chunk=LEN_TASK)
    local = tag[walk["perm"]] == 1
    return args, walk, ref, local


@pytest.mark.parametrize("variant,max_tol,rms_tol", [("dp", 1e-12, 1e-12), ("sp", 1e-3, 1e-5)])
def test_reference_fmm_task_through_dropin(gpu, case, variant, max_tol, rms_tol):
    args, walk, ref, local = case
    out = O.RefWalk(f"libref_dropin_{variant}.so").run(*args, collect_acc=True)
    assert np.array_equal(out["perm"], walk["perm"])
    assert out["kernel_seconds"] > 0
    rms, mx = rel_err(out["acc"], ref, local)
    assert mx <= max_tol and rms <= rms_tol, (rms, mx)


@pytest.mark.parametrize("variant,max_tol,rms_tol", [("dp", 1e-12, 1e-12), ("sp", 1e-3, 1e-5)])
def test_multi_pack_entry_point(gpu, variant, max_tol, rms_tol):
    """p2ppack_compute_gpu with four subtree packs and an overlapping
    inter-subtree pack (the reference's INTRA_LB protocol, src/fmm.c:1245-1250,
    src/gpu_entry.cu:211-386), then get_last_kntime + devMemcpyDH_updateAcc:
    every particle receives its pairs once, as the oracle computes them on
    the whole list."""
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    tl = W.prepare(pos, cfg)
    mass = 1.0 / pos.shape[1]
    leaf_base = 5  # a biased leaf pointer, as PhotoNs' first_leaf
    packs = lb_packs(tl, 4, leaf_base)
    assert len(packs) == 5 and sum(len(p["task_t"]) for p in packs) == tl.ntask
    ref, _ = O.p2p_lists(O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass), tl.pos,
                         tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    got, ksec = O.ref_pack_run(f"libref_dropin_{variant}.so", tl.pos, tl.leaf_ipart, tl.leaf_npart, leaf_base,
                               cfg.split_radius, cfg.eps, mass, packs)
    assert ksec > 0
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert mx <= max_tol and rms <= rms_tol, (rms, mx)


def test_unmoved_particles_are_not_uploaded_again(gpu):
    """The drop-in keeps the previous pass's positions (page-locked staging
    and device copy) and uploads only the 65536-particle chunks that changed:
    a second pass over the same particles uploads nothing and gives the same
    accelerations; after a few particles move, the pass uploads only their
    chunks and equals the pass that uploads everything (after devfree)."""
    import ctypes

    cfg = W.ref_dropin_config(64, 128, 32)
    pos = W.lattice_gaussian(64, 0.2, W.rng(7))
    allpos, tag = W.with_ghosts(pos, cfg)
    n = allpos.shape[1]
    mass = 1.0 / pos.shape[1]
    rest = (cfg.maxleaf, cfg.box, cfg.split_radius, cfg.cutoff_radius, cfg.eps, mass, cfg.open_angle, 10 ** 7)
    lib = O.RefWalk("libref_dropin_dp.so")
    uploaded = lib.L.p2p_dropin_last_upload_bytes
    uploaded.restype = ctypes.c_int64
    full = 24 * n
    lib.L.devfree()
    a = lib.run(allpos, tag, *rest, collect_acc=True)
    assert uploaded() == full
    b = lib.run(allpos, tag, *rest, collect_acc=True)
    assert uploaded() == 0
    assert np.array_equal(a["acc"], b["acc"])
    moved = allpos.copy()
    idx = np.nonzero(tag == 1)[0][[10, 5000, 200000]]
    moved[:, idx] += 1e-9
    c = lib.run(moved, tag, *rest, collect_acc=True)
    got = uploaded()
    assert 0 < got <= full
    if np.array_equal(c["perm"], a["perm"]):  # the tree kept its order: three chunks at most
        assert got <= 3 * 24 * 65536
    lib.L.devfree()
    d = lib.run(moved, tag, *rest, collect_acc=True)
    assert uploaded() == full
    assert np.array_equal(c["acc"], d["acc"])


@pytest.mark.parametrize("lib,mode,level,chunk", [
    ("dp", "pack", 2, 0), ("dp", "pack", 0, 0), ("dp", "task", 1, 3000), ("dp", "task", -1, 7919),
    ("act", "task", 2, 3000), ("act", "task", -1, 5000), ("act", "task", 255, 3000)])
def test_active_level_entry_points(gpu, lib, mode, level, chunk):
    """p2ppack_compute_act_gpu and task_compute_p2p_act_gpu
    (src/gpu_active.impl.h) through the reference's globals: the particles
    of the level receive the oracle's forces on the whole list (rows whose
    sink leaf has none of them are not computed), every other particle's acc
    is left as it was, bit for bit. The act library is the FP64 form built
    with ACT_OPT."""
    if not O.ref_available(f"libref_dropin_{lib}.so"):
        pytest.skip(f"libref_dropin_{lib}.so not built")
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    tl = W.prepare(pos, cfg)
    mass = 1.0 / pos.shape[1]
    g = np.random.default_rng(11)
    act = act_levels(tl, g)
    leaf_base = 5
    packs = lb_packs(tl, 4, leaf_base)
    ref, _ = O.p2p_lists(O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass), tl.pos,
                         tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    acc0 = g.normal(size=ref.shape) * np.linalg.norm(ref, axis=0)  # each particle's own scale
    got = O.ref_act_run(f"libref_dropin_{lib}.so", tl.pos, tl.leaf_ipart, tl.leaf_npart, leaf_base,
                        cfg.split_radius, cfg.eps, mass, packs, act, level, mode, chunk, acc0)
    upd = act_updates(act, level, lib == "act")
    if level not in (0, -1):
        assert 0 < upd.sum() < upd.size
    assert np.array_equal(got[:, ~upd], acc0[:, ~upd])
    rms, mx = rel_err(got - acc0, ref, upd & (tl.tag == 1))
    assert mx <= 1e-11 and rms <= 1e-12, (rms, mx)

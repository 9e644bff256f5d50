"""Device list walk (p2p_pass_submit_walk) against the serial host walk
(libphotons_lists.so, checked against the reference's src/fmm.c in
test_lists.py): the CSR rows equal the stable-sorted serial list entry for
entry, so the pass results equal the list path's bit for bit."""
import ctypes

import numpy as np
import pytest

from photons_p2p import abi, lists as L, workloads as W
from photons_p2p.p2p import DeviceWalkTree, P2PError, Session, params_for

pytestmark = pytest.mark.gpu


def case(name):
    if name == "c1":
        cfg, pos = W.c1_config(), W.c1_positions()
    elif name == "ref_dropin":
        cfg, pos = W.ref_dropin_config(), W.c1_positions()
    else:  # clustered 64^3: deeper, uneven tree
        side = 64
        cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=1 / (40 * side))
        pos = W.c2_positions(side)
    allpos, tag = W.with_ghosts(pos, cfg)
    tree = L.Tree(allpos, tag, cfg.maxleaf, cfg.box)
    tt, ts = tree.walk(cfg.cutoff_radius, cfg.open_angle)
    return cfg, tree, tt, ts


def sorted_rows(tree, tt, ts):
    order = np.argsort(tt, kind="stable")
    off = np.zeros(tree.nleaf + 1, np.int64)
    off[1:] = np.cumsum(np.bincount(tt, minlength=tree.nleaf))
    return off, ts[order]


@pytest.mark.parametrize("name", ["c1", "ref_dropin", "c2_64"])
@pytest.mark.parametrize("form", [abi.FORM_PLAIN_FP64, abi.FORM_SPLIT])
def test_walk_rows_and_pass_equal_list_path(gpu, name, form):
    cfg, tree, tt, ts = case(name)
    with tree:
        mass = 1.0 / int(tree.tag.sum())
        dev = DeviceWalkTree(tree, f"cuda:{gpu}")
        with Session(gpu, params_for(cfg, form, mass)) as s:
            want, _ = s.force_pass(tree.pos, tree.leaf_ipart, tree.leaf_npart, tt, ts)
            want_pairs, want_eval = s.pair_count(), s.evaluated_pairs()
            got, _, ntask = s.force_pass_walk(tree, dev, cfg.cutoff_radius, cfg.open_angle)
            assert ntask == len(tt)
            assert s.pair_count() == want_pairs and s.evaluated_pairs() == want_eval
            off, src = s.rows()
    want_off, want_src = sorted_rows(tree, tt, ts)
    assert np.array_equal(off, want_off)
    assert np.array_equal(src, want_src)
    # same rows in the same order: the same sums
    assert np.array_equal(got, want)


def test_walk_repeats_and_respects_mask_of_sinks(gpu):
    """Two walks in a row give the same rows; leaves without a local particle
    (ghost-only) get empty rows."""
    cfg, tree, tt, ts = case("c1")
    with tree:
        dev = DeviceWalkTree(tree, f"cuda:{gpu}")
        with Session(gpu, params_for(cfg, abi.FORM_SPLIT, 1.0 / int(tree.tag.sum()))) as s:
            a, _, _ = s.force_pass_walk(tree, dev, cfg.cutoff_radius, cfg.open_angle)
            off1, src1 = s.rows()
            b, _, _ = s.force_pass_walk(tree, dev, cfg.cutoff_radius, cfg.open_angle)
            off2, src2 = s.rows()
    assert np.array_equal(a, b) and np.array_equal(off1, off2) and np.array_equal(src1, src2)
    ghost_only = tree.leaf_active < 0
    assert ghost_only.any()
    assert np.all(np.diff(off1)[ghost_only] == 0)


def test_walk_rejects_a_malformed_tree_without_fault(gpu):
    """A child code pointing outside the node table is reported (P2P_ERR_ARG)
    before anything reads through it; the session stays usable."""
    import torch

    cfg, tree, tt, ts = case("c1")
    with tree:
        dev = DeviceWalkTree(tree, f"cuda:{gpu}")
        son = dev._t[0]
        bad = son.clone()
        bad[3, 1] = 2 * (son.shape[0] + 1000) + 1  # a node id past the table
        dev.struct.son = bad.data_ptr()
        with Session(gpu, params_for(cfg, abi.FORM_SPLIT, 1.0 / int(tree.tag.sum()))) as s:
            s.begin(tree.pos, tree.leaf_ipart, tree.leaf_npart)
            with pytest.raises(P2PError) as ei:
                s.submit_walk(dev, cfg.cutoff_radius, cfg.open_angle)
            assert ei.value.status == abi.P2P_ERR_ARG
            # closing the pass reports the same fault
            assert s.lib.p2p_pass_end(s.h, ctypes.byref(ctypes.c_double())) == abi.P2P_ERR_ARG
            torch.cuda.synchronize()
            # the same session runs a good walk afterwards
            dev.struct.son = son.data_ptr()
            got, _, ntask = s.force_pass_walk(tree, dev, cfg.cutoff_radius, cfg.open_angle)
            assert ntask == len(tt) and np.isfinite(got).all()

"""The device kd-tree (p2p_dtree_build) against the caller-side tree build
(host/p2p_lists.cpp, equal to the reference's build_kdtree / center_kdtree,
src/fmm.c:69-327, entry for entry): particle order, leaf ranges, active
flags, node child codes, first leaves, and node and leaf boxes equal bit for
bit; the P2P pass walked on the device tree equals the pass on the host
tree's lists.

Cases: the reference's drop-in settings (32^3 lattice, leaf cap 32), the
clustered mix at 64^3 and 128^3 (2.6M particles with ghosts: nodes above
2048 particles split level-wide), leaf caps 8 and 256, a box smaller than one
leaf (the root is still split), and many coincident particles (mean splits
that move one particle at a time)."""
import numpy as np
import pytest

from conftest import rel_err
from photons_p2p import abi, lists as L, workloads as W
from photons_p2p.p2p import DeviceTree, Session, params_for

pytestmark = pytest.mark.gpu


def _dev(a, torch, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def compare(pos, tag, maxleaf, boxsize):
    import torch

    dev = torch.device("cuda", 0)
    with L.Tree(pos, tag, maxleaf, boxsize) as host, Session(0) as s:
        son, first, center, width = host.nodes()
        with DeviceTree(s, _dev(pos, torch, dev), _dev(np.asarray(tag, np.int32), torch, dev), maxleaf,
                        boxsize) as t:
            d = t.download()
        assert t.nleaf == host.nleaf and t.nnode == son.shape[0]
        assert np.array_equal(d["perm"], host.perm)
        assert np.array_equal(d["pos"], host.pos)
        for k in ("leaf_ipart", "leaf_npart", "leaf_active", "leaf_center", "leaf_width"):
            assert np.array_equal(d[k], getattr(host, k)), k
        assert np.array_equal(d["son"], son)
        assert np.array_equal(d["node_first"], first)
        assert np.array_equal(d["node_center"], center)
        assert np.array_equal(d["node_width"], width)
    return t


@pytest.mark.parametrize("side,maxleaf", [(32, 32), (32, 8), (24, 256)])
def test_lattice_trees_equal_host(gpu, side, maxleaf):
    cfg = W.ref_dropin_config(side, 2 * side, maxleaf)
    pos = W.lattice_gaussian(side, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    compare(allpos, tag, maxleaf, cfg.box)


@pytest.mark.parametrize("side", [64, 128])
def test_clustered_trees_equal_host(gpu, side):
    cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=1.0 / (40 * side))
    allpos, tag = W.with_ghosts(W.c2_positions(side), cfg)
    compare(allpos, tag, cfg.maxleaf, cfg.box)


def test_box_smaller_than_a_leaf(gpu):
    pos = np.random.default_rng(3).random((3, 20))
    compare(pos, np.ones(20, np.int32), 32, 1.0)


def test_coincident_particles(gpu):
    g = np.random.default_rng(4)
    pos = g.random((3, 3000))
    pos[:, 500:2500] = 0.25  # 2000 particles at one point
    tag = (g.random(3000) < 0.7).astype(np.int32)
    compare(pos, tag, 16, 1.0)


def test_pass_on_device_tree_equals_host_lists(gpu):
    """Device tree -> device walk -> pair kernel, against the pass on the host
    tree's list (32^3 lattice, the reference's drop-in settings: clamp
    softening, open angle 0.4): the same pair count and forces (plain FP64
    bit for bit up to summation order; split form to its FP32 rounding)."""
    import torch

    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    tl = W.prepare(pos, cfg)
    mass = 1.0 / pos.shape[1]
    dev = torch.device("cuda", 0)
    for form in (abi.FORM_PLAIN_FP64, abi.FORM_SPLIT):
        with Session(0, params_for(cfg, form, mass)) as s:
            ref, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
            ref_pairs = s.pair_count()
            with DeviceTree(s, _dev(allpos, torch, dev), _dev(tag, torch, dev), cfg.maxleaf, cfg.box) as t:
                d_pos, d_perm, d_ip, d_np = t.device_arrays()
                lib = s.lib
                assert lib.p2p_pass_begin_device(s.h, t.npart, d_pos, None, t.nleaf, d_ip, d_np) == 0
                s._nleaf = t.nleaf
                s.npart = t.npart
                ntask = s.submit_walk(t, cfg.cutoff_radius, cfg.open_angle)
                s.end()
                got = np.zeros((3, t.npart))
                s.accumulate(got)
                assert ntask == tl.ntask and s.pair_count() == ref_pairs
                # the result in the input order of the positions
                d_out = torch.empty((3, t.npart), dtype=torch.float64, device=dev)
                t.unpermute(s.result_device(), d_out.data_ptr())
                s.lib.p2p_session_synchronize(s.h)
                back = d_out.cpu().numpy()
                assert np.array_equal(back[:, tl.perm], got)
        rms, mx = rel_err(got, ref, tl.tag == 1)
        assert mx <= (1e-13 if form == abi.FORM_PLAIN_FP64 else 1e-5), (form, rms, mx)


def test_rebuild_in_place_equals_fresh_builds(gpu):
    """p2p_dtree_rebuild: one tree object rebuilt over a sequence of inputs
    (larger, smaller, the first again, moved particles) equals the host tree
    of each input entry for entry, and a rebuild that fits the tree's arrays
    keeps them (no allocation)."""
    import torch

    dev = torch.device("cuda", 0)
    cases = []
    for side in (24, 32, 16):
        cfg = W.ref_dropin_config(side, 2 * side, 32)
        allpos, tag = W.with_ghosts(W.lattice_gaussian(side, 0.2, W.rng(side)), cfg)
        cases.append((allpos, tag, cfg))
    moved = cases[1][0] + W.rng(5).normal(scale=1e-4, size=cases[1][0].shape)
    cases += [cases[0], (moved, cases[1][1], cases[1][2])]
    with Session(0) as s:
        tree = None
        for i, (pos, tag, cfg) in enumerate(cases):
            p, t = _dev(pos, torch, dev), _dev(np.asarray(tag, np.int32), torch, dev)
            if tree is None:
                tree = DeviceTree(s, p, t, 32, cfg.box)
            else:
                before = tree.device_arrays()
                tree.rebuild(p, t, 32, cfg.box)
                if i in (2, 3):  # smaller than the largest input so far: the arrays are kept
                    assert tree.device_arrays() == before
            d = tree.download()
            with L.Tree(pos, tag, 32, cfg.box) as host:
                son, first, center, width = host.nodes()
                assert tree.npart == pos.shape[1] and tree.nleaf == host.nleaf and tree.nnode == son.shape[0]
                assert np.array_equal(d["perm"], host.perm) and np.array_equal(d["pos"], host.pos)
                for k in ("leaf_ipart", "leaf_npart", "leaf_active", "leaf_center", "leaf_width"):
                    assert np.array_equal(d[k], getattr(host, k)), (i, k)
                assert np.array_equal(d["son"], son) and np.array_equal(d["node_first"], first)
                assert np.array_equal(d["node_center"], center) and np.array_equal(d["node_width"], width)
        tree.close()

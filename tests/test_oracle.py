"""The CPU oracle, pinned to the reference's own arithmetic.

golden/ fixtures were produced by the reference's pair functions and walk
compiled for the host (tests/golden/make_golden.py); the live comparisons run
when oracle/_ref is present.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from photons_p2p import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
need_ref = pytest.mark.skipif(not O.ref_available("libref_pair.so"),
                              reason="oracle/_ref (reference pair functions) not built")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_known_pairs_bit_exact():
    g = load("pairs_known.npz")
    for k in range(g["r"].shape[0]):
        prm = O.params(int(g["soft_mode"][k]), float(g["soften"]), float(g["split_radius"]),
                       float(g["x_cut"][k]), 1.0)
        out = O.pair(prm, g["ii"][k], g["jj"][k])
        assert np.array_equal(out, g["out"][k]), (k, out, g["out"][k])


def test_self_pair_is_zero():
    for mode in (O.SOFT_CLAMP, O.SOFT_PLUMMER):
        prm = O.params(mode, 1e-3, 0.01, 2.8125, 1.0)
        assert np.all(O.pair(prm, [0.2, 0.3, 0.4], [0.2, 0.3, 0.4]) == 0.0)


def test_clamp_vs_plummer_inside_softening():
    """Clamp: force grows linearly with r inside eps (r/eps^3); Plummer:
    r/(r^2+eps^2)^(3/2). Both approach 1/r^2 far outside eps."""
    from math import erfc, exp, pi, sqrt

    eps, rs = 1e-3, 0.05
    for r in (1e-4, 5e-4):
        c = O.pair(O.params(O.SOFT_CLAMP, eps, rs, 2.8125, 1.0), [0, 0, 0], [r, 0, 0])[0]
        x = eps / (2 * rs)
        assert c == pytest.approx(r / eps ** 3 * (erfc(x) + 2 / sqrt(pi) * x * exp(-x * x)), rel=1e-12)
        p = O.pair(O.params(O.SOFT_PLUMMER, eps, rs, 2.8125, 1.0), [0, 0, 0], [r, 0, 0])[0]
        R = sqrt(r * r + eps * eps)
        x = R / (2 * rs)
        assert p == pytest.approx(r / R ** 3 * (erfc(x) + 2 / sqrt(pi) * x * exp(-x * x)), rel=1e-12)


def test_cutoff_edges():
    rs = 0.01
    prm = O.params(O.SOFT_PLUMMER, 1e-9, rs, 2.25, 1.0)
    just_in = O.pair(prm, [0, 0, 0], [2 * rs * 2.25 * (1 - 1e-9), 0, 0])[0]
    just_out = O.pair(prm, [0, 0, 0], [2 * rs * 2.25 * (1 + 1e-9), 0, 0])[0]
    assert just_in > 0 and just_out == 0.0


def test_golden_dropin12_lists_oracle_bit_exact():
    g = load("dropin12.npz")
    pos = g["input_pos"][:, g["perm"]]
    m, eps, rs = float(g["mass"]), float(g["soften"]), float(g["split_radius"])
    args = (pos, g["leaf_ipart"], g["leaf_npart"], g["task_t"], g["task_s"])
    acc, pairs = O.p2p_lists(O.params(O.SOFT_CLAMP, eps, rs, 2.8125, m), *args,
                             chunk=int(g["len_task"]))
    assert pairs == int(g["pairs"])
    assert np.array_equal(acc, g["acc_clamp_cut"])
    acc, _ = O.p2p_lists(O.params(O.SOFT_PLUMMER, eps, rs, 2.8125, m), *args, chunk=int(g["len_task"]))
    assert np.array_equal(acc, g["acc_plummer"])
    # the reference's production FP32 SPI arithmetic stays within 1e-3 of FP64
    loc = g["input_tag"][g["perm"]] == 1
    d = np.linalg.norm(g["acc_spi_fp32"] - g["acc_clamp_cut"], axis=0)[loc]
    n = np.linalg.norm(g["acc_clamp_cut"], axis=0)[loc]
    assert np.max(d / n) < 1e-3


def test_pair_count_matches_golden():
    g = load("dropin12.npz")
    assert O.pair_count(g["leaf_npart"], g["task_t"], g["task_s"]) == int(g["pairs"])


@need_ref
@pytest.mark.parametrize("variant,mode,xcut", [("dp_cut", 0, 2.8125), ("dp", 0, 0.0), ("dp", 1, 2.8125)])
def test_oracle_matches_reference_pair_functions_live(variant, mode, xcut):
    cfg = W.ref_dropin_config(16, 32, 32)
    pos = W.lattice_gaussian(16, 0.25, W.rng(21))
    tl = W.prepare(pos, cfg)
    m = 1.0 / pos.shape[1]
    args = (tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    ref, rp = O.ref_p2p_lists(variant, mode, cfg.eps, cfg.split_radius, m, *args, chunk=4321)
    got, gp = O.p2p_lists(O.params(mode, cfg.eps, cfg.split_radius, xcut, m), *args, chunk=4321)
    assert rp == gp
    assert np.array_equal(got, ref)


def test_direct_oracle_equals_complete_list_oracle():
    """With open angle 0 and x_cut * 2 r_s equal to the list cutoff, the
    list-based sum over ghosts equals the direct minimum-image sum."""
    cfg = W.scaled(W.c1_config(), n_side=12, mesh=24, eps=1.0 / (40 * 12))
    pos = W.lattice_gaussian(12, 0.2, W.rng(3))
    tl = W.prepare(pos, cfg)
    m = 1.0 / pos.shape[1]
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, m)
    acc, _ = O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    sinks = np.arange(pos.shape[1], dtype=np.int32)
    ref = O.direct(prm, pos, cfg.box, sinks)
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    got = acc[:, slot[sinks]]
    rel = np.linalg.norm(got - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert rel.max() < 1e-11


def test_masses_equal_scaled_mass():
    cfg = W.ref_dropin_config(10, 20, 16)
    pos = W.lattice_gaussian(10, 0.2, W.rng(4))
    tl = W.prepare(pos, cfg)
    prm = O.params(0, cfg.eps, cfg.split_radius, cfg.x_cut, 0.25)
    a, _ = O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    b, _ = O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s,
                       masses=np.full(tl.npart, 0.25))
    assert np.allclose(a, b, rtol=1e-13, atol=0)

"""The reference's own far field of the short-range force (p2m, m2m, the M2L
walk and m2l, l2l, l2p: src/operator.c, src/fmm.c:812-957 and :1188-1217),
compiled from its sources by oracle/build_ref.sh and driven by
oracle/ref_walk_harness.c (ref_harness_fmm): the oracle of the GPU far field.

Known answers about the reference itself, checked here on the CPU:
  * every leaf's monopole is its particles' mass;
  * its m2l tests `abs(r2) <= 1e-15` with the integer abs() of <stdlib.h>
    (src/operator.c:340-344), so in a unit box, where every M2L distance is
    below 1, the M2L tasks are made but the far field is exactly zero; in a
    box of 1000 the same particles give a non-zero far field;
  * with the drop-in settings on a lattice (r_s = 1.25 cells, cutoff 4.5
    r_s, open angle 0.4) no pair of boxes within the cutoff is well
    separated: no M2L task at all."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from photons_p2p import workloads as W

pytestmark = pytest.mark.skipif(not O.ref_available("libref_walk.so"),
                                reason="oracle/_ref walk harness not built")


def quiet(fn):
    """Runs fn with the process's stdout closed (the reference's m2l prints a
    line for every task it skips)."""
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return fn()
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)


def clustered(side, box):
    cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=box / (40 * side), open_angle=0.4, box=box)
    pos = W.c2_positions(side) * box
    allpos, tag = W.with_ghosts(pos, cfg)
    return cfg, allpos, tag, 1.0 / pos.shape[1]


def ref_fmm(cfg, allpos, tag, mass):
    return quiet(lambda: O.RefWalk("libref_walk.so").fmm(allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius,
                                                         cfg.cutoff_radius, cfg.eps, mass, cfg.open_angle))


def test_unit_box_far_field_is_zero_in_the_reference():
    cfg, allpos, tag, mass = clustered(64, 1.0)
    r = ref_fmm(cfg, allpos, tag, mass)
    assert np.allclose(r["leaf_M"][:, 0], r["leaf_npart"] * mass, rtol=1e-14, atol=0)
    big = clustered(64, 1000.0)
    rb = ref_fmm(*big)
    assert rb["n_m2l"] > 0 and np.abs(rb["acc"]).max() > 0
    assert r["n_m2l"] == rb["n_m2l"]
    assert not np.any(r["acc"])


def test_lattice_drop_in_settings_make_no_m2l():
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    r = ref_fmm(cfg, allpos, tag, 1.0 / pos.shape[1])
    assert r["n_m2l"] == 0 and not np.any(r["acc"])

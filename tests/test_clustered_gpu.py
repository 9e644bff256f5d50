"""The FP32 forms and the plain FP64 form on the clustered mix (60% uniform,
40% in NFW halos: the 256^3 configuration's draw at 128^3, 2.1M particles)
against the FP64 direct oracle on sampled local sinks.

Bars (per-particle relative force error |a - a_direct| / |a_direct|):
  chosen FP32/FP64-split form, every packed lane mapping: rms <= 1e-5, max <= 1e-3
  Kahan-compensated FP32 form:                            rms <= 1e-5, max <= 1e-3
  plain FP64 form:                                        max <= 1e-10
The lists are complete within the cutoff (open angle 0, x_cut = list cutoff),
so the pass equals the direct minimum-image sum of the truncated kernel; the
direct sum (oracle/p2p_oracle.c, oracle_direct) is independent of the tree.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O
from photons_p2p import abi, workloads as W
from photons_p2p.p2p import Session, params_for

pytestmark = pytest.mark.gpu

SIDE = 128
NSINK = 3000


@pytest.fixture(scope="module")
def clustered():
    cfg = W.scaled(W.c2_config(), name="c2_clustered_128^3", n_side=SIDE, mesh=SIDE, eps=1.0 / (40 * SIDE))
    pos = W.c2_positions(SIDE)
    tl = W.prepare(pos, cfg)
    n = pos.shape[1]
    mass = 1.0 / n
    sinks = W.rng(88).choice(n, NSINK, replace=False).astype(np.int32)
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)
    ref = O.direct(prm, pos, cfg.box, sinks)
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    return cfg, tl, mass, slot[sinks], ref


def run(cfg, tl, mass, form, variant=0):
    prm = params_for(cfg, form, mass)
    prm.kernel_variant = variant
    with Session(0, prm) as s:
        acc, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
        assert s.pair_count() == tl.pair_count()
        evaluated = s.evaluated_pairs()
    return acc, evaluated


def test_plain_vs_direct(gpu, clustered):
    cfg, tl, mass, rows, ref = clustered
    acc, _ = run(cfg, tl, mass, abi.FORM_PLAIN_FP64)
    rms, mx = rel_err(acc[:, rows], ref)
    assert mx <= 1e-10, (rms, mx)


@pytest.mark.parametrize("variant", [abi.VARIANT_SOURCE_LANES_X2, abi.VARIANT_SOURCE_LANES_X2_S16,
                                     abi.VARIANT_SINK_LANES_X2, abi.VARIANT_SINK_REGS])
def test_split_vs_direct(gpu, clustered, variant):
    cfg, tl, mass, rows, ref = clustered
    acc, evaluated = run(cfg, tl, mass, abi.FORM_SPLIT, variant)
    rms, mx = rel_err(acc[:, rows], ref)
    assert rms <= 1e-5 and mx <= 1e-3, (rms, mx)
    assert 0 < evaluated < tl.pair_count()


@pytest.mark.parametrize("variant", [abi.VARIANT_SOURCE_LANES_X2, abi.VARIANT_SINK_REGS])
def test_kahan_vs_direct(gpu, clustered, variant):
    cfg, tl, mass, rows, ref = clustered
    acc, _ = run(cfg, tl, mass, abi.FORM_KAHAN_FP32, variant)
    rms, mx = rel_err(acc[:, rows], ref)
    assert rms <= 1e-5 and mx <= 1e-3, (rms, mx)


def test_sink_regs_drops_more_pairs_than_entry_skip(gpu, clustered):
    """The sink-register kernel drops single source particles beyond the
    cutoff from a whole sink slice: it evaluates fewer pairs than the
    entry-level skip of the source-lane kernel, and the forces agree to the
    FP32 forms' rounding."""
    cfg, tl, mass = clustered[:3]
    a, ev_x2 = run(cfg, tl, mass, abi.FORM_SPLIT, abi.VARIANT_SOURCE_LANES_X2)
    b, ev_sr = run(cfg, tl, mass, abi.FORM_SPLIT, abi.VARIANT_SINK_REGS)
    assert ev_sr < ev_x2
    rms, mx = rel_err(b, a, tl.tag == 1)
    assert rms <= 1e-6 and mx <= 1e-4, (rms, mx)

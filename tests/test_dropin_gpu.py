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

"""Serving: an ensemble of small periodic boxes through p2p_server.

Each box's result must be the same alone and in the mix: a box computed in a
launch of its own and the same box packed with others (and sharing the GPU
with a second in-flight launch) agree to 1e-12 relative (they are computed by
the same rows in the same order; equality is expected). Results also match
the single-pass session path on the same box (FP64 form: 1e-12; FP32 forms:
rms 1e-6, max 1e-4, the FP32 rounding of box vs. kernel units) and the FP64
direct oracle within the chosen form's bound.
"""
import copy
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O
from photons_p2p import abi, p2p, serve, workloads as W
from photons_p2p.p2p import P2PError

MIX_TOL = 1e-12
NBOX = 10


@pytest.fixture(scope="module")
def ensemble():
    boxes = W.c4_boxes(nbox=NBOX, seed_offset=11, n_range=(16, 24))
    lists = [serve.box_lists(b) for b in boxes]
    return boxes, lists


def n_local(lists):
    return int(lists.tag.sum())


def locals_in_order(tl, acc):
    """Tree-order (3, npart) accelerations -> the local particles in their
    original order, the layout a server request returns."""
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    return acc[:, slot[:n_local(tl)]]


def make_server(form, ensemble, **kw):
    boxes, lists = ensemble
    kw.setdefault("hbm_bytes", 2 << 30)
    eps_over_rs = boxes[0].cfg.eps / boxes[0].cfg.split_radius
    srv = serve.Server(serve.serving_shape(form, eps_over_rs), **kw)
    for b, tl in zip(boxes, lists):
        srv.add_box(tl, 0.5 / b.cfg.split_radius, 1.0 / n_local(tl))
    return srv


def alone(srv, k):
    out, _ = srv.wait(srv.submit(k))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("form", [abi.FORM_SPLIT, abi.FORM_PLAIN_FP64])
def test_same_alone_and_in_the_mix(gpu, ensemble, form):
    with make_server(form, ensemble, device=gpu, slots=2) as srv:
        ref = [alone(srv, k) for k in range(NBOX)]
        s0 = srv.stats()
        order = np.random.default_rng(3).permutation(np.tile(np.arange(NBOX), 3))
        tickets = [(srv.submit(int(k)), int(k)) for k in order]
        for t, k in tickets:
            out, lat = srv.wait(t)
            assert lat > 0
            assert rel_err(out, ref[k])[1] <= MIX_TOL
        s1 = srv.stats()
        launches = s1["launches"] - s0["launches"]
        assert s1["requests_done"] - s0["requests_done"] == len(order)
        assert launches < len(order), "requests were not packed"
        assert s1["builds"] == NBOX and s1["evictions"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("form", [abi.FORM_SPLIT, abi.FORM_PLAIN_FP64, abi.FORM_KAHAN_FP32])
def test_server_matches_session(gpu, ensemble, form):
    boxes, lists = ensemble
    with make_server(form, ensemble, device=gpu) as srv:
        tickets = [srv.submit(k) for k in range(NBOX)]
        got = [srv.wait(t)[0] for t in tickets]
    with p2p.Session(gpu) as s:
        for k, (b, tl) in enumerate(zip(boxes, lists)):
            s.set_params(p2p.params_for(b.cfg, form, 1.0 / n_local(tl)))
            want, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
            assert got[k].shape == (3, n_local(tl))
            rms, mx = rel_err(got[k], locals_in_order(tl, want))
            if form == abi.FORM_PLAIN_FP64:
                assert mx <= 1e-12, (k, mx)
            else:
                assert rms <= 1e-6 and mx <= 1e-4, (k, rms, mx)


@pytest.mark.gpu
def test_server_vs_direct_oracle(gpu, ensemble):
    boxes, lists = ensemble
    k = 3
    b, tl = boxes[k], lists[k]
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu) as srv:
        got = alone(srv, k)
    nloc = n_local(tl)
    prm = O.params(b.cfg.soft_mode, b.cfg.eps, b.cfg.split_radius, b.cfg.x_cut, 1.0 / nloc)
    sinks = np.arange(0, nloc, 7)
    ref = O.direct(prm, b.pos, b.cfg.box, sinks)
    rms, mx = rel_err(got[:, sinks], ref)
    assert rms <= 1e-5 and mx <= 1e-3


@pytest.mark.gpu
def test_admission_by_footprint_and_eviction(gpu, ensemble):
    boxes, lists = ensemble
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu) as big:
        ref = [alone(big, k) for k in range(NBOX)]
        sizes = [big.box_bytes(k) for k in range(NBOX)]
    rpp = max(tl.ntask / tl.npart for tl in lists)
    ppl = min(tl.npart / tl.nleaf for tl in lists)
    budget = int(3.2 * max(sizes))
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu, slots=2, hbm_bytes=budget,
                     rows_per_particle=rpp, particles_per_leaf=ppl) as srv:
        order = np.tile(np.arange(NBOX), 2)
        tickets = [(srv.submit(int(k)), int(k)) for k in order]
        for t, k in tickets:
            out, _ = srv.wait(t)
            assert rel_err(out, ref[k])[1] <= MIX_TOL
        st = srv.stats()
        assert st["evictions"] > 0 and st["builds"] >= NBOX
        assert st["resident_boxes"] < NBOX
        assert st["resident_bytes"] <= st["capacity_bytes"]
        # evicted boxes are rebuilt when asked for again, with the same result
        for k in range(NBOX):
            assert rel_err(alone(srv, k), ref[k])[1] <= MIX_TOL
        assert srv.stats()["builds"] > st["builds"]


@pytest.mark.gpu
def test_preload_releases_host_arrays(gpu, ensemble):
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu) as srv:
        want = alone(srv, 2)
        srv.preload(4)
        assert srv.boxes[4].keep == ()
        got4 = alone(srv, 4)
        assert np.isfinite(got4).all()
        assert rel_err(alone(srv, 2), want)[1] <= MIX_TOL
        assert srv.stats()["resident_boxes"] >= 2


@pytest.mark.gpu
def test_all_particles_in_slot_order(gpu, ensemble):
    """Without a result map a request returns every particle in tree order,
    equal to the session pass."""
    boxes, lists = ensemble
    k = 1
    b, tl = boxes[k], lists[k]
    eps_over_rs = b.cfg.eps / b.cfg.split_radius
    with serve.Server(serve.serving_shape(abi.FORM_PLAIN_FP64, eps_over_rs), device=gpu,
                      hbm_bytes=1 << 30) as srv:
        srv.add_box(tl, 0.5 / b.cfg.split_radius, 1.0 / n_local(tl), locals_only=False)
        got = alone(srv, 0)
    with p2p.Session(gpu, p2p.params_for(b.cfg, abi.FORM_PLAIN_FP64, 1.0 / n_local(tl))) as s:
        want, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    assert got.shape == want.shape
    assert rel_err(got, want)[1] <= 1e-12


@pytest.mark.gpu
def test_poisson_driver(gpu, ensemble):
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu, slots=2) as srv:
        r = serve.run_poisson(srv, rate_hz=2000.0, n_requests=60, seed=1)
    assert r["requests"] == 60 and 0 < r["p50_ms"] <= r["p99_ms"]
    assert r["launches"] >= 1 and r["pairs_per_s"] > 0


@pytest.mark.gpu
def test_server_errors(gpu, ensemble):
    boxes, lists = ensemble
    tl = lists[0]
    with make_server(abi.FORM_SPLIT, ensemble, device=gpu, hbm_bytes=64 << 20) as srv:
        lib = srv.lib
        # result buffer must be page-locked
        out = np.zeros(3 * tl.npart)
        t = ctypes.c_int64()
        st = lib.p2p_server_submit(srv.h, 0, out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(t))
        assert st == abi.P2P_ERR_ARG
        # leaf range outside the box
        tl_bad = copy.copy(tl)
        tl_bad.leaf_ipart = tl.leaf_ipart.copy()
        tl_bad.leaf_ipart[-1] = tl.npart
        with pytest.raises(P2PError) as ei:
            srv.add_box(tl_bad, 0.5 / boxes[0].cfg.split_radius, 1.0)
        assert ei.value.status == abi.P2P_ERR_RANGE
        # unknown box
        assert lib.p2p_server_preload(srv.h, 99) == abi.P2P_ERR_ARG


@pytest.mark.gpu
def test_box_larger_than_arena(gpu, ensemble):
    boxes, lists = ensemble
    k = int(np.argmax([tl.npart for tl in lists]))
    eps_over_rs = boxes[0].cfg.eps / boxes[0].cfg.split_radius
    small = max(tl.npart for tl in lists) * 60  # bytes: too few for the largest box's lists
    with serve.Server(serve.serving_shape(abi.FORM_SPLIT, eps_over_rs), device=gpu,
                      hbm_bytes=small, rows_per_particle=1.0) as srv:
        with pytest.raises(P2PError) as ei:
            srv.add_box(lists[k], 0.5 / boxes[k].cfg.split_radius, 1.0)
        assert ei.value.status == abi.P2P_ERR_CAPACITY


@pytest.mark.gpu
def test_batching_window_packs_and_keeps_results(gpu, ensemble):
    """With a batching window, requests submitted one after another within
    it share one launch, each result equals the box computed alone, a lone
    request waits out the window, and min_pack_pairs launches a pack at once."""
    import time

    with make_server(abi.FORM_SPLIT, ensemble, device=gpu, slots=1) as srv:
        ref = [alone(srv, k) for k in range(4)]
        srv.set_batching(400.0)
        s0 = srv.stats()
        tickets = []
        for k in range(4):
            tickets.append(srv.submit(k))
            time.sleep(0.01)
        for k, t in enumerate(tickets):
            out, lat = srv.wait(t)
            assert rel_err(out, ref[k])[1] <= MIX_TOL
        s1 = srv.stats()
        assert s1["launches"] - s0["launches"] == 1
        assert s1["boxes_launched"] - s0["boxes_launched"] == 4
        # a lone request of a resident box waits out the window (a box not yet
        # built has no pair count and launches at once)
        _, lat = srv.wait(srv.submit(0))
        assert lat >= 0.4
        # one request of any size reaches a 1-pair threshold: no waiting
        srv.set_batching(5000.0, 1.0)
        _, lat = srv.wait(srv.submit(1))
        assert lat < 2.0
        srv.set_batching(0.0)
        with pytest.raises(P2PError):
            srv.set_batching(-1.0)

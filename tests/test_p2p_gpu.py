"""Parity of the CUDA P2P pass against the CPU oracle (through the C ABI).

Tolerances (per-particle relative force error |a - a_ref| / |a_ref| over local
particles):
  plain FP64 form vs the reference-order oracle:   max <= 1e-12
  split FP32/FP64 form vs the plain FP64 form:     rms <= 1e-5, max <= 1e-3
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O
from photons_p2p import abi, workloads as W
from photons_p2p.p2p import P2PError, Session, make_params, params_for

pytestmark = pytest.mark.gpu

PLAIN_MAX = 1e-12
SPLIT_RMS = 1e-5
SPLIT_MAX = 1e-3


@pytest.fixture(scope="module")
def dropin32():
    """32^3 particles with the reference's own pass settings (clamp softening,
    GPUCUTOFF, open angle 0.4, r_s 1.25 cells)."""
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    tl = W.prepare(pos, cfg)
    return cfg, tl, 1.0 / pos.shape[1]


@pytest.fixture(scope="module")
def c1():
    cfg = W.c1_config()
    pos = W.c1_positions()
    tl = W.prepare(pos, cfg)
    return cfg, tl, 1.0 / pos.shape[1], pos


def oracle_acc(cfg, tl, mass, chunk=0, masses=None):
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)
    acc, pairs = O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s,
                             masses=masses, chunk=chunk)
    return acc, pairs


def gpu_acc(cfg, tl, mass, form, chunk=0, masses=None, **launch):
    with Session(0) as s:
        prm = params_for(cfg, form, mass)
        for k, v in launch.items():
            setattr(prm, k, v)
        s.set_params(prm)
        acc, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s,
                              masses=masses, chunk=chunk)
        return acc, s.pair_count()


def test_plain_matches_oracle_dropin32(gpu, dropin32):
    cfg, tl, m = dropin32
    ref, pairs = oracle_acc(cfg, tl, m, chunk=40000)
    got, gpairs = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64, chunk=40000)
    assert gpairs == pairs == tl.pair_count()
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert mx <= PLAIN_MAX, (rms, mx)


def test_plain_matches_oracle_c1_plummer(gpu, c1):
    cfg, tl, m, _ = c1
    ref, _ = oracle_acc(cfg, tl, m)
    got, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64)
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert mx <= PLAIN_MAX, (rms, mx)


VARIANTS = [abi.VARIANT_SINK_LANES, abi.VARIANT_SOURCE_LANES, abi.VARIANT_SOURCE_LANES_X2,
            abi.VARIANT_SOURCE_LANES_X2_S16, abi.VARIANT_SINK_LANES_X2, abi.VARIANT_SINK_REGS,
            abi.VARIANT_SINK_REGS8]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("which", ["dropin32", "c1"])
def test_split_vs_plain(gpu, which, variant, request):
    cfg, tl, m = request.getfixturevalue(which)[:3]
    plain, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64)
    split, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, kernel_variant=variant)
    rms, mx = rel_err(split, plain, tl.tag == 1)
    assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (rms, mx)


@pytest.mark.parametrize("form", [abi.FORM_KAHAN_FP32, abi.FORM_NAIVE_FP32])
@pytest.mark.parametrize("variant", VARIANTS)
def test_fp32_study_forms(gpu, c1, form, variant):
    """The precision-study forms stay close to FP64 on a unit box (their
    differences show at large coordinates, see the precision stress test)."""
    cfg, tl, m = c1[:3]
    plain, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64)
    got, _ = gpu_acc(cfg, tl, m, form, kernel_variant=variant)
    rms, mx = rel_err(got, plain, tl.tag == 1)
    assert rms <= 1e-4 and mx <= 1e-2, (rms, mx)


def test_plain_equals_direct_oracle_c1(gpu, c1):
    """Complete lists (open angle 0, x_cut = list cutoff) make the pass equal
    to the FP64 direct minimum-image sum, independent of the tree."""
    cfg, tl, m, pos = c1
    got, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64)
    g = W.rng(77)
    n = pos.shape[1]
    sinks = g.choice(n, 2000, replace=False).astype(np.int32)
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, m)
    ref = O.direct(prm, pos, cfg.box, sinks)
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    rms, mx = rel_err(got[:, slot[sinks]], ref)
    assert mx <= 1e-10, (rms, mx)


def test_masses_per_particle(gpu, dropin32):
    cfg, tl, m = dropin32
    g = W.rng(5)
    masses = g.uniform(0.5, 1.5, tl.npart) * m
    ref, _ = oracle_acc(cfg, tl, m, masses=masses)
    got, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64, masses=masses)
    assert rel_err(got, ref, tl.tag == 1)[1] <= PLAIN_MAX
    split, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, masses=masses)
    rms, mx = rel_err(split, got, tl.tag == 1)
    assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (rms, mx)


@pytest.mark.parametrize("form", [abi.FORM_PLAIN_FP64, abi.FORM_SPLIT])
def test_chunked_submits_equal_single(gpu, dropin32, form):
    cfg, tl, m = dropin32
    one, _ = gpu_acc(cfg, tl, m, form)
    many, _ = gpu_acc(cfg, tl, m, form, chunk=7777)
    rms, mx = rel_err(many, one, tl.tag == 1)
    # chunks regroup each row's sources, so FP32 partial sums differ in their
    # last bits for the split form; FP64 sums only reorder
    if form == abi.FORM_PLAIN_FP64:
        assert mx <= 1e-13, (rms, mx)
    else:
        assert rms <= 1e-6 and mx <= 1e-4, (rms, mx)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("warps,stage,bps", [(1, 32, 0), (2, 64, 1), (4, 512, 0)])
def test_launch_shapes(gpu, dropin32, warps, stage, bps, variant):
    cfg, tl, m = dropin32
    ref, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, kernel_variant=abi.VARIANT_SINK_LANES)
    got, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, warps_per_block=warps, stage_sources=stage,
                     blocks_per_sm=bps, kernel_variant=variant)
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert mx <= 1e-5, (rms, mx)


@pytest.mark.parametrize("variant", [abi.VARIANT_SINK_REGS, abi.VARIANT_SINK_REGS8])
@pytest.mark.parametrize("leaf_warps", [2, 4])
@pytest.mark.parametrize("maxleaf", [32, 64])
def test_warps_per_leaf(gpu, variant, leaf_warps, maxleaf):
    """A sink leaf's row spread over 2 or 4 warps (each a contiguous share of
    its entries, partial forces added with atomics), with 32- and 64-sink
    tiles, at leaf caps 32 and 64: the same forces as one warp per leaf (to
    the atomics' reassociation) and within the FP32 form's bars of the FP64
    form; pair counts unchanged."""
    cfg = W.ref_dropin_config(32, 64, maxleaf)
    pos = W.lattice_gaussian(32, 0.2, W.rng(5))
    tl = W.prepare(pos, cfg)
    m = 1.0 / pos.shape[1]
    one, p1 = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, kernel_variant=abi.VARIANT_SINK_REGS)
    got, p2 = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, kernel_variant=variant, warps_per_leaf=leaf_warps)
    assert p1 == p2
    rms, mx = rel_err(got, one, tl.tag == 1)
    assert mx <= 1e-5, (rms, mx)
    plain, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64)
    rms, mx = rel_err(got, plain, tl.tag == 1)
    assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (rms, mx)


def test_warps_per_leaf_rejects_other_values(gpu):
    cfg = W.ref_dropin_config(32, 64, 32)
    with Session(0) as s:
        prm = params_for(cfg, abi.FORM_SPLIT, 1.0)
        prm.warps_per_leaf = 3
        with pytest.raises(P2PError):
            s.set_params(prm)


def test_big_leaves_maxleaf256(gpu):
    """The reference's default MAXLEAF = 256: sink leaves span several warp
    slices and source leaves overflow a small staging buffer."""
    cfg = W.ref_dropin_config(24, 32, 256)
    pos = W.lattice_gaussian(24, 0.3, W.rng(11))
    tl = W.prepare(pos, cfg)
    assert tl.leaf_npart.max() > 64
    m = 1.0 / pos.shape[1]
    ref, _ = oracle_acc(cfg, tl, m)
    got, _ = gpu_acc(cfg, tl, m, abi.FORM_PLAIN_FP64, stage_sources=64)
    assert rel_err(got, ref, tl.tag == 1)[1] <= PLAIN_MAX
    for variant in VARIANTS:
        split, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT, stage_sources=64, kernel_variant=variant)
        rms, mx = rel_err(split, got, tl.tag == 1)
        assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (variant, rms, mx)


def test_empty_list_and_zero_particles(gpu):
    with Session(0) as s:
        s.set_params(make_params())
        pos = np.random.default_rng(0).random((3, 10))
        acc, _ = s.force_pass(pos, [0], [10], np.zeros(0, np.int32), np.zeros(0, np.int32))
        assert np.all(acc == 0)
        assert s.pair_count() == 0
        acc, _ = s.force_pass(np.zeros((3, 0)), [], [], np.zeros(0, np.int32), np.zeros(0, np.int32))
        assert acc.shape == (3, 0)


def test_two_body_known_answer(gpu):
    """Two particles at separation r, one leaf each; compare to the closed
    form m * g(r/(2 r_s)) / r^2 and to the oracle's pair function."""
    from math import erfc, exp, pi, sqrt

    rs, eps, m = 0.01, 1e-4, 0.5
    for r in (0.003, 0.02, 0.0449, 0.0451):
        pos = np.array([[0.1, 0.1 + r], [0.2, 0.2], [0.3, 0.3]])
        for form in (abi.FORM_PLAIN_FP64, abi.FORM_SPLIT):
            with Session(0, make_params(form=form, soft_mode=abi.SOFT_PLUMMER, soften=eps,
                                        split_radius=rs, x_cut=2.25, mass=m)) as s:
                acc, _ = s.force_pass(pos, [0, 1], [1, 1], np.array([0, 0, 1, 1], np.int32),
                                      np.array([0, 1, 0, 1], np.int32))
            R = sqrt(r * r + eps * eps)
            x = R / (2 * rs)
            want = 0.0 if x > 2.25 else m * r * (erfc(x) + 2 / sqrt(pi) * x * exp(-x * x)) / R ** 3
            tol = 1e-13 if form == abi.FORM_PLAIN_FP64 else 1e-5
            if want == 0.0:
                assert acc[0, 0] == 0.0 and acc[0, 1] == 0.0
            else:
                assert abs(acc[0, 0] - want) <= tol * want
                assert abs(acc[0, 1] + want) <= tol * want
            assert np.all(acc[1:, :] == 0.0)


def test_out_of_range_ids_report_without_fault(gpu):
    """Bad leaf ids in a list are skipped on the device and reported."""
    pos = np.random.default_rng(1).random((3, 40))
    with Session(0, make_params()) as s:
        s.begin(pos, [0, 20], [20, 20])
        s.submit(np.array([0, 1, 7, -3], np.int32), np.array([1, 0, 0, 1], np.int32))
        with pytest.raises(P2PError) as e:
            s.end()
        assert e.value.status == abi.P2P_ERR_RANGE
    with Session(0, make_params()) as s:
        with pytest.raises(P2PError) as e:
            s.begin(pos, [0, 30], [20, 20])  # second leaf runs past npart
        assert e.value.status == abi.P2P_ERR_RANGE


def test_protocol_errors(gpu):
    with Session(0, make_params()) as s:
        with pytest.raises(P2PError) as e:
            s.submit(np.zeros(1, np.int32), np.zeros(1, np.int32))
        assert e.value.status == abi.P2P_ERR_STATE
        with pytest.raises(P2PError) as e:
            s.set_params(make_params(soften=0.0))
        assert e.value.status == abi.P2P_ERR_ARG


def test_deterministic_repeat(gpu, dropin32):
    cfg, tl, m = dropin32
    a, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT)
    b, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT)
    rms, mx = rel_err(a, b, tl.tag == 1)
    assert mx <= 1e-12, (rms, mx)


def test_run_device_graph_matches_host_path(gpu, dropin32):
    torch = pytest.importorskip("torch")
    cfg, tl, m = dropin32
    host, _ = gpu_acc(cfg, tl, m, abi.FORM_SPLIT)
    dev = torch.device("cuda", 0)
    d_pos = torch.from_numpy(np.ascontiguousarray(tl.pos)).to(dev)
    d_ip = torch.from_numpy(tl.leaf_ipart).to(dev)
    d_np = torch.from_numpy(tl.leaf_npart).to(dev)
    d_t = torch.from_numpy(tl.task_t).to(dev)
    d_s = torch.from_numpy(tl.task_s).to(dev)
    torch.cuda.synchronize()
    with Session(0, params_for(cfg, abi.FORM_SPLIT, m)) as s:
        for _ in range(3):  # first call captures the graph, the others replay it
            s.run_device(tl.npart, d_pos.data_ptr(), tl.nleaf, d_ip.data_ptr(), d_np.data_ptr(),
                         tl.ntask, d_t.data_ptr(), d_s.data_ptr())
            s.end()
            out = np.zeros((3, tl.npart))
            s.accumulate(out)
            rms, mx = rel_err(out, host, tl.tag == 1)
            assert mx <= 1e-12, (rms, mx)
            assert s.pair_count() == tl.pair_count()


@pytest.mark.parametrize("variant", [abi.VARIANT_SOURCE_LANES_X2, abi.VARIANT_SINK_LANES_X2,
                                     abi.VARIANT_SINK_REGS])
def test_skipped_entries_change_nothing(gpu, c1, variant):
    """The packed kernels skip list entries whose particles lie wholly beyond
    the cutoff. The skipped pairs are counted (evaluated <= listed, and some
    are skipped on this lattice), and the forces agree with the scalar
    source-lane kernel, which evaluates every listed pair, to FP32 rounding."""
    cfg, tl, mass, _ = c1
    with Session(gpu) as s:
        prm = params_for(cfg, abi.FORM_SPLIT, mass)
        prm.kernel_variant = variant
        s.set_params(prm)
        got, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
        listed, evaluated = s.pair_count(), s.evaluated_pairs()
        prm.kernel_variant = abi.VARIANT_SOURCE_LANES
        s.set_params(prm)
        ref, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
        assert s.evaluated_pairs() == s.pair_count() == listed == tl.pair_count()
    assert 0 < evaluated < listed
    # the scalar kernel decides cutoff-band pairs in FP32, so single particles
    # may differ by up to the two forms' bounds together
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert rms <= 1e-6 and mx <= 2e-3


def test_pipelined_host_submit_matches_resident_pass(gpu):
    """A host list longer than 2^26 entries is uploaded in pieces on a copy
    stream while earlier pieces compute; the result equals the resident
    single-chunk pass up to the FP32 grouping of the pieces' partial sums."""
    import torch

    side = 128
    cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=1 / (40 * side), maxleaf=16)
    tl = W.prepare(W.c2_positions(side), cfg)
    assert tl.ntask > 2 ** 26
    mass = 1.0 / int(tl.tag.sum())
    dev = torch.device("cuda", gpu)
    d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)]
    with Session(gpu, params_for(cfg, abi.FORM_SPLIT, mass)) as s:
        got, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
        assert s.pair_count() == tl.pair_count()
        s.run_device(tl.npart, d[0].data_ptr(), tl.nleaf, d[1].data_ptr(), d[2].data_ptr(), tl.ntask,
                     d[3].data_ptr(), d[4].data_ptr())
        s.end()
        ref = np.zeros((3, tl.npart))
        s.accumulate(ref)
    rms, mx = rel_err(got, ref, tl.tag == 1)
    assert rms <= 1e-6 and mx <= 1e-4, (rms, mx)


def test_plain_matches_oracle_with_ten_bit_radix(gpu):
    """More than 2^16 leaves: the CSR build sorts with two 10-bit radix digits.
    The rows of every 97th sink leaf of a 128^3 clustered pass, through the
    plain FP64 form, against the reference-order oracle."""
    side = 128
    cfg = W.scaled(W.c2_config(), n_side=side, mesh=side, eps=1 / (40 * side))
    tl = W.prepare(W.c2_positions(side), cfg)
    assert 2 ** 16 <= tl.nleaf < 2 ** 20
    keep = (tl.task_t % 97) == 0
    tt, ts = tl.task_t[keep], tl.task_s[keep]
    mass = 1.0 / int(tl.tag.sum())
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)
    ref, pairs = O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tt, ts)
    with Session(gpu, params_for(cfg, abi.FORM_PLAIN_FP64, mass)) as s:
        got, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tt, ts)
        assert s.pair_count() == pairs
    sinks = np.zeros(tl.npart, bool)
    for l in np.unique(tt):
        sinks[tl.leaf_ipart[l]:tl.leaf_ipart[l] + tl.leaf_npart[l]] = True
    rms, mx = rel_err(got, ref, sinks)
    assert mx <= PLAIN_MAX, mx


def test_throughput_probes(gpu):
    """The FP32 and FP64 throughput probes whose results are the rooflines'
    peaks: positive, below the B200's nominal figures at 1965 MHz (74.4 FP32,
    37.2 FP64 TFLOP/s) with margin, FP64 slower than FP32."""
    with Session(gpu) as s:
        f32 = s.measure_fp32_peak()
        f64 = s.measure_fp64_peak()
    assert 10.0 < f32 < 80.0, f32
    assert 5.0 < f64 < 42.0, f64
    assert f64 < f32


def test_autotune_on_the_gpu(gpu, dropin32, tmp_path):
    """tune() times the candidates on a row sample, keeps a shape whose pass
    matches the FP64 form within the split form's bars, and a second call
    with the same histogram is answered from the JSON cache."""
    from photons_p2p import autotune

    cfg, tl, mass = dropin32
    cache = str(tmp_path / "tune.json")
    prm, rec = autotune.tune(cfg, tl, abi.FORM_SPLIT, mass, sample_pairs=tl.pair_count() / 4, cache_path=cache,
                             min_rows=64)
    assert not rec["cached"] and rec["candidates"] >= len(autotune.CANDIDATES) // 2
    assert rec["sample_pairs"] < tl.pair_count()
    assert (prm.kernel_variant, prm.stage_sources, prm.warps_per_block, prm.warps_per_leaf) == \
        (rec["variant"], rec["stage"], rec["warps"], rec["leaf_warps"])
    prm2, rec2 = autotune.tune(cfg, tl, abi.FORM_SPLIT, mass, cache_path=cache)
    assert rec2["cached"] and rec2["variant"] == rec["variant"] and prm2.warps_per_leaf == prm.warps_per_leaf
    with Session(0) as s:
        s.set_params(prm)
        acc, _ = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)
    plain, _ = gpu_acc(cfg, tl, mass, abi.FORM_PLAIN_FP64)
    rms, mx = rel_err(acc, plain, tl.tag == 1)
    assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (rms, mx)

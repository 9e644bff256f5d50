"""Benchmark of the B200 P2P short-range force pass.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--workload c2|c1|c2_128|c4|pm|fmm] [--form split|plain]

A step is one force pass over the workload's interaction lists. The default
workload is the 256^3 clustered configuration (60% uniform, 40% in 2,000 NFW
halos, leaves <= 32, mesh 256, r_s 1.2 cells, cutoff 4.5 r_s, Plummer
eps 1/40 spacing), generated from a fixed seed (no dataset). Its lists come
from the caller-side tree build + walk (the reference's src/fmm.c algorithm).

  value    pair-interactions/s of the chosen FP32/FP64-split form, inputs
           resident in HBM, the whole pass (frame prep, CSR build, pair
           kernel) replayed as a CUDA graph, device time from CUDA events,
           L2 flushed between steps (inputs are also larger than L2)
  accuracy the chosen form's per-particle force error against the plain
           FP64 form on the same inputs (rms and max of |da| / |a|)
  accuracy_vs_oracle  the chosen and the plain form against the FP64 direct
           minimum-image sum (the oracle) on 10^4 random local sinks
  e2e      the same metric through the C ABI on pinned host buffers:
           H2D of positions, leaves and lists, the pass, D2H of the forces
  roofline FP32 pipe: pairs/s x flops-per-pair (counted from the kernel
           source, FMA = 2) / the FP32 FFMA peak measured in-process
  pm       the PM long-range force (deposit, FFT, Green's function, FFT,
           gradient, interpolation) on the workload's particles and mesh:
           device ms per phase, the deposit and force kernels' HBM roofline, the
           numpy PM oracle beside the GPU on the 32^3 / mesh 64^3 workload
  serving  48 boxes of the serving ensemble resident in one server:
           saturation throughput, then Poisson arrivals at half of it,
           p50 / p99 request latency (submit to result in host memory),
           with the batching window on (launches wait up to 3 mean service
           times for other requests to share them) and, beside it, off

--workload c4 runs the serving configuration alone: 512 boxes, Poisson
arrivals at 0.25, 0.5, 1, 2 and 4 times the measured saturation rate.
--workload pm runs the PM leg alone (256^3 clustered particles, mesh 256^3).
--workload fmm runs the far field within the cutoff (P2M, M2M, M2L, L2L,
L2P) on the clustered particles with open angle 0.4, beside the reference's
own M2L timed on one host core.

With --gpus N > 1 (torchrun, one rank per GPU) every rank runs its own
independent box (replicas, no collective on the data path); the timed
region is bracketed by barriers and the max over ranks is reported.
--impl reference times the reference's own P2P arithmetic (P2P_core_lite,
FP32 SPI, compiled for the host from the reference sources into
oracle/_ref) on the host cores, over a bounded sample of the same lists:
the rows of every k-th sink leaf, about 2e9 pair interactions (the default
run's cpu_baseline is the same sample, with the first sink rows' figure
beside it).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [REPO, os.path.join(REPO, "photons-on-mt3000_b200")]

from photons_p2p import abi, workloads as W  # noqa: E402

METRIC = "pair-interactions/s at rms force err\u22641e-5 vs plain; ensemble p50/p99 latency"


def flops_per_pair(soft_mode, degree, masses=False):
    """FP32 flops of one pair in pair_split (p2p_kernels.cuh), FMA = 2:
    dx,dy,dz 3 FADD; u: 3 FFMA (Plummer) or FMUL + 2 FFMA (+FMNMX, clamp);
    rinv^3 2 FMUL; t = u - u0 1 FADD; Horner `degree` FFMA; f 1 FADD;
    acc 3 FFMA. MUFU rsqrt and the cutoff select are not flops."""
    u = 6 if soft_mode == abi.SOFT_PLUMMER else 5
    return 3 + u + 2 + 1 + 2 * degree + 1 + 6 + (1 if masses else 0)


def build_workload(name, rank=0):
    if name == "c2":
        cfg, pos = W.c2_config(), W.c2_positions()
    elif name == "c2_128":
        cfg = W.scaled(W.c2_config(), name="c2_clustered_128^3", n_side=128, mesh=128,
                       eps=1.0 / (40 * 128))
        pos = W.c2_positions(128)
    elif name == "c1":
        cfg, pos = W.c1_config(), W.c1_positions()
    else:
        raise SystemExit(f"unknown workload {name}")
    if rank:
        # replicas: each rank's box is the same configuration, its own draw
        g = W.rng(1000 + rank)
        pos = np.mod(pos + g.random((3, 1)), 1.0) * cfg.box + cfg.origin
    tl = W.prepare(pos, cfg)
    return cfg, pos.shape[1], tl, pos


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_hbm_peak():
    """The pool's measured copy bandwidth (GB/s) from MEASURED_PEAKS.json, or
    the earlier measurement 6650 GB/s when the file is absent."""
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def load_traffic(workload, form_name):
    """DRAM bytes per launch of the pair kernel from the committed ncu summary
    for this workload (None when no capture covers it)."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(f"{workload}:{form_name}")
    except (OSError, ValueError):
        return None


def load_fp64_flops(workload):
    """FP64 flops per listed pair of the plain form's pair kernel (DFMA x 2 +
    DADD + DMUL per pair, CUDA's erfc/exp/rsqrt included) from the committed
    ncu summary, or None."""
    path = os.path.join(REPO, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(f"{workload}:plain_fp64:fp64_flops_per_pair")
    except (OSError, ValueError):
        return None


def combine_ranks(total_s, e2e_s, pairs, dist, device):
    """Whole-job figures of a replica run: the slowest rank's times (max over
    ranks) and the pair interactions of all ranks (sum)."""
    if not dist:
        return float(total_s), float(e2e_s), float(pairs)
    import torch

    t = torch.tensor([total_s, e2e_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    pt = torch.tensor([float(pairs)], dtype=torch.float64, device=device)
    dist.all_reduce(pt, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(pt[0])


def plain_roofline(workload, pairs, kernel_ms, fp64_peak, fp32_peak):
    """The plain FP64 form's pair kernel against the measured FP64 and FP32
    peaks: FP64 flops per pair counted by ncu (the form's own arithmetic
    calls CUDA's FP64 erfc, exp and rsqrt, so its flops are counted where they
    execute rather than from the source)."""
    f64 = load_fp64_flops(workload)
    if not f64:
        return {"bound": "fp64", "peak": fp64_peak, "unit": "TFLOP/s", "flops_per_pair": None}
    achieved = pairs / (kernel_ms * 1e-3) * f64 / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak, "frac_of_fp32_peak": achieved / fp32_peak,
            "fp32_peak": fp32_peak, "flops_per_pair": f64,
            "flops_source": "ncu: 2 DFMA + DADD + DMUL per listed pair (128^3 capture)",
            "peak_source": "DFMA chain microbenchmark in-process (measured)"}


def walk_leg(sess, cfg, raw_pos, tl, dev, d_pos, d_ip, d_np, pairs, steps=3):
    """The P2P lists walked on the GPU (p2p_pass_submit_walk) against the
    caller's serial walk on the host cores: the host walk's time, and whole
    passes (frame prep, device walk, pair kernel) on resident particles."""
    from photons_p2p import lists as L
    from photons_p2p.p2p import DeviceWalkTree, kernel_launch_count

    allpos, tag = W.with_ghosts(raw_pos, cfg)
    t0 = time.time()
    tree = L.Tree(allpos, tag, cfg.maxleaf, cfg.box)
    tree_s = time.time() - t0
    with tree:
        if not (np.array_equal(tree.leaf_ipart, tl.leaf_ipart) and np.array_equal(tree.perm, tl.perm)):
            raise RuntimeError("walk leg: the tree differs from the pass's tree")
        t0 = time.time()
        tt, _ = tree.walk(cfg.cutoff_radius, cfg.open_angle)
        host_walk_s = time.time() - t0
        ntask_host = len(tt)
        del tt
        dtree = DeviceWalkTree(tree, dev)
        lib = sess.lib
        times, kern, ntask = [], [], 0
        l0 = kernel_launch_count()
        for k in range(steps + 1):
            if lib.p2p_pass_begin_device(sess.h, tl.npart, d_pos.data_ptr(), None, tl.nleaf, d_ip.data_ptr(),
                                         d_np.data_ptr()):
                raise RuntimeError(lib.p2p_last_error().decode())
            ntask = sess.submit_walk(dtree, cfg.cutoff_radius, cfg.open_angle)
            sec = sess.end()
            if k:  # the first pass warms up
                times.append(sec)
                kern.append(sess.last_kernel_ms())
        launches = (kernel_launch_count() - l0) // (steps + 1)
        walk_pairs = sess.pair_count()
        host_perm, host_ip = tree.perm.copy(), tree.leaf_ipart.copy()
    pass_s, kern_ms = float(np.mean(times)), float(np.mean(kern))
    out = {"host_tree_s": round(tree_s, 2), "host_walk_s": round(host_walk_s, 2),
           "host_walk_cores": L.num_threads(), "entries": int(ntask),
           "entries_equal_host": bool(ntask == ntask_host), "pairs_equal": bool(walk_pairs == pairs),
           "pass_ms": 1e3 * pass_s, "pair_kernel_ms": kern_ms,
           "walk_and_prep_ms": 1e3 * pass_s - kern_ms, "pairs_per_s": pairs / pass_s,
           "gpu_launches_per_pass": int(launches)}
    out["device_tree"] = device_tree_leg(sess, cfg, allpos, tag, dev, host_perm, host_ip, pairs, steps)
    return out


def device_tree_leg(sess, cfg, allpos, tag, dev, host_perm, host_ip, pairs, steps=3):
    """Tree, walk and pass all on the GPU from the particles (with ghosts) in
    device memory: p2p_dtree_build (the reference's kd-tree, built on the
    GPU), then p2p_pass_begin_device + p2p_pass_submit_walk on its arrays.
    Times the tree build (CUDA events) and the whole sequence (wall clock
    around the calls, which wait for the GPU)."""
    import torch

    from photons_p2p.p2p import DeviceTree

    d_all = torch.from_numpy(np.ascontiguousarray(allpos)).to(dev)
    d_tag = torch.from_numpy(np.ascontiguousarray(tag, dtype=np.int32)).to(dev)
    torch.cuda.synchronize()
    build_ms, total_s, equal = [], [], True
    lib = sess.lib
    for k in range(steps + 1):
        t0 = time.perf_counter()
        with DeviceTree(sess, d_all, d_tag, cfg.maxleaf, cfg.box) as t:
            d_pos, _, d_ip, d_np = t.device_arrays()
            if lib.p2p_pass_begin_device(sess.h, t.npart, d_pos, None, t.nleaf, d_ip, d_np):
                raise RuntimeError(lib.p2p_last_error().decode())
            sess.submit_walk(t, cfg.cutoff_radius, cfg.open_angle)
            sess.end()
            el = time.perf_counter() - t0
            if k == 0:  # the first build is checked against the host tree
                d = t.download()
                equal = bool(np.array_equal(d["perm"], host_perm) and np.array_equal(d["leaf_ipart"], host_ip))
                got_pairs = sess.pair_count()
            else:
                build_ms.append(t.build_ms)
                total_s.append(el)
    out = {"tree_ms": float(np.mean(build_ms)), "tree_walk_pass_ms": 1e3 * float(np.mean(total_s)),
           "tree_equal_host": equal, "pairs_equal": bool(got_pairs == pairs),
           "pairs_per_s": pairs / float(np.mean(total_s))}
    out["e2e_particles"] = particles_e2e(sess, cfg, allpos, tag, dev, pairs, steps)
    return out


def pm_leg(sess, cfg, raw_pos, dev, hbm_peak, cpu=True, steps=5, warmup=3):
    """The PM long-range force (p2p_pm_forces) on the workload's local
    particles and mesh: device times per phase (CUDA events on the session's
    stream), in the particles' input order and sorted by mesh cell (the order
    a tree walk leaves them in), the deposit and force kernels against the
    HBM roofline of their algorithmic bytes, and the numpy oracle beside the
    GPU on the lattice drop-in workload (32^3 particles, mesh 64^3)."""
    import torch

    from oracle import pm_oracle as PMO
    from photons_p2p.p2p import ParticleMesh

    n = raw_pos.shape[1]
    mass = 1.0 / n
    cell = np.minimum((raw_pos * (cfg.mesh / cfg.box)).astype(np.int64), cfg.mesh - 1)
    order = np.argsort((cell[0] * cfg.mesh + cell[1]) * cfg.mesh + cell[2], kind="stable")
    out = {"mesh": cfg.mesh, "particles": n}

    def timed(pm, pos, nsteps, nwarm):
        d_pos = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
        d_acc = torch.empty_like(d_pos)
        torch.cuda.synchronize()
        rows = []
        for k in range(nwarm + nsteps):
            pm.forces(d_pos, None, mass, d_acc)
            t = pm.timings()
            if k >= nwarm:
                rows.append(t)
        return {key: float(np.mean([r[key] for r in rows])) for key in rows[0]}

    with ParticleMesh(sess, cfg.mesh, cfg.box, cfg.split_radius) as pm:
        out["input_order_ms"] = timed(pm, raw_pos, steps, warmup)
        out["cell_sorted_ms"] = timed(pm, raw_pos[:, order], steps, warmup)
    ms = out["cell_sorted_ms"]
    out["particles_per_s"] = n / (ms["total"] * 1e-3)
    # algorithmic HBM bytes: deposit reads positions (24 B a particle) and
    # writes the mass mesh (8 B a cell, cleared and summed); the gradient
    # reads the potential (8 B a cell) and writes the interleaved gradient
    # (32 B); interpolation reads positions and the gradient mesh once and
    # writes accelerations (24 B a particle)
    cells = float(cfg.mesh) ** 3
    for name, nbytes in (("deposit", 24.0 * n + 16.0 * cells), ("gradient", 40.0 * cells),
                         ("interp", 48.0 * n + 32.0 * cells)):
        achieved = nbytes / (ms[name] * 1e-3) / 1e9
        out[f"{name}_roofline"] = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                                   "frac": achieved / hbm_peak, "bytes": nbytes}
    if not cpu:
        return out
    # the oracle beside the GPU on the lattice drop-in workload
    c1 = W.c1_config()
    p1 = W.c1_positions()
    t0 = time.perf_counter()
    PMO.pm_forces(p1, None, 1.0 / p1.shape[1], c1.mesh, c1.box, c1.split_radius)
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    with ParticleMesh(sess, c1.mesh, c1.box, c1.split_radius) as pm:
        gpu1 = timed(pm, p1, steps, warmup)
    out["lattice_32^3_mesh_64^3"] = {"gpu_ms": gpu1["total"], "cpu_oracle_ms": cpu_ms,
                                     "cpu_oracle": "numpy, 1 thread (the reference's PM needs MPI and 2DECOMP&FFT)"}
    return out


def _stdout_closed(fn):
    """fn() with the process's stdout closed (the reference's m2l prints a
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


def run_fmm(args, local):
    """The far field within the cutoff (p2p_fmm_far) on the clustered
    particles with the reference's open angle 0.4: at 256^3 in the unit box
    with every M2L task applied (min_r2 = 1e-15), and at 128^3 in a box of
    1000, where the reference's own FMM applies its tasks (min_r2 = 1, its
    integer-abs test), beside the reference's task_compute_m2l and l2p timed
    on one host core (its own dtime_m2l timer)."""
    import torch

    from photons_p2p.p2p import DeviceTree, FarField, Session

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    warm = max(3, args.warmup)

    def gpu(cfg, allpos, tag, mass, min_r2):
        d_all = torch.from_numpy(np.ascontiguousarray(allpos)).to(dev)
        d_tag = torch.from_numpy(np.ascontiguousarray(tag, dtype=np.int32)).to(dev)
        torch.cuda.synchronize()
        with Session(local) as s, DeviceTree(s, d_all, d_tag, cfg.maxleaf, cfg.box) as t, FarField(s) as ff:
            d_pos, _, d_ip, d_np = t.device_arrays()
            acc = torch.empty((3, t.npart), dtype=torch.float64, device=dev)
            rows, wall = [], []
            for k in range(warm + args.steps):
                a = time.perf_counter()
                ff.far(t.struct, d_pos, d_ip, d_np, t.npart, mass, cfg.split_radius, cfg.cutoff_radius,
                       cfg.open_angle, min_r2, acc.data_ptr())
                el = time.perf_counter() - a
                st = ff.stats()
                if k >= warm:
                    rows.append(st["ms"])
                    wall.append(el)
            ms = {key: float(np.mean([r[key] for r in rows])) for key in rows[0]}
            return {"particles_with_ghosts": int(t.npart), "leaves": int(t.nleaf), "nodes": int(t.nnode),
                    "m2l_tasks": st["n_m2l"], "m2l_applied": st["n_applied"], "walk_levels": st["levels"],
                    "device_ms": ms, "wall_ms": 1e3 * float(np.mean(wall)),
                    "m2l_tasks_per_s": st["n_m2l"] / (ms["m2l"] * 1e-3) if ms["m2l"] > 0 else None}

    cfg = W.scaled(W.c2_config(), open_angle=0.4)
    pos = W.c2_positions()
    allpos, tag = W.with_ghosts(pos, cfg)
    out = {"workload": "fmm_clustered_256^3_open_0.4", "steps": args.steps, "warmup": warm,
           "unit_box_256": gpu(cfg, allpos, tag, 1.0 / pos.shape[1], 1e-15)}
    del allpos, tag, pos
    cfgb = W.scaled(W.c2_config(), n_side=128, mesh=128, eps=1000.0 / (40 * 128), open_angle=0.4, box=1000.0)
    posb = W.c2_positions(128) * 1000.0
    allb, tagb = W.with_ghosts(posb, cfgb)
    massb = 1.0 / posb.shape[1]
    out["box_1000_128"] = g = gpu(cfgb, allb, tagb, massb, 1.0)
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        if O.ref_available("libref_walk.so"):
            r = _stdout_closed(lambda: O.RefWalk("libref_walk.so").fmm(
                allb, tagb, cfgb.maxleaf, cfgb.box, cfgb.split_radius, cfgb.cutoff_radius, cfgb.eps, massb,
                cfgb.open_angle))
            out["cpu_baseline"] = {"kind": "reference", "cores": 1, "sample": "the 128^3 box-1000 case, whole",
                                   "m2l_s": r["m2l_s"], "l2p_s": r["l2p_s"], "m2l_tasks": r["n_m2l"],
                                   "m2l_tasks_per_s": r["n_m2l"] / r["m2l_s"] if r["m2l_s"] > 0 else None,
                                   "gpu_m2l_speedup": (r["m2l_s"] * 1e3) / g["device_ms"]["m2l"]
                                   if g["device_ms"]["m2l"] > 0 else None}
        else:
            out["cpu_baseline"] = {"unavailable": "oracle/_ref not built"}
    return out


def particles_e2e(sess, cfg, allpos, tag, dev, pairs, steps=3):
    """End to end from particles to forces through the C ABI: positions and
    tags (with ghosts) from page-locked host memory to the device, the tree
    (p2p_dtree_build, then p2p_dtree_rebuild in place), the list walk and the
    pass (p2p_pass_submit_walk), the forces back to input order
    (p2p_dtree_unpermute) and to page-locked host memory for the local
    particles; wall clock around it all, every step."""
    import torch

    from photons_p2p.p2p import DeviceTree

    n = allpos.shape[1]
    nlocal = int(np.count_nonzero(tag))
    h_pos = torch.from_numpy(np.ascontiguousarray(allpos)).pin_memory()
    h_tag = torch.from_numpy(np.ascontiguousarray(tag, dtype=np.int32)).pin_memory()
    h_out = torch.empty((3, nlocal), dtype=torch.float64).pin_memory()
    d_pos = torch.empty((3, n), dtype=torch.float64, device=dev)
    d_tag = torch.empty(n, dtype=torch.int32, device=dev)
    d_out = torch.empty((3, n), dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(sess.stream, device=dev)
    lib = sess.lib
    times = []
    t = None
    try:
        for k in range(steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with torch.cuda.stream(stream):
                d_pos.copy_(h_pos, non_blocking=True)
                d_tag.copy_(h_tag, non_blocking=True)
            if t is None:  # the warm-up step builds the tree; the timed steps rebuild it in place
                t = DeviceTree(sess, d_pos, d_tag, cfg.maxleaf, cfg.box)
            else:
                t.rebuild(d_pos, d_tag, cfg.maxleaf, cfg.box)
            dp, _, dip, dnp = t.device_arrays()
            if lib.p2p_pass_begin_device(sess.h, t.npart, dp, None, t.nleaf, dip, dnp):
                raise RuntimeError(lib.p2p_last_error().decode())
            sess.submit_walk(t, cfg.cutoff_radius, cfg.open_angle)
            sess.end()
            t.unpermute(sess.result_device(), d_out.data_ptr())
            with torch.cuda.stream(stream):
                h_out.copy_(d_out[:, :nlocal], non_blocking=True)
            stream.synchronize()
            if k:
                times.append(time.perf_counter() - t0)
    finally:
        if t is not None:
            t.close()
    e = float(np.mean(times))
    return {"value": pairs / e, "unit": "pairs/s", "ms": 1e3 * e,
            "h2d_bytes_per_step": int(h_pos.numel() * 8 + h_tag.numel() * 4),
            "d2h_bytes_per_step": int(h_out.numel() * 8)}


def run_ours(args, rank, world, dist):
    import torch

    from photons_p2p.p2p import Session, kernel_launch_count, params_for

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t0 = time.time()
    cfg, nlocal, tl, raw_pos = build_workload(args.workload, rank)
    prep_s = time.time() - t0
    mass = 1.0 / nlocal
    P = tl.pair_count()
    form = abi.FORM_SPLIT if args.form == "split" else abi.FORM_PLAIN_FP64

    d_pos = torch.from_numpy(np.ascontiguousarray(tl.pos)).to(dev)
    d_ip = torch.from_numpy(tl.leaf_ipart).to(dev)
    d_np = torch.from_numpy(tl.leaf_npart).to(dev)
    d_t = torch.from_numpy(tl.task_t).to(dev)
    d_s = torch.from_numpy(tl.task_s).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()

    def resident_passes(sess, steps, warmup, sampler=None):
        stream = torch.cuda.ExternalStream(sess.stream, device=dev)
        args_dev = (tl.npart, d_pos.data_ptr(), tl.nleaf, d_ip.data_ptr(), d_np.data_ptr(),
                    tl.ntask, d_t.data_ptr(), d_s.data_ptr())
        for _ in range(warmup):
            sess.run_device(*args_dev)
            sess.end()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        pass_s, kern_ms = [], []
        l0 = kernel_launch_count()
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1)  # L2 flush, outside the pass events
                sess.run_device(*args_dev)
                pass_s.append(sess.end())
                kern_ms.append(sess.last_kernel_ms())
        launches = kernel_launch_count() - l0
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return pass_s, kern_ms, launches

    def result(sess):
        out = np.empty((3, tl.npart))
        if sess.lib.p2p_pass_result(sess.h, out.ctypes.data_as(ctypes.c_void_p)):
            raise RuntimeError(sess.lib.p2p_last_error().decode())
        return out

    # launch shape: the autotuner's pick for this leaf-size histogram (FP32 forms)
    prm, tuned = params_for(cfg, form, mass), None
    if form != abi.FORM_PLAIN_FP64 and not args.no_tune:
        from photons_p2p import autotune

        prm, rec = autotune.tune(cfg, tl, form, mass, device=local, sample_pairs=args.tune_pairs,
                                 cache_path=args.tune_cache)
        tuned = {k: rec.get(k, 1) for k in ("key", "variant", "stage", "warps", "leaf_warps", "sample_pairs",
                                             "cached")}
    with Session(local) as sess:
        fp32_peak = sess.measure_fp32_peak()
        fp64_peak = sess.measure_fp64_peak()
        sess.set_params(prm)
        degree = sess.poly_degree
        sampler = ClockSampler(local)
        pass_s, kern_ms, launches = resident_passes(sess, args.steps, args.warmup, sampler)
        clocks = sampler.summary()
        acc_form = result(sess)
        acc_plain = None
        evaluated = sess.evaluated_pairs()
        # the plain FP64 form on the same inputs: the split/plain ratio and the
        # chosen form's force error against it (local particles)
        plain, accuracy = None, None
        if form == abi.FORM_SPLIT and not args.skip_plain:
            sess.set_params(params_for(cfg, abi.FORM_PLAIN_FP64, mass))
            p_s, p_k, _ = resident_passes(sess, max(1, min(args.steps, 3)), 1)
            plain = {"value": P / float(np.mean(p_s)), "kernel_ms": float(np.mean(p_k))}
            plain["roofline"] = plain_roofline(args.workload, P, plain["kernel_ms"], fp64_peak, fp32_peak)
            loc = tl.tag == 1
            acc_plain = result(sess)
            num = np.linalg.norm(acc_form - acc_plain, axis=0)[loc]
            den = np.linalg.norm(acc_plain, axis=0)[loc]
            rel = num / np.where(den > 0, den, 1.0)
            accuracy = {"vs": "plain_fp64", "rms": float(np.sqrt(np.mean(rel ** 2))),
                        "max": float(rel.max()), "particles": int(loc.sum())}
            sess.set_params(prm)

        # e2e through the C ABI on pinned host buffers
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        h_pos, h_ip, h_np, h_t, h_s = (pin(tl.pos), pin(tl.leaf_ipart), pin(tl.leaf_npart),
                                       pin(tl.task_t), pin(tl.task_s))
        h_out = torch.zeros((3, tl.npart), dtype=torch.float64).pin_memory()
        lib = sess.lib

        def e2e_pass():
            ok = lib.p2p_pass_begin(sess.h, tl.npart, h_pos.data_ptr(), None, tl.nleaf,
                                    h_ip.data_ptr(), h_np.data_ptr())
            ok |= lib.p2p_pass_submit(sess.h, tl.ntask, h_t.data_ptr(), h_s.data_ptr())
            ok |= lib.p2p_pass_end(sess.h, ctypes.byref(ctypes.c_double()))
            ok |= lib.p2p_pass_result(sess.h, h_out.data_ptr())
            if ok:
                raise RuntimeError(lib.p2p_last_error().decode())

        for _ in range(max(1, args.warmup)):
            e2e_pass()
        e2e_t = []
        for _ in range(max(1, min(args.steps, 5))):
            a = time.perf_counter()
            e2e_pass()
            e2e_t.append(time.perf_counter() - a)
        h2d = tl.pos.nbytes + tl.leaf_ipart.nbytes + tl.leaf_npart.nbytes + tl.task_t.nbytes + tl.task_s.nbytes
        d2h = 3 * tl.npart * 8
        walk = None
        if not args.no_walk:
            walk = walk_leg(sess, cfg, raw_pos, tl, dev, d_pos, d_ip, d_np, P)
        pm = None
        if not args.no_pm:
            pm = pm_leg(sess, cfg, raw_pos, dev, measured_hbm_peak(),
                        cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)

    mean_pass = float(np.mean(pass_s))
    mean_kernel_ms = float(np.mean(kern_ms))
    total_s = float(np.sum(pass_s))
    e2e_mean = float(np.mean(e2e_t))
    total_s, e2e_mean, P_all = combine_ranks(total_s, e2e_mean, P, dist, dev)
    value = P_all * args.steps / total_s
    F = flops_per_pair(cfg.soft_mode, degree) if form != abi.FORM_PLAIN_FP64 else None
    kernel_pairs_per_s = P / (mean_kernel_ms * 1e-3)
    roofline = None
    if form == abi.FORM_PLAIN_FP64:
        roofline = plain_roofline(args.workload, P, mean_kernel_ms, fp64_peak, fp32_peak)
    if F:
        # flops of the pairs the kernel evaluates (entries wholly beyond the
        # cutoff are skipped: counted in the metric's pairs, not in the flops)
        achieved = evaluated / (mean_kernel_ms * 1e-3) * F / 1e12
        traffic = load_traffic(args.workload, abi.FORM_NAMES[form])
        roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak, "traffic": traffic,
                    "flops_per_pair": F, "peak_source": "FFMA chain microbenchmark in-process (measured)"}
    out = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 leaf offsets + f64 accumulation)" if form == abi.FORM_SPLIT else "f64",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": cfg.name, "form": abi.FORM_NAMES[form], "n_local": nlocal,
                   "n_with_ghosts": int(tl.npart), "n_leaf": int(tl.nleaf), "n_task": int(tl.ntask),
                   "pairs_per_pass": int(P), "pairs_evaluated_per_pass": int(evaluated),
                   "leaf_cap": cfg.maxleaf, "mesh": cfg.mesh,
                   "r_s": cfg.split_radius, "x_cut": cfg.x_cut, "eps": cfg.eps, "soft": "plummer"
                   if cfg.soft_mode == abi.SOFT_PLUMMER else "clamp", "open_angle": cfg.open_angle,
                   "poly_degree": degree, "launch_shape": tuned or "default",
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MB flush between steps; inputs > L2", "host_prep_s": round(prep_s, 1)},
        "kernel_ms": mean_kernel_ms,
        "kernel_pairs_per_s": kernel_pairs_per_s,
        "roofline": roofline,
        "plain_fp64": plain,
        "split_over_plain": (value / plain["value"]) if plain else None,
        "device_walk": walk,
        "pm": pm,
        "accuracy": accuracy,
        "e2e": {"value": P_all / e2e_mean, "unit": "pairs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    forms = {abi.FORM_NAMES[form]: acc_form}
    if acc_plain is not None:
        forms["plain_fp64"] = acc_plain
    return out, cfg, tl, nlocal, raw_pos, forms


C4_EPS_OVER_RS = (1.0 / 40) / 1.2  # serving boxes: eps = 1/(40 n), r_s = 1.2 / n


def serving_ensemble(srv, nbox, log=None):
    """Registers and preloads serving boxes 0..nbox-1 (their host lists are
    dropped once resident); returns (particles, pair interactions) totals."""
    from photons_p2p import serve

    npart = pairs = 0
    for b in range(nbox):
        box = W.c4_box(b)
        tl = serve.box_lists(box)
        k = srv.add_box(tl, 0.5 / box.cfg.split_radius, 1.0 / int(tl.tag.sum()))
        srv.preload(k)
        npart += tl.npart
        pairs += srv.boxes[k].pairs
        if log and (b + 1) % 64 == 0:
            log(f"[serving] {b + 1}/{nbox} boxes resident")
    return npart, pairs


def serving_measure(srv, rates_frac, requests, seed=10, window_service_times=0.0):
    """Saturation throughput (a burst of 2 requests per box), then Poisson
    arrivals at the given fractions of it. window_service_times > 0 sets the
    server's batching window to that many mean service times (1 / saturation
    request rate) after the saturation run, with a pack launching without
    waiting once it holds 3 mean requests' pair interactions."""
    from photons_p2p import serve

    nbox = len(srv.boxes)
    srv.set_batching(0.0)
    sat = serve.run_poisson(srv, 1e9, 2 * nbox, seed=seed, reserve=2)
    window = None
    if window_service_times > 0:
        mean_s = 1.0 / sat["requests_per_s"]
        mean_pairs = sat["pairs_per_s"] / sat["requests_per_s"]
        window = {"batch_window_ms": 1e3 * window_service_times * mean_s, "min_pack_pairs": 3.0 * mean_pairs,
                  "service_times": window_service_times}
        srv.set_batching(window["batch_window_ms"], window["min_pack_pairs"])
    rows = []
    for i, f in enumerate(rates_frac):
        rate = f * sat["requests_per_s"]
        n = requests(rate) if callable(requests) else requests
        r = serve.run_poisson(srv, rate, int(n), seed=seed + 1 + i)
        r["rate_frac"] = f
        r["window"] = window
        rows.append(r)
    srv.set_batching(0.0)
    return sat, rows


def run_serving_leg(local, nbox=48, window_service_times=3.0):
    """The serving summary of the default run: nbox ensemble boxes, one full
    grid slot, Poisson arrivals at half the measured saturation rate, with
    and without the batching window (window_service_times mean service
    times; launches wait for company up to that long)."""
    from photons_p2p import serve

    t0 = time.time()
    shape = serve.serving_shape(abi.FORM_SPLIT, C4_EPS_OVER_RS)
    with serve.Server(shape, device=local, slots=1, full_grid=True, hbm_bytes=40 << 30) as srv:
        npart, pairs = serving_ensemble(srv, nbox)
        prep = time.time() - t0
        sat, rows = serving_measure(srv, [0.5], 4 * nbox)
        _, wrows = serving_measure(srv, [0.5], 4 * nbox, seed=20, window_service_times=window_service_times)
    keys = ("rate_hz", "requests", "p50_ms", "p99_ms", "requests_per_s", "pairs_per_s", "boxes_per_launch")
    r, w = rows[0], wrows[0]
    out = {"boxes": nbox, "particles": int(npart), "slots": 1, "max_pack": 32,
           "saturation_pairs_per_s": sat["pairs_per_s"],
           "saturation_requests_per_s": sat["requests_per_s"], "rate_frac_of_saturation": 0.5,
           "host_prep_s": round(prep, 1)}
    # headline: the batching window on (packs under load); beside it the
    # same arrivals' rate with the window off (lowest latency at low load)
    out.update({k: w[k] for k in keys})
    out["p99_over_p50"] = w["p99_ms"] / w["p50_ms"]
    out["batch_window"] = w["window"]
    out["no_window"] = {k: r[k] for k in keys}
    out["no_window"]["p99_over_p50"] = r["p99_ms"] / r["p50_ms"]
    return out


def run_serving_sweep(args, local):
    """Serving configuration: 512 boxes (n^3, n log-uniform in [32, 128],
    lattice + Gaussian + 0-200 NFW halos), Poisson arrivals at 0.25, 0.5, 1,
    2 and 4 times the measured saturation throughput."""
    from photons_p2p import serve

    t0 = time.time()
    shape = serve.serving_shape(abi.FORM_SPLIT, C4_EPS_OVER_RS)
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    with serve.Server(shape, device=local, slots=args.slots, full_grid=True,
                      hbm_bytes=int(args.hbm_gb * (1 << 30))) as srv:
        npart, pairs = serving_ensemble(srv, args.boxes, log)
        prep = time.time() - t0
        st0 = srv.stats()
        sampler = ClockSampler(local)
        with sampler:
            sat, rows = serving_measure(srv, [0.25, 0.5, 1.0, 2.0, 4.0],
                                        lambda rate: min(3000, max(200, rate * 6.0)),
                                        window_service_times=args.window)
        st1 = srv.stats()
    for r in rows:
        log(f"[serving] {r['rate_frac']:.2f}x sat ({r['rate_hz']:.0f}/s): p50 {r['p50_ms']:.2f} ms "
            f"p99 {r['p99_ms']:.2f} ms  {r['requests_per_s']:.1f} req/s  {r['pairs_per_s']:.3e} pairs/s")
    sweep = [{k: r[k] for k in ("rate_frac", "rate_hz", "requests", "p50_ms", "p99_ms", "mean_ms",
                                "max_ms", "requests_per_s", "pairs_per_s", "boxes_per_launch",
                                "launches")} for r in rows]
    out = {
        "metric": METRIC, "value": sat["pairs_per_s"], "unit": "pairs/s", "n_gpus": 1,
        "steps": len(rows), "warmup": 1, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 leaf offsets + f64 accumulation)",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"c4_serving_{args.boxes}_boxes", "boxes": args.boxes,
                   "particles_with_ghosts": int(npart), "pairs_per_round": int(pairs),
                   "slots": args.slots, "max_pack": 32, "hbm_budget_gb": args.hbm_gb,
                   "batch_window": rows[0]["window"],
                   "resident_gb": st1["resident_bytes"] / 1e9, "host_prep_s": round(prep, 1),
                   "l2": "inputs > L2 (boxes resident, 126 MB L2)"},
        "serving": {"saturation_pairs_per_s": sat["pairs_per_s"],
                    "saturation_requests_per_s": sat["requests_per_s"],
                    "saturation_p50_ms": sat["p50_ms"], "saturation_p99_ms": sat["p99_ms"],
                    "sweep": sweep, "launches": st1["launches"] - st0["launches"],
                    "kernel_s": (st1["kernel_ms"] - st0["kernel_ms"]) / 1e3},
        "gpu_launches": int(3 * (st1["launches"] - st0["launches"])),
        "clocks": sampler.summary(),
        "cpu_baseline": None,
    }
    return out


def run_batching(args, local):
    """Batching configuration: side^3 particles (512^3 = 134M by default) of
    the uniform / NFW mix with 20,000 halos (scaled by volume below 512),
    leaf cap swept; for each cap the walk runs in groups of sink leaves
    (bounded host memory) straight into device-resident list chunks, the
    autotuner picks the launch shape on a sample, and whole passes (frame
    prep, per-chunk CSR build, persistent pair kernel) are timed with CUDA
    events, inputs resident in HBM."""
    import torch

    from photons_p2p import autotune
    from photons_p2p.lists import Tree
    from photons_p2p.p2p import Session, _check

    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    dev = torch.device("cuda", local)
    torch.cuda.set_device(local)
    side = args.side
    t0 = time.time()
    nh = max(1, int(round(20000 * (side / 512.0) ** 3)))
    pos, _ = W.clustered(side ** 3, 0.4, nh, (4.0, 12.0), W.rng(3))
    base = W.scaled(W.c3_config(32), n_side=side, mesh=side, eps=1.0 / (40 * side))
    allpos, tag = W.with_ghosts(pos, base)
    nlocal = pos.shape[1]
    del pos
    mass = 1.0 / nlocal
    log(f"[batching] {side}^3: {allpos.shape[1]} particles with ghosts, {time.time() - t0:.1f} s")
    records = []
    caps = [int(c) for c in args.leaf_caps.split(",")]
    cache = args.tune_cache
    for cap in caps:
        cfg = W.scaled(base, name=f"c3_batching_{side}^3_leaf{cap}", maxleaf=cap)
        t1 = time.time()
        with Tree(allpos, tag, cap, cfg.box) as tree:
            nleaf = tree.nleaf
            # rows per sink leaf from a 1/64 sample walk sets the group count
            probe = np.zeros(nleaf, np.uint8)
            probe[::64] = 1
            tt, _ = tree.walk(cfg.cutoff_radius, cfg.open_angle, probe)
            est = len(tt) * 64
            groups = max(1, int(np.ceil(est / args.chunk_rows)))
            bounds = np.linspace(0, nleaf, groups + 1).astype(np.int64)
            chunks, pairs, rows = [], 0, 0
            npl = tree.leaf_npart.astype(np.int64)
            sample_lists = None
            for g in range(groups):
                m = np.zeros(nleaf, np.uint8)
                m[bounds[g]:bounds[g + 1]] = 1
                tt, ts = tree.walk(cfg.cutoff_radius, cfg.open_angle, m)
                if not len(tt):
                    continue
                pairs += int(np.dot(npl[tt], npl[ts]))
                rows += len(tt)
                if sample_lists is None:
                    sample_lists = tree.lists(tt, ts)
                chunks.append((torch.from_numpy(tt).to(dev), torch.from_numpy(ts).to(dev)))
                del tt, ts
            lists_s = time.time() - t1
            d_pos = torch.from_numpy(tree.pos).to(dev)
            d_ip = torch.from_numpy(tree.leaf_ipart).to(dev)
            d_np = torch.from_numpy(tree.leaf_npart).to(dev)
            npart = tree.pos.shape[1]
            qs = np.percentile(tree.leaf_npart, [0, 25, 50, 75, 100]).tolist()
            mean_leaf = float(tree.leaf_npart.mean())
        log(f"[batching] cap {cap}: {nleaf} leaves (mean {mean_leaf:.1f}), {rows:.3e} rows in "
            f"{len(chunks)} chunks, {pairs:.3e} pairs, lists {lists_s:.1f} s")
        params, rec = autotune.tune(cfg, sample_lists, abi.FORM_SPLIT, mass, device=local,
                                    sample_pairs=args.tune_pairs, cache_path=cache, log=log)
        del sample_lists
        with Session(local, params) as sess:
            lib = sess.lib

            def one_pass():
                _check(lib, lib.p2p_pass_begin_device(sess.h, npart, d_pos.data_ptr(), None, nleaf,
                                                      d_ip.data_ptr(), d_np.data_ptr()))
                for ct, cs in chunks:
                    _check(lib, lib.p2p_pass_submit_device(sess.h, ct.numel(), ct.data_ptr(), cs.data_ptr()))
                return sess.end()

            for _ in range(args.warmup):
                one_pass()
            secs = [one_pass() for _ in range(args.steps)]
        pass_s = float(np.mean(secs))
        r = {"leaf_cap": cap, "leaves": int(nleaf), "leaf_npart_q0_25_50_75_100": qs,
             "mean_leaf": mean_leaf, "rows": int(rows), "rows_per_sink_leaf": rows / max(1, nleaf),
             "chunks": len(chunks), "pairs": int(pairs), "pass_s": pass_s, "pairs_per_s": pairs / pass_s,
             "tuned": {k: rec.get(k, 1) for k in ("key", "variant", "stage", "warps", "leaf_warps", "cached")},
             "lists_host_s": round(lists_s, 1)}
        log(f"[batching] cap {cap}: pass {pass_s:.3f} s  {pairs / pass_s:.3e} pairs/s  shape "
            f"{rec['variant']}/{rec['stage']}/{rec['warps']}")
        records.append(r)
        del chunks, d_pos, d_ip, d_np
        torch.cuda.empty_cache()
    head = next((r for r in records if r["leaf_cap"] == 32), records[0])
    return {
        "metric": METRIC, "value": head["pairs_per_s"], "unit": "pairs/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * head["pass_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 leaf offsets + f64 accumulation)", "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"c3_batching_{side}^3", "n_local": int(nlocal),
                   "n_with_ghosts": int(allpos.shape[1]), "halos": nh, "leaf_caps": caps,
                   "value_leaf_cap": head["leaf_cap"], "chunk_rows": args.chunk_rows,
                   "l2": "inputs > L2"},
        "batching": records, "cpu_baseline": None,
    }


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def cpu_reference_sample(cfg, tl, mass, target_pairs, strided=True):
    """A bounded sample of the pass for the CPU legs, about target_pairs pair
    interactions of whole sink rows: strided, the rows of every k-th sink
    leaf across the whole box (the autotuner's sample); else the rows of the
    first sink leaves in leaf-id order (one corner of the box)."""
    if strided:
        from photons_p2p import autotune

        tt, ts, pairs = autotune.sample_rows(tl.leaf_npart, tl.task_t, tl.task_s, target_pairs)
        k = max(1, int(tl.pair_count() // max(target_pairs, 1.0)))
        return tt, ts, pairs, f"rows of every {k}-th sink leaf"
    npart = tl.leaf_npart.astype(np.int64)
    per_sink = np.bincount(tl.task_t, weights=(npart[tl.task_t] * npart[tl.task_s]).astype(np.float64),
                           minlength=tl.nleaf)
    cum = np.cumsum(per_sink)
    last = min(int(np.searchsorted(cum, target_pairs)), tl.nleaf - 1)
    sel = tl.task_t <= last
    return tl.task_t[sel], tl.task_s[sel], int(round(cum[last])), "first sink rows"


def time_cpu(cfg, tl, mass, target_pairs, steps=1, strided=True):
    from oracle import oracle as O

    tt, ts, pairs, how = cpu_reference_sample(cfg, tl, mass, target_pairs, strided)
    if O.ref_available("libref_pair.so"):
        kind = "reference"
        soft = 0 if cfg.soft_mode == abi.SOFT_CLAMP else 1

        def run():
            O.ref_p2p_lists("sp_spi", soft, cfg.eps, cfg.split_radius, mass, tl.pos, tl.leaf_ipart,
                            tl.leaf_npart, tt, ts)
        what = "reference P2P_core_lite/P2P_core_1 FP32 SPI+GPUCUTOFF (src/gpu_kernel.impl.h, host-compiled), OpenMP over sink leaves"
    else:
        kind = "port"
        prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)

        def run():
            O.p2p_lists(prm, tl.pos, tl.leaf_ipart, tl.leaf_npart, tt, ts)
        what = "oracle/p2p_oracle.c FP64 restatement, OpenMP over sink leaves"
    times = []
    for _ in range(steps):
        a = time.perf_counter()
        run()
        times.append(time.perf_counter() - a)
    v = pairs / float(np.mean(times))
    return {"value": v, "unit": "pairs/s", "cores": O.num_threads(), "kind": kind,
            "sample": f"{pairs:.3g} pair interactions ({len(tt)} list entries, {how} of {cfg.name}); {what}"}, times


def accuracy_vs_oracle(cfg, raw_pos, tl, mass, forms, nsink=10000, seed=91):
    """Per-particle relative force error of each form's pass against the FP64
    direct minimum-image sum of the same truncated kernel (the oracle,
    oracle/p2p_oracle.c oracle_direct), on nsink randomly drawn local sinks.
    forms: {name: (3, npart) result in tree order}."""
    from oracle import oracle as O

    n = raw_pos.shape[1]
    sinks = np.sort(np.random.default_rng(seed).choice(n, min(nsink, n), replace=False)).astype(np.int32)
    prm = O.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)
    t0 = time.time()
    ref = O.direct(prm, raw_pos, cfg.box, sinks)
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    den = np.linalg.norm(ref, axis=0)
    out = {"vs": "fp64 direct minimum-image sum (oracle)", "sinks": int(sinks.size),
           "oracle_s": round(time.time() - t0, 1)}
    for name, acc in forms.items():
        if acc is None:
            continue
        rel = np.linalg.norm(acc[:, slot[sinks]] - ref, axis=0) / np.where(den > 0, den, 1.0)
        out[name] = {"rms": float(np.sqrt(np.mean(rel ** 2))), "max": float(rel.max())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--form", choices=["split", "plain"], default="split")
    ap.add_argument("--cpu-pairs", type=float, default=2e9)
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving summary")
    ap.add_argument("--no-walk", action="store_true", help="skip the device list walk leg")
    ap.add_argument("--no-pm", action="store_true", help="skip the PM long-range leg")
    ap.add_argument("--no-tune", action="store_true", help="default launch shape, no autotuning")
    ap.add_argument("--boxes", type=int, default=512, help="c4: ensemble size")
    ap.add_argument("--slots", type=int, default=1, help="c4: server launch slots")
    ap.add_argument("--window", type=float, default=0.0,
                    help="c4: batching window in mean service times (0: off)")
    ap.add_argument("--hbm-gb", type=float, default=100.0, help="c4: server arena size")
    ap.add_argument("--side", type=int, default=512, help="c3: particles per side")
    ap.add_argument("--leaf-caps", default="16,32,64", help="c3: leaf caps to sweep")
    ap.add_argument("--chunk-rows", type=float, default=1.0e9, help="c3: list entries per chunk")
    ap.add_argument("--tune-pairs", type=float, default=1e10,
                    help="autotuner sample size (pair interactions; enough rows that every warp gets several)")
    ap.add_argument("--tune-cache", default=None, help="c3: autotuner cache (JSON)")
    args = ap.parse_args()
    if args.warmup < 3:
        print("note: fewer than 3 warm-up steps requested", file=sys.stderr)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist

    if args.impl == "reference":
        if rank == 0:
            t0 = time.time()
            cfg, nlocal, tl, _ = build_workload(args.workload, 0)
            mass = 1.0 / nlocal
            if args.warmup:
                time_cpu(cfg, tl, mass, min(args.cpu_pairs, 2e8))
            cb, times = time_cpu(cfg, tl, mass, args.cpu_pairs, steps=args.steps)
            out = {"metric": METRIC, "value": cb["value"], "unit": "pairs/s", "n_gpus": args.gpus,
                   "steps": args.steps, "warmup": args.warmup,
                   "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
                   "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                   "data": "synthetic (seeded; no dataset)",
                   "config": {"workload": cfg.name, "host_prep_s": round(time.time() - t0, 1)},
                   "impl": "reference", "cpu_baseline": cb,
                   "e2e": {"value": cb["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}}
            print(json.dumps(out), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload == "c3":
        if rank == 0:
            print(json.dumps(run_batching(args, int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload == "fmm":
        if rank == 0:
            print(json.dumps(run_fmm(args, int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload == "pm":
        # the PM long-range force alone on the 256^3 clustered particles and
        # mesh (the default workload's PM leg, without the P2P pass)
        if rank == 0:
            import torch

            from photons_p2p.p2p import Session

            local = int(os.environ.get("LOCAL_RANK", "0"))
            torch.cuda.set_device(local)
            with Session(local) as sess:
                pm = pm_leg(sess, W.c2_config(), W.c2_positions(), torch.device("cuda", local),
                            measured_hbm_peak(), cpu=not args.no_cpu_baseline, steps=args.steps,
                            warmup=args.warmup)
            print(json.dumps({"workload": "pm_clustered_256^3_mesh_256^3", "pm": pm}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload == "c4":
        if rank == 0:
            print(json.dumps(run_serving_sweep(args, int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    out, cfg, tl, nlocal, raw_pos, forms = run_ours(args, rank, world, dist)
    if world == 1 and not args.no_serving and args.workload == "c2":
        out["serving"] = run_serving_leg(int(os.environ.get("LOCAL_RANK", "0")))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU leg: the reference's own pair arithmetic timed on the host
        # cores over a strided sample (the first-rows sample beside it), and
        # the oracle as the checker of the GPU forms' results
        cb, _ = time_cpu(cfg, tl, 1.0 / nlocal, args.cpu_pairs)
        first, _ = time_cpu(cfg, tl, 1.0 / nlocal, args.cpu_pairs, strided=False)
        cb["first_rows_value"] = first["value"]
        cb["first_rows_sample"] = first["sample"]
        out["cpu_baseline"] = cb
        out["accuracy_vs_oracle"] = accuracy_vs_oracle(cfg, raw_pos, tl, 1.0 / nlocal, forms)
    elif rank == 0:
        out["cpu_baseline"] = None
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Precision stress study of the P2P pass's arithmetic forms.

Workload: 2^26 particles in a periodic unit box whose origin is shifted to
1.0 (coordinates in [1, 2), where an FP32 ulp is 1.19e-7 of the box), 90% in
500 NFW halos (concentration U[10, 20]), 10% uniform; Plummer softening
eps = 1/200 lattice spacing; mesh 406, r_s = 1.2 cells, cutoff 4.5 r_s.
A random sample of local particles (10^5 by default) is drawn; the walk keeps
only the list rows of the leaves holding them, every form runs the pass on
those rows, and each sampled particle's acceleration is compared with the
FP64 direct minimum-image sum of the same truncated kernel (the oracle):

  plain_fp64   FP64 throughout (the drop-in form)
  naive_fp32   FP32 pair math on global coordinates, FP32 accumulation
  split        FP32 pair math on leaf-local coordinates, FP64 centre offsets,
               FP64 accumulation (the chosen form)
  kahan_fp32   as split but Kahan-compensated FP32 accumulation

Per form it reports rms / max / percentiles of the relative error
|a - a_direct| / |a_direct| and a histogram over decades. The oracle is the
checker here; this file sits with the tests for that reason.

  python tests/precision_stress.py --n 67108864 --sinks 100000 --json out.json

The oracle's part (minutes of CPU) can run apart from the GPU part:
--oracle-only --oracle-cache f.npz computes it without a GPU, and a later run
given the same --oracle-cache reuses it.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(_HERE)
for _p in (_REPO, os.path.join(_REPO, "photons-on-mt3000_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from oracle import oracle  # noqa: E402
from photons_p2p import abi, p2p, workloads as W  # noqa: E402
from photons_p2p.lists import build_tree_lists  # noqa: E402

FORMS = [("plain_fp64", abi.FORM_PLAIN_FP64), ("naive_fp32", abi.FORM_NAIVE_FP32),
         ("split", abi.FORM_SPLIT), ("kahan_fp32", abi.FORM_KAHAN_FP32)]
DECADES = np.arange(-17, 1)  # histogram edges 10^-17 .. 10^0, plus under/overflow


def stress_config(n_total):
    """The stress configuration at n_total particles (2^26 at full size): the
    lattice-equivalent spacing, mesh and softening follow n_total^(1/3)."""
    base = W.c5_config()
    side = round(n_total ** (1.0 / 3.0))
    if n_total == 2 ** 26:
        return base
    return W.scaled(base, name=f"c5_stress_{n_total}", n_side=side, mesh=side,
                    eps=1.0 / (200 * side))


def error_stats(got, ref):
    num = np.linalg.norm(got - ref, axis=0)
    den = np.linalg.norm(ref, axis=0)
    rel = num / np.where(den > 0, den, 1.0)
    with np.errstate(divide="ignore"):
        lg = np.log10(np.maximum(rel, 1e-300))
    hist, _ = np.histogram(np.clip(lg, DECADES[0] - 0.5, DECADES[-1] + 0.5),
                           bins=np.concatenate([[-400], DECADES, [400]]))
    return {
        "rms": float(np.sqrt(np.mean(rel ** 2))),
        "max": float(rel.max()),
        "p50": float(np.percentile(rel, 50)),
        "p99": float(np.percentile(rel, 99)),
        "p99.9": float(np.percentile(rel, 99.9)),
        "hist_decades": {"edges_log10": DECADES.tolist(), "counts": hist.tolist()},
    }


def direct_reference(cfg, pos, sinks, mass, cache=None, log=print):
    """FP64 direct oracle for the sampled sinks; with `cache` (an .npz path)
    the result is reused when the file holds the same sinks and settings,
    and written otherwise."""
    key = np.array([pos.shape[1], cfg.eps, cfg.split_radius, cfg.x_cut, cfg.box, cfg.origin])
    if cache and os.path.exists(cache):
        z = np.load(cache)
        if np.array_equal(z["key"], key) and np.array_equal(z["sinks"], sinks):
            log(f"[stress] FP64 direct oracle from {cache}")
            return z["acc"], float(z["seconds"]), int(z["threads"])
    t1 = time.time()
    oprm = oracle.params(cfg.soft_mode, cfg.eps, cfg.split_radius, cfg.x_cut, mass)
    ref = oracle.direct(oprm, pos, cfg.box, sinks)
    sec, thr = time.time() - t1, oracle.num_threads()
    log(f"[stress] FP64 direct oracle: {sec:.1f} s on {thr} threads")
    if cache:
        np.savez(cache, key=key, sinks=sinks, acc=ref, seconds=sec, threads=thr)
    return ref, sec, thr


def run(n_total=2 ** 26, nsink=100_000, seed=7, forms=FORMS, device=0, log=print,
        oracle_cache=None, oracle_only=False, chunk=1 << 27):
    cfg = stress_config(n_total)
    t0 = time.time()
    pos = W.c5_positions(n_total)
    n = pos.shape[1]
    mass = 1.0 / n
    sinks = np.sort(np.random.default_rng(seed).choice(n, size=min(nsink, n), replace=False))
    if oracle_only:
        ref, sec, thr = direct_reference(cfg, pos, sinks, mass, oracle_cache, log)
        return {"config": cfg.name, "n": n, "sinks": int(sinks.size), "oracle_s": sec,
                "oracle_threads": thr}
    allpos, tag = W.with_ghosts(pos, cfg)
    tl = build_tree_lists(allpos, tag, cfg.maxleaf, cfg.box, cfg.cutoff_radius, cfg.open_angle,
                          sink_particles=sinks)
    slot = np.empty(tl.npart, np.int64)
    slot[tl.perm] = np.arange(tl.npart)
    sink_slots = slot[sinks]
    log(f"[stress] n={n} ghosts={tl.npart - n} leaves={tl.nleaf} rows={tl.ntask} "
        f"pairs={tl.pair_count():.3e} setup {time.time() - t0:.1f}s")

    out = {"config": cfg.name, "n": n, "sinks": int(sinks.size), "seed": seed,
           "origin": cfg.origin, "eps": cfg.eps, "split_radius": cfg.split_radius,
           "pairs": tl.pair_count(), "forms": {}}
    accs = {}
    for name, form in forms:
        prm = p2p.params_for(cfg, form, mass)
        with p2p.Session(device, prm) as s:
            acc, sec = s.force_pass(tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s,
                                    chunk=chunk)
        accs[name] = acc[:, sink_slots]
        out["forms"][name] = {"gpu_s": sec}
        log(f"[stress] {name}: {sec:.3f} s on the GPU")

    del tl
    ref, out["oracle_s"], out["oracle_threads"] = direct_reference(cfg, pos, sinks, mass,
                                                                   oracle_cache, log)
    for name, _ in forms:
        st = error_stats(accs[name], ref)
        out["forms"][name].update(st)
        log(f"[stress] {name:11s} rms {st['rms']:.3e} max {st['max']:.3e} "
            f"p99 {st['p99']:.3e} p99.9 {st['p99.9']:.3e}")
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, default=2 ** 26)
    ap.add_argument("--sinks", type=int, default=100_000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--json", default=None)
    ap.add_argument("--oracle-cache", default=None,
                    help=".npz holding (or receiving) the FP64 direct oracle's result")
    ap.add_argument("--oracle-only", action="store_true",
                    help="only compute the oracle into --oracle-cache (no GPU needed)")
    a = ap.parse_args()
    out = run(a.n, a.sinks, a.seed, oracle_cache=a.oracle_cache, oracle_only=a.oracle_only)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

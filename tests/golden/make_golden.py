"""Generates the golden fixtures in this directory from the reference's own
code compiled for the host (oracle/_ref, built by oracle/build_ref.sh from the
reference sources):

  dropin12.npz   12^3 particles + periodic ghosts with the reference's pass
                 settings; the reference's tree build and P2P walk
                 (src/fmm.c via oracle/ref_walk_harness.c) give the particle
                 order, leaves and list chunks (LEN_TASK = 3000); the
                 reference's pair functions (src/gpu_kernel.impl.h, host
                 compiled) give the accelerations:
                   acc_clamp_cut    P2P_core_lite, FP64, GPUCUTOFF
                   acc_plummer      P2P_core_1, FP64 (zero beyond x > 2.8125)
                   acc_spi_fp32     P2P_core_lite, FP32, SPI tables, GPUCUTOFF
  pairs_known.npz single pairs through the reference's pair functions around
                 the softening length and the cutoff.

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "photons-on-mt3000_b200")]

from oracle import oracle as O  # noqa: E402
from photons_p2p import workloads as W  # noqa: E402

LEN_TASK = 3000


def make_dropin12():
    cfg = W.ref_dropin_config(12, 24, 32)
    pos = W.lattice_gaussian(12, 0.2, W.rng(1))
    allpos, tag = W.with_ghosts(pos, cfg)
    mass = 1.0 / pos.shape[1]
    walk = O.RefWalk("libref_walk.so")
    r = walk.run(allpos, tag, cfg.maxleaf, cfg.box, cfg.split_radius, cfg.cutoff_radius, cfg.eps,
                 mass, cfg.open_angle, LEN_TASK)
    tree_pos = allpos[:, r["perm"]]
    args = (tree_pos, r["leaf_ipart"], r["leaf_npart"], r["task_t"], r["task_s"])
    acc_cut, pairs = O.ref_p2p_lists("dp_cut", 0, cfg.eps, cfg.split_radius, mass, *args, chunk=LEN_TASK)
    acc_plum, _ = O.ref_p2p_lists("dp", 1, cfg.eps, cfg.split_radius, mass, *args, chunk=LEN_TASK)
    acc_spi, _ = O.ref_p2p_lists("sp_spi", 0, cfg.eps, cfg.split_radius, mass, *args, chunk=LEN_TASK)
    np.savez_compressed(
        os.path.join(HERE, "dropin12.npz"),
        input_pos=allpos, input_tag=tag, maxleaf=cfg.maxleaf, box=cfg.box,
        split_radius=cfg.split_radius, cutoff_radius=cfg.cutoff_radius, soften=cfg.eps,
        mass=mass, open_angle=cfg.open_angle, len_task=LEN_TASK,
        perm=r["perm"], leaf_ipart=r["leaf_ipart"], leaf_npart=r["leaf_npart"],
        leaf_active=r["leaf_active"], leaf_center=r["leaf_center"], leaf_width=r["leaf_width"],
        task_t=r["task_t"], task_s=r["task_s"], chunk_end=r["chunk_end"], pairs=pairs,
        acc_clamp_cut=acc_cut, acc_plummer=acc_plum, acc_spi_fp32=acc_spi)


def make_pairs():
    rs, eps = 0.01, 1e-3
    rows = []
    # below, at and above the softening length; across the cutoffs x = 2.25, 2.8125
    radii = [0.0, 2e-4, 9.99e-4, 1e-3, 1.001e-3, 5e-3, 0.01, 0.02, 0.0449, 0.045, 0.0451,
             0.0562, 0.05625, 0.0563, 0.07]
    for r in radii:
        ii = np.array([0.3, 0.4, 0.5])
        jj = ii + r * np.array([0.6, 0.0, 0.8])
        for variant, mode in (("dp_cut", 0), ("dp", 0), ("dp", 1)):
            out = O.ref_pair(variant, mode, eps, rs, ii, jj)
            rows.append((r, {"dp_cut": 2.8125, "dp": 0.0}[variant] if mode == 0 else 2.8125, mode,
                         ii, jj, out))
    np.savez_compressed(
        os.path.join(HERE, "pairs_known.npz"), soften=eps, split_radius=rs,
        r=np.array([x[0] for x in rows]), x_cut=np.array([x[1] for x in rows]),
        soft_mode=np.array([x[2] for x in rows], np.int32), ii=np.array([x[3] for x in rows]),
        jj=np.array([x[4] for x in rows]), out=np.array([x[5] for x in rows]))


if __name__ == "__main__":
    if not O.ref_available("libref_walk.so") or not O.ref_available("libref_pair.so"):
        sys.exit("oracle/_ref is not built; run oracle/build_ref.sh first")
    make_dropin12()
    make_pairs()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")

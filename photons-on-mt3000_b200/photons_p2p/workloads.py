"""Seeded synthetic particle sets for the P2P pass.

No public dataset is involved: each configuration below is generated from a
fixed seed (numpy PCG64, master seed 20261203, configuration k uses seed + k)
with the shapes, sizes and distributions the configurations name:

  c1_plain      32^3 lattice + Gaussian displacement (sigma 0.2 spacing),
                mesh 64, r_s 1.2 cells, cutoff 4.5 r_s, Plummer eps 1/40 spacing
  c2_clustered  256^3: 60% uniform, 40% in 2,000 NFW halos (c ~ U[4,12],
                truncated at r200, counts ~ M^-1.9 on [100, 20000] rescaled to
                the 40%), mesh 256, r_s 1.2 cells, eps 1/40 spacing
  c3_batching   512^3, same mix with 20,000 halos, mesh 512, leaf cap swept
  c4 boxes      serving ensemble boxes, n^3 with n log-uniform in [32, 128],
                lattice + Gaussian (sigma U[0.1,0.4] spacing) + 0-200 halos
  c5_stress     2^26: 90% in 500 NFW halos (c ~ U[10,20]), 10% uniform,
                eps 1/200 spacing, mesh 406, box origin shifted to 1.0
  ref_dropin    c1 particles with the reference's own force-pass settings
                (src/setparam.c:16-35: SoftenScale 0.03 cells clamp softening,
                r_s 1.25 cells, GPUCUTOFF x > 2.8125, open angle 0.4)

The configurations c1..c5 use x_cut = 2.25 (pair cutoff r = 4.5 r_s, equal to
the list cutoff) and open angle 0 so the lists hold every leaf pair within the
cutoff; the pass then equals a direct minimum-image sum of the truncated
kernel and can be checked against the FP64 direct oracle.
"""
from dataclasses import dataclass, replace

import numpy as np

MASTER_SEED = 20261203

SOFT_CLAMP = 0
SOFT_PLUMMER = 1


@dataclass(frozen=True)
class PassConfig:
    name: str
    n_side: int            # particles per side of the lattice-equivalent (spacing 1/n_side)
    mesh: int              # PM mesh cells per side (sets r_s)
    rs_cells: float        # split radius in mesh cells
    cutoff_rs: float       # list cutoff in units of r_s (cutoffRadius)
    soft_mode: int
    eps: float             # softening length (box units)
    x_cut: float           # per-pair cutoff on x = r/(2 r_s); 0 = none
    maxleaf: int
    open_angle: float
    box: float = 1.0
    origin: float = 0.0

    @property
    def split_radius(self):
        return self.rs_cells * self.box / self.mesh

    @property
    def cutoff_radius(self):
        return self.cutoff_rs * self.split_radius


def c1_config():
    return PassConfig("c1_plain_32^3", 32, 64, 1.2, 4.5, SOFT_PLUMMER, 1.0 / (40 * 32), 2.25, 32, 0.0)


def c2_config():
    return PassConfig("c2_clustered_256^3", 256, 256, 1.2, 4.5, SOFT_PLUMMER, 1.0 / (40 * 256), 2.25,
                      32, 0.0)


def c3_config(maxleaf=32):
    return PassConfig(f"c3_batching_512^3_leaf{maxleaf}", 512, 512, 1.2, 4.5, SOFT_PLUMMER,
                      1.0 / (40 * 512), 2.25, maxleaf, 0.0)


def c5_config():
    n_side = round((2 ** 26) ** (1.0 / 3.0))
    return PassConfig("c5_stress_2^26", n_side, 406, 1.2, 4.5, SOFT_PLUMMER, 1.0 / (200 * n_side),
                      2.25, 32, 0.0, box=1.0, origin=1.0)


def ref_dropin_config(n_side=32, mesh=64, maxleaf=32):
    """The reference's production force-pass settings (src/setparam.c:13-35,
    src/gpu_kernel.impl.h:192-196): SoftenScale = 1.5*0.02*L/mesh with clamp
    softening, r_s = 1.25 cells, cutoff 4.5 r_s, GPUCUTOFF at x > 2.8125,
    open angle 0.4."""
    return PassConfig(f"ref_dropin_{n_side}^3", n_side, mesh, 1.25, 4.5, SOFT_CLAMP,
                      1.5 * 0.02 / mesh, 2.8125, maxleaf, 0.4)


def rng(k):
    return np.random.Generator(np.random.PCG64(MASTER_SEED + k))


def lattice_gaussian(n_side, sigma_cells, g, box=1.0, origin=0.0):
    """Regular lattice (i+1/2)/n plus Gaussian displacement, wrapped."""
    i = (np.arange(n_side) + 0.5) / n_side
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()])
    pos += g.normal(0.0, sigma_cells / n_side, size=pos.shape)
    pos = np.mod(pos, 1.0) * box + origin
    return pos


def halo_counts(nhalo, total, g, lo=100.0, hi=20000.0, slope=1.9):
    """Counts drawn from dN/dM ~ M^-slope on [lo, hi], rescaled so they sum to
    `total` (the stated particle fraction); realised min/max are returned
    through the counts themselves."""
    a = 1.0 - slope
    u = g.random(nhalo)
    m = (lo ** a + u * (hi ** a - lo ** a)) ** (1.0 / a)
    n = np.floor(m * (total / m.sum())).astype(np.int64)
    n = np.maximum(n, 1)
    short = int(total - n.sum())
    if short > 0:
        idx = np.argsort(-(m * (total / m.sum()) - n))[:short]
        n[idx] += 1
    elif short < 0:
        for k in np.argsort(-n)[: -short]:
            n[k] -= 1
    return n


def nfw_halo(n, mass, conc, centre, g):
    """n particles of an NFW halo of mass `mass` (unit-mass box, mean density
    1), concentration conc, truncated at r200 = (3 M / (4 pi 200))^(1/3);
    radii from the inverse of m(s) = ln(1+s) - s/(1+s) (closed form through
    the Lambert W function), isotropic directions."""
    from scipy.special import lambertw

    r200 = (3.0 * mass / (4.0 * np.pi * 200.0)) ** (1.0 / 3.0)
    rs = r200 / conc
    mmax = np.log1p(conc) - conc / (1.0 + conc)
    u = g.random(n) * mmax
    w = lambertw(-np.exp(-u - 1.0), 0).real
    s = -1.0 / w - 1.0
    r = s * rs
    v = g.normal(size=(3, n))
    v /= np.linalg.norm(v, axis=0)
    return centre[:, None] + r * v


def clustered(n_total, frac_halo, nhalo, conc_range, g, box=1.0, origin=0.0):
    n_halo_total = int(round(frac_halo * n_total))
    n_uni = n_total - n_halo_total
    parts = [g.random((3, n_uni))]
    counts = halo_counts(nhalo, n_halo_total, g)
    centres = g.random((nhalo, 3))
    concs = g.uniform(conc_range[0], conc_range[1], nhalo)
    for k in range(nhalo):
        parts.append(nfw_halo(int(counts[k]), counts[k] / n_total, concs[k], centres[k], g))
    pos = np.concatenate(parts, axis=1)
    pos = np.mod(pos, 1.0) * box + origin
    return pos, counts


def c1_positions():
    cfg = c1_config()
    return lattice_gaussian(cfg.n_side, 0.2, rng(1))


def c2_positions(scale_side=None):
    """C2 particles. scale_side < 256 draws the same mix at a smaller size
    (halo count scaled by volume) for tests."""
    side = scale_side or 256
    nh = max(1, int(round(2000 * (side / 256.0) ** 3)))
    pos, _ = clustered(side ** 3, 0.4, nh, (4.0, 12.0), rng(2))
    return pos


def c3_positions():
    pos, _ = clustered(512 ** 3, 0.4, 20000, (4.0, 12.0), rng(3))
    return pos


def c5_positions(n_total=2 ** 26):
    cfg = c5_config()
    nh = max(1, int(round(500 * n_total / 2 ** 26)))
    pos, _ = clustered(n_total, 0.9, nh, (10.0, 20.0), rng(5), box=cfg.box, origin=cfg.origin)
    return pos


@dataclass
class ServingBox:
    box_id: int
    n_side: int
    pos: np.ndarray
    cfg: PassConfig


def c4_box(b, seed_offset=0, n_range=(32, 128)):
    """Box b of the serving ensemble (independent periodic unit box, its own
    seed): n^3 lattice points, n log-uniform in n_range, Gaussian displacement
    sigma ~ U[0.1, 0.4] spacing, plus 0-200 NFW halos (c ~ U[4, 12], counts
    from dN/dM ~ M^-1.9 on [100, 20000], total capped at n^3 / 2)."""
    g = np.random.Generator(np.random.PCG64([MASTER_SEED + 4, seed_offset, b]))
    n = int(round(np.exp(g.uniform(np.log(n_range[0]), np.log(n_range[1])))))
    sigma = g.uniform(0.1, 0.4)
    pos = lattice_gaussian(n, sigma, g)
    nh = int(g.integers(0, 201))
    if nh:
        cap = n ** 3 // 2
        lo, hi, a = 100.0, 20000.0, -0.9
        m = (lo ** a + g.random(nh) * (hi ** a - lo ** a)) ** (1.0 / a)
        cnt = np.maximum(1, np.round(m)).astype(np.int64)
        if cnt.sum() > cap:
            cnt = np.maximum(1, np.floor(cnt * (cap / cnt.sum()))).astype(np.int64)
        centres = g.random((nh, 3))
        concs = g.uniform(4.0, 12.0, nh)
        ntot = n ** 3 + int(cnt.sum())
        extra = [nfw_halo(int(cnt[k]), cnt[k] / ntot, concs[k], centres[k], g) for k in range(nh)]
        pos = np.mod(np.concatenate([pos] + extra, axis=1), 1.0)
    cfg = PassConfig(f"c4_box{b}_{n}^3", n, n, 1.2, 4.5, SOFT_PLUMMER, 1.0 / (40 * n), 2.25, 32, 0.0)
    return ServingBox(b, n, pos, cfg)


def c4_boxes(nbox=512, seed_offset=0, n_range=(32, 128)):
    """Serving ensemble: independent periodic unit boxes (c4_box 0..nbox-1)."""
    return [c4_box(b, seed_offset, n_range) for b in range(nbox)]


def with_ghosts(pos, cfg):
    """Append periodic ghost images within the list cutoff; returns (pos, tag)."""
    from .lists import make_ghosts

    gpos, _ = make_ghosts(pos, cfg.origin, cfg.box, cfg.cutoff_radius)
    allpos = np.concatenate([pos, gpos], axis=1)
    tag = np.concatenate([np.ones(pos.shape[1], np.int32), np.zeros(gpos.shape[1], np.int32)])
    return allpos, tag


def prepare(pos, cfg):
    """Ghosts + tree + lists for one pass (what PhotoNs' gravity step does
    before it calls the P2P entry point)."""
    from .lists import build_tree_lists

    allpos, tag = with_ghosts(pos, cfg)
    return build_tree_lists(allpos, tag, cfg.maxleaf, cfg.box, cfg.cutoff_radius, cfg.open_angle)


def scaled(cfg, **kw):
    return replace(cfg, **kw)

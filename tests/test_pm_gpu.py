"""The GPU PM long-range force (p2p_pm_*, csrc/p2p_pm.cu) against the PM
oracle (oracle/pm_oracle.py, PhotoNs' partmesh_kick force part,
src/partmesh.c:96-1450 with src/conv.f90:239-330).

The deposit's FP64 atomics sum in another order than the oracle's loop, and
cuFFT and numpy's FFT round differently; the rest is the same arithmetic in
the same order. Bounds: mass mesh within 1e-12 of its largest cell,
potential within 1e-11 of its largest value, accelerations within 1e-10 of
their rms.

Cases: the lattice drop-in workload (32^3 particles, mesh 64^3, r_s = 1.2
cells), a third of the particles tagged out (mesh 32^3), the clustered mix at
128^3 on a 128^3 mesh, no particles, and at the full 256^3 clustered size on
a 256^3 mesh the size-independent checks: total mass, total momentum zero,
the potential of the GPU's own deposit through the oracle's FFT and Green's
function, and 20,000 sampled particles interpolated from it."""
import numpy as np
import pytest

from oracle import pm_oracle as P
from photons_p2p import workloads as W
from photons_p2p.p2p import P2PError, ParticleMesh, Session

pytestmark = pytest.mark.gpu


def run(pos, tag, mass, nmesh, box, rs):
    import torch

    dev = torch.device("cuda", 0)
    with Session(0) as s, ParticleMesh(s, nmesh, box, rs) as pm:
        p = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).to(dev)
        t = None if tag is None else torch.from_numpy(np.asarray(tag, np.int32)).to(dev)
        acc = torch.empty_like(p)
        torch.cuda.synchronize()
        pm.forces(p, t, mass, acc)
        mass_mesh, phi = pm.download()
        ms = pm.timings()
        return acc.cpu().numpy(), mass_mesh, phi, ms


def check_against_oracle(pos, tag, mass, nmesh, box, rs):
    acc, mass_mesh, phi, _ = run(pos, tag, mass, nmesh, box, rs)
    ref_mass = P.deposit(pos, tag, mass, nmesh, box)
    assert np.abs(mass_mesh - ref_mass).max() <= 1e-12 * np.abs(ref_mass).max()
    ref_phi = P.potential(P.density(ref_mass, box), box, rs)
    assert np.abs(phi - ref_phi).max() <= 1e-11 * np.abs(ref_phi).max()
    ref_acc = P.interpolate(P.gradient(ref_phi, box), pos, tag, nmesh, box)
    rms = np.sqrt((ref_acc ** 2).sum(0).mean())
    assert np.abs(acc - ref_acc).max() <= 1e-10 * rms
    if tag is not None:
        assert np.all(acc[:, np.asarray(tag) != 1] == 0.0)
    return acc


def test_lattice_drop_in_config(gpu):
    cfg = W.c1_config()
    pos = W.c1_positions()
    check_against_oracle(pos, None, 1.0 / pos.shape[1], cfg.mesh, cfg.box, cfg.split_radius)


def test_tagged_particles(gpu):
    pos = W.lattice_gaussian(24, 0.3, W.rng(11))
    tag = (W.rng(12).uniform(size=pos.shape[1]) < 0.67).astype(np.int32)
    check_against_oracle(pos, tag, 1.0 / pos.shape[1], 32, 1.0, 1.2 / 32)


def test_clustered_128(gpu):
    pos = W.c2_positions(128)
    check_against_oracle(pos, None, 1.0 / pos.shape[1], 128, 1.0, 1.2 / 128)


def test_no_particles(gpu):
    acc, mass_mesh, phi, _ = run(np.zeros((3, 0)), None, 1.0, 16, 1.0, 1.2 / 16)
    assert acc.shape == (3, 0) and not mass_mesh.any() and not phi.any()


def test_bad_mesh_rejected(gpu):
    with Session(0) as s:
        for n in (3, 7, 2048):
            with pytest.raises(P2PError):
                ParticleMesh(s, n, 1.0, 0.01)


def test_clustered_256_full_size(gpu):
    cfg = W.c2_config()
    pos = W.c2_positions()
    n = pos.shape[1]
    mass = 1.0 / n
    acc, mass_mesh, phi, ms = run(pos, None, mass, cfg.mesh, cfg.box, cfg.split_radius)
    assert abs(mass_mesh.sum() - 1.0) < 1e-9
    mag = np.linalg.norm(acc, axis=0)
    assert np.abs(acc.sum(1)).max() < 1e-9 * mag.sum()
    ref_phi = P.potential(P.density(mass_mesh, cfg.box), cfg.box, cfg.split_radius)
    assert np.abs(phi - ref_phi).max() <= 1e-11 * np.abs(ref_phi).max()
    sample = W.rng(13).choice(n, 20000, replace=False)
    ref = P.interpolate(P.gradient(ref_phi, cfg.box), pos[:, sample], None, cfg.mesh, cfg.box)
    rms = np.sqrt((ref ** 2).sum(0).mean())
    assert np.abs(acc[:, sample] - ref).max() <= 1e-10 * rms
    assert ms["total"] > 0

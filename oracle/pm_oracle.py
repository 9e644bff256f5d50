"""TEST INFRASTRUCTURE ONLY: numpy restatement of PhotoNs' particle-mesh (PM)
long-range force for one periodic domain, the checker of the GPU PM
(photons-on-mt3000_b200/csrc/p2p_pm.cu). Only tests/ and bench.py's CPU leg
use it.

The reference splits the mesh over MPI sub-domains with halos; on a single
periodic domain every halo read is a periodic wrap, which is what this
restatement does. Steps (FP64 throughout):

  deposit   cloud-in-cell: particle n (tag 1) at cell i = int(x N / L) adds
            m (1 - w)(...) to its cell and m w (...) to the neighbour on the
            side of its offset w = |x N / L - (i + 1/2)|, per axis
            (src/partmesh.c:96-204), then every cell times (N / L)^3, mass
            per cell to density (src/partmesh.c:319-327)
  convolve  real-to-complex FFT, times G(l, m, n) = pref exp(-k2 s2) / k2 /
            (sinc_x sinc_y sinc_z)^4 with k2 = l^2 + m^2 + n^2 (integer wave
            numbers, l > N/2 wrapped to l - N), s2 = (2 pi r_s / L)^2,
            pref = L^2 / (pi N^3), sinc(l) = sin(pi l / N) / (pi l / N) (1 at
            l = 0), zero mode 0; complex-to-real inverse without normalisation
            (src/conv.f90:239-330)
  gradient  at each of the particle's 8 cloud-in-cell cells and per axis,
            f1 h (M[+1] - M[-1]) - f2 h (M[+2] - M[-2]) with f1 = 4/3,
            f2 = 1/6, h = N / (2 L) (src/partmesh.c:1116-1262)
  interp    the 8 cell values weighted as in the deposit
            (src/partmesh.c:1415-1450)
The result is the long-range acceleration of every particle with tag 1
(0 for others), in the reference's units.
"""
import numpy as np


def cic_cells(pos, nmesh, box):
    """Per particle and axis: cell index, neighbour index (both wrapped), and
    the neighbour's weight w (the cell's weight is 1 - w)."""
    norm = nmesh / box
    delta = 1.0 / norm
    i = (pos * norm).astype(np.int64)  # (int) truncation; pos >= 0
    w = (pos - (i + 0.5) * delta) * norm
    nb = np.where(w > 0, i + 1, i - 1)
    w = np.abs(w)
    return np.mod(i, nmesh), np.mod(nb, nmesh), w


def deposit(pos, tag, mass, nmesh, box):
    """(nmesh, nmesh, nmesh) mass per cell, index [x, y, z]."""
    sel = tag == 1 if tag is not None else np.ones(pos.shape[1], bool)
    c, nb, w = cic_cells(pos[:, sel], nmesh, box)
    mesh = np.zeros((nmesh,) * 3)
    for sx in (0, 1):
        ix = nb[0] if sx else c[0]
        wx = w[0] if sx else 1.0 - w[0]
        for sy in (0, 1):
            iy = nb[1] if sy else c[1]
            wy = w[1] if sy else 1.0 - w[1]
            for sz in (0, 1):
                iz = nb[2] if sz else c[2]
                wz = w[2] if sz else 1.0 - w[2]
                np.add.at(mesh, (ix, iy, iz), mass * wx * wy * wz)
    return mesh


def green(nmesh, box, split_radius):
    """The Green's function on the r2c half spectrum (last axis halved)."""
    n = nmesh
    l = np.arange(n)
    l = np.where(l > n // 2, l - n, l).astype(np.float64)
    lz = np.arange(n // 2 + 1).astype(np.float64)

    def sinc(v):
        a = np.pi * v / n
        out = np.ones_like(v)
        nz = v != 0
        out[nz] = np.sin(a[nz]) / a[nz]
        return out

    fx, fy, fz = sinc(l)[:, None, None], sinc(l)[None, :, None], sinc(lz)[None, None, :]
    k2 = l[:, None, None] ** 2 + l[None, :, None] ** 2 + lz[None, None, :] ** 2
    s2 = (2 * np.pi * split_radius / box) ** 2
    pref = box * box / (np.pi * n ** 3)
    with np.errstate(divide="ignore", invalid="ignore"):
        ff = 1.0 / (fx * fy * fz)
        g = pref * np.exp(-k2 * s2) / k2 * ff ** 4
    g[0, 0, 0] = 0.0
    return g


def density(mesh, box):
    """Mass per cell to density: times (N / L)^3 (src/partmesh.c:319-327)."""
    renormal = mesh.shape[0] / box
    return mesh * (renormal * renormal * renormal)


def potential(rho_mesh, box, split_radius):
    n = rho_mesh.shape[0]
    rho = np.fft.rfftn(rho_mesh)
    return np.fft.irfftn(rho * green(n, box, split_radius), s=rho_mesh.shape, axes=(0, 1, 2)) * n ** 3


def gradient(phi, box):
    """(3, n, n, n): the 4-point difference along each axis, periodic."""
    n = phi.shape[0]
    h = 0.5 * n / box
    f1, f2 = 4.0 / 3.0, 1.0 / 6.0
    out = np.empty((3,) + phi.shape)
    for a in range(3):
        d1 = np.roll(phi, -1, axis=a) - np.roll(phi, 1, axis=a)
        d2 = np.roll(phi, -2, axis=a) - np.roll(phi, 2, axis=a)
        out[a] = f1 * h * d1 - f2 * h * d2
    return out


def interpolate(grad, pos, tag, nmesh, box):
    n = pos.shape[1]
    sel = tag == 1 if tag is not None else np.ones(n, bool)
    c, nb, w = cic_cells(pos[:, sel], nmesh, box)
    acc = np.zeros((3, n))
    out = np.zeros((3, int(sel.sum())))
    for sx in (0, 1):
        ix = nb[0] if sx else c[0]
        wx = w[0] if sx else 1.0 - w[0]
        for sy in (0, 1):
            iy = nb[1] if sy else c[1]
            wy = w[1] if sy else 1.0 - w[1]
            for sz in (0, 1):
                iz = nb[2] if sz else c[2]
                wz = w[2] if sz else 1.0 - w[2]
                wt = wx * wy * wz
                for a in range(3):
                    out[a] += wt * grad[a][ix, iy, iz]
    acc[:, sel] = out
    return acc


def pm_forces(pos, tag, mass, nmesh, box, split_radius):
    """Long-range accelerations (3, n) of the particles with tag 1."""
    mesh = density(deposit(pos, tag, mass, nmesh, box), box)
    phi = potential(mesh, box, split_radius)
    return interpolate(gradient(phi, box), pos, tag, nmesh, box)

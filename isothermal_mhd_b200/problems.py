"""Initial conditions for periodic boxes (host side, numpy float64).

Every function returns ``(q, bface, qpass)`` with shapes ``(7, nz, ny, nx)``,
``(3, nz, ny, nx)`` and ``(npass, nz, ny, nx)`` (x fastest, unpadded); use
:func:`pad` to add the reference's ghost layers.  Cell (i,j,k), 0-based, has
its centre at ((i+1/2) dx, (j+1/2) dx, (k+1/2) dx) with dx = 1/max(n), face B
``bface[d]`` sits on the upper face of the cell, and the cell-centred field is
the average of the two faces, as the reference's test problems set it
(e.g. 3D_MPI/src/init_domain_mod.f90:539-549).
"""
from __future__ import annotations

import numpy as np

TWOPI = 2.0 * np.pi


def _grid(n):
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    dx = 1.0 / max(nx, ny, nz)
    xc = (np.arange(nx) + 0.5) * dx
    yc = (np.arange(ny) + 0.5) * dx
    zc = (np.arange(nz) + 0.5) * dx
    return (nx, ny, nz), dx, xc, yc, zc


def cell_centred_b(bface):
    """Cell-centred B as the face average (init_domain_mod.f90:539-549)."""
    bx, by, bz = bface
    return np.stack([0.5 * (bx + np.roll(bx, 1, axis=2)),
                     0.5 * (by + np.roll(by, 1, axis=1)),
                     0.5 * (bz + np.roll(bz, 1, axis=0))])


def curl_edge(ax, ay, az, dx):
    """Face B of the discrete curl of an edge-centred vector potential.

    ax[k,j,i] lives on edge (i, j+1/2, k+1/2), ay on (i+1/2, j, k+1/2), az on
    (i+1/2, j+1/2, k); the result's discrete divergence telescopes to zero.
    """
    bx = (az - np.roll(az, 1, axis=1)) / dx - (ay - np.roll(ay, 1, axis=0)) / dx
    by = (ax - np.roll(ax, 1, axis=0)) / dx - (az - np.roll(az, 1, axis=2)) / dx
    bz = (ay - np.roll(ay, 1, axis=2)) / dx - (ax - np.roll(ax, 1, axis=1)) / dx
    return np.stack([bx, by, bz])


def smooth_wave_box(n, npass=1):
    """64^3 parity configuration: rho = 1 + 0.1 sin 2pi x,
    v = 0.1 (sin 2pi y, sin 2pi z, sin 2pi x), B = (1/sqrt2, 1/sqrt2, 0) + curl A
    with A = 0.05 (cos 2pi z, cos 2pi x, cos 2pi y) on cell edges, and one
    passive scalar equal to 1 for x < 1/2 and 0 elsewhere."""
    (nx, ny, nz), dx, xc, yc, zc = _grid(n)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    rho = 1.0 + 0.1 * np.sin(TWOPI * X)
    vx = 0.1 * np.sin(TWOPI * Y)
    vy = 0.1 * np.sin(TWOPI * Z)
    vz = 0.1 * np.sin(TWOPI * X)
    xf = (np.arange(nx) + 1.0) * dx
    yf = (np.arange(ny) + 1.0) * dx
    zf = (np.arange(nz) + 1.0) * dx
    shape = (nz, ny, nx)
    ax = np.broadcast_to(0.05 * np.cos(TWOPI * zf)[:, None, None], shape)
    ay = np.broadcast_to(0.05 * np.cos(TWOPI * xf)[None, None, :], shape)
    az = np.broadcast_to(0.05 * np.cos(TWOPI * yf)[None, :, None], shape)
    b = curl_edge(ax, ay, az, dx)
    b[0] += 1.0 / np.sqrt(2.0)
    b[1] += 1.0 / np.sqrt(2.0)
    q = np.empty((7,) + shape)
    q[0] = rho
    q[1], q[2], q[3] = rho * vx, rho * vy, rho * vz
    q[4:7] = cell_centred_b(b)
    p = np.zeros((npass,) + shape)
    if npass:
        p[0] = np.where(X < 0.5, 1.0, 0.0)
        for m in range(1, npass):
            p[m] = np.where(Y < 0.5, 1.0, 0.0)
    return q, b, p


def uniform_box(n, rho=1.0, v=(0.0, 0.0, 0.0), b0=(1.0, 0.0, 0.0), npass=0, pass_value=1.0):
    (nx, ny, nz), dx, xc, yc, zc = _grid(n)
    shape = (nz, ny, nx)
    q = np.zeros((7,) + shape)
    q[0] = rho
    for d in range(3):
        q[1 + d] = rho * v[d]
        q[4 + d] = b0[d]
    b = np.stack([np.full(shape, float(b0[d])) for d in range(3)])
    p = np.full((npass,) + shape, float(pass_value))
    return q, b, p


def alfven_wave(n, npass=0):
    """Standing Alfven wave of init_domain_mod.f90:483-553: rho = 1,
    v_z = B_z = 0.01 sin(2pi(2x + 2y)), B_x = 1."""
    (nx, ny, nz), dx, xc, yc, zc = _grid(n)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    shape = (nz, ny, nx)
    kx, ky = 2.0 * TWOPI, 2.0 * TWOPI
    vz = 0.01 * 1.0 * np.sin(kx * X + ky * Y)
    q = np.zeros((7,) + shape)
    q[0] = 1.0
    q[3] = vz
    b = np.zeros((3,) + shape)
    b[0] = 1.0
    b[2] = vz
    q[4:7] = cell_centred_b(b)
    p = np.zeros((npass,) + shape)
    return q, b, p


def shock_tube(n, axis=0, left=(1.0, 0.0, 0.0, 0.0, 0.75, 1.0, 0.0), right=(0.2, 0.0, 0.0, 0.0, 0.75, -1.0, 0.0),
               npass=0):
    """Planar Riemann problem along `axis` (cyclic frame: normal, t1, t2).

    left/right = (rho, v_n, v_t1, v_t2, B_n, B_t1, B_t2); both interfaces of
    the periodic box (x_n = 1/2 and x_n = 0) are discontinuities.
    """
    (nx, ny, nz), dx, xc, yc, zc = _grid(n)
    shape = (nz, ny, nx)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    coord = (X, Y, Z)[axis]
    L = coord < 0.5
    q = np.zeros((7,) + shape)
    b = np.zeros((3,) + shape)
    comps = [axis, (axis + 1) % 3, (axis + 2) % 3]
    for side, st in ((L, left), (~L, right)):
        rho, vn, vt1, vt2, bn, bt1, bt2 = st
        q[0][side] = rho
        for r, vv in zip(comps, (vn, vt1, vt2)):
            q[1 + r][side] = rho * vv
        for r, bb in zip(comps, (bn, bt1, bt2)):
            b[r][side] = bb
    q[4:7] = cell_centred_b(b)
    p = np.zeros((npass,) + shape)
    if npass:
        p[0] = L.astype(float)
    return q, b, p


def pad(a, g):
    """Add g periodic ghost layers on each side of every spatial axis
    (the reference's layout after boundary_conditions())."""
    if g == 0:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(np.pad(a, ((0, 0), (g, g), (g, g), (g, g)), mode="wrap"))


def unpad(a, g):
    if g == 0:
        return a
    return a[:, g:-g, g:-g, g:-g]

"""Turbulence forcing fields (host side) for the kick of add_random_force.

The reference regenerates a Gaussian random velocity field after every drive
step (generate_rand_force, 3D_MPI/src/turb_driver_mod.f90:197-391) and adds it,
normalised to a fixed kinetic-energy injection with zero net momentum, once
per dt_turb (add_random_force :395-457).  The kick itself runs on the GPU
(imhd_step with drive_next = 1); this module only produces the field delv.

:class:`OUForcing` is the solenoidal Ornstein-Uhlenbeck generator of the
driven-turbulence configuration: Fourier amplitudes on the shells
kmin <= |k| <= kmax (integer wave vectors of the unit box), projected
perpendicular to k, evolved as an OU process with correlation time `tcorr`
and evaluated on the cell centres with a real inverse FFT.
"""
from __future__ import annotations

import numpy as np

try:
    import scipy.fft as _fft
    _HAVE_SCIPY = True
except Exception:  # pragma: no cover
    import numpy.fft as _fft
    _HAVE_SCIPY = False


def shell_modes(kmin=1.0, kmax=2.0):
    """Integer wave vectors with kmin <= |k| <= kmax, one of each +/- pair
    (the member with its first non-zero component positive)."""
    r = int(np.floor(kmax))
    out = []
    for kz in range(-r, r + 1):
        for ky in range(-r, r + 1):
            for kx in range(-r, r + 1):
                k2 = kx * kx + ky * ky + kz * kz
                if k2 < kmin * kmin - 1e-12 or k2 > kmax * kmax + 1e-12:
                    continue
                first = next(c for c in (kx, ky, kz) if c != 0)
                if first > 0:
                    out.append((kx, ky, kz))
    return np.array(out, dtype=np.int64)


class OUForcing:
    """Solenoidal Gaussian random field with Ornstein-Uhlenbeck time correlation."""

    def __init__(self, n, kmin=1.0, kmax=2.0, tcorr=0.5, seed=20261203, solenoidal=True):
        self.n = (n, n, n) if np.isscalar(n) else tuple(n)
        self.modes = shell_modes(kmin, kmax)
        self.tcorr = float(tcorr)
        self.solenoidal = solenoidal
        self.rng = np.random.default_rng(seed)
        self.amp = self._draw()          # stationary start

    def _project(self, a):
        if not self.solenoidal:
            return a
        k = self.modes.astype(np.float64)
        khat = k / np.linalg.norm(k, axis=1, keepdims=True)
        return a - khat * np.sum(khat * a, axis=1, keepdims=True)

    def _draw(self):
        m = len(self.modes)
        a = (self.rng.standard_normal((m, 3)) + 1j * self.rng.standard_normal((m, 3))) / np.sqrt(2.0)
        return self._project(a)

    def advance(self, dt):
        """OU update a <- f a + sqrt(1 - f^2) xi, f = exp(-dt/tcorr)."""
        f = np.exp(-float(dt) / self.tcorr)
        self.amp = f * self.amp + np.sqrt(max(0.0, 1.0 - f * f)) * self._draw()

    def device_modes(self, rms=1.0):
        """(kvec int32 (m,3), amp float64 (m,6), scale) for imhd_fourier_field:
        the same field as :meth:`field` on the device.  The cell-centre phase is
        applied there; the rms of |v| over the grid is 2 sum_m |a_m|^2 exactly
        for wave numbers below the Nyquist limit, so the scale is analytic."""
        kv = self.modes.astype(np.int32)
        amp = np.empty((len(kv), 6))
        amp[:, 0::2] = self.amp.real
        amp[:, 1::2] = self.amp.imag
        power = 2.0 * float(np.sum(np.abs(self.amp) ** 2))
        return kv, amp, (rms / np.sqrt(power) if power > 0 else 0.0)

    def field(self, rms=1.0):
        """Real field v(x) = sum_k 2 Re(a_k exp(2 pi i k.x)) on the cell centres,
        shape (3, nz, ny, nx), scaled to the given rms of |v|."""
        nx, ny, nz = self.n
        L = 1.0 / max(nx, ny, nz)           # dx; box length along axis d is n_d * dx
        out = np.empty((3, nz, ny, nx))
        for c in range(3):
            spec = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
            for (kx, ky, kz), a in zip(self.modes, self.amp[:, c]):
                # cell centres sit at (i+1/2) dx: fold the half-cell phase into a
                ph = np.exp(1j * np.pi * (kx / nx + ky / ny + kz / nz) * (max(nx, ny, nz) * L))
                if kx > 0:      # irfftn adds the conjugate (-k) half itself
                    spec[kz % nz, ky % ny, kx] += a * ph
                else:   # kx == 0: Hermitian pair in the kx = 0 plane
                    spec[kz % nz, ky % ny, 0] += a * ph
                    spec[(-kz) % nz, (-ky) % ny, 0] += np.conj(a * ph)
            if _HAVE_SCIPY:
                out[c] = _fft.irfftn(spec, s=(nz, ny, nx), axes=(0, 1, 2), norm="forward", workers=-1)
            else:
                out[c] = _fft.irfftn(spec, s=(nz, ny, nx), axes=(0, 1, 2), norm="forward")
        cur = np.sqrt(np.mean(np.sum(out * out, axis=0)))
        if cur > 0:
            out *= rms / cur
        return out


def turbulent_box(n, mach=2.0, b0=(0.5, 0.0, 0.0), npass=2, sound_speed=1.0, seed=20261203, forcing=None):
    """Driven-turbulence initial state: rho = 1, uniform B0, velocity = one
    realisation of the OU forcing field scaled to rms Mach `mach`, passive
    scalars uniform random on [0, 1) from `seed`."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
    shape = (nz, ny, nx)
    f = forcing or OUForcing(n, seed=seed)
    v = f.field(rms=mach * sound_speed)
    q = np.zeros((7,) + shape)
    q[0] = 1.0
    q[1:4] = v
    for d in range(3):
        q[4 + d] = b0[d]
    b = np.stack([np.full(shape, float(b0[d])) for d in range(3)])
    rng = np.random.default_rng(seed + 1)
    p = rng.random((npass,) + shape)
    return q, b, p

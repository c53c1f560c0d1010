"""Host-side logic without a GPU: initial conditions, layouts, the forcing
generator and the driver loop (against a fake box)."""
import numpy as np
import pytest

from isothermal_mhd_b200 import driver, forcing, problems


def divb(b):
    bx, by, bz = b
    return (bx - np.roll(bx, 1, 2)) + (by - np.roll(by, 1, 1)) + (bz - np.roll(bz, 1, 0))


def test_smooth_box_is_divergence_free_and_face_averaged():
    q, b, p = problems.smooth_wave_box((16, 20, 12), npass=1)
    assert np.max(np.abs(divb(b))) < 1e-12
    np.testing.assert_array_equal(q[4:7], problems.cell_centred_b(b))
    assert q.shape == (7, 12, 20, 16) and p.shape == (1, 12, 20, 16)
    assert set(np.unique(p)) == {0.0, 1.0}


def test_pad_roundtrip_is_periodic():
    a = np.random.default_rng(0).random((3, 5, 6, 7))
    pa = problems.pad(a, 2)
    assert pa.shape == (3, 9, 10, 11)
    np.testing.assert_array_equal(problems.unpad(pa, 2), a)
    np.testing.assert_array_equal(pa[:, :, :, 0], pa[:, :, :, 7])   # ghost i=-1 is image of i=n-1


def test_ou_field_is_solenoidal_and_normalised():
    n = 32
    f = forcing.OUForcing(n, seed=7)
    v = f.field(rms=2.0)
    assert np.isclose(np.sqrt(np.mean(np.sum(v * v, axis=0))), 2.0)
    # spectral divergence vanishes
    k = np.fft.fftfreq(n) * n
    K = np.meshgrid(k, k, k, indexing="ij")   # (kz, ky, kx)
    div = K[2] * np.fft.fftn(v[0]) + K[1] * np.fft.fftn(v[1]) + K[0] * np.fft.fftn(v[2])
    assert np.max(np.abs(div)) < 1e-8 * np.max(np.abs(np.fft.fftn(v[0])))
    # only shells 1 <= |k| <= 2 carry power
    P = np.abs(np.fft.fftn(v[0])) ** 2
    kk = np.sqrt(K[0] ** 2 + K[1] ** 2 + K[2] ** 2)
    assert P[(kk > 2.01) | (kk < 0.99)].sum() < 1e-20 * P.sum() + 1e-30


def test_ou_field_equals_direct_mode_sum():
    # v(x) = sum_m 2 Re(a_m exp(2 pi i k_m.x)) at the cell centres of a
    # non-cubic box, and the analytic scale of device_modes gives its rms
    n = (10, 8, 6)
    f = forcing.OUForcing(n, seed=4)
    v = f.field(rms=1.5)
    kv, amp, scale = f.device_modes(rms=1.5)
    nx, ny, nz = n
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    d = np.zeros((3, nz, ny, nx))
    for (kx, ky, kz), a in zip(kv, amp):
        ph = 2 * np.pi * (kx * x + ky * y + kz * z)
        for c in range(3):
            d[c] += 2.0 * (a[2 * c] * np.cos(ph) - a[2 * c + 1] * np.sin(ph))
    np.testing.assert_allclose(v, scale * d, rtol=0, atol=1e-12)


def test_ou_process_decorrelates_with_tcorr():
    f = forcing.OUForcing(16, tcorr=0.5, seed=3)
    a0 = f.amp.copy()
    f.advance(0.05)
    c_short = np.real(np.vdot(a0, f.amp)) / np.vdot(a0, a0).real
    for _ in range(40):
        f.advance(0.05)
    c_long = np.real(np.vdot(a0, f.amp)) / np.vdot(a0, a0).real
    assert c_short > 0.8 and abs(c_long) < 0.4


def test_turbulent_box_mach_and_passives():
    q, b, p = forcing.turbulent_box(16, mach=2.0, npass=2, seed=11)
    v = q[1:4] / q[0]
    assert np.isclose(np.sqrt(np.mean(np.sum(v * v, axis=0))), 2.0)
    assert p.shape == (2, 16, 16, 16) and p.min() >= 0 and p.max() < 1
    assert np.all(q[4] == 0.5) and np.all(b[0] == 0.5)


class FakeBox:
    """Records the dt / drive sequence the driver produces."""

    class C:
        dt_turb = 0.05

    def __init__(self, dt_next):
        self.cfg = self.C()
        self.calls = []
        self.forces = 0
        self.dt_next = dt_next

    def step(self, dt, drive):
        self.calls.append((dt, drive))
        return self.dt_next * (0.5 if drive else 1.0)

    def set_force(self, f):
        self.forces += 1


def test_driver_matches_reference_schedule():
    # dt = 0.02 each step; drive when t_turb in (t, t + dt]; dt halves on a drive
    box = FakeBox(0.02)
    rec = driver.run(box, t_end=0.2, maxsteps=1000, dt0=0.02, forcing=lambda: None, dt_turb=0.05)
    t = 0.0
    t_turb = 0.05
    for dt, drive in box.calls:
        expect = (t_turb > t) and (t_turb <= t + (2 * dt if drive else dt))
        assert drive == expect
        if drive:
            t_turb = max(t_turb + 0.05, t + 1e-2 * 2 * dt)
        t += dt
    assert abs(rec.t - 0.2) < 1e-12
    assert box.forces == 1 + len(rec.drive_steps)


def test_driver_step_count_rule():
    box = FakeBox(1e-3)
    rec = driver.run(box, t_end=10.0, maxsteps=11)
    assert rec.steps == 10 and len(box.calls) == 10
    assert box.calls[0][0] == 1e-15

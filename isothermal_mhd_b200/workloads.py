"""Seeded synthetic workloads of many boxes: the mixed-size batch and the
request stream of the serving loop.

Every box is driven isothermal-MHD turbulence on its own periodic unit-edge
grid: rho = 1, cs = 1, a uniform field B0, an initial velocity that is one
realisation of the solenoidal OU forcing field (shells 1 <= |k| <= 2) scaled
to the box's rms Mach number, and a forcing field from the next realisation.
Both fields are evaluated on the device from their Fourier modes
(imhd_fourier_field), so building a box needs no host arrays.

The forcing amplitude is set through the energy-injection rate of
add_random_force (turb_driver_mod.f90:395-457): edot = mach^3, the
dissipation rate v^3/L of turbulence at rms speed v = mach * cs on the box
scale L = 1.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import forcing

C3_EDGES = (32, 48, 64, 96, 128)
C4_EDGES = (32, 64, 96, 128, 192)
C4_WEIGHTS = (0.35, 0.30, 0.20, 0.10, 0.05)


@dataclass
class BoxSpec:
    n: int
    b0: tuple
    mach: float
    riemann: str = "roe"
    npass: int = 0
    steps: int = 50
    seed: int = 0
    dt_turb: float = 0.05
    arrival: float = 0.0          # seconds after the start of a request stream
    recon: str = "plm"

    @property
    def edot(self):
        return self.mach ** 3

    @property
    def cells(self):
        return self.n ** 3

    def fields(self):
        """(kv, amp_velocity, scale_velocity, amp_force, scale_force): Fourier
        modes of the initial velocity (rms = mach) and of the force field
        (rms 1; add_random_force rescales it to edot)."""
        f = forcing.OUForcing(self.n, seed=self.seed)
        kv, av, sv = f.device_modes(rms=self.mach)
        f.advance(self.dt_turb)
        _, af, sf = f.device_modes(rms=1.0)
        return kv, av, sv, af, sf


def _b0(rng, lo=0.1, hi=2.0):
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    return tuple(float(x) for x in rng.uniform(lo, hi) * d)


def batched_boxes(nbox=512, steps=50, seed=20261203, edges=C3_EDGES):
    """Mixed-size batch: edges uniform on `edges`, |B0| uniform on [0.1, 2]
    along a random unit vector, rms Mach uniform on [0.5, 5], Roe, no passive
    scalars, `steps` steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nbox):
        out.append(BoxSpec(n=int(rng.choice(edges)), b0=_b0(rng), mach=float(rng.uniform(0.5, 5.0)), riemann="roe",
                           npass=0, steps=steps, seed=seed + 1 + i))
    return out


@dataclass
class RequestStream:
    specs: list = field(default_factory=list)

    @property
    def total_cells_steps(self):
        return sum(s.cells * s.steps for s in self.specs)


def request_stream(nreq=400, rate=200.0, seed=20261204, edges=C4_EDGES, weights=C4_WEIGHTS, npass=0):
    """Poisson arrivals at `rate` requests/s; edge from `edges` with
    `weights`; steps uniform on [20, 200]; |B0| and Mach as the batch;
    Roe or HLLD with probability 1/2 each."""
    rng = np.random.default_rng(seed)
    t = 0.0
    specs = []
    for i in range(nreq):
        t += float(rng.exponential(1.0 / rate))
        specs.append(BoxSpec(n=int(rng.choice(edges, p=weights)), b0=_b0(rng), mach=float(rng.uniform(0.5, 5.0)),
                             riemann="roe" if rng.random() < 0.5 else "hlld", npass=npass,
                             steps=int(rng.integers(20, 201)), seed=seed + 1 + i, arrival=t))
    return RequestStream(specs)

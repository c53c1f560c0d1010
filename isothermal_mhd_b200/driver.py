"""Host time loop mirroring the reference driver (3D_MPI/src/driver.f90:35-186).

Per step: decide whether this is a drive step (driver.f90:57-70: t_turb in
(t_old, t_old + dt], then t_turb advances and dt halves), call
:meth:`Box.step` (copy_velocity, vanleer_solve_3d, passive_solve_3d, the
periodic fill and compute_new_time_step in one C-ABI call), advance the clock,
regenerate the force after a drive step (driver.f90:102-111), and clamp the
new dt to the remaining time (finish_mpi_reductions, driver.f90:475).
The first step runs with dt = 1e-15 as main_init sets it (driver.f90:249).
"""
from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class RunRecord:
    t: float = 0.0
    steps: int = 0
    dts: list = field(default_factory=list)
    drive_steps: list = field(default_factory=list)


def run(box, t_end, maxsteps, dt0=1.0e-15, forcing=None, dt_turb=None, t0=0.0, record_dt=True, on_step=None,
        seeds=(1234, 5678, 9123), k_max=2):
    """Advance `box` like the reference's main loop; returns a RunRecord.

    maxsteps follows the reference's counter: tsteps starts at 1 and the loop
    runs while tsteps < maxsteps, so maxsteps = N + 1 gives N steps.
    `forcing` is a callable returning the next delv field (3, nz+2g, ny+2g,
    nx+2g), "ref" for the reference's generator on the device (seeded with
    `seeds`, a new field before the run and after every drive step, as
    driver.f90:336-339 and :102-105), "device" for a force field already on
    the device (set by Box.fourier_field; every drive reuses it), or None for
    an undriven run.
    """
    rec = RunRecord(t=t0)
    t_sim = t0
    tsteps = 1
    my_dt = dt0
    dt_turb = box.cfg.dt_turb if dt_turb is None else dt_turb
    t_turb = t_sim + dt_turb
    host_field = callable(forcing)
    ref = forcing == "ref"
    if host_field:
        box.set_force(forcing())
    if ref:
        box.init_turb(seeds, k_max)
        box.generate_force()
    while t_sim < t_end and tsteps < maxsteps:
        t_old = t_sim
        drive_next = False
        if forcing is not None and (t_turb > t_old) and (t_turb <= t_old + my_dt):
            drive_next = True
            t_turb = max(t_turb + dt_turb, t_sim + 1.0e-2 * my_dt)
            my_dt = 0.5 * my_dt
        dt_new = box.step(my_dt, drive_next)
        if record_dt:
            rec.dts.append(my_dt)
        if drive_next:
            rec.drive_steps.append(tsteps)
        t_sim = t_sim + my_dt
        tsteps += 1
        if drive_next and host_field:
            box.set_force(forcing())
        if drive_next and ref:
            box.generate_force()
        my_dt = min(t_end - t_sim, dt_new)
        if on_step is not None:
            on_step(tsteps, t_sim, my_dt)
    rec.t = t_sim
    rec.steps = tsteps - 1
    return rec

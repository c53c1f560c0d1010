"""One periodic box split into z slabs over ranks, with halo planes.

The reference decomposes its box over MPI ranks and exchanges ghost layers
of width nb = 6 every step (mpi_domain_mod.f90:618-649, 674-3091).  Here a
rank owns planes [z0, z0 + nz_local) of the global box and holds them in a
device box of nz_local + 2*H planes: its own planes at [H, H + nz_local) and
H copies of each neighbour's planes around them.  A step runs over the whole
slab (with the box's periodic wrap in z, which corrupts only the outer
planes); the own planes come out exact when H covers the step's dependency
radius, and one exchange per step refreshes the halos.  Only the own planes
enter the speed maxima (imhd_set_geometry), so the new dt, min-reduced over
ranks, equals the single-box dt, and the whole run equals the single-box run
bit for bit in FP64.

Forcing: on a drive step every slab adds up its forcing sums over its own
planes (imhd_force_sums) and all ranks' totals set the kick's normalisation
(imhd_set_force_sums), as the reference's all-reduce of get_rho_turb's sums
does (turb_driver_mod.f90:184-189, 402-415).  The totals are added in a
different order than one box adds its cells, so driven slab runs equal the
single box to FP64 rounding rather than bit for bit.  The dt after a drive
step is the minimum of the ranks' dts, each from its own max(c, smax +
delv_max), as the reference's ranks take it (driver.f90:432-448 and the
MIN all-reduce of share_dt); it can exceed one box's dt when smax and
delv_max peak on different ranks.  With passive scalars
a drive step differs at the global z boundary: a slab's halo planes are
kicked with the rest, so the passive corrector of the planes next to the
global boundary reads kicked velocities across it, where one box reads the
unforced periodic image (the reference's ranks, for their part, read
unforced ghost velocities at every rank boundary, turb_driver_mod.f90:
437-453, passive_mod.f90:227-239).

Dependency radius of one step along z: the half-step state needs the start
state within 2 planes, the corrector's fluxes and corner EMFs need the
half-step state within 3 (PLM) or 4 (PPM) planes, and the passive corrector
reads the new velocities one plane further out.

:class:`LocalSlabs` runs all ranks in one process on one device (the
exchange is a device copy); :class:`RankSlab` is one rank of a
torch.distributed job (NCCL between GPUs; any backend for the host logic).
"""
from __future__ import annotations

import numpy as np


def halo_width(recon="plm", npass=0):
    """Halo planes a slab needs for one exact step."""
    r = 6 if recon in ("ppm", "ppm-prim") else 5
    return r + (1 if npass else 0)


class Decomposition:
    """z slabs of a global (nx, ny, nz) box over `nranks` ranks."""

    def __init__(self, n, nranks, halo):
        self.nx, self.ny, self.nz = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
        self.nranks = int(nranks)
        self.halo = int(halo)
        base, extra = divmod(self.nz, self.nranks)
        self.counts = [base + (1 if r < extra else 0) for r in range(self.nranks)]
        self.starts = [sum(self.counts[:r]) for r in range(self.nranks)]
        if min(self.counts) < self.halo:
            raise ValueError("every slab needs at least `halo` planes (nz / nranks >= %d)" % self.halo)
        self.dx = 1.0 / max(self.nx, self.ny, self.nz)

    def local_nz(self, r):
        return self.counts[r] + 2 * self.halo

    def neighbours(self, r):
        return (r - 1) % self.nranks, (r + 1) % self.nranks

    def global_planes(self, r):
        """Global plane index of every local plane of rank r (periodic)."""
        return [(self.starts[r] - self.halo + t) % self.nz for t in range(self.local_nz(r))]

    def scatter(self, a, r, axis=-3):
        """Slab of rank r (with halos) of a global field array (z on `axis`)."""
        return np.take(a, self.global_planes(r), axis=axis)

    def gather(self, parts, axis=-3):
        """Global field array from the own planes of every rank's slab."""
        h = self.halo
        own = [np.take(p, range(h, h + self.counts[r]), axis=axis) for r, p in enumerate(parts)]
        return np.concatenate(own, axis=axis)

    def exchange_plan(self, r):
        """(send_lo_z0, send_hi_z0, recv_lo_z0, recv_hi_z0, nplanes) in local
        planes: the first own planes go down, the last own planes go up; the
        bottom halo comes from below, the top halo from above."""
        h, c = self.halo, self.counts[r]
        return h, c, 0, h + c, h


def _box_for(dec, r, **kw):
    from .box import Box
    box = Box((dec.nx, dec.ny, dec.local_nz(r)), **kw)
    box.set_geometry(dec.dx, dec.halo, dec.halo + dec.counts[r])
    return box


class LocalSlabs:
    """All ranks' slabs in one process on one device; the exchange is a
    device copy.  Same results as one box of the global size."""

    def __init__(self, n, nranks, precision=64, riemann="roe", recon="plm", npass=0, cour=0.4, halo=None, **kw):
        self.dec = Decomposition(n, nranks, halo if halo is not None else halo_width(recon, npass))
        self.npass = npass
        self.boxes = [_box_for(self.dec, r, precision=precision, riemann=riemann, recon=recon, npass=npass,
                               cour=cour, **kw) for r in range(nranks)]

    def upload(self, q, b, p=None):
        for r, box in enumerate(self.boxes):
            box.upload(self.dec.scatter(q, r), self.dec.scatter(b, r),
                       self.dec.scatter(p, r) if self.npass else None)

    def download(self):
        parts = [box.download() for box in self.boxes]
        q = self.dec.gather([p[0] for p in parts])
        b = self.dec.gather([p[1] for p in parts])
        p = self.dec.gather([p[2] for p in parts]) if self.npass else None
        return q, b, p

    def set_force(self, delv):
        """Force field of the global box (3, nz, ny, nx): every slab gets its
        planes and halos."""
        for r, box in enumerate(self.boxes):
            box.set_force(np.ascontiguousarray(self.dec.scatter(delv, r)))

    def exchange(self):
        import torch
        bufs = []
        for r, box in enumerate(self.boxes):
            slo, shi, _, _, npl = self.dec.exchange_plan(r)
            bufs.append((box.pack_planes(slo, npl), box.pack_planes(shi, npl)))
        for r, box in enumerate(self.boxes):
            lo, hi = self.dec.neighbours(r)
            _, _, rlo, rhi, npl = self.dec.exchange_plan(r)
            box.unpack_planes(rlo, npl, bufs[lo][1])     # lower neighbour's top planes
            box.unpack_planes(rhi, npl, bufs[hi][0])     # upper neighbour's bottom planes
        del bufs
        torch.cuda.synchronize()

    def step(self, dt, drive=False):
        """One step of every slab, the halo exchange; the global next dt.  A
        drive step first adds up the slabs' forcing sums (in rank order)."""
        if drive:
            total = np.zeros(5)
            for box in self.boxes:
                total = total + box.force_sums()
            for box in self.boxes:
                box.set_force_sums(total)
        dts = [box.step(dt, drive) for box in self.boxes]
        self.exchange()
        return min(dts)

    def close(self):
        for box in self.boxes:
            box.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class RankSlab:
    """This rank's slab in a torch.distributed job: exchange by point-to-point
    messages to the z neighbours, new dt by a MIN all-reduce.  `box` is any
    object with pack_planes / unpack_planes / step (a Box on GPU)."""

    def __init__(self, dec, rank, box, dist, device=None):
        self.dec, self.rank, self.box, self.dist = dec, rank, box, dist
        self.device = device

    def exchange(self):
        dist = self.dist
        r = self.rank
        lo, hi = self.dec.neighbours(r)
        slo, shi, rlo, rhi, npl = self.dec.exchange_plan(r)
        send_lo = self.box.pack_planes(slo, npl)
        send_hi = self.box.pack_planes(shi, npl)
        if self.dec.nranks == 1:
            self.box.unpack_planes(rlo, npl, send_hi)
            self.box.unpack_planes(rhi, npl, send_lo)
            return
        recv_lo = send_hi.new_empty(send_hi.shape)
        recv_hi = send_lo.new_empty(send_lo.shape)
        # sends up, then down; receives from below, then from above: with two
        # ranks both messages go to the same peer and match in this order
        ops = [dist.P2POp(dist.isend, send_hi, hi), dist.P2POp(dist.isend, send_lo, lo),
               dist.P2POp(dist.irecv, recv_lo, lo), dist.P2POp(dist.irecv, recv_hi, hi)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        self.box.unpack_planes(rlo, npl, recv_lo)
        self.box.unpack_planes(rhi, npl, recv_hi)

    def step(self, dt, drive=False):
        import torch
        if drive:
            # all ranks' forcing sums (a SUM all-reduce) set the kick of this drive step
            s = torch.tensor(np.asarray(self.box.force_sums(), dtype=np.float64), device=self.device)
            self.dist.all_reduce(s, op=self.dist.ReduceOp.SUM)
            self.box.set_force_sums(s.cpu().numpy())
        dt_local = self.box.step(dt, drive)
        self.exchange()
        t = torch.tensor([dt_local], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())

"""A box split into z-slabs: the reference's proc_z ranks
(SRC/setup_MPI.F90:112-131, SRC/bcond.comm.step3.F90:77-297) without MPI.

Each slab is a ``BGK3D`` context with ``proc_z > 1``. Its step kernel stores
the five populations that cross each z face straight into the neighbouring
slab's ghost planes (device memory of the same GPU, or of a peer GPU reached
through CUDA IPC and NVLink), so the exchange needs no messages: only a
barrier between steps (the library's contract, ``include/bgk3d.h``
"z-slabs"). Two drivers:

- ``LocalSlabs``: every slab in this process (one or several devices); the
  barrier is device-side: each slab's stream waits for the events its two
  neighbours recorded after their step (no host wait).
- ``DistSlabs``: one slab per process under ``torch.distributed`` (one
  process per GPU). The ghost buffers are shared as CUDA IPC handles
  (``all_gather_object``); the barrier is a one-element all-reduce on the
  slab's stream (NCCL) or a stream synchronisation plus ``dist.barrier``
  (gloo).

Diagnostics of a slab are its contribution to the global means; the global
record is their sum (``combine_diagnostics``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import BgkDiag, check
from .solver import BGK3D

# fields of bgk_diag that add up over the slabs (contributions to global
# means, sums and counts); t and itime are the same on every slab
ADDITIVE = ("rho_mean", "ux_mean", "uy_mean", "uz_mean", "ke_mean", "tke_norm", "diss", "tke", "eps_strain",
            "nonfinite")


def slab_range(lz: int, proc_z: int, coord_z: int) -> tuple[int, int]:
    """(first global plane, planes) of slab coord_z; lz must divide evenly
    (the reference's check, SRC/input.F90:66-82)."""
    if proc_z < 1 or not 0 <= coord_z < proc_z or lz % proc_z:
        raise ValueError(f"lz = {lz} does not split into {proc_z} slabs (coord {coord_z})")
    n = lz // proc_z
    return coord_z * n, n


def split_z(a, global_shape, proc_z: int) -> list:
    """A (lz, ly, lx) global array (any layout numpy can reshape to it) as
    the proc_z slabs' views, slab r holding planes slab_range(lz, proc_z, r)."""
    lx, ly, lz = global_shape
    a = np.asarray(a).reshape(lz, ly, lx)
    out = []
    for r in range(proc_z):
        z0, n = slab_range(lz, proc_z, r)
        out.append(a[z0:z0 + n])
    return out


def neighbours(coord_z: int, proc_z: int) -> tuple[int, int]:
    """Slabs below and above, periodic in z."""
    return (coord_z - 1) % proc_z, (coord_z + 1) % proc_z


def fp16_scale_for_velocity(u, v, w) -> float:
    """A power-of-two FP16 scale 2^floor(log2(65504 / (4 m))) from the largest
    equilibrium deviation m = max |w_q (3 c.u + 4.5 (c.u)^2 - 1.5 |u|^2)| of a
    velocity field at rho = 1 (host estimate, the same on every slab once the
    maxima are combined)."""
    cx = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)
    cy = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], float)
    cz = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], float)
    wq = np.where(np.abs(cx) + np.abs(cy) + np.abs(cz) == 2, 1 / 36, 1 / 18)
    wq[18] = 1 / 3
    u, v, w = (np.asarray(a, dtype=np.float64).reshape(-1) for a in (u, v, w))
    usq = u * u + v * v + w * w
    m = 0.0
    for q in range(19):
        cu = cx[q] * u + cy[q] * v + cz[q] * w
        m = max(m, float(np.max(np.abs(wq[q] * (3 * cu + 4.5 * cu * cu - 1.5 * usq)))))
    return scale_for_max(m)


def scale_for_max(m: float) -> float:
    if not m > 0 or not np.isfinite(m):
        return 1.0
    return float(2.0 ** np.floor(np.log2(65504.0 / (4.0 * m))))


def diagnostic_raw(box: BGK3D, itime: int) -> dict:
    """Diagnostics of one slab (its contributions) at a diagnostic step
    (itime a multiple of icheck, SRC/diagnostic.F90:37); non-finite cells
    are counted instead of raising."""
    d = BgkDiag()
    rc = box._lib.bgk_diagnostic(box._h, itime, C.byref(d))
    if rc == _abi.BGK_SKIPPED:
        raise ValueError(f"itime {itime} is not a diagnostic step (icheck = {box.params.icheck})")
    if rc not in (_abi.BGK_OK, _abi.BGK_ERR_NONFINITE):
        check(rc, "bgk_diagnostic")
    return d.as_dict()


def combine_diagnostics(parts: list[dict]) -> dict:
    """Global diagnostics from the slabs' contributions."""
    out = dict(parts[0])
    for k in ADDITIVE:
        out[k] = sum(p[k] for p in parts)
    out["enstrophy"] = float("nan")  # needs the whole box
    return out


class LocalSlabs:
    """All z-slabs of one box in this process, on `devices` (round robin)."""

    def __init__(self, lx: int, ly: int, lz: int, proc_z: int, devices=(0,), **kw):
        if proc_z < 2:
            raise ValueError("LocalSlabs needs proc_z >= 2")
        self.proc_z = proc_z
        self.global_shape = (lx, ly, lz)
        self.slabs = [BGK3D(lx, ly, lz, proc_z=proc_z, coord_z=r, device=devices[r % len(devices)], **kw)
                      for r in range(proc_z)]
        bufs = [s.halo_buffer()[0] for s in self.slabs]
        for r, s in enumerate(self.slabs):
            lo, hi = neighbours(r, proc_z)
            s.halo_connect(bufs[lo], bufs[hi])

    def close(self):
        for s in self.slabs:
            s.close()

    def barrier(self):
        """Each slab's next work waits, on the device, for its neighbours'
        queued work (they read and write each other's ghost planes)."""
        for s in self.slabs:
            s.record_event()
        for r, s in enumerate(self.slabs):
            lo, hi = neighbours(r, self.proc_z)
            s.wait_event(self.slabs[lo])
            if hi != lo:
                s.wait_event(self.slabs[hi])

    def synchronize(self):
        for s in self.slabs:
            s.synchronize()

    def prime(self):
        for s in self.slabs:
            s.halo_prime()
        self.barrier()

    def _split(self, a):
        return split_z(a, self.global_shape, self.proc_z)

    def init(self):
        for s in self.slabs:
            s.init()
        self.prime()

    def init_velocity(self, u, v, w, rho: float = 1.0):
        parts = [self._split(a) for a in (u, v, w)]
        for r, s in enumerate(self.slabs):
            s.init_velocity(parts[0][r], parts[1][r], parts[2][r], rho)
        self.prime()

    def set_populations(self, pops):
        lx, ly, lz = self.global_shape
        pops = np.asarray(pops).reshape(19, lz, ly, lx)
        for r, s in enumerate(self.slabs):
            z0, n = slab_range(lz, self.proc_z, r)
            s.set_populations(pops[:, z0:z0 + n])
        self.prime()

    def step(self, itime: int = 0):
        for s in self.slabs:
            s.col_MC(itime)
        self.barrier()

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()

    def populations(self) -> np.ndarray:
        return np.concatenate([s.populations() for s in self.slabs], axis=1)

    def deviations(self) -> np.ndarray:
        return np.concatenate([s.deviations() for s in self.slabs], axis=1)

    def diagnostic(self, itime: int) -> dict:
        return combine_diagnostics([diagnostic_raw(s, itime) for s in self.slabs])


class DistSlabs:
    """One z-slab per process of a ``torch.distributed`` group (rank = coord_z).

    ``box_factory(**kw)`` builds the slab context (``BGK3D`` by default; tests
    on the host pass a stand-in with the same halo methods)."""

    def __init__(self, lx: int, ly: int, lz: int, device: int = 0, box_factory=None, **kw):
        import torch.distributed as dist

        self.dist = dist
        self.rank, self.proc_z = dist.get_rank(), dist.get_world_size()
        if self.proc_z < 2:
            raise ValueError("DistSlabs needs a group of >= 2 processes")
        self.backend = dist.get_backend()
        self.device = device
        make = box_factory or BGK3D
        self.box = make(lx=lx, ly=ly, lz=lz, proc_z=self.proc_z, coord_z=self.rank, device=device, **kw)
        handles = [None] * self.proc_z
        dist.all_gather_object(handles, self.box.halo_ipc_handle())
        lo, hi = neighbours(self.rank, self.proc_z)
        opened = {}
        for r in (lo, hi):
            if r not in opened:
                opened[r] = self.box.halo_ipc_open(handles[r])
        self.box.halo_connect(opened[lo], opened[hi])
        self._flag = None

    def close(self):
        self.box.close()

    def barrier(self):
        """Every slab's queued work completes before any slab's next call."""
        if self.backend == "nccl":
            import torch

            if self._flag is None:
                self._flag = torch.zeros(1, device=f"cuda:{self.device}")
            s = torch.cuda.ExternalStream(self.box.stream, device=f"cuda:{self.device}")
            with torch.cuda.stream(s):
                self.dist.all_reduce(self._flag)
        else:
            self.box.synchronize()
            self.dist.barrier()

    def prime(self):
        self.box.halo_prime()
        self.barrier()

    def init(self):
        self.box.init()
        self.prime()

    def init_velocity(self, u, v, w, rho: float = 1.0):
        """u, v, w: this slab's planes (lz/proc_z, ly, lx)."""
        self.box.init_velocity(u, v, w, rho)
        self.prime()

    def step(self, itime: int = 0):
        self.box.col_MC(itime)
        self.barrier()

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()

    def diagnostic(self, itime: int) -> dict:
        """Global diagnostics (the same record on every rank)."""
        import torch

        mine = diagnostic_raw(self.box, itime) if isinstance(self.box, BGK3D) else self.box.diagnostic_raw(itime)
        vals = torch.tensor([float(mine[k]) for k in ADDITIVE], dtype=torch.float64)
        if self.backend == "nccl":
            vals = vals.to(f"cuda:{self.device}")
        self.dist.all_reduce(vals)
        out = dict(mine)
        for k, v in zip(ADDITIVE, vals.cpu().tolist()):
            out[k] = v
        out["nonfinite"] = int(round(out["nonfinite"]))
        out["enstrophy"] = float("nan")
        return out

"""Host logic of the z-slab decomposition, on CPU: partitioning, the FP16
scale agreed by all slabs, and the DistSlabs driver over a two- and
three-process gloo group with a stand-in for the slab context (handle
exchange, neighbour wiring, barriers, global diagnostics)."""
import datetime
import os
import socket

import numpy as np
import pytest


def test_slab_range_and_neighbours():
    from bgk3d_hit_b200.slabs import neighbours, slab_range

    assert [slab_range(24, 3, r) for r in range(3)] == [(0, 8), (8, 8), (16, 8)]
    assert slab_range(4, 4, 3) == (3, 1)
    for bad in ((25, 3, 0), (24, 3, 3), (24, 0, 0), (24, 3, -1)):
        with pytest.raises(ValueError):
            slab_range(*bad)
    assert neighbours(0, 4) == (3, 1) and neighbours(3, 4) == (2, 0) and neighbours(0, 2) == (1, 1)


def test_split_z_gives_contiguous_plane_blocks():
    from bgk3d_hit_b200.slabs import split_z

    lx, ly, lz = 3, 2, 12
    a = np.arange(lx * ly * lz, dtype=float)
    parts = split_z(a, (lx, ly, lz), 4)
    assert [p.shape for p in parts] == [(3, 2, 3)] * 4
    assert np.array_equal(np.concatenate(parts, axis=0).reshape(-1), a)
    assert parts[1][0, 0, 0] == 3 * lx * ly  # slab 1 starts at global plane 3


def test_fp16_scale_for_velocity_bounds_the_stored_values():
    from bgk3d_hit_b200.hit import hit_velocity
    from bgk3d_hit_b200.slabs import fp16_scale_for_velocity, scale_for_max

    u = hit_velocity(16, 2, 0.05, 1)
    s = fp16_scale_for_velocity(*u)
    assert s == 2.0 ** round(np.log2(s))
    c = [(1, -1, 0), (1, 0, -1), (1, 1, 0), (1, 0, 1), (1, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), (0, 1, -1)]
    c = c + [tuple(-x for x in v) for v in c]
    m = 0.0
    usq = u[0] ** 2 + u[1] ** 2 + u[2] ** 2
    for cx, cy, cz in c:
        w = 1 / 18 if abs(cx) + abs(cy) + abs(cz) == 1 else 1 / 36
        cu = cx * u[0] + cy * u[1] + cz * u[2]
        m = max(m, float(np.abs(w * (3 * cu + 4.5 * cu * cu - 1.5 * usq)).max()))
    m = max(m, float(np.abs(-0.5 * usq).max()))  # rest population, w = 1/3
    # 4x headroom below the largest binary16 value, and less than 8x
    assert 4.0 * m * s <= 65504.0 < 8.0 * m * s
    assert scale_for_max(0.0) == 1.0 and scale_for_max(float("nan")) == 1.0
    assert scale_for_max(65504.0 / 4.0) == 1.0


class FakeSlab:
    """Stands in for a BGK3D z-slab: records the halo calls."""

    def __init__(self, lx, ly, lz, proc_z, coord_z, device, **kw):
        self.coord_z, self.proc_z = coord_z, proc_z
        self.calls = []
        self.connected = None
        self.stream = 0

    def halo_ipc_handle(self):
        return bytes([self.coord_z]) * 64

    def halo_ipc_open(self, handle):
        self.calls.append(("open", handle[0]))
        return 1000 + handle[0]  # a fake device pointer naming the peer

    def halo_connect(self, below, above):
        self.connected = (below, above)

    def halo_prime(self):
        self.calls.append(("prime",))

    def init(self):
        self.calls.append(("init",))

    def col_MC(self, itime):
        self.calls.append(("step", itime))

    def synchronize(self):
        self.calls.append(("sync",))

    def diagnostic_raw(self, itime):
        r = self.coord_z + 1
        return {"itime": itime, "rho_mean": 0.25 * r, "ux_mean": 1e-3 * r, "uy_mean": 0.0, "uz_mean": -1e-3,
                "ke_mean": 1e-4 * r, "t": 0.5, "tke_norm": 0.1 * r, "diss": 2.0 * r, "tke": 3.0 * r,
                "enstrophy": 0.0, "eps_strain": 1e-6 * r, "nonfinite": r - 1}

    def close(self):
        pass


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from bgk3d_hit_b200.slabs import DistSlabs

        ds = DistSlabs(8, 8, 8 * world, device=0, box_factory=FakeSlab)
        ds.init()
        ds.step(1)
        ds.step(2)
        d = ds.diagnostic(2)
        b = ds.box
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([b.connected[0], b.connected[1], d["rho_mean"], d["diss"], d["nonfinite"],
                          d["t"], sum(1 for c in b.calls if c[0] == "open"),
                          sum(1 for c in b.calls if c[0] == "sync")], dtype=float))
        ds.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dist_slabs_wiring_and_diagnostics_over_gloo(tmp_path, world):
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    tot_rho = sum(0.25 * (r + 1) for r in range(world))
    tot_diss = sum(2.0 * (r + 1) for r in range(world))
    tot_nf = sum(r for r in range(world))
    for r in range(world):
        below, above, rho, diss, nf, t, nopen, nsync = np.load(tmp_path / f"r{r}.npy")
        # each slab is wired to the IPC mappings of coord_z - 1 and coord_z + 1
        assert below == 1000 + (r - 1) % world and above == 1000 + (r + 1) % world
        # a neighbour that is both below and above (two slabs) is mapped once
        assert nopen == (1 if world == 2 else 2)
        assert rho == pytest.approx(tot_rho) and diss == pytest.approx(tot_diss) and nf == tot_nf
        assert t == 0.5
        # gloo barrier: the slab's stream is synchronised after prime and each step
        assert nsync == 3

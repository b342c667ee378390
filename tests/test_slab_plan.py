"""Host logic of the slab decomposition (dns_slab_ranges / dns_slab_segments).

The plan partitions the operator slots (both pencils kz', Nz - kz' of each on
one rank) and the Py wall-normal planes over R ranks, and lists the blocks
of the two exchanges of a step.  Checked here on the CPU: every (pencil,
plane) pair travels exactly once, both ends list the same segments in the
same order, and a backward (6 fields) plus forward (3 fields) exchange
executed from the plan over gloo all_to_all with two and three ranks
reproduces the global arrays.  The device step does not use the plan yet.
"""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import load_package

GRIDS = [(48, 48, 128), (24, 36, 64), (384, 384, 512), (576, 576, 768)]


def _geom(mx, my, mz):
    Nx, Nz, Py = mx // 3 * 2, my // 3 * 2, mz // 2 + 1
    return Nx // 2 + 1, Nz, Py


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("R", [1, 2, 3, 4, 7])
def test_plan_covers_every_pencil_and_plane_once(grid, R):
    pkg = load_package()
    Kx, Nz, Py = _geom(*grid)
    own = np.full(Nz, -1)
    cover = np.zeros((Nz, Py), dtype=np.int64)
    counts = []
    for r in range(R):
        s0, s1, y0, y1, npen = pkg.slab_ranges(*grid, R, r)
        counts.append(npen)
        seen = 0
        for sg in pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS):
            kz = np.arange(sg["kz0"], sg["kz0"] + sg["nkz"])
            cover[kz, sg["y0"]:sg["y0"] + sg["ny"]] += 1
            if sg["peer"] == 0:
                assert np.all(own[kz] == -1)
                own[kz] = r
                assert sg["local_row0"] == seen
                seen += sg["nkz"] * Kx
            # slots: both pencils of every slot of this rank
            for k in kz:
                kzs = k if k <= Nz // 2 else Nz - k
                assert s0 <= kzs < s1
        assert seen == npen
        # the plane owner lists the same segments, per peer, in the same order
        for s in range(R):
            mine = [dict(g, peer=s) for g in pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS)
                    if g["peer"] == s]
            theirs = [dict(g, peer=s) for g in pkg.slab_segments(*grid, R, s, pkg.SLAB_PLANES)
                      if g["peer"] == r]
            assert mine == theirs
    assert np.all(own >= 0)
    assert np.all(cover == 1)
    assert sum(counts) == Kx * Nz and max(counts) - min(counts) <= 2 * Kx


def test_plan_rejects_bad_arguments():
    pkg = load_package()
    with pytest.raises(pkg.DnsError):
        pkg.slab_ranges(48, 48, 128, 2, 2)
    with pytest.raises(pkg.DnsError):
        pkg.slab_ranges(48, 48, 128, 100, 0)  # more ranks than slots
    with pytest.raises(pkg.DnsError):
        pkg.slab_segments(48, 48, 130, 2, 0, pkg.SLAB_PENCILS)


def _exchange(pkg, grid, R, r, G, dist, torch):
    """Backward then forward exchange of rank r, executed from the plan."""
    Kx, Nz, Py = _geom(*grid)
    pen = pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS)
    pla = pkg.slab_segments(*grid, R, r, pkg.SLAB_PLANES)
    s0, s1, y0, y1, npen = pkg.slab_ranges(*grid, R, r)
    # local pencil buffer [f][local pencil][Py], runs in increasing kz
    runs = sorted({(g["kz0"], g["nkz"], g["local_row0"]) for g in pen})
    loc = np.zeros((6, npen, Py))
    for kz0, nkz, row0 in runs:
        loc[:, row0:row0 + nkz * Kx] = G[:, kz0 * Kx:(kz0 + nkz) * Kx]

    def a2a(send_parts, recv_sizes):
        sb = torch.from_numpy(np.concatenate([p.ravel() for p in send_parts]))
        rb = torch.empty(sum(recv_sizes), dtype=torch.float64)
        dist.all_to_all_single(rb, sb, output_split_sizes=recv_sizes,
                               input_split_sizes=[p.size for p in send_parts])
        return rb.numpy()

    # backward: pencils -> planes, 6 fields
    nf = 6
    send = []
    for s in range(R):
        blocks = [loc[f, g["local_row0"]:g["local_row0"] + g["nkz"] * Kx, g["y0"]:g["y0"] + g["ny"]]
                  for f in range(nf) for g in pen if g["peer"] == s]
        send.append(np.concatenate([b.ravel() for b in blocks]) if blocks else np.zeros(0))
    rsz = [nf * sum(g["nkz"] * Kx * g["ny"] for g in pla if g["peer"] == s) for s in range(R)]
    buf = a2a(send, rsz)
    ny = y1 - y0
    planes = np.full((6, Kx * Nz, ny), np.nan)
    off = 0
    for s in range(R):
        for f in range(nf):
            for g in (g for g in pla if g["peer"] == s):
                n = g["nkz"] * Kx * g["ny"]
                planes[f, g["kz0"] * Kx:(g["kz0"] + g["nkz"]) * Kx, :] = buf[off:off + n].reshape(-1, ny)
                off += n
    assert off == buf.size
    assert np.array_equal(planes, G[:, :, y0:y1])
    # forward: planes -> pencils, 3 fields (the spanwise pass's output)
    nf = 3
    send = []
    for s in range(R):
        blocks = [planes[f, g["kz0"] * Kx:(g["kz0"] + g["nkz"]) * Kx, :]
                  for f in range(nf) for g in pla if g["peer"] == s]
        send.append(np.concatenate([b.ravel() for b in blocks]) if blocks else np.zeros(0))
    rsz = [nf * sum(g["nkz"] * Kx * g["ny"] for g in pen if g["peer"] == s) for s in range(R)]
    buf = a2a(send, rsz)
    back = np.full((3, npen, Py), np.nan)
    off = 0
    for s in range(R):
        for f in range(nf):
            for g in (g for g in pen if g["peer"] == s):
                n = g["nkz"] * Kx * g["ny"]
                back[f, g["local_row0"]:g["local_row0"] + g["nkz"] * Kx, g["y0"]:g["y0"] + g["ny"]] = \
                    buf[off:off + n].reshape(-1, g["ny"])
                off += n
    assert np.array_equal(back, loc[:3])


def _worker(rank, world, port, grid, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pkg = load_package()
        Kx, Nz, Py = _geom(*grid)
        G = np.random.default_rng(5).standard_normal((6, Kx * Nz, Py))
        _exchange(pkg, grid, world, rank, G, dist, torch)
        q.put((rank, "ok"))
    except Exception as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,grid", [(2, (48, 48, 128)), (3, (24, 36, 64))])
def test_exchange_round_trip_gloo(world, grid):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, grid, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res == {r: "ok" for r in range(world)}

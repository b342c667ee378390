"""Host logic of the slab decomposition (dns_slab_ranges / dns_slab_segments).

The plan partitions the operator slots (both pencils kz', Nz - kz' of each on
one rank) and the Py wall-normal planes over R ranks, and lists the blocks
of the two exchanges of a step.  Checked here on the CPU: every (pencil,
plane) pair travels exactly once, both ends list the same segments in the
same order, and a backward (6 fields) plus forward (3 fields) exchange
executed from the plan over gloo all_to_all with two and three ranks
reproduces the global arrays, and the oracle's nonlinear phase run
decomposed by the plan (wall-normal transforms on each rank's pencils,
spanwise/streamwise transforms and the Lamb vector on its planes) equals the
undecomposed one.  The device step does not use the plan yet.
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


def _a2a(dist, torch, send_parts, recv_sizes):
    sb = torch.from_numpy(np.concatenate([np.ravel(x) for x in send_parts]))
    rb = torch.empty(sum(recv_sizes), dtype=sb.dtype)
    dist.all_to_all_single(rb, sb, output_split_sizes=recv_sizes,
                           input_split_sizes=[int(np.size(x)) for x in send_parts])
    return rb.numpy()


def pencils_to_planes(pkg, grid, R, r, loc, dist, torch):
    """Backward exchange executed from the plan: loc[f][local pencil][Py]
    -> planes[f][pencil][ny of this rank]."""
    Kx, Nz, Py = _geom(*grid)
    pen = pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS)
    pla = pkg.slab_segments(*grid, R, r, pkg.SLAB_PLANES)
    nf = loc.shape[0]
    send = []
    for s in range(R):
        blocks = [loc[f, g["local_row0"]:g["local_row0"] + g["nkz"] * Kx, g["y0"]:g["y0"] + g["ny"]]
                  for f in range(nf) for g in pen if g["peer"] == s]
        send.append(np.concatenate([x.ravel() for x in blocks]) if blocks else np.zeros(0, loc.dtype))
    rsz = [nf * sum(g["nkz"] * Kx * g["ny"] for g in pla if g["peer"] == s) for s in range(R)]
    buf = _a2a(dist, torch, send, rsz)
    _, _, y0, y1, _ = pkg.slab_ranges(*grid, R, r)
    planes = np.full((nf, Kx * Nz, y1 - y0), np.nan, dtype=loc.dtype)
    off = 0
    for s in range(R):
        for f in range(nf):
            for g in (g for g in pla if g["peer"] == s):
                n = g["nkz"] * Kx * g["ny"]
                planes[f, g["kz0"] * Kx:(g["kz0"] + g["nkz"]) * Kx] = buf[off:off + n].reshape(-1, y1 - y0)
                off += n
    assert off == buf.size
    return planes


def planes_to_pencils(pkg, grid, R, r, planes, dist, torch):
    """Forward exchange executed from the plan: planes[f][pencil][ny] ->
    loc[f][local pencil][Py]."""
    Kx, Nz, Py = _geom(*grid)
    pen = pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS)
    pla = pkg.slab_segments(*grid, R, r, pkg.SLAB_PLANES)
    nf = planes.shape[0]
    send = []
    for s in range(R):
        blocks = [planes[f, g["kz0"] * Kx:(g["kz0"] + g["nkz"]) * Kx]
                  for f in range(nf) for g in pla if g["peer"] == s]
        send.append(np.concatenate([x.ravel() for x in blocks]) if blocks else np.zeros(0, planes.dtype))
    rsz = [nf * sum(g["nkz"] * Kx * g["ny"] for g in pen if g["peer"] == s) for s in range(R)]
    buf = _a2a(dist, torch, send, rsz)
    npen = pkg.slab_ranges(*grid, R, r)[4]
    loc = np.full((nf, npen, Py), np.nan, dtype=planes.dtype)
    off = 0
    for s in range(R):
        for f in range(nf):
            for g in (g for g in pen if g["peer"] == s):
                n = g["nkz"] * Kx * g["ny"]
                loc[f, g["local_row0"]:g["local_row0"] + g["nkz"] * Kx, g["y0"]:g["y0"] + g["ny"]] = \
                    buf[off:off + n].reshape(-1, g["ny"])
                off += n
    assert off == buf.size
    return loc


def local_pencils(pkg, grid, R, r):
    """Global pencil indices of rank r's local buffer rows, in order."""
    Kx = _geom(*grid)[0]
    runs = sorted({(g["kz0"], g["nkz"], g["local_row0"])
                   for g in pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS)}, key=lambda t: t[2])
    return np.concatenate([np.arange(kz0 * Kx, (kz0 + nkz) * Kx) for kz0, nkz, _ in runs])


def _exchange(pkg, grid, R, r, G, dist, torch):
    """Backward then forward exchange of rank r, executed from the plan."""
    rows = local_pencils(pkg, grid, R, r)
    loc = G[:, rows]
    y0, y1 = pkg.slab_ranges(*grid, R, r)[2:4]
    planes = pencils_to_planes(pkg, grid, R, r, loc, dist, torch)
    assert np.array_equal(planes, G[:, :, y0:y1])
    back = planes_to_pencils(pkg, grid, R, r, planes[:3], dist, torch)
    assert np.array_equal(back, loc[:3])


def decomposed_nonlinear(pkg, pb, R, r, dist, torch):
    """The oracle's nonlinear phase run as the slab decomposition would run
    the step: wall-normal transforms on this rank's pencils only, the
    spanwise/streamwise transforms and the Lamb vector on its planes only
    (other planes zero), data moved between the two by the plan's exchanges.
    Returns (rows, Nv, No) for this rank's pencils."""
    from oracle import rpcf_oracle as O
    sz, p = pb.sz, pb.p
    grid = (sz.mx, sz.my, sz.mz)
    rows = local_pencils(pkg, grid, R, r)
    H = sz.ny * sz.hnx
    fields = pb.spectral_fields()
    loc = np.zeros((6, rows.size, sz.pz), dtype=np.complex128)
    for f, F in enumerate(fields):
        S = np.zeros((rows.size, sz.mz), dtype=np.complex128)
        S[:, :sz.nz] = F.reshape(H, sz.nz)[rows]
        loc[f] = O.cheby_s2p(S, sz.mz, pad=True)[:, :sz.pz]
    planes = pencils_to_planes(pkg, grid, R, r, loc, dist, torch)
    y0, y1 = pkg.slab_ranges(*grid, R, r)[2:4]
    phys = []
    for f in range(6):
        S = np.zeros((sz.ny, sz.hnx, sz.mz), dtype=np.complex128)
        S[:, :, y0:y1] = planes[f].reshape(sz.ny, sz.hnx, y1 - y0)
        C = O.set_zeros(O.transpose_backward(S, sz), sz)
        phys.append(O.c2r_2d(C, sz))
    lx, ly, lz = O.lamb(*phys, sz, p.Ro, p.prof)
    out = np.zeros((3, H, y1 - y0), dtype=np.complex128)
    for f, L in enumerate((lx, ly, lz)):
        S = O.transpose_forward(O.r2c_2d(L, sz), sz)
        out[f] = S[:, :, y0:y1].reshape(H, y1 - y0)
    back = planes_to_pencils(pkg, grid, R, r, out, dist, torch)
    tl = []
    for f in range(3):
        S = np.zeros((rows.size, sz.mz), dtype=np.complex128)
        S[:, :sz.pz] = back[f]
        T = np.zeros((H, sz.mz), dtype=np.complex128)
        T[rows] = O.cheby_p2s(S, sz.mz, pad=True)
        tl.append(T.reshape(sz.ny, sz.hnx, sz.mz))
    hv, ho = O.rhs_nonlinear(*tl, sz, pb.aphi, pb.beta)
    res = []
    for h in (hv, ho):
        Hh = np.zeros((rows.size, sz.mz), dtype=np.complex128)
        Hh[:, :sz.nz] = h.reshape(H, sz.nz)[rows]
        res.append(O.cheby_s2p(Hh, sz.mz, pad=False)[:, :sz.nz])
    return rows, res[0], res[1]


class _FakeRank:
    """Stand-in for a SlabContext in the driver test: exchange sizes from the
    plan (as dns_slab_exchange_bytes computes them: 6 fields back, 3 fields
    forward, 8 bytes per value), parts that write peer-tagged bytes into the
    send buffer and check what the all-to-all delivered."""

    def __init__(self, pkg, grid, R, r, torch):
        Kx = _geom(*grid)[0]
        self.torch, self.R, self.r, self.checked, self.bufs = torch, R, r, 0, None
        self.sizes = {x: ([0] * R, [0] * R) for x in (0, 1)}
        for sg in pkg.slab_segments(*grid, R, r, pkg.SLAB_PENCILS):
            b = sg["nkz"] * Kx * sg["ny"] * 8
            self.sizes[0][0][sg["peer"]] += 6 * b
            self.sizes[1][1][sg["peer"]] += 3 * b
        for sg in pkg.slab_segments(*grid, R, r, pkg.SLAB_PLANES):
            b = sg["nkz"] * Kx * sg["ny"] * 8
            self.sizes[0][1][sg["peer"]] += 6 * b
            self.sizes[1][0][sg["peer"]] += 3 * b

    def exchange_bytes(self, x):
        return self.sizes[x]

    def _fill(self, x):
        off = 0
        for s, n in enumerate(self.sizes[x][0]):
            self.bufs.send[off:off + n] = (self.r * 16 + s + 64 * x) & 0xFF
            off += n

    def _check(self, x):
        off = 0
        for p, n in enumerate(self.sizes[x][1]):
            assert bool(self.torch.all(self.bufs.recv[off:off + n] == ((p * 16 + self.r + 64 * x) & 0xFF)))
            off += n
        self.checked += 1

    def part(self, part, send_ptr, recv_ptr, boot=False):
        if part == 0:
            self._fill(0)
        elif part == 1:
            self._check(0)
            self._fill(1)
        else:
            self._check(1)


def _worker(rank, world, port, grid, q, mode="exchange"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pkg = load_package()
        if mode == "driver":
            import importlib
            slab = importlib.import_module(pkg.__name__ + ".slab")
            fake = _FakeRank(pkg, grid, world, rank, torch)
            fake.bufs = slab.SlabBuffers(fake, device="cpu")
            slab.step_dist(fake, boot=True, bufs=fake.bufs)
            slab.step_dist(fake, 2, bufs=fake.bufs)
            assert fake.checked == 6, fake.checked
        elif mode == "exchange":
            Kx, Nz, Py = _geom(*grid)
            G = np.random.default_rng(5).standard_normal((6, Kx * Nz, Py))
            _exchange(pkg, grid, world, rank, G, dist, torch)
        else:
            from oracle import rpcf_oracle as O
            pb = O.Problem(O.Params(*grid, Re=1300.0, Ro=0.1, dt=0.005))
            sz = pb.sz
            V0, O0 = pkg.seeded_state(sz.nx, sz.nz, sz.ny, 4.0, 2.0, 0.05, 0)
            pb.set_state(V0, O0)
            rows, Nv, No = decomposed_nonlinear(pkg, pb, world, rank, dist, torch)
            Nv_ref, No_ref = pb.nonlinear()
            H = sz.ny * sz.hnx
            ev = np.max(np.abs(Nv - Nv_ref.reshape(H, -1)[rows])) / np.max(np.abs(Nv_ref))
            eo = np.max(np.abs(No - No_ref.reshape(H, -1)[rows])) / np.max(np.abs(No_ref))
            assert ev < 1e-13 and eo < 1e-13, (ev, eo)
        q.put((rank, "ok"))
    except Exception as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(world, grid, mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, grid, q, mode)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert res == {r: "ok" for r in range(world)}


@pytest.mark.parametrize("world,grid", [(2, (48, 48, 128)), (3, (24, 36, 64))])
def test_exchange_round_trip_gloo(world, grid):
    _spawn(world, grid, "exchange")


@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_nonlinear_matches_oracle_gloo(world):
    """The nonlinear phase decomposed by the plan (pencil passes on the
    rank's pencils, plane passes on its planes, the two exchanges between)
    equals the undecomposed oracle on every rank's pencils."""
    _spawn(world, (48, 48, 128), "nonlinear")


@pytest.mark.parametrize("world,grid", [(2, (48, 48, 128)), (3, (24, 36, 64))])
def test_step_dist_driver_gloo(world, grid):
    """slab.step_dist, the NCCL driver of the decomposed step, on gloo ranks:
    the all-to-all byte splits of both exchanges agree at both ends and every
    peer's bytes arrive where the receiving part reads them, for a bootstrap
    and two steps."""
    _spawn(world, grid, "driver")

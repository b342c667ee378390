"""Drivers of the slab-decomposed step (``SlabContext``, ``dns_slab_part``):
the two exchanges between its three parts, either on one device (copies
between the ranks' buffers, every rank's context on that device) or across
processes (an NCCL all-to-all through ``torch.distributed``, one rank per
GPU).  The packed buffers are byte tensors on the device; their layout is
the library's (per peer, per field, the segments in plan order)."""
import torch

from .abi import SLAB_XZ, SLAB_Y1, SLAB_Y3


class SlabBuffers:
    """Send and receive buffers of one rank and the bytes per peer of both
    exchanges."""

    def __init__(self, ctx, device=None):
        self.split = {x: ctx.exchange_bytes(x) for x in (0, 1)}
        ns = max(sum(self.split[0][0]), sum(self.split[1][0]), 16)
        nr = max(sum(self.split[0][1]), sum(self.split[1][1]), 16)
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send = torch.empty(ns, dtype=torch.uint8, device=dev)
        self.recv = torch.empty(nr, dtype=torch.uint8, device=dev)


def _offsets(sizes):
    out, o = [], 0
    for n in sizes:
        out.append(o)
        o += n
    return out


def step_local(ctxs, nsteps=1, boot=False, bufs=None):
    """Run all ranks of a decomposition on one device, rank after rank, with
    the exchanges as device copies between their buffers.  boot: the
    bootstrap (one pass, the AB2 history only).  Synchronous."""
    ctxs = list(ctxs)
    bufs = bufs or [SlabBuffers(c) for c in ctxs]
    R = len(ctxs)
    for _ in range(1 if boot else nsteps):
        for part, x in ((SLAB_Y3, 0), (SLAB_XZ, 1), (SLAB_Y1, None)):
            for c, b in zip(ctxs, bufs):
                c.part(part, b.send.data_ptr(), b.recv.data_ptr(), boot)
            if x is None:
                break
            for c in ctxs:
                c.synchronize()
            for s in range(R):
                recv_sizes = bufs[s].split[x][1]
                roff = _offsets(recv_sizes)
                for r in range(R):
                    send_sizes = bufs[r].split[x][0]
                    n = send_sizes[s]
                    if n != recv_sizes[r]:
                        raise RuntimeError(f"exchange {x}: rank {r} sends {n} bytes to {s}, which expects "
                                           f"{recv_sizes[r]}")
                    so = _offsets(send_sizes)[s]
                    bufs[s].recv[roff[r]:roff[r] + n].copy_(bufs[r].send[so:so + n])
            torch.cuda.synchronize()
    for c in ctxs:
        c.synchronize()
    return bufs


def step_dist(ctx, nsteps=1, boot=False, bufs=None, group=None):
    """This process's rank of a decomposition across processes: the parts on
    the context's stream, the exchanges as all-to-all collectives of
    torch.distributed (NCCL) ordered on the same stream.  Asynchronous on
    that stream; returns the buffers for reuse."""
    import contextlib

    import torch.distributed as dist
    bufs = bufs or SlabBuffers(ctx)
    on_gpu = bufs.send.is_cuda
    with (torch.cuda.stream(torch.cuda.ExternalStream(ctx.stream)) if on_gpu else contextlib.nullcontext()):
        for _ in range(1 if boot else nsteps):
            for part, x in ((SLAB_Y3, 0), (SLAB_XZ, 1), (SLAB_Y1, None)):
                ctx.part(part, bufs.send.data_ptr(), bufs.recv.data_ptr(), boot)
                if x is None:
                    break
                snd, rcv = bufs.split[x]
                dist.all_to_all_single(bufs.recv[:sum(rcv)], bufs.send[:sum(snd)], output_split_sizes=rcv,
                                       input_split_sizes=snd, group=group)
    return bufs

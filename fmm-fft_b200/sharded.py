"""Sharded single transform: one FMM-FFT of N points over G devices (fmmfft_shard_*).

The library computes each shard's phases (include/fmmfft.h, "sharded transform"); this module
moves the data between them, the part the reference does with MPI (src/fmmfft.c:517-618 halo
exchanges, :452-453 the section-sum reduction, :970 the all-to-all):

  exchanges   before phase 0: the x halos (each shard gets the last `halo` points of the shard
              before it and the first `halo` of the one after it, cyclically);
              between 0 and 1: all-reduce (sum) of the P section sums, all-gather of the coarse
              expansions; between 1 and 2: one all-to-all of the combined rows.

Two transports implement the same four exchanges:

  DistTransport   one shard per rank of a torch.distributed process group (NCCL over NVLink on
                  GPUs): batched isend/irecv for the halos, all_reduce, all_gather, all_to_all;
  LocalTransport  G shards in one process on one device, each exchange a set of device copies in
                  stream order (the G shards' phases run one after another: nothing waits on
                  another shard's kernels).

Device memory of a shard is viewed as torch tensors through __cuda_array_interface__ (no copy).
torch is plumbing here; the transform's arithmetic is the library's.
"""
import os
import sys

import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import fmmfft  # noqa: E402


class _DevArray:
    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _views(shard):
    """torch views of a shard's exchange buffers."""
    bb = shard.buffers()
    f64 = shard.precision == "f64"
    rtype, cdt = ("<f8", torch.complex128) if f64 else ("<f4", torch.complex64)
    G = shard.G

    def real(name, n):
        return torch.as_tensor(_DevArray(bb[name], n, rtype), device="cuda")

    def cplx(name, n):  # complex buffers as views of their (re, im) pairs
        return real(name, 2 * n).view(cdt)
    return {"x_ext": cplx("x_ext", bb["x_ext_elems"]), "halo": bb["halo_elems"],
            "sums": cplx("sums", shard.P), "phi_send": real("phi_send", bb["phi_elems"]),
            "phi_all": real("phi_all", bb["phi_elems"] * G), "z_send": cplx("z_send", bb["z_elems"]),
            "z_recv": cplx("z_recv", bb["z_elems"]), "y": cplx("y", bb["y_elems"])}


# ------------------------------------------------------------------------ exchanges
class DistTransport:
    """The four exchanges between the ranks of a process group, this rank's shard's tensors."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.G, self.g = dist.get_world_size(group), dist.get_rank(group)

    def halos(self, block, left, right):
        """left <- the last len(left) of rank g-1's block, right <- the first len(right) of rank g+1's."""
        d, G, g = self.dist, self.G, self.g
        nxt, prv = (g + 1) % G, (g - 1) % G
        h = left.numel()
        ops = [d.P2POp(d.isend, block[-h:].contiguous(), nxt, self.group),
               d.P2POp(d.isend, block[:h].contiguous(), prv, self.group),
               d.P2POp(d.irecv, left, prv, self.group), d.P2POp(d.irecv, right, nxt, self.group)]
        for r in d.batch_isend_irecv(ops):
            r.wait()

    def sum(self, t):
        self.dist.all_reduce(t, group=self.group)

    def gather(self, send, out):
        self.dist.all_gather(list(out.chunk(self.G)), send, group=self.group)

    def alltoall(self, send, recv):
        self.dist.all_to_all_single(recv, send, group=self.group)


class LocalTransport:
    """The same four exchanges over lists of every shard's tensors, in this process."""

    def __init__(self, G):
        self.G = G

    def halos(self, blocks, lefts, rights):
        G = self.G
        for g in range(G):
            h = lefts[g].numel()
            lefts[g].copy_(blocks[(g - 1) % G][-h:])
            rights[g].copy_(blocks[(g + 1) % G][:h])

    def sum(self, ts):
        tot = ts[0].clone()
        for t in ts[1:]:
            tot += t
        for t in ts:
            t.copy_(tot)

    def gather(self, sends, outs):
        cat = torch.cat(list(sends))
        for o in outs:
            o.copy_(cat)

    def alltoall(self, sends, recvs):
        G = self.G
        for h in range(G):
            recvs[h].copy_(torch.cat([sends[g].chunk(G)[h] for g in range(G)]))


# ------------------------------------------------------------------------ drivers
def forward_rank(shard, block, transport, stream=None):
    """This rank's shard: its block of N/G input points (a device tensor) -> its N/G outputs (a
    view of the shard's output buffer, valid until the shard's next transform)."""
    v = _views(shard)
    st = stream or torch.cuda.current_stream()
    h = v["halo"]
    x = v["x_ext"]
    x[h:h + block.numel()].copy_(block)
    transport.halos(block, x[:h], x[h + block.numel():])
    shard.phase(0, st.cuda_stream)
    transport.sum(v["sums"])
    transport.gather(v["phi_send"], v["phi_all"])
    shard.phase(1, st.cuda_stream)
    transport.alltoall(v["z_send"], v["z_recv"])
    shard.phase(2, st.cuda_stream)
    return v["y"]


def forward_emulated(shards, x, stream=None):
    """All G shards in this process on one device: x (N points, device tensor) -> y (N points),
    each shard's phases run in turn with the exchanges between them as device copies."""
    G = len(shards)
    tr = LocalTransport(G)
    st = stream or torch.cuda.current_stream()
    vs = [_views(s) for s in shards]
    blocks = list(x.chunk(G))
    for v, blk in zip(vs, blocks):
        v["x_ext"][v["halo"]:v["halo"] + blk.numel()].copy_(blk)
    tr.halos(blocks, [v["x_ext"][:v["halo"]] for v in vs],
             [v["x_ext"][v["halo"] + blk.numel():] for v, blk in zip(vs, blocks)])
    for s in shards:
        s.phase(0, st.cuda_stream)
    tr.sum([v["sums"] for v in vs])
    tr.gather([v["phi_send"] for v in vs], [v["phi_all"] for v in vs])
    for s in shards:
        s.phase(1, st.cuda_stream)
    tr.alltoall([v["z_send"] for v in vs], [v["z_recv"] for v in vs])
    for s in shards:
        s.phase(2, st.cuda_stream)
    return torch.cat([v["y"] for v in vs])

"""The exchanges of the sharded transform (fmm-fft_b200/sharded.py) between world-size 2 and 4
gloo process groups on CPU: the halo ring, the all-reduce of the section sums, the all-gather of
the coarse expansions and the all-to-all of the combined rows, each rank with its own tensors
(DistTransport, the calls a multi-GPU job makes under NCCL), must give every rank exactly what the
in-process transport (LocalTransport, the one the single-device GPU tests run) gives it for the
same data.  No GPU: the shards' phases are the library's and run in the GPU tests."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "fmm-fft_b200"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data(G, seed=7):
    import torch
    g = torch.Generator().manual_seed(seed)
    nb, halo, nphi, nz = 48, 12, 20, 32  # per shard: block, halo, phi reals, z (G | nz)
    blocks = [torch.randn(nb, 2, generator=g).view(torch.complex64).squeeze(-1) for _ in range(G)]
    sums = [torch.randn(16, 2, generator=g, dtype=torch.float64).view(torch.complex128).squeeze(-1) for _ in range(G)]
    phis = [torch.randn(nphi, generator=g) for _ in range(G)]
    zs = [torch.randn(nz, 2, generator=g).view(torch.complex64).squeeze(-1) for _ in range(G)]
    return blocks, halo, sums, phis, zs


def _rank(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    try:
        import datetime

        import torch
        import torch.distributed as dist
        import sharded
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
        blocks, halo, sums, phis, zs = _data(world)
        tr = sharded.DistTransport()
        left, right = torch.empty(halo, dtype=torch.complex64), torch.empty(halo, dtype=torch.complex64)
        tr.halos(blocks[rank], left, right)
        s = sums[rank].clone()
        tr.sum(s)
        out = torch.empty(phis[0].numel() * world)
        tr.gather(phis[rank], out)
        rz = torch.empty_like(zs[rank])
        tr.alltoall(zs[rank], rz)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank,) + tuple(t.numpy() for t in (left, right, s, out, rz)))  # by value
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put((rank, "error", repr(e)))


@pytest.mark.parametrize("world", [2, 4])
def test_dist_exchanges_equal_local_exchanges(world):
    import torch
    import torch.multiprocessing as mp
    import sharded
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = {}
    for _ in range(world):
        item = q.get(timeout=120)
        assert not (isinstance(item[1], str) and item[1] == "error"), item
        got[item[0]] = item[1:]
    for p in ps:
        p.join(timeout=60)
    blocks, halo, sums, phis, zs = _data(world)
    tr = sharded.LocalTransport(world)
    lefts = [torch.empty(halo, dtype=torch.complex64) for _ in range(world)]
    rights = [torch.empty(halo, dtype=torch.complex64) for _ in range(world)]
    tr.halos(blocks, lefts, rights)
    ss = [s.clone() for s in sums]
    tr.sum(ss)
    outs = [torch.empty(phis[0].numel() * world) for _ in range(world)]
    tr.gather(phis, outs)
    rzs = [torch.empty_like(z) for z in zs]
    tr.alltoall(zs, rzs)
    for r in range(world):
        left, right, s, out, rz = (torch.from_numpy(a) for a in got[r])
        assert torch.equal(left, lefts[r]) and torch.equal(right, rights[r])
        assert torch.allclose(s, ss[r], rtol=0, atol=1e-12)
        assert torch.equal(out, outs[r])
        assert torch.equal(rz, rzs[r])

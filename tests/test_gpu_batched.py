"""Batched plans: many transforms of one shape in one launch sequence (fmmfft_execute_many).

Every transform of a batch must give bitwise the same output as its own execute on a plan of
capacity 1: the tree stages contract the rows of all transforms at once, the other stages take
the transform as a grid dimension, and the routing of each stage (tensor cores, coarse tree,
CUDA cores) depends on one transform's row counts only.  Shapes cover the tensor-core path, the
CUDA-core FP32 and FP64 paths, the coarse-tree kernel (forced), the leaf for b not a multiple of
8 (rowgemm + half-shift pass), P < 16 (the shared-memory combine) and one-pass local FFTs."""
import os

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


CASES = [(1 << 16, 16, 16, 32, "f32_tc"), (1 << 16, 16, 16, 32, "f32"), (1 << 14, 4, 12, 16, "f64"),
         (1 << 15, 8, 10, 4, "f32"), (1 << 18, 64, 24, 32, "f32_tc"), (4096, 8, 8, 16, "f32_tc"),
         (1 << 17, 32, 20, 32, "f32_tc")]


def _run_batched(fm, N, P, T, b, prec, nbt, monkeypatch=None):
    import torch
    dt = torch.complex128 if prec == "f64" else torch.complex64
    xs = [ol.seeded_input(N, 1000 + i) for i in range(nbt)]
    single = fm.Plan(N, P, T, b, prec)
    ref = []
    for x in xs:
        d = torch.from_numpy(x).to(dt).cuda()
        o = torch.empty_like(d)
        single.execute_ptr(d.data_ptr(), o.data_ptr())
        torch.cuda.synchronize()
        ref.append(o.cpu().numpy())
    single.check()
    single.close()
    plan = fm.Plan(N, P, T, b, prec, max_transforms=nbt)
    xin = torch.from_numpy(np.concatenate(xs)).to(dt).cuda()
    out = torch.empty_like(xin)
    plan.execute_many_ptr(nbt, xin.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    plan.check()
    got = out.cpu().numpy().reshape(nbt, N)
    # the graph form too, on the same plan and buffers
    out2 = torch.empty_like(xin)
    plan.execute_many_ptr(nbt, xin.data_ptr(), out2.data_ptr(), graph=True)
    torch.cuda.synchronize()
    plan.check()
    got2 = out2.cpu().numpy().reshape(nbt, N)
    plan.close()
    return xs, ref, got, got2


@pytest.mark.parametrize("N,P,T,b,prec", CASES)
@pytest.mark.parametrize("nbt", [1, 3, 8])
def test_batch_equals_alone_bitwise(fm, N, P, T, b, prec, nbt):
    xs, ref, got, got2 = _run_batched(fm, N, P, T, b, prec, nbt)
    for i in range(nbt):
        assert np.array_equal(got[i], ref[i]), (i, ol.rel_l2(got[i], ref[i]))
        assert np.array_equal(got2[i], ref[i]), i
    if prec == "f64":  # the FMM's own result at this order (its truncation is above 1e-12)
        assert ol.rel_l2(got[-1], ol.forward(xs[-1], P, T, b)) < 1e-12
    else:
        assert ol.rel_l2(got[-1].astype(np.complex128), np.fft.fft(xs[-1])) < 1e-6


def test_batch_with_coarse_tree_and_tc_everywhere(fm, monkeypatch):
    """The coarse-tree kernel (forced below 4096 rows) and every stage on the tensor
    cores, with S2M as its own stage, in a batch of 5."""
    monkeypatch.setenv("FMMFFT_COARSE_ROWS", "4096")
    monkeypatch.setenv("FMMFFT_TC_MIN_ROWS", "1")
    monkeypatch.setenv("FMMFFT_FUSE_S2M", "0")
    xs, ref, got, got2 = _run_batched(fm, 1 << 16, 16, 16, 32, "f32_tc", 5)
    for i in range(5):
        assert np.array_equal(got[i], ref[i]), i
        assert np.array_equal(got2[i], ref[i]), i


def test_plan_bytes_matches_plan(fm):
    for args in [(1 << 16, 16, 16, 32, "f32_tc", 4), (1 << 18, 64, 24, 32, "f32", 1),
                 (1 << 14, 4, 12, 16, "f64", 2)]:
        est = fm.plan_bytes(*args)
        plan = fm.Plan(*args[:5], max_transforms=args[5])
        assert plan.device_bytes == est, args
        plan.close()


def test_uneven_batch_grouped_by_shape_one_graph(fm):
    """Transforms of uneven sizes grouped by shape: one batched launch sequence per shape, all
    groups as branches of one graph (fmmfft_batch_create_many); every transform bitwise equal to
    its own execute, and within 1e-6 of the FP64 FFT."""
    import torch
    rng = np.random.Generator(np.random.PCG64(12))
    jobs = []
    while len(jobs) < 30:
        N = 1 << int(rng.integers(12, 18))
        P = int(rng.choice([8, 16, 32, 64]))
        if N // P >= 256:
            jobs.append((N, P, 16, 32))
    groups = {}
    for i, j in enumerate(jobs):
        groups.setdefault(j, []).append(i)
    shapes = sorted(groups)
    xs = {i: ol.seeded_input(j[0], 700 + i) for i, j in enumerate(jobs)}
    plans = [fm.Plan(*sh, "f32_tc", max_transforms=len(groups[sh])) for sh in shapes]
    xin = [torch.from_numpy(np.concatenate([xs[i] for i in groups[sh]])).to(torch.complex64).cuda()
           for sh in shapes]
    yout = [torch.empty_like(x) for x in xin]
    batch = fm.Batch(plans, [x.data_ptr() for x in xin], [y.data_ptr() for y in yout], nbranch=5,
                     counts=[len(groups[sh]) for sh in shapes])
    batch.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream().cuda_stream
    for gi, sh in enumerate(shapes):
        alone_plan = fm.Plan(*sh, "f32_tc")
        N = sh[0]
        for j, i in enumerate(groups[sh]):
            d = xin[gi][j * N:(j + 1) * N]
            alone = torch.empty_like(d)
            alone_plan.execute_ptr(d.data_ptr(), alone.data_ptr(), s)
            torch.cuda.synchronize()
            got = yout[gi][j * N:(j + 1) * N]
            assert torch.equal(alone, got), (sh, j)
            assert ol.rel_l2(got.cpu().numpy(), np.fft.fft(xs[i])) < 1e-6
        alone_plan.close()
    batch.close()


@pytest.mark.parametrize("N,P,T,b,prec", [(1 << 18, 64, 24, 32, "f32_tc"), (1 << 14, 4, 12, 16, "f64"),
                                          (4096, 8, 8, 16, "f32_tc"), (1 << 15, 8, 10, 4, "f32"),
                                          (1 << 16, 16, 16, 32, "f32")])
def test_execute_many_ptrs_equals_contiguous(fm, N, P, T, b, prec):
    """fmmfft_execute_many_ptrs: transforms in buffers of their own (here scattered, one of them
    in place) give bitwise the outputs of the contiguous batched execute, for the two-pass and the
    one-pass local FFTs (4096 = 8 x 512), the block-DC bins of FP32 plans and an FP64 plan."""
    import torch
    dt = torch.complex128 if prec == "f64" else torch.complex64
    nbt = 3
    xs = [ol.seeded_input(N, 2000 + i) for i in range(nbt)]
    plan = fm.Plan(N, P, T, b, prec, max_transforms=nbt)
    s = torch.cuda.current_stream().cuda_stream
    cin = torch.from_numpy(np.concatenate(xs)).to(dt).cuda()
    cout = torch.empty_like(cin)
    plan.execute_many_ptr(nbt, cin.data_ptr(), cout.data_ptr(), s)
    ins = [torch.from_numpy(x).to(dt).cuda() for x in xs]
    outs = [torch.empty_like(d) for d in ins]
    outs[1] = ins[1]  # in place
    plan.execute_many_ptrs([d.data_ptr() for d in ins], [o.data_ptr() for o in outs], s)
    torch.cuda.synchronize()
    for i in range(nbt):
        assert torch.equal(outs[i], cout[i * N:(i + 1) * N]), f"transform {i} differs"
    plan.close()

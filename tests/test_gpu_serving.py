"""Graphs, batches and the request server (batched and served transforms) on the GPU.

Each transform is checked against the plain per-call execute of the same plan (bitwise: the
graph replays the same kernels) and against an FP64 FFT (rel-L2 <= 1e-6 for FP32 plans)."""
import numpy as np
import pytest

import oracle_lib as ol
from gpu_util import run_device

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


def _dev(x, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(dt).cuda()


def test_graph_execute_equals_plain_execute(fm):
    import torch
    for N, P, T, b, prec in [(1 << 16, 16, 16, 32, "f32"), (1 << 18, 64, 24, 32, "f32_tc"),
                             (1 << 14, 4, 16, 256, "f64")]:
        x = ol.seeded_input(N, N)
        dt = torch.complex128 if prec == "f64" else torch.complex64
        d = _dev(x, dt)
        y1, y2 = torch.empty_like(d), torch.empty_like(d)
        plan = fm.Plan(N, P, T, b, prec)
        s = torch.cuda.current_stream().cuda_stream
        plan.execute_ptr(d.data_ptr(), y1.data_ptr(), s)
        for _ in range(3):  # first call captures, the rest replay
            y2.zero_()
            plan.execute_graph_ptr(d.data_ptr(), y2.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(y1, y2)


def _uneven_jobs(n, seed):
    """Sizes as in the uneven-batch workload: N log-uniform over powers of two 2^12..2^22, P from
    {8, 16, 32, 64} with M >= 256, p = 16 (scaled down in count for a test)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    jobs = []
    while len(jobs) < n:
        lg = int(rng.integers(12, 19))
        P = int(rng.choice([8, 16, 32, 64]))
        N = 1 << lg
        if N // P < 256:
            continue
        b = 32 if N // P >= 128 else 8
        jobs.append((N, P, 16, b))
    return jobs


def test_uneven_batch_one_graph(fm):
    import torch
    jobs = _uneven_jobs(40, 3)
    plans = {}
    for N, P, T, b in jobs:
        plans.setdefault((N, P, T, b), fm.Plan(N, P, T, b, "f32"))
    xs = [ol.seeded_input(N, 100 + i) for i, (N, P, T, b) in enumerate(jobs)]
    din = [_dev(x, torch.complex64) for x in xs]
    dout = [torch.empty_like(d) for d in din]
    batch = fm.Batch([plans[j] for j in jobs], [d.data_ptr() for d in din],
                     [d.data_ptr() for d in dout], nbranch=6)
    batch.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream().cuda_stream
    for i, (job, x) in enumerate(zip(jobs, xs)):
        alone = torch.empty_like(din[i])
        plans[job].execute_ptr(din[i].data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, dout[i]), job
        assert ol.rel_l2(dout[i].cpu().numpy(), np.fft.fft(x)) < TOL, job
    batch.close()


def test_server_mix_equals_alone(fm):
    """Requests submitted back to back overlap on 4 streams; each result must be bitwise the
    result of the same request run alone."""
    import torch
    jobs = _uneven_jobs(24, 5) + [(1 << 20, 64, 20, 32), (1 << 16, 8, 8, 32)]
    precs = ["f32_tc" if i % 3 == 0 else "f32" for i in range(len(jobs))]
    xs = [ol.seeded_input(N, 900 + i) for i, (N, P, T, b) in enumerate(jobs)]
    din = [_dev(x, torch.complex64) for x in xs]
    mixed = [torch.empty_like(d) for d in din]
    srv = fm.Server(8 << 30, nstreams=4)
    tickets = [srv.submit(N, P, T, b, pr, din[i].data_ptr(), mixed[i].data_ptr())
               for i, ((N, P, T, b), pr) in enumerate(zip(jobs, precs))]
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    assert st["plans"] >= 1 and st["hbm_used"] <= 8 << 30
    srv.close()
    s = torch.cuda.current_stream().cuda_stream
    for i, ((N, P, T, b), pr) in enumerate(zip(jobs, precs)):
        plan = fm.Plan(N, P, T, b, pr)
        alone = torch.empty_like(din[i])
        plan.execute_ptr(din[i].data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, mixed[i]), (N, P, T, b, pr)
        assert ol.rel_l2(mixed[i].cpu().numpy(), np.fft.fft(xs[i])) < TOL


def test_server_admission_by_budget(fm):
    """Plans are admitted under the HBM budget: an idle plan is evicted to make room for a new
    shape, and a request whose plan cannot fit even then is refused (FMMFFT_ERR_BUSY) before
    anything is allocated: the device's free memory is the same before and after."""
    import torch
    N, P, T, b = 1 << 24, 64, 16, 32
    one = fm.plan_bytes(N, P, T, b, "f32", max_transforms=4)  # the server's plan of this shape
    x = _dev(ol.seeded_input(N, 1), torch.complex64)
    y = torch.empty_like(x)
    srv = fm.Server(int(one * 1.5), nstreams=1)  # room for one resident plan of this size
    t = srv.submit(N, P, T, b, "f32", x.data_ptr(), y.data_ptr())
    srv.wait(t)
    assert srv.stats()["plans"] == 1
    # a different shape needs a new plan: the idle one is evicted to make room
    x2 = _dev(ol.seeded_input(N // 2, 2), torch.complex64)
    y2 = torch.empty_like(x2)
    t2 = srv.submit(N // 2, P, T, b, "f32", x2.data_ptr(), y2.data_ptr())
    srv.wait(t2)
    assert srv.stats()["plans"] == 1
    assert ol.rel_l2(y2.cpu().numpy(), np.fft.fft(x2.cpu().numpy())) < TOL
    # a plan larger than the whole budget is refused, not built: nothing is allocated
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with pytest.raises(fm.FmmFftError) as ei:
        srv.submit(4 * N, P, T, b, "f32", x.data_ptr(), y.data_ptr())
    assert ei.value.status == 7
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert srv.stats()["plans"] == 1
    srv.close()


def test_server_batches_concurrent_requests(fm):
    """Continuous batching: 40 requests of one small shape submitted back to back leave in
    batches (several transforms per launch sequence) and each result is bitwise the result of
    the request run alone; requests of another shape interleaved with them are unaffected."""
    import torch
    N, P, T, b = 1 << 14, 16, 16, 32
    xs = [ol.seeded_input(N, 300 + i) for i in range(40)]
    din = [_dev(x, torch.complex64) for x in xs]
    dout = [torch.empty_like(d) for d in din]
    N2 = 1 << 16
    x2 = [ol.seeded_input(N2, 500 + i) for i in range(6)]
    d2 = [_dev(x, torch.complex64) for x in x2]
    o2 = [torch.empty_like(d) for d in d2]
    srv = fm.Server(4 << 30, nstreams=3)
    tickets = []
    for i in range(40):
        tickets.append(srv.submit(N, P, T, b, "f32_tc", din[i].data_ptr(), dout[i].data_ptr()))
        if i % 7 == 0:
            j = i // 7
            tickets.append(srv.submit(N2, 32, 20, 32, "f32_tc", d2[j].data_ptr(), o2[j].data_ptr()))
    for t in tickets:
        srv.wait(t)
    nreq, nlaunch = srv.counts()
    assert nreq == len(tickets) and nlaunch < nreq, (nreq, nlaunch)
    srv.close()
    plan = fm.Plan(N, P, T, b, "f32_tc")
    s = torch.cuda.current_stream().cuda_stream
    for i in range(40):
        alone = torch.empty_like(din[i])
        plan.execute_ptr(din[i].data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, dout[i]), i
    plan.close()
    plan2 = fm.Plan(N2, 32, 20, 32, "f32_tc")
    for j in range(6):
        alone = torch.empty_like(d2[j])
        plan2.execute_ptr(d2[j].data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, o2[j]), j
        assert ol.rel_l2(o2[j].cpu().numpy(), np.fft.fft(x2[j])) < TOL
    plan2.close()


@pytest.mark.parametrize("which", [0], ids=["mbarrier_with_tmem"])
def test_bounded_wait_gives_up_and_reports_timeout(fm, which):
    """The device waits are bounded: a wait for an event that never comes (an mbarrier nobody
    arrives on while the kernel holds tensor memory, as the tensor-core kernels' waits do), with
    a 2 ms limit, gives up, frees what it holds and returns.  The plan's check reports
    FMMFFT_ERR_TIMEOUT once (the status is cleared by reading it), and the plan still computes
    the right transform afterwards."""
    N, P, T, b = 1 << 14, 16, 16, 32
    plan = fm.Plan(N, P, T, b, "f32_tc")
    x = ol.seeded_input(N, 3)
    y0 = run_device(plan, x)
    plan.check()
    plan.selftest_wait(which, 2000)
    with pytest.raises(fm.FmmFftError) as ei:
        plan.check()
    assert ei.value.status == 6  # FMMFFT_ERR_TIMEOUT
    plan.check()  # cleared
    y1 = run_device(plan, x)
    plan.check()
    assert np.array_equal(y0, y1)
    plan.close()


def test_server_reserve_makes_plans_resident(fm):
    """reserve builds a shape's plans (and their batch graphs) before any request: the plan
    count reaches the reserved number at once and requests that follow make no new plan; results
    are bitwise those of the plan run alone.  A reserve beyond the budget is refused."""
    import torch
    N, P, T, b = 1 << 14, 16, 16, 32
    srv = fm.Server(4 << 30, nstreams=3)
    srv.reserve(N, P, T, b, "f32_tc", 2)
    assert srv.stats()["plans"] == 2
    srv.reserve(N, P, T, b, "f32_tc", 2)  # already resident: nothing more
    assert srv.stats()["plans"] == 2
    xs = [ol.seeded_input(N, 700 + i) for i in range(12)]
    din = [_dev(x, torch.complex64) for x in xs]
    dout = [torch.empty_like(d) for d in din]
    ts = [srv.submit(N, P, T, b, "f32_tc", d.data_ptr(), o.data_ptr()) for d, o in zip(din, dout)]
    for t in ts:
        srv.wait(t)
    assert srv.stats()["plans"] <= 3
    plan = fm.Plan(N, P, T, b, "f32_tc")
    s = torch.cuda.current_stream().cuda_stream
    for d, o in zip(din, dout):
        alone = torch.empty_like(d)
        plan.execute_ptr(d.data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, o)
    plan.close()
    srv.close()
    big = fm.plan_bytes(1 << 24, 64, 16, 32, "f32", max_transforms=4)  # the server's plan of this shape
    small = fm.Server(int(big * 1.5), nstreams=3)
    with pytest.raises(fm.FmmFftError) as ei:
        small.reserve(1 << 24, 64, 16, 32, "f32", 3)  # room for one of the three
    assert ei.value.status == 7
    assert small.stats()["plans"] == 1
    small.close()


def test_server_large_requests_batch_in_their_own_buffers(fm):
    """Requests of 2^22 samples batch (up to four per launch sequence) with each request read and
    written in its own buffers: six submitted back to back leave in fewer launches than requests,
    and each result is bitwise that of the request run alone on a plan of its shape."""
    import torch
    N, P, T, b = 1 << 22, 64, 20, 32
    xs = [ol.seeded_input(N, 900 + i) for i in range(6)]
    din = [_dev(x, torch.complex64) for x in xs]
    dout = [torch.empty_like(d) for d in din]
    srv = fm.Server(32 << 30, nstreams=1)
    srv.reserve(N, P, T, b, "f32_tc", 1)
    ts = [srv.submit(N, P, T, b, "f32_tc", d.data_ptr(), o.data_ptr()) for d, o in zip(din, dout)]
    for t in ts:
        srv.wait(t)
    nreq, nlaunch = srv.counts()
    assert nreq == 6 and nlaunch < 6, (nreq, nlaunch)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    s = torch.cuda.current_stream().cuda_stream
    for d, o in zip(din, dout):
        alone = torch.empty_like(d)
        plan.execute_ptr(d.data_ptr(), alone.data_ptr(), s)
        torch.cuda.synchronize()
        assert torch.equal(alone, o)
    plan.close()
    srv.close()

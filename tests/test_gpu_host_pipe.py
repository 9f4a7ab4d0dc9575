"""The pipelined host execute (fmmfft_execute_host_many): a sequence of host-resident transforms
with copy-in, execute and copy-out overlapped on three streams.  Every output is bitwise what the
one-at-a-time host execute gives, for page-locked and pageable buffers, in place and out of
place, and for more transforms than staging buffers (the buffers are reused in turn)."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
@pytest.mark.parametrize("prec", ["f32_tc", "f64"])
def test_host_many_equals_host_one_at_a_time(fm, prec, pinned):
    import torch
    N, P, T, b = 1 << 18, 64, 16, 32
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    plan = fm.Plan(N, P, T, b, prec)
    n = 7  # more than the three staging buffers
    xs = [torch.from_numpy(ol.seeded_input(N, 900 + i)).to(cdt) for i in range(n)]
    if pinned:
        xs = [x.pin_memory() for x in xs]
    outs = [torch.empty_like(x) for x in xs]
    if pinned:
        outs = [o.pin_memory() for o in outs]
    plan.execute_host_many_ptr([x.data_ptr() for x in xs], [o.data_ptr() for o in outs])
    for i in range(n):
        one = torch.empty_like(xs[i])
        plan.execute_host_ptr(xs[i].data_ptr(), one.data_ptr())
        assert torch.equal(one, outs[i]), i
        tol = 1e-12 if prec == "f64" else 1e-6
        assert ol.rel_l2(outs[i].numpy(), np.fft.fft(xs[i].numpy())) < tol
    # in place, and an empty sequence
    ys = [x.clone() for x in xs[:4]]
    plan.execute_host_many_ptr([y.data_ptr() for y in ys], [y.data_ptr() for y in ys])
    for i in range(4):
        assert torch.equal(ys[i], outs[i])
    plan.execute_host_many_ptr([], [])
    plan.close()

"""The allocation-free entry point, fmmfft_execute_noalloc, against the regular plan path.

Some callers of this library cannot call cudaMalloc: they run under a device-memory budget
that someone else owns, or in a phase where they may not allocate at all.  For them the library
keeps the operator tables and the workspace of one transform in a static device array and
allocates nothing.  This file checks, through the C-ABI, that the entry point gives the same
result as fmmfft_execute on an FMMFFT_F32 plan (rel-L2 <= 1e-6, the FP32 tolerance used by
every FP32 parity test), on two calls in a row (the second call runs on the array the first one
left behind), for a one-pass and a two-pass local-FFT size, and that sizes beyond the array's
limit are refused.  The file is named to be collected last.
"""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-6


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


def _plan_result(fm, plan, x):
    import torch
    d_in = torch.from_numpy(x).to(torch.complex64).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute_ptr(d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().astype(np.complex128)


def _noalloc_result(fm, N, P, T, b, x):
    import torch
    d_in = torch.from_numpy(x).to(torch.complex64).cuda()
    d_out = torch.empty_like(d_in)
    fm.execute_noalloc(N, P, T, b, d_in.data_ptr(), d_out.data_ptr(),
                       torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("N,P,T,b", [(1 << 18, 64, 24, 32),   # M = 4096: one FFT pass
                                     (1 << 18, 16, 16, 32)])  # M = 16384: two FFT passes
def test_noalloc_matches_plan_on_two_calls_in_a_row(fm, N, P, T, b):
    plan = fm.Plan(N, P, T, b, "f32")
    xs = [ol.seeded_input(N, 100 + k) for k in range(2)]
    refs = [_plan_result(fm, plan, x) for x in xs]
    plan.close()
    for x, ref in zip(xs, refs):  # two calls in a row on the shared array
        got = _noalloc_result(fm, N, P, T, b, x)
        assert ol.rel_l2(got, ref) <= TOL_F32
        assert ol.rel_l2(got, np.fft.fft(x)) <= TOL_F32


def test_noalloc_refuses_sizes_beyond_its_array(fm):
    import torch
    N, P, T, b = 1 << 22, 64, 24, 32  # tables + workspace far above 32 MiB
    d = torch.empty(16, dtype=torch.complex64, device="cuda")
    with pytest.raises(fm.FmmFftError) as ei:
        fm.execute_noalloc(N, P, T, b, d.data_ptr(), d.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    assert ei.value.status == 1
    assert "32" in str(ei.value) or "limit" in str(ei.value)

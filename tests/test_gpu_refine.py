"""The optional FP64 residual-correction pass (fmmfft_execute_refined) of complex64 plans.

One step y = y1 + F~(x - F64^-1(y1) / N) moves the result from FP32-level agreement with the FP64
FMM-FFT (the reference's arithmetic) to about the square of it: against the FP64 plan's own
output the refined result must agree to 1e-11 (FP32 plans agree to ~1e-7), and against the FP64
FFT it reaches the FMM's truncation at that order."""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


@pytest.mark.parametrize("N,P,T,b,prec", [(1 << 16, 16, 16, 32, "f32"), (1 << 20, 64, 24, 32, "f32_tc"),
                                          (1 << 18, 256, 20, 16, "f32_tc")])
def test_refined_matches_fp64_fmm(fm, accuracy_report, N, P, T, b, prec):
    import torch
    x = ol.seeded_input(N, 77).astype(np.complex64)
    x128 = x.astype(np.complex128)
    p64 = fm.Plan(N, P, T, b, "f64")
    d64 = torch.from_numpy(x128).cuda()
    o64 = torch.empty_like(d64)
    p64.execute_ptr(d64.data_ptr(), o64.data_ptr())
    torch.cuda.synchronize()
    y64 = o64.cpu().numpy()
    p64.close()
    plan = fm.Plan(N, P, T, b, prec)
    plan.enable_refinement()
    d = torch.from_numpy(x).cuda()
    y1 = torch.empty_like(d)
    plan.execute_ptr(d.data_ptr(), y1.data_ptr())
    out = torch.empty(N, dtype=torch.complex128, device="cuda")
    plan.execute_refined_ptr(d.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    plan.check()
    yr = out.cpu().numpy()
    e1 = ol.rel_l2(y1.cpu().numpy().astype(np.complex128), y64)
    er = ol.rel_l2(yr, y64)
    ef = ol.rel_l2(yr, np.fft.fft(x128))
    accuracy_report(f"N={N} P={P} T={T} b={b} {prec}: plain vs FP64 FMM {e1:.3e}; refined vs FP64 FMM "
                    f"{er:.3e}, vs FP64 FFT {ef:.3e}")
    assert e1 < 1e-6
    assert er < 1e-11, er
    assert ef < max(1e-9, 2 * ol.rel_l2(y64, np.fft.fft(x128)))
    plan.close()

"""Accuracy at the sizes and orders of the headline workloads, through the C-ABI.

* Precision sweep shapes: N = 2^26 complex64, P = 256, b = 32, terms in {8, 16, 24, 32}, input a
  sum of 32 off-bin tones plus 1e-3 white noise (seeded).  Each FP32 plan (CUDA cores and split
  TF32 on the tensor cores) is compared with the FP64 plan of the same order, which is the
  reference's arithmetic at that order (the FP64 plans match the oracle and the reference's
  golden vectors to 1e-12 in test_gpu_parity.py): rel-L2 <= 1e-6.  Against the FP64 FFT of the
  same input the FP64 plan shows the FMM's own truncation at that order; from 16 terms on that is
  below 1e-6 and the FP32 plans must be within 1e-6 of the FFT too.
* 32 terms through every tensor-core stage at small sizes (M2L K = 160, leaf K = T + 3b),
  stage by stage against the FP64 oracle.
* The single large transform (N = 2^24, P = 64, 24 terms, b = 32, seed 0) against the output of
  the reference itself (src/fmmfft.c built against the project's MPI/FFTW shims, oracle/_ref),
  when that library was built.
Each case prints its rel-L2 and max error (max |y - ref| / max |ref|) in the run's summary.
"""
import os

import numpy as np
import pytest

import oracle_lib as ol
from gpu_util import run_device

pytestmark = pytest.mark.gpu
TOL = 1e-6
TOL_STAGE = 1e-4


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


def max_err(y, ref):
    return float(np.max(np.abs(y - ref)) / np.max(np.abs(ref)))


@pytest.fixture(scope="module")
def sweep_input():
    N = 1 << 26
    x = ol.tone_input(N, 2026).astype(np.complex64).astype(np.complex128)
    return x, np.fft.fft(x)


@pytest.mark.parametrize("T", [8, 16, 24, 32])
def test_sweep_shape_n2p26_p256(fm, sweep_input, accuracy_report, T):
    x, ref = sweep_input
    N, P, b = x.size, 256, 32
    p64 = fm.Plan(N, P, T, b, "f64")
    y64 = run_device(p64, x)
    p64.close()
    trunc = ol.rel_l2(y64, ref)
    accuracy_report(f"N=2^26 P=256 T={T} b=32 tones: f64 plan vs FP64 FFT rel-L2 {trunc:.3e} "
                    f"max {max_err(y64, ref):.3e}")
    for prec in ("f32", "f32_tc"):
        plan = fm.Plan(N, P, T, b, prec)
        y = run_device(plan, x)
        plan.check()
        plan.close()
        e64 = ol.rel_l2(y, y64)
        efft = ol.rel_l2(y, ref)
        accuracy_report(f"N=2^26 P=256 T={T} b=32 tones: {prec} vs f64 plan rel-L2 {e64:.3e} "
                        f"max {max_err(y, y64):.3e}; vs FP64 FFT rel-L2 {efft:.3e}")
        assert e64 < TOL, (prec, e64)
        if T >= 16:
            assert trunc < TOL
            assert efft < TOL, (prec, efft)


T32_CASES = [(65536, 16, 32, 32), (1 << 18, 64, 32, 32), (1 << 18, 256, 32, 16), (1 << 18, 8, 32, 64)]


@pytest.mark.parametrize("N,P,T,b", T32_CASES)
def test_32_terms_every_tensor_core_stage(fm, monkeypatch, accuracy_report, N, P, T, b):
    monkeypatch.setenv("FMMFFT_TC_MIN_ROWS", "1")   # read when the plan is made
    monkeypatch.setenv("FMMFFT_FUSE_S2M", "0")      # S2M as its own tensor-core stage
    x = ol.seeded_input(N, 71 + N % 53)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    y = run_device(plan, x)
    plan.check()
    d = plan.debug_fetch()
    M = N // P
    n = (M // b).bit_length() - 1
    for lev in range(2, n + 1):
        gp = fm.level_planar(d["phi"], P, T, n, lev)
        gs = fm.level_planar(d["psi"], P, T, n, lev)
        gp = (gp[:, 0] + 1j * gp[:, 1]).transpose(1, 0, 2)
        gs = (gs[:, 0] + 1j * gs[:, 1]).transpose(1, 0, 2)
        assert ol.rel_l2(gp, o["phi"][ol.level_slice(lev)]) < TOL_STAGE, ("phi", lev)
        assert ol.rel_l2(gs, o["psi"][ol.level_slice(lev)]) < TOL_STAGE, ("psi", lev)
    assert ol.rel_l2(d["u"], o["u"]) < TOL_STAGE
    e = ol.rel_l2(y, o["y"])
    accuracy_report(f"N={N} P={P} T=32 b={b} f32_tc every stage on the tensor cores: vs oracle "
                    f"rel-L2 {e:.3e} max {max_err(y, o['y']):.3e}")
    assert e < TOL


def test_single_large_transform_vs_reference_output(fm, accuracy_report):
    """N = 2^24 complex64, P = 64, 24 terms, b = 32, seed 0: the FP32 plans against the
    reference's own FMM output for the same input (P = 64 thread-ranks on the host CPU)."""
    if ol.load_reference() is None:
        pytest.skip("oracle/_ref (the shim-built reference) was not built")
    N, P, T, b = 1 << 24, 64, 24, 32
    x = ol.seeded_input(N, 0).astype(np.complex64).astype(np.complex128)
    yr = ol.reference_forward(x, P, T, b)
    for prec in ("f32", "f32_tc"):
        plan = fm.Plan(N, P, T, b, prec)
        y = run_device(plan, x)
        plan.check()
        plan.close()
        e = ol.rel_l2(y, yr)
        accuracy_report(f"N=2^24 P=64 T=24 b=32 normal: {prec} vs reference output rel-L2 {e:.3e} "
                        f"max {max_err(y, yr):.3e}")
        assert e < TOL, (prec, e)


BF16_CASES = [(65536, 16, 8, 32), (1 << 18, 64, 8, 32), (1 << 18, 256, 12, 16), (1 << 16, 8, 16, 64)]


@pytest.mark.parametrize("N,P,T,b", BF16_CASES)
def test_bf16x3_tensor_core_stages(fm, monkeypatch, accuracy_report, N, P, T, b):
    """BF16x3 (BF16 hi + lo operands, three products, FP32 accumulation) on every tensor-core
    stage, for the 1e-4 accuracy class: stage outputs and the transform against the FP64 oracle
    of the same order, rel-L2 <= 1e-4."""
    monkeypatch.setenv("FMMFFT_TC_MIN_ROWS", "1")
    monkeypatch.setenv("FMMFFT_FUSE_S2M", "0")
    x = ol.seeded_input(N, 91 + N % 41)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "bf16x3")
    y = run_device(plan, x)
    plan.check()
    d = plan.debug_fetch()
    M = N // P
    n = (M // b).bit_length() - 1
    for lev in range(2, n + 1):
        gs = fm.level_planar(d["psi"], P, T, n, lev)
        gs = (gs[:, 0] + 1j * gs[:, 1]).transpose(1, 0, 2)
        assert ol.rel_l2(gs, o["psi"][ol.level_slice(lev)]) < 1e-3, ("psi", lev)
    eu = ol.rel_l2(d["u"], o["u"])
    e = ol.rel_l2(y, o["y"])
    accuracy_report(f"N={N} P={P} T={T} b={b} bf16x3 every stage on the tensor cores: u rel-L2 {eu:.3e}, "
                    f"y vs oracle rel-L2 {e:.3e} max {max_err(y, o['y']):.3e}")
    assert e < 1e-4


@pytest.mark.parametrize("N,P,T,b", [(1 << 20, 64, 24, 32), (1 << 22, 16, 20, 32), (1 << 18, 256, 16, 16)])
def test_compensated_twiddles(fm, monkeypatch, accuracy_report, N, P, T, b):
    """The FP32 FFT passes (the combine's length-P DFT and the size-M FFTs) with twiddles carried
    as FP32 hi + lo pairs (the tensor-core plans' default) against single FP32 twiddles: both
    within 1e-6 of the FP64 FFT; the errors of both are reported."""
    x = ol.seeded_input(N, 19 + N % 13)
    ref = np.fft.fft(x.astype(np.complex64).astype(np.complex128))
    errs = {}
    for comp in ("1", "0"):
        monkeypatch.setenv("FMMFFT_COMP_TWIDDLES", comp)
        plan = fm.Plan(N, P, T, b, "f32_tc")
        y = run_device(plan, x)
        plan.check()
        plan.close()
        errs[comp] = (ol.rel_l2(y, ref), max_err(y, ref))
    accuracy_report(f"N={N} P={P} T={T} b={b} f32_tc: compensated twiddles rel-L2 {errs['1'][0]:.3e} "
                    f"max {errs['1'][1]:.3e}; single FP32 twiddles rel-L2 {errs['0'][0]:.3e} max {errs['0'][1]:.3e}")
    assert errs["1"][0] < TOL and errs["0"][0] < TOL

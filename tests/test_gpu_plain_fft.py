"""GPU parity of the plain size-N FFT (fmmfft_fft_*), the comparator that stands where the
reference's FFTW programs stand (src/fftw_serial.c:53-58, src/fftw_mpi.c:54-58).

The oracle is the project's FP64 FFT (oracle/fft64.c, the FFTW stand-in the shim-built
reference links) cross-checked by numpy.  Tolerances: complex128 plans rel-L2 <= 1e-12,
complex64 plans rel-L2 <= 1e-6 (the accuracy bar of the FP32 FMM-FFT).
"""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12
TOL_F32 = 1e-6

# one, two and three passes, and the edges between them (4096 | 8192, 2^21 | 2^22)
SIZES = [16, 64, 512, 4096, 8192, 1 << 14, 1 << 17, 1 << 21, 1 << 22, 1 << 24]


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


def _oracle_fft(x):
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    assert ol.load().orc_fft64(len(y), y.ctypes.data) == 0
    return y


def _run(fm, N, prec, x):
    import torch
    dt = torch.complex128 if prec == "f64" else torch.complex64
    f = fm.PlainFFT(N, prec)
    xd = torch.from_numpy(x).to(dt).cuda()
    yd = torch.empty_like(xd)
    f.execute_ptr(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    f.close()
    return yd.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("N", SIZES)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_plain_fft_matches_oracle(fm, N, prec):
    x = ol.seeded_input(N, 7)
    ref = _oracle_fft(x)
    if N <= 1 << 16:
        assert ol.rel_l2(ref, np.fft.fft(x)) < 1e-13
    got = _run(fm, N, prec, x)
    assert ol.rel_l2(got, ref) < (TOL_F64 if prec == "f64" else TOL_F32)


def test_plain_fft_agrees_with_fmmfft(fm):
    """Two different algorithms, the same transform: plain FFT and FMM-FFT (FP64)."""
    import torch
    N = 1 << 16
    x = ol.seeded_input(N, 3)
    plan = fm.Plan(N, 16, 16, 32, "f64")
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    plan.execute_ptr(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = _run(fm, N, "f64", x)
    assert ol.rel_l2(yd.cpu().numpy(), got) < 1e-12


def test_plain_fft_linearity_full_size(fm):
    """At 2^24: FFT(a x + b y) = a FFT(x) + b FFT(y), and the DC bin is the sum."""
    N = 1 << 24
    x = ol.seeded_input(N, 11)
    y = ol.seeded_input(N, 12)
    a, b = 0.75 - 0.5j, -1.25 + 2.0j
    fx, fy = _run(fm, N, "f32", x), _run(fm, N, "f32", y)
    fz = _run(fm, N, "f32", a * x + b * y)
    assert ol.rel_l2(fz, a * fx + b * fy) < 2e-6
    assert abs(fx[0] - x.sum()) / np.abs(x).sum() < 1e-6


def test_plain_fft_rejects_bad_sizes_and_in_place(fm):
    import torch
    for bad in (8, 12, 3 << 10, 1 << 31):
        with pytest.raises(fm.FmmFftError):
            fm.PlainFFT(bad, "f32")
    f = fm.PlainFFT(1024, "f32")
    xd = torch.zeros(1024, dtype=torch.complex64, device="cuda")
    with pytest.raises(fm.FmmFftError):
        f.execute_ptr(xd.data_ptr(), xd.data_ptr())
    assert f.device_bytes() >= 1024 * 8
    f.close()

"""CPU tests of the oracle itself: it must agree with the reference before it can check the GPU.

Pins (reference = 97amarnathk/fmm-fft src/fmmfft.c):
  * golden vectors made by running the unmodified reference (tests/golden/make_golden.py);
  * the reference's own recorded error envelope (plotting/raw_data/cluster_output_error.csv);
  * the shim-built reference itself, when oracle/_ref was built in this container;
  * the dense FP64 DFT (numpy pocketfft).
"""
import csv
import glob
import hashlib
import os

import numpy as np
import pytest

import oracle_lib as ol

GOLDEN_FILES = sorted(glob.glob(os.path.join(ol.GOLDEN, "ref_forward_*.npz")))


def test_golden_files_present():
    assert len(GOLDEN_FILES) >= 8


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=os.path.basename)
def test_oracle_matches_reference_golden_vectors(path):
    g = np.load(path)
    N, P, T, b, seed = (int(g[k]) for k in ("N", "P", "terms", "b", "seed"))
    x = ol.seeded_input(N, seed)
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g["x_sha256"])
    y = ol.forward(x, P, T, b)
    ref = g["y"]
    # same algorithm in FP64, different summation grouping only: a few ulps
    assert ol.rel_l2(y, ref) < 1e-14
    assert np.max(np.abs(y - ref)) < 1e-13 * np.max(np.abs(ref))


def _recorded_rows(max_n):
    with open(os.path.join(ol.GOLDEN, "recorded_error_envelope.csv")) as f:
        rows = [r for r in csv.DictReader(f)]
    return [r for r in rows if int(r["N"]) <= max_n]


@pytest.mark.parametrize("row", _recorded_rows(2 ** 20), ids=lambda r: f"N{r['N']}_P{r['P']}")
def test_recorded_error_envelope(row):
    """Ramp input x[i] = i + 1 (fmmfft_error.c:1236-1247), b = 32, T = 15: the max pointwise
    relative error of block 0 against an FP64 FFT, printed with %lf (fmmfft_error.c:1267),
    must equal the reference's recorded value."""
    N, P, b, T = (int(row[k]) for k in ("N", "P", "b", "T"))
    M = N // P
    x = np.arange(1, N + 1).astype(np.complex128)
    y = ol.forward(x, P, T, b)
    yf = np.fft.fft(x)
    lib = ol.load()
    err = lib.orc_max_error_percent(y.ctypes.data, yf.ctypes.data, M)
    assert "%f" % err == row["err_percent"]


@pytest.mark.slow
@pytest.mark.parametrize("row", [r for r in _recorded_rows(2 ** 22) if int(r["N"]) > 2 ** 20],
                         ids=lambda r: f"N{r['N']}_P{r['P']}")
def test_recorded_error_envelope_large(row):
    test_recorded_error_envelope(row)


@pytest.mark.parametrize("N,P,T,b", [(1024, 4, 16, 16), (4096, 8, 20, 32), (8192, 2, 16, 64),
                                     (16384, 16, 24, 32), (65536, 4, 16, 2048)])
def test_oracle_vs_dense_fp64_dft(N, P, T, b):
    x = ol.seeded_input(N, 11)
    y = ol.forward(x, P, T, b)
    assert ol.rel_l2(y, np.fft.fft(x)) < 1e-11


def test_fft64_vs_numpy():
    lib = ol.load()
    for n in (1, 2, 8, 1024, 1 << 15):
        x = ol.seeded_input(n, n)
        y = x.copy()
        assert lib.orc_fft64(n, y.ctypes.data) == 0
        assert ol.rel_l2(y, np.fft.fft(x)) < 1e-14 * max(1.0, np.log2(n))


def test_oracle_rejects_bad_parameters():
    lib = ol.load()
    for M, P, T, b in [(1024, 3, 8, 16), (1000, 4, 8, 8), (64, 4, 8, 32), (1024, 4, 1, 16),
                       (1024, 4, 8, 1), (1024, 1, 8, 16)]:
        assert not lib.orc_plan_create(M, P, T, b)


def test_intermediates_identity():
    """z_r = DFT over sections of the pre-twiddled u (the combine of fmmfft.c:956-968 is a
    length-P DFT with twiddles); y = FFT_M(z_r) per block."""
    N, P, T, b = 4096, 8, 12, 16
    M = N // P
    x = ol.seeded_input(N, 3)
    o = ol.forward_ex(x, P, T, b)
    sc = np.arange(1, P)
    c = -np.exp(-1j * np.pi * sc / P) * np.sin(np.pi * sc / P)
    w = np.zeros((P, M), np.complex128)
    w[0] = x[0::P]
    w[1:] = c[:, None] * (o["u"] - o["ssum"][:, None])
    z = np.fft.fft(w, axis=0)
    assert ol.rel_l2(z, o["z"]) < 1e-14
    assert ol.rel_l2(np.fft.fft(o["z"], axis=1).ravel(), o["y"]) < 1e-14
    assert np.allclose(o["ssum"], 1j / M * x.reshape(M, P)[:, 1:].sum(axis=0), rtol=1e-13)


ref_needed = pytest.mark.skipif(ol.load_reference() is None,
                                reason="shim-built reference (oracle/_ref) not built here")


@ref_needed
@pytest.mark.parametrize("N,P,T,b", [(256, 2, 8, 8), (2048, 4, 10, 8), (4096, 8, 12, 16),
                                     (8192, 8, 9, 32), (32768, 64, 8, 8), (4096, 16, 6, 16)])
def test_oracle_vs_shim_built_reference(N, P, T, b):
    ref = ol.load_reference()
    x = ol.seeded_input(N, N + P)
    yr = np.zeros(N, np.complex128)
    assert ref.fmmref_forward(N, P, T, b, x.ctypes.data, yr.ctypes.data, 1, None) == 0
    assert ol.rel_l2(ol.forward(x, P, T, b), yr) < 1e-14


@ref_needed
@pytest.mark.parametrize("M,P,T,b", [(256, 4, 8, 8), (1024, 8, 12, 16), (2048, 2, 16, 32),
                                     (16384, 4, 16, 2048), (4096, 64, 24, 32)])
def test_operators_bitwise_equal_to_reference(M, P, T, b):
    """Every operator mfti builds (fmmfft.c:337-382) agrees bit for bit."""
    ref = ol.load_reference()
    lib = ol.load()
    wl = ref.fmmref_wlen(M, P, T, b)
    assert wl == lib.orc_getwlen2(M, T, P, b)
    assert ref.fmmref_vlen(M, P, T, b) == lib.orc_getvlen(M, T, P, b)
    w_ref = np.zeros(wl)
    v_ref = np.zeros(ref.fmmref_vlen(M, P, T, b))
    ref.fmmref_mfti(M, P, T, b, w_ref.ctypes.data, v_ref.ctypes.data)
    pl = lib.orc_plan_create(M, P, T, b)
    w = np.zeros(wl)
    assert lib.orc_fill_reference_w(pl, w.ctypes.data, wl) == 0
    lib.orc_plan_destroy(pl)
    n = (M // b).bit_length() - 1
    n_ops = 8 * T * T * (n - 2) + T * T + T * b + T * (P - 1) * b + T * P // 2 \
        + 3 * b * P // 2 + 3 * b * (b - 1) * (P - 1) + 3 * b * P // 2 + T + 2 * (P - 1) * P
    assert np.array_equal(w[:n_ops].view(np.uint64), w_ref[:n_ops].view(np.uint64))

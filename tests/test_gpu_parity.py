"""GPU parity: the sm_100a FMM-FFT through the C-ABI against the oracle and the reference.

Tolerances: FP64 plans agree with the reference's FP64 result to
rel-L2 <= 1e-12; FP32 plans (complex64) agree with the FP64 oracle / FP64 DFT to rel-L2 <= 1e-6.
"""
import glob
import os

import numpy as np
import pytest

import oracle_lib as ol
from gpu_util import run_device

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12
TOL_F32 = 1e-6

GOLDEN_FILES = sorted(glob.glob(os.path.join(ol.GOLDEN, "ref_forward_*.npz")))


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=os.path.basename)
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_golden_reference_vectors(fm, path, prec):
    g = np.load(path)
    N, P, T, b, seed = (int(g[k]) for k in ("N", "P", "terms", "b", "seed"))
    x = ol.seeded_input(N, seed)
    plan = fm.Plan(N, P, T, b, prec)
    y = run_device(plan, x)
    err = ol.rel_l2(y, g["y"])
    assert err < (TOL_F64 if prec == "f64" else TOL_F32), err


CASES = [  # (N, P, terms, b): t = s/P in {<1, 1, 2, >2}, P = 2, n = 2, odd log2 sizes
    (64, 2, 4, 4), (256, 4, 6, 8), (512, 8, 8, 4), (2048, 2, 8, 64), (4096, 16, 10, 16),
    (8192, 4, 12, 256), (16384, 64, 8, 16), (32768, 8, 16, 32), (65536, 32, 12, 16),
    (131072, 128, 10, 8), (1 << 18, 4, 16, 1024),
]


@pytest.mark.parametrize("N,P,T,b", CASES)
def test_f64_matches_oracle_stagewise(fm, N, P, T, b):
    x = ol.seeded_input(N, N + 7 * P)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f64")
    y = run_device(plan, x)
    assert ol.rel_l2(y, o["y"]) < TOL_F64
    d = plan.debug_fetch()
    M = N // P
    s = M // b
    n = s.bit_length() - 1
    # expansions, every level, against the oracle (planar -> box-major)
    for lev in range(2, n + 1):
        ref_phi = o["phi"][ol.level_slice(lev)]  # [boxes, P-1, T]
        ref_psi = o["psi"][ol.level_slice(lev)]
        got_phi = fm.level_planar(d["phi"], P, T, n, lev)  # [P-1, 2, boxes, T]
        got_psi = fm.level_planar(d["psi"], P, T, n, lev)
        gp = (got_phi[:, 0] + 1j * got_phi[:, 1]).transpose(1, 0, 2)
        gs = (got_psi[:, 0] + 1j * got_psi[:, 1]).transpose(1, 0, 2)
        assert ol.rel_l2(gp, ref_phi) < TOL_F64, lev
        assert ol.rel_l2(gs, ref_psi) < TOL_F64, lev
    assert ol.rel_l2(d["z"], o["z"]) < TOL_F64


@pytest.mark.parametrize("N,P,T,b", CASES)
def test_f32_matches_oracle(fm, N, P, T, b):
    x = ol.seeded_input(N, N + 3 * P)
    yo = ol.forward(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f32")
    y = run_device(plan, x)
    assert ol.rel_l2(y, yo) < TOL_F32


def test_inverse_is_unnormalised_idft(fm):
    N, P, T, b = 16384, 8, 16, 32
    x = ol.seeded_input(N, 5)
    for prec, tol in (("f64", TOL_F64), ("f32", TOL_F32)):
        plan = fm.Plan(N, P, T, b, prec)
        y = run_device(plan, x, inverse=True)
        ref = np.fft.ifft(x) * N
        assert ol.rel_l2(y, ref) < tol


def test_compat_mfti_mft_host_path(fm):
    """The reference's own calling sequence (fmmfft.c:1222-1260) through the C-ABI with host
    buffers: getwlen2/getvlen sizes, mfti fills w, mft transforms qr in place."""
    g = np.load(os.path.join(ol.GOLDEN, "ref_forward_N65536_P4_T16_b2048.npz"))
    N, P, T, b, seed = (int(g[k]) for k in ("N", "P", "terms", "b", "seed"))
    lq = N // P
    w = np.zeros(fm.getwlen2(lq, T, P, b))
    v = np.zeros(fm.getvlen(lq, T, P, b))
    fm.mfti(lq, P, T, b, w, v)
    qr = ol.seeded_input(N, seed)
    fm.mft(lq, qr, 1, P, 0, T, b, w, v)
    assert ol.rel_l2(qr, g["y"]) < TOL_F64


def test_in_place_execution(fm):
    import torch
    N, P, T, b = 65536, 16, 12, 32
    x = ol.seeded_input(N, 9)
    plan = fm.Plan(N, P, T, b, "f32")
    d = torch.from_numpy(x).to(torch.complex64).cuda()
    plan.execute_ptr(d.data_ptr(), d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ol.rel_l2(d.cpu().numpy(), np.fft.fft(x)) < TOL_F32


def test_config2_full_size_vs_fp64_fft(fm):
    """N = 2^24 complex64, P = 64, p = 24, b = 32: rel-L2 and max error against an FP64 FFT."""
    N, P, T, b = 1 << 24, 64, 24, 32
    x = ol.seeded_input(N, 0)
    plan = fm.Plan(N, P, T, b, "f32")
    y = run_device(plan, x)
    ref = np.fft.fft(x)
    assert ol.rel_l2(y, ref) < TOL_F32
    assert np.max(np.abs(y - ref)) / np.max(np.abs(ref)) < 1e-5


def test_repeat_runs_bitwise_deterministic(fm):
    N, P, T, b = 1 << 18, 64, 16, 32
    x = ol.seeded_input(N, 1)
    plan = fm.Plan(N, P, T, b, "f32")
    y1 = run_device(plan, x)
    y2 = run_device(plan, x)
    assert np.array_equal(y1, y2)


def test_plan_made_before_a_smaller_one_still_runs(fm):
    """Kernel-wide launch limits set while making a plan must not depend on the plan made last:
    a 24-term plan, then a 4-term plan, then the 24-term plan executes (the coarse-tree kernel
    takes shared memory that grows with the terms)."""
    N, P, b = 1 << 23, 64, 32
    x = ol.seeded_input(N, 21)
    big = fm.Plan(N, P, 24, b, "f32")
    small = fm.Plan(N, P, 4, b, "f32")
    y = run_device(big, x)
    assert ol.rel_l2(y, np.fft.fft(x)) < TOL_F32
    y2 = run_device(small, x)
    assert np.all(np.isfinite(y2))


COARSE_CASES = [(4096, 16, 10, 16), (32768, 8, 7, 32), (65536, 32, 12, 16), (131072, 4, 9, 16)]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,P,T,b", COARSE_CASES)
def test_coarse_tree_kernel_forced(fm, monkeypatch, N, P, T, b, prec):
    """Every tree level the coarse-tree kernel takes (FMMFFT_COARSE_ROWS above every level's row
    count, read when the plan is made: levels up to 64 boxes per plane, one block per plane)
    there.  The level operators are prefetched into shared memory while the level before runs:
    in 16-byte pieces for even T, one element per copy for odd T.  Same tolerances as the
    plans' own paths."""
    monkeypatch.setenv("FMMFFT_COARSE_ROWS", str(1 << 40))
    x = ol.seeded_input(N, N + 3 * P)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, prec)
    plan.profile_start(1)
    y = run_device(plan, x)
    _, stages = plan.profile_stop()
    assert stages["coarse_tree"][1] == 1, stages
    assert ol.rel_l2(y, o["y"]) < (TOL_F64 if prec == "f64" else TOL_F32)


@pytest.mark.parametrize("lq,p,T,b", [(4096, 4, 12, 32), (16384, 16, 16, 32), (2048, 8, 10, 16)])
def test_mft_rank_mode_per_rank_blocks(fm, lq, p, T, b):
    """The reference's SPMD calling pattern: p threads call mft, each with ONLY its own block
    (rank myid's lq values); every block comes back holding that rank's outputs, equal to the
    full-vector call's and to the reference's golden outputs where the shape has one."""
    import threading
    N = lq * p
    x = ol.seeded_input(N, 5 + p)
    full = x.copy()
    fm.mft(lq, full, 1, p, 0, T, b)
    blocks = [x[r * lq:(r + 1) * lq].copy() for r in range(p)]
    res = {}

    def rank(r):
        try:
            fm.mft(lq, blocks[r], 1, p, r, T, b)
            res[r] = 0
        except fm.FmmFftError as e:
            res[r] = e.status

    fm.mft_rank_mode(True)
    try:
        th = [threading.Thread(target=rank, args=(r,)) for r in range(p)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        fm.mft_rank_mode(False)
    assert all(v == 0 for v in res.values()) and len(res) == p, res
    got = np.concatenate(blocks)
    assert np.array_equal(got, full)
    assert ol.rel_l2(got, ol.forward(x, p, T, b)) < TOL_F64


def test_execute_blocks_device_and_host(fm):
    """Block-distributed I/O: P separate device blocks (and P host blocks) in, P blocks out,
    bitwise the result of the contiguous execute."""
    import torch
    N, P, T, b = 1 << 16, 16, 16, 32
    x = ol.seeded_input(N, 41)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    y = run_device(plan, x)
    M = N // P
    xs = [torch.from_numpy(x[r * M:(r + 1) * M]).to(torch.complex64).cuda() for r in range(P)]
    ys = [torch.empty_like(t) for t in xs]
    plan.execute_blocks_ptr([t.data_ptr() for t in xs], [t.data_ptr() for t in ys])
    torch.cuda.synchronize()
    got = np.concatenate([t.cpu().numpy() for t in ys]).astype(np.complex128)
    assert np.array_equal(got, y)
    hx = [np.ascontiguousarray(x[r * M:(r + 1) * M].astype(np.complex64)) for r in range(P)]
    plan.execute_blocks_ptr([a.ctypes.data for a in hx], [a.ctypes.data for a in hx], host=True)
    assert np.array_equal(np.concatenate(hx).astype(np.complex128), y)
    plan.close()

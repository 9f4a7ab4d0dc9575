"""Host-side parts of bench.py, without a GPU: the algorithmic bytes that the roofline divides by,
and the seeded workloads of the serving and uneven-batch measurements (deterministic, within the
stated distributions, and shapes that a plan accepts)."""
import os
import sys

import numpy as np
import pytest

import oracle_lib as ol

sys.path.insert(0, ol.REPO)


@pytest.fixture(scope="module")
def bench():
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        import bench as b
    finally:
        sys.argv = argv
    return b


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    if not os.path.exists(fmmfft.LIB_PATH):
        import build_lib  # fmm-fft_b200/build_lib.py
        build_lib.build()
    fmmfft.load()
    return fmmfft


def test_stage_bytes_of_the_headline_transform(bench):
    """N = 2^24 complex64, P = 64, 24 terms, b = 32: each stage's arrays counted once."""
    sb = bench.stage_bytes(1 << 24, 64, 24, 32, 8)
    M, S1, R = (1 << 24) // 64, 63, 4
    lv = lambda l: 2 * S1 * 24 * (1 << l) * R  # one level of expansions, both planes
    n = 13  # 2^13 leaf boxes per section
    assert sb["sections"] == (1 << 24) * 8 + 2 * 64 * M * R + lv(n)  # x in, planar sections + S2M out
    assert sb["s2m"] == 0  # fused into the sections pass
    assert sb["leaf_l2t_near"] == lv(n) + 2 * S1 * M * R + 2 * S1 * M * R
    assert sb["combine_dftP"] == 2 * M * R + 2 * S1 * M * R + (1 << 24) * 8
    assert sb["fft_pass1"] == sb["fft_pass2"] == 2 * (1 << 24) * 8
    # every tree level is counted once between the fine-level launches and the coarse-tree launch
    assert sb["m2m"] + sb["coarse_tree"] + sb["m2l_l2l"] == \
        sum(lv(l + 1) + lv(l) for l in range(2, n)) + 2 * lv(2) + sum(lv(l - 1) + 2 * lv(l) for l in range(3, n + 1))
    # the figures the design's roofline table quotes
    assert (sb["sections"], sb["m2m"], sb["m2l_l2l"], sb["leaf_l2t_near"]) == \
        (367525888, 294948864, 491581440, 363331584)


def test_serving_requests_are_seeded_poisson_arrivals(bench):
    a, b = bench.serving_requests(10000, 2000, 7), bench.serving_requests(10000, 2000, 7)
    assert a == b
    t = np.array([r[0] for r in a])
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / len(t) - 1e-4) < 1e-5  # mean gap 1 / rate
    lgN = np.array([int(r[1]).bit_length() - 1 for r in a])
    assert lgN.min() == 10 and lgN.max() == 24
    assert {r[3] for r in a} == set(bench.SERVE_CLASSES.values())
    for (_, N, P, T, b) in a:
        assert P == max(2, min(64, N // 512)) and b == 32


def test_serving_and_uneven_shapes_are_plannable(bench, fm):
    shapes = {r[1:] for r in bench.serving_requests(50000, 600, 7)} | set(bench.uneven_jobs(200, 3))
    for (N, P, T, b) in shapes:
        assert fm.plan_bytes(N, P, T, b, "f32_tc") > 0
    for (N, P, T, b) in bench.uneven_jobs(200, 3):
        assert 1 << 12 <= N <= 1 << 22 and N // P >= 256

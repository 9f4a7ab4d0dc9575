"""fmmfft_plan_bytes on the host (no GPU): the device bytes a plan will hold, which the request
server's HBM admission compares with its budget before it allocates anything.

The figure must cover the plan's workspace as laid out in HBM -- planar sections xt[2P][M], the
far+near field u[2(P-1)][M], the combine's z[P][M] and the FFT's tmp[P][M], multipole and local
expansions phi / psi of every level (2 (P-1) planes x T terms x (2^(n+1) - 1) boxes), the per-tile
section sums -- once per transform of a batched plan, plus operator tables shared by the batch; and
refuse the shapes a plan refuses."""
import os

import pytest

import oracle_lib as ol  # noqa: F401  (puts the package on sys.path)


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    if not os.path.exists(fmmfft.LIB_PATH):
        import build_lib  # fmm-fft_b200/build_lib.py
        build_lib.build()
    fmmfft.load()
    return fmmfft


def workspace_floor(N, P, T, b, real_bytes):
    """Bytes of one transform's large arrays (the ones that scale with N), and an allowance for
    what may come with them: the expansions of levels 0 and 1 and the per-tile section sums."""
    M, S1 = N // P, P - 1
    s = M // b
    n = s.bit_length() - 1
    R, C = real_bytes, 2 * real_bytes
    tile = max(1, 2048 // P)  # points per sections tile
    levels = 2 * S1 * T * ((1 << (n + 1)) - 4) * R  # levels 2..n
    floor = (2 * P * M * R           # xt
             + 2 * S1 * M * R        # u
             + 2 * P * M * C         # z, tmp
             + 2 * levels)           # phi, psi
    extra = 2 * 2 * S1 * T * 3 * R + (M // tile) * P * C
    return floor, extra


SHAPES = [(1 << 24, 64, 24, 32), (1 << 22, 64, 20, 32), (1 << 20, 256, 16, 16), (1 << 18, 16, 8, 8)]


@pytest.mark.parametrize("N,P,T,b", SHAPES)
@pytest.mark.parametrize("prec,rb", [("f64", 8), ("f32", 4), ("f32_tc", 4), ("bf16x3", 4)])
def test_plan_bytes_cover_the_workspace_per_transform(fm, N, P, T, b, prec, rb):
    one, two, four = (fm.plan_bytes(N, P, T, b, prec, k) for k in (1, 2, 4))
    per = two - one
    # affine in the batch (to the arrays' 256-byte alignment): workspace per transform, operators once
    assert abs((four - two) - 2 * per) <= 16 * 256
    floor, extra = workspace_floor(N, P, T, b, rb)
    assert floor <= per <= (floor + extra) * 1.01 + (1 << 20), (per, floor, extra)
    ops = one - per  # operator tables (and, on tensor-core plans, their shared-memory images)
    assert 0 < ops < max(64 << 20, per // 4)


def test_fp64_workspace_is_twice_fp32(fm):
    N, P, T, b = 1 << 22, 64, 20, 32
    per = {p: fm.plan_bytes(N, P, T, b, p, 2) - fm.plan_bytes(N, P, T, b, p, 1) for p in ("f64", "f32")}
    assert abs(per["f64"] - 2 * per["f32"]) <= 64 * 1024


@pytest.mark.parametrize("N,P,T,b", [(1 << 24, 48, 24, 32), (1 << 24, 64, 24, 33), (1 << 24, 64, 0, 32),
                                     (100, 64, 24, 32), (1 << 24, 2048, 24, 32), (1 << 12, 64, 24, 32)])
def test_plan_bytes_refuses_what_a_plan_refuses(fm, N, P, T, b):
    with pytest.raises(fm.FmmFftError):
        fm.plan_bytes(N, P, T, b, "f32")

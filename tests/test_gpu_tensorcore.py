"""The split-TF32 tcgen05 path (FMMFFT_F32_TC) against the FP64 oracle, stage by stage.

FMMFFT_TC_MIN_ROWS=1 (set before the plans are made) sends every eligible stage, however small,
through the tensor-core kernel so that small cases cover it; the default threshold only routes
stages with >= 4096 rows there.  Each test runs for the default per-stage kernels (16-lane row
form for S2M, M2M and M2L, the neighbour-sum form for the leaf) and for each tensor-core kernel
forced on every stage (FMMFFT_TC_FORM row, row16 and ws, the warp-specialised one), with S2M as
its own stage (FMMFFT_FUSE_S2M=0) so that it runs on the tensor cores.  Tolerance: rel-L2 <= 1e-6
against FP64, as for FP32 plans.
"""
import os

import numpy as np
import pytest

import oracle_lib as ol
from gpu_util import run_device

pytestmark = pytest.mark.gpu
TOL = 1e-6          # the transform's output and z, against FP64
TOL_STAGE = 1e-4    # intermediate expansions: the TF32 split leaves ~2^-22 per product, and with few
                    # terms and wide boxes (S2M with K = b = 128) cancellation magnifies it

CASES = [(4096, 4, 8, 16), (16384, 8, 12, 32), (65536, 16, 16, 32), (65536, 64, 24, 32),
         (1 << 18, 4, 20, 64), (1 << 18, 32, 24, 16), (1 << 18, 2, 8, 128)]


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


FORMS = ["default", "row", "row16", "ws"]


@pytest.fixture(params=FORMS)
def force_tc(request):
    """Every eligible stage on the tensor cores, in the default per-stage forms or in one form
    forced on every stage: the 32-lane row form, the 16-lane row form or the warp-specialised
    kernel (FMMFFT_TC_FORM=row / row16 / ws)."""
    saved = {k: os.environ.get(k) for k in ("FMMFFT_TC_MIN_ROWS", "FMMFFT_TC_FORM", "FMMFFT_FUSE_S2M")}
    os.environ["FMMFFT_TC_MIN_ROWS"] = "1"
    if request.param == "default":
        os.environ.pop("FMMFFT_TC_FORM", None)
    else:
        os.environ["FMMFFT_TC_FORM"] = request.param
    os.environ["FMMFFT_FUSE_S2M"] = "0"  # S2M as its own tensor-core stage
    yield request.param
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


@pytest.mark.parametrize("N,P,T,b", CASES)
def test_tc_stagewise_vs_oracle(fm, force_tc, N, P, T, b):
    x = ol.seeded_input(N, 17 + N % 97)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    y = run_device(plan, x)
    plan.check()
    d = plan.debug_fetch()
    M = N // P
    s = M // b
    n = s.bit_length() - 1
    for lev in range(2, n + 1):
        gp = fm.level_planar(d["phi"], P, T, n, lev)
        gs = fm.level_planar(d["psi"], P, T, n, lev)
        gp = (gp[:, 0] + 1j * gp[:, 1]).transpose(1, 0, 2)
        gs = (gs[:, 0] + 1j * gs[:, 1]).transpose(1, 0, 2)
        assert ol.rel_l2(gp, o["phi"][ol.level_slice(lev)]) < TOL_STAGE, ("phi", lev)
        assert ol.rel_l2(gs, o["psi"][ol.level_slice(lev)]) < TOL_STAGE, ("psi", lev)
    assert ol.rel_l2(d["u"], o["u"]) < TOL_STAGE
    assert ol.rel_l2(d["z"], o["z"]) < TOL
    assert ol.rel_l2(y, o["y"]) < TOL


@pytest.fixture(params=FORMS)
def tc_form(request):
    """Default routing (stages of >= 4096 rows on the tensor cores) in each kernel form."""
    saved = os.environ.get("FMMFFT_TC_FORM")
    if request.param == "default":
        os.environ.pop("FMMFFT_TC_FORM", None)
    else:
        os.environ["FMMFFT_TC_FORM"] = request.param
    yield request.param
    if saved is None:
        os.environ.pop("FMMFFT_TC_FORM", None)
    else:
        os.environ["FMMFFT_TC_FORM"] = saved


def test_tc_config2_full_size(fm, tc_form):
    """N = 2^24 complex64, P = 64, p = 24, b = 32 with the default routing."""
    N, P, T, b = 1 << 24, 64, 24, 32
    x = ol.seeded_input(N, 0)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    y = run_device(plan, x)
    plan.check()
    ref = np.fft.fft(x)
    assert ol.rel_l2(y, ref) < TOL
    assert np.max(np.abs(y - ref)) / np.max(np.abs(ref)) < 1e-5


def test_tc_matches_plain_f32(fm):
    N, P, T, b = 1 << 20, 64, 16, 32
    x = ol.seeded_input(N, 4)
    y1 = run_device(fm.Plan(N, P, T, b, "f32"), x)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    y2 = run_device(plan, x)
    plan.check()
    assert ol.rel_l2(y2, y1) < TOL


LEAF_CASES = [(4096, 4, 8, 16), (16384, 8, 12, 32), (65536, 16, 16, 32), (65536, 64, 24, 32),
              (1 << 18, 32, 24, 16), (1 << 18, 256, 12, 16), (1 << 20, 128, 24, 32), (1 << 20, 1024, 16, 8)]


@pytest.mark.parametrize("leaf_form", ["neighbour_sum", "window_rows"])
@pytest.mark.parametrize("N,P,T,b", LEAF_CASES)
def test_tc_leaf_with_half_shift_column(fm, monkeypatch, N, P, T, b, leaf_form):
    """The leaf contraction on the tensor cores at every size (FMMFFT_TC_MIN_ROWS=1, read when
    the plan is made), in both forms.  Window rows (FMMFFT_LEAF_FORM=row): a row holds its box's
    expansion and the 3-box sample window, and the operator carries one extra output column, the
    next box's half-shifted first point for sections sc >= P/2, which the epilogue stores in place
    of the in-box value (sc > P/2) or leaves for the sc = P/2 mean.  Neighbour sums (default for
    b <= 32): a row holds its own box only, the operator has blocks for the box and its two
    neighbours (and three half-shift columns), and the epilogue adds the blocks of adjacent rows
    (shuffles within a warp, shared memory across warps, tiles of 126 output rows with wrap).
    The half-shift stage is then the sc = P/2 mean alone.  The near-field weights grow like P/pi
    against O(1) sums, hence the large-P cases.  u (the leaf output) and the transform against
    the FP64 oracle.  The autotuner is off so that the per-stage routing under test runs."""
    monkeypatch.setenv("FMMFFT_TC_MIN_ROWS", "1")
    monkeypatch.setenv("FMMFFT_AUTOTUNE", "0")
    if leaf_form == "window_rows":
        monkeypatch.setenv("FMMFFT_LEAF_FORM", "row")
    x = ol.seeded_input(N, 29 + N % 89)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    assert "leaf_form=" + leaf_form in plan.describe(), plan.describe()
    plan.profile_start(1)
    y = run_device(plan, x)
    _, stages = plan.profile_stop()
    plan.check()
    assert stages["leaf_halfshift"][1] == 1, stages
    d = plan.debug_fetch()
    assert ol.rel_l2(d["u"], o["u"]) < TOL_STAGE
    assert ol.rel_l2(y, o["y"]) < TOL


def test_tc_leaf_off_by_stage_mask(fm, monkeypatch):
    """FMMFFT_TC_STAGES=7 (S2M, M2M, M2L; no leaf) keeps the leaf on the CUDA cores: the direct
    leaf evaluates the half-shifted points itself, so no half-shift stage runs, and the result
    is the FP32 leaf's."""
    monkeypatch.setenv("FMMFFT_TC_STAGES", "7")
    N, P, T, b = 1 << 18, 64, 24, 32  # 2s = 256 leaf rows: the tensor cores' by default
    x = ol.seeded_input(N, 31)
    o = ol.forward_ex(x, P, T, b)
    plan = fm.Plan(N, P, T, b, "f32_tc")
    plan.profile_start(1)
    y = run_device(plan, x)
    _, stages = plan.profile_stop()
    plan.check()
    assert stages["leaf_halfshift"][1] == 0, stages
    assert ol.rel_l2(y, o["y"]) < TOL

"""The sharded single transform (fmmfft_shard_*, fmm-fft_b200/sharded.py), its G shards run in one
process on one device with the exchanges as device copies (every GPU call of this build has one
GPU; the exchanges' multi-rank form is tested on CPU in test_sharded_transport.py).

Each shard computes with the single-device kernels over its strip (own boxes plus s/(2G) boxes of
halo a side) and the global tree's coarse levels; the result must be the transform's: FP64 shards
against the single-device FP64 plan to 1e-12 and against FP64 FFT to the FMM's own truncation,
FP32 and split-TF32 shards against the FP64 FFT to the FP32 bar of 1e-6 and against their own
single-device plan.  Shapes: 2, 4 and 8 shards, several P and b, the coarse level at the top of a
small tree (G = 2) and deep inside a large one (G = 8, N = 2^22)."""
import os
import sys

import numpy as np
import pytest

import oracle_lib as ol

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "fmm-fft_b200"))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    fmmfft.load()
    return fmmfft


CASES = [
    (1 << 16, 16, 16, 32, "f64", 2), (1 << 16, 16, 16, 32, "f64", 4), (1 << 16, 16, 16, 32, "f64", 8),
    (1 << 18, 64, 20, 32, "f32", 4), (1 << 20, 64, 24, 32, "f32_tc", 2), (1 << 20, 64, 24, 32, "f32_tc", 8),
    (1 << 22, 64, 24, 32, "f32_tc", 8), (1 << 19, 32, 16, 16, "f32_tc", 4),
]


@pytest.mark.parametrize("N,P,T,b,prec,G", CASES)
def test_sharded_equals_single_device(fm, N, P, T, b, prec, G):
    import torch
    import sharded
    dt = torch.complex128 if prec == "f64" else torch.complex64
    x = ol.seeded_input(N, 31)
    d = torch.from_numpy(x).to(dt).cuda()
    shards = [fm.Shard(N, P, T, b, prec, G, g) for g in range(G)]
    y = sharded.forward_emulated(shards, d)
    torch.cuda.synchronize()
    ys = y.cpu().numpy().astype(np.complex128)
    plan = fm.Plan(N, P, T, b, prec)
    one = torch.empty_like(d)
    plan.execute_ptr(d.data_ptr(), one.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    y1 = one.cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(x)
    e_plan, e_fft = ol.rel_l2(ys, y1), ol.rel_l2(ys, ref)
    print(f"N={N} P={P} T={T} b={b} {prec} G={G}: sharded vs one-device plan rel-L2 {e_plan:.3e}, "
          f"vs FP64 FFT {e_fft:.3e} (one-device plan vs FFT {ol.rel_l2(y1, ref):.3e})")
    if prec == "f64":
        assert e_plan < 1e-12
        assert e_fft < 10 * ol.rel_l2(y1, ref) + 1e-13
    else:
        assert e_fft < 1e-6
        assert e_plan < 1e-6
    # a second transform through the same shards (their buffers are reused)
    y2 = sharded.forward_emulated(shards, d)
    torch.cuda.synchronize()
    assert torch.equal(y2, y)
    for s in shards:
        s.close()
    plan.close()


def test_sharded_shape_checks(fm):
    """Shapes a shard cannot split are refused: G not a power of two, P not a multiple of 2G,
    fewer than 8 leaf boxes per shard."""
    for args in ((1 << 16, 16, 16, 32, "f32", 3, 0), (1 << 16, 16, 16, 32, "f32", 16, 0),
                 (1 << 12, 16, 16, 32, "f32", 2, 0), (1 << 16, 16, 16, 32, "f32", 2, 2)):
        with pytest.raises(fm.FmmFftError):
            fm.Shard(*args)

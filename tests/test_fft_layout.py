"""The register FFT pass's shared exchange layout, checked on the host.

`fft_lp`, `fft_swz` and `fft_smem_elems` are taken verbatim from
fmm-fft_b200/csrc/fmmfft_kernels.cu and compiled for the CPU with g++ (the CUDA qualifiers
defined away), so the functions checked are the ones the kernel uses.  The test then replays
k_fft_reg's shared-memory accesses (the first stage's stores, each later stage's loads, stage
twiddles and stores, the transposing exchange when the output order differs, the 4-step twiddle
steps) for the thread orders the kernel uses, and checks:

  * bounds: every index of sequence w lies in [w LP, w LP + L), and is a permutation of those L
    slots (no two elements share a slot), and the stage-twiddle and twiddle-step regions fit in
    fft_smem_elems(L, W);
  * bank conflicts: with 8-byte elements a warp's access is served per half-warp, 16 distinct
    slots (index mod 16) a wavefront; at the FMM-FFT's shapes -- the two size-512 passes with 8
    sequences a block and the combine over P sections with min(32, 4096 / P) columns -- every
    access takes the minimum number of wavefronts (the combine at P = 1024 and 2048, 4 and 2
    columns a block, within 1.25 times it).

The thread orders and the access index expressions restate k_fft_reg (one thread per 8 points of
a sequence: t = position, w = sequence; along the sequence when the input is contiguous, across
sequences otherwise); the per-sequence bit-0 flip kw = (W == 8 ? (w >> 2) & 1 : 0) is the
kernel's.  No GPU is needed."""
import ctypes
import os
import re
import shutil
import subprocess
from collections import defaultdict

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "fmm-fft_b200", "csrc", "fmmfft_kernels.cu")


def _function(text, name):
    """Source of the function `name` (signature through its closing brace)."""
    m = re.search(r"(?:__host__\s+)?__device__\s+__forceinline__\s+[\w:]+\s+" + name + r"\s*\(", text)
    assert m, name
    i = text.index("{", m.end())
    depth = 0
    for j in range(i, len(text)):
        depth += text[j] == "{"
        depth -= text[j] == "}"
        if depth == 0:
            return text[m.start():j + 1]
    raise AssertionError(name)


@pytest.fixture(scope="module")
def lay(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not found")
    text = open(SRC).read()
    body = "\n".join(_function(text, n) for n in ("fft_lp", "fft_swz", "fft_smem_elems"))
    d = tmp_path_factory.mktemp("fftlayout")
    cpp = d / "layout.cpp"
    cpp.write_text("#define __host__\n#define __device__\n#define __forceinline__ inline\n#include <cstddef>\n"
                   + body + "\n"
                   'extern "C" int t_lp(int L, int W) { return fft_lp(L, W); }\n'
                   'extern "C" int t_swz(int i, int kw) { return fft_swz(i, kw); }\n'
                   'extern "C" long t_smem(int L, int W) { return (long)fft_smem_elems(L, W); }\n')
    so = d / "layout.so"
    subprocess.run(["g++", "-O1", "-shared", "-fPIC", "-o", str(so), str(cpp)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.t_smem.restype = ctypes.c_long
    return lib


def _stages(L):
    lg = L.bit_length() - 1
    ns0 = {0: 8, 2: 4, 1: 2}[lg % 3]
    out, Ns = [], ns0
    while Ns <= L // 8:
        out.append(Ns)
        Ns <<= 3
    return ns0, out


def _accesses(L, W, tin, tout, post, lay):
    """(region, thread order, index function of (t, w)) for every shared access of one pass."""
    q = L // 8
    LP = lay.t_lp(L, W)
    lg = L.bit_length() - 1

    def x(w, i):  # exchange buffer
        return w * LP + lay.t_swz(i, (w >> 2) & 1 if W == 8 else 0)
    ns0, stages = _stages(L)
    acc = []
    if ns0 == 8:
        acc += [("x", tin, lambda t, w, r=r: x(w, 8 * t + r)) for r in range(8)]
    elif ns0 == 4:
        for r in range(4):
            acc += [("x", tin, lambda t, w, r=r: x(w, 4 * t + r)), ("x", tin, lambda t, w, r=r: x(w, 4 * (t + q) + r))]
    else:
        for m in range(4):
            acc += [("x", tin, lambda t, w, m=m: x(w, 2 * (t + m * q))),
                    ("x", tin, lambda t, w, m=m: x(w, 2 * (t + m * q) + 1))]
    lNs = ns0.bit_length() - 1
    for si, Ns in enumerate(stages):
        acc += [("x", tin, lambda t, w, r=r: x(w, t + r * q)) for r in range(8)]
        acc += [("tw", tin, lambda t, w, r=r, Ns=Ns: (Ns - ns0) + 7 * (t & (Ns - 1)) + r - 1) for r in range(1, 8)]
        if si == len(stages) - 1:
            break
        acc += [("x", tin, lambda t, w, r=r, Ns=Ns, l=lNs: x(w, ((t >> l) << (l + 3)) + (t & (Ns - 1)) + (r << l)))
                for r in range(8)]
        lNs += 3
    if tout != tin:
        acc += [("x", tin, lambda t, w, r=r: x(w, t + r * q)) for r in range(8)]
        acc += [("x", tout, lambda t, w, r=r: x(w, t + r * q)) for r in range(8)]
    if post:
        acc += [("twq", tout, lambda t, w, r=r: w * 9 + r) for r in range(8)]
    assert lNs + 3 == lg
    return acc


def _thread(L, W, order, tid):
    q = L // 8
    if order:
        return tid & (q - 1), tid >> (q.bit_length() - 1)
    return tid >> (W.bit_length() - 1), tid & (W - 1)


def _wavefronts(L, W, tin, tout, post, lay):
    """(wavefronts, minimum) over one block's shared accesses, by region offsets in elements."""
    thr = W * (L // 8)
    LP = lay.t_lp(L, W)
    base = {"x": 0, "tw": W * LP, "twq": W * LP + L + L // 16 + 1}
    tot = ideal = 0
    for region, order, f in _accesses(L, W, tin, tout, post, lay):
        for wb in range(0, thr, 32):
            lanes = [_thread(L, W, order, tid) for tid in range(wb, min(wb + 32, thr))]
            for half in (lanes[:16], lanes[16:]):
                if not half:
                    continue
                slots = defaultdict(set)
                for t, w in half:
                    a = base[region] + f(t, w)
                    slots[a % 16].add(a)
                tot += max(len(s) for s in slots.values())
                ideal += 1
    return tot, ideal


def _shapes():
    """Every (L, W) a register pass runs with: FFT passes (W = min(16, 4096 / L), fewer when a
    row holds fewer sequences) and the combine over P sections."""
    out = set()
    for L in (16, 32, 64, 128, 256, 512, 1024, 2048, 4096):
        for W in (1, 2, 4, 8, 16):
            if W * L // 8 <= 512:
                out.add((L, W))
    for P in (16, 32, 64, 128, 256, 512, 1024, 2048, 4096):
        out.add((P, min(32, 4096 // P)))
    return sorted(out)


@pytest.mark.parametrize("L,W", _shapes())
def test_exchange_indices_are_a_permutation_within_bounds(lay, L, W):
    LP = lay.t_lp(L, W)
    assert LP >= L
    ns0, stages = _stages(L)
    n_tw = sum(7 * Ns for Ns in stages)
    assert n_tw == L - ns0 <= L + L // 16 + 1  # stage twiddles fit their region
    assert lay.t_smem(L, W) == W * LP + L + L // 16 + 1 + 9 * W
    for w in range(W):
        kw = (w >> 2) & 1 if W == 8 else 0
        idx = [lay.t_swz(i, kw) for i in range(L)]
        assert sorted(idx) == list(range(L)), (L, W, w)
        assert all(w * LP + i < W * LP for i in idx)


@pytest.mark.parametrize("tin,tout,post", [(False, False, True), (True, False, False), (True, True, False)])
def test_fmm_fft_passes_are_free_of_bank_conflicts(lay, tin, tout, post):
    """The 2^18-point FFTs of the N = 2^24 plan: two size-512 passes, 8 sequences a block (pass 1
    across sequences with the 4-step twiddle, pass 2 along them with a transposing store)."""
    tot, ideal = _wavefronts(512, 8, tin, tout, post, lay)
    assert tot == ideal, (tot, ideal)


@pytest.mark.parametrize("P", [16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_combine_is_free_of_bank_conflicts(lay, P):
    tot, ideal = _wavefronts(P, min(32, 4096 // P), False, False, False, lay)
    if P in (1024, 2048):  # 4 / 2 columns: the first stage's stores meet twice in some rows
        assert tot <= 1.25 * ideal, (P, tot, ideal)
    else:
        assert tot == ideal, (P, tot, ideal)

"""ctypes access to the CPU oracle (oracle/liboracle_fmmfft.so) for the tests.

The oracle is the checker: tests compare the GPU path with it; nothing here is product code.
The shared library is built on first use with the committed recipe (oracle/Makefile) when it
is missing, e.g. on a fresh machine.
"""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORC_SO = os.path.join(ORACLE_DIR, "liboracle_fmmfft.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libfmmfft_ref.so")
GOLDEN = os.path.join(REPO, "tests", "golden")

_L, _VP = ctypes.c_long, ctypes.c_void_p
_lib = None
_ref = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORC_SO):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR, "liboracle_fmmfft.so"], check=True)
        lib = ctypes.CDLL(ORC_SO)
        lib.orc_forward.argtypes = [_L, _L, _L, _L, _VP, _VP]
        lib.orc_plan_create.argtypes = [_L, _L, _L, _L]
        lib.orc_plan_create.restype = _VP
        lib.orc_plan_destroy.argtypes = [_VP]
        lib.orc_forward_ex.argtypes = [_VP] * 8
        lib.orc_fill_reference_w.argtypes = [_VP, _VP, _L]
        lib.orc_getwlen2.argtypes = [_L, _L, _L, _L]
        lib.orc_getwlen2.restype = _L
        lib.orc_getvlen.argtypes = [_L, _L, _L, _L]
        lib.orc_getvlen.restype = _L
        lib.orc_fft64.argtypes = [_L, _VP]
        lib.orc_max_error_percent.argtypes = [_VP, _VP, _L]
        lib.orc_max_error_percent.restype = ctypes.c_double
        _lib = lib
    return _lib


def load_reference():
    """The shim-built reference (oracle/_ref), or None where it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        lib = ctypes.CDLL(REF_SO)
        lib.fmmref_forward.argtypes = [_L, _L, _L, _L, _VP, _VP, ctypes.c_int, _VP]
        lib.fmmref_wlen.argtypes = [_L, _L, _L, _L]
        lib.fmmref_wlen.restype = _L
        lib.fmmref_vlen.argtypes = [_L, _L, _L, _L]
        lib.fmmref_vlen.restype = _L
        lib.fmmref_mfti.argtypes = [_L, _L, _L, _L, _VP, _VP]
        _ref = lib
    return _ref


def seeded_input(n, seed):
    """iid standard-normal real and imaginary parts from numpy PCG64(seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    re_ = rng.standard_normal(n)
    im_ = rng.standard_normal(n)
    return (re_ + 1j * im_).astype(np.complex128)


def forward(x, P, terms, b):
    lib = load()
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros_like(x)
    rc = lib.orc_forward(x.size, P, terms, b, x.ctypes.data, y.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle rejected N={x.size} P={P} terms={terms} b={b} (rc={rc})")
    return y


def forward_ex(x, P, terms, b):
    """Output plus intermediates: dict(y, u[P-1,M], z[P,M], phi, psi [nbox,P-1,terms], ssum)."""
    lib = load()
    x = np.ascontiguousarray(x, dtype=np.complex128)
    N = x.size
    M = N // P
    pl = lib.orc_plan_create(M, P, terms, b)
    if not pl:
        raise ValueError("oracle rejected parameters")
    s = M // b
    n = s.bit_length() - 1
    nbox = (2 << n) - 4
    out = dict(
        y=np.zeros(N, np.complex128),
        u=np.zeros((P - 1, M), np.complex128),
        z=np.zeros((P, M), np.complex128),
        phi=np.zeros((nbox, P - 1, terms), np.complex128),
        psi=np.zeros((nbox, P - 1, terms), np.complex128),
        ssum=np.zeros(P - 1, np.complex128),
    )
    try:
        rc = lib.orc_forward_ex(pl, x.ctypes.data, *(out[k].ctypes.data for k in
                                                     ("y", "u", "z", "phi", "psi", "ssum")))
    finally:
        lib.orc_plan_destroy(pl)
    if rc != 0:
        raise RuntimeError(f"oracle failed rc={rc}")
    return out


def level_slice(n_level):
    """Box range of level l in the oracle's phi/psi arrays (levels 2..n)."""
    return slice((1 << n_level) - 4, (1 << (n_level + 1)) - 4)


def rel_l2(a, ref):
    a = np.asarray(a)
    ref = np.asarray(ref)
    return float(np.linalg.norm((a - ref).ravel()) / np.linalg.norm(ref.ravel()))


def tone_input(n, seed, ntones=32, noise=1e-3):
    """Sum of `ntones` unit-modulus tones at real (off-bin) frequencies f_k ~ U[0, n) with random
    phases, plus noise * (g_re + i g_im), g iid N(0, 1); numpy PCG64(seed).  Evaluated in FP64 in
    blocks of 2^16 points: exp(2 pi i f (n0 + j) / n) = exp(2 pi i f n0 / n) exp(2 pi i f j / n)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    f = rng.uniform(0.0, float(n), ntones)
    ph = rng.uniform(0.0, 2 * np.pi, ntones)
    g = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    blk = min(n, 1 << 16)
    j = np.arange(blk, dtype=np.float64)
    base = np.exp(2j * np.pi * np.outer(f, j) / n)          # [ntones][blk]
    x = np.empty(n, np.complex128)
    for n0 in range(0, n, blk):
        c = np.exp(1j * (ph + 2 * np.pi * f * (n0 / n)))       # [ntones]
        x[n0:n0 + blk] = c @ base
    x += noise * g
    return x


def reference_forward(x, P, terms, b):
    """Output of the shim-built reference (oracle/_ref: src/fmmfft.c unmodified, P thread-ranks)
    for input x, or None where it was not built."""
    lib = load_reference()
    if lib is None:
        return None
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros_like(x)
    rc = lib.fmmref_forward(x.size, P, terms, b, x.ctypes.data, y.ctypes.data, 1, None)
    if rc != 0:
        raise RuntimeError(f"reference run failed rc={rc}")
    return y

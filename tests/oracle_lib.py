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

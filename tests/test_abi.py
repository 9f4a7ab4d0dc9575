"""CPU tests of the C-ABI library: it loads, exports what include/fmmfft.h declares, and its
host-side (no GPU) behaviour matches the reference: workspace sizes, the operator buffer that
mfti fills, and parameter validation."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as ol

REPO = ol.REPO
HEADER = os.path.join(REPO, "include", "fmmfft.h")


@pytest.fixture(scope="module")
def fm():
    import fmmfft
    if not os.path.exists(fmmfft.LIB_PATH):
        import build_lib  # fmm-fft_b200/build_lib.py
        build_lib.build()
    fmmfft.load()
    return fmmfft


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(l for l in txt.splitlines() if not l.strip().startswith("#"))
    names = []
    for stmt in txt.split(";"):
        s = " ".join(stmt.split())
        if not s or s.startswith("typedef") or "{" in s or "}" in s:
            continue
        m = re.match(r"^(?:extern\s+\"C\"\s*)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", s)
        if m:
            names.append(m.group(1))
    return names


def test_header_declares_the_reference_entry_points():
    names = header_functions()
    for ref in ("getwlen2", "getvlen", "mfti", "mft"):
        assert ref in names


def test_library_exports_every_declared_symbol(fm):
    lib = ctypes.CDLL(fm.LIB_PATH)
    names = header_functions()
    assert len(names) >= 13
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(names) == sorted(fm.EXPORTS)


@pytest.mark.parametrize("lq,terms,p,b", [(16384, 16, 4, 2048), (262144, 24, 64, 32),
                                          (1024, 15, 8, 32), (256, 8, 2, 16)])
def test_workspace_sizes_match_reference(fm, lq, terms, p, b):
    lib = ol.load()
    assert fm.getwlen2(lq, terms, p, b) == lib.orc_getwlen2(lq, terms, p, b)
    assert fm.getvlen(lq, terms, p, b) == lib.orc_getvlen(lq, terms, p, b)
    ref = ol.load_reference()
    if ref is not None:
        assert fm.getwlen2(lq, terms, p, b) == ref.fmmref_wlen(lq, p, terms, b)
        assert fm.getvlen(lq, terms, p, b) == ref.fmmref_vlen(lq, p, terms, b)


@pytest.mark.parametrize("lq,p,terms,b", [(256, 4, 8, 8), (1024, 8, 12, 16), (2048, 2, 16, 32),
                                          (4096, 64, 24, 32), (16384, 4, 16, 2048)])
def test_mfti_operators_bitwise_equal_to_reference(fm, lq, p, terms, b):
    """mfti fills w on the host before it makes the device plan; without a GPU the plan step
    reports ERR_NO_DEVICE, and w must still be the reference's operators, bit for bit."""
    wl = fm.getwlen2(lq, terms, p, b)
    w = np.zeros(wl)
    os.environ["FMMFFT_QUIET"] = "1"
    try:
        fm.mfti(lq, p, terms, b, w)
    except fm.FmmFftError as e:
        assert e.status == 4  # no device here
    lib = ol.load()
    pl = lib.orc_plan_create(lq, p, terms, b)
    w_orc = np.zeros(wl)
    lib.orc_fill_reference_w(pl, w_orc.ctypes.data, wl)
    lib.orc_plan_destroy(pl)
    n = (lq // b).bit_length() - 1
    n_ops = wl - (p * (p - 1) + b + 3 * terms + 1)  # operator part of getwlen2 (:1160-1183)
    assert np.array_equal(w[:n_ops].view(np.uint64), w_orc[:n_ops].view(np.uint64))
    ref = ol.load_reference()
    if ref is not None:
        w_ref = np.zeros(wl)
        v_ref = np.zeros(ref.fmmref_vlen(lq, p, terms, b))
        ref.fmmref_mfti(lq, p, terms, b, w_ref.ctypes.data, v_ref.ctypes.data)
        n_cmp = n_ops - p * (p - 1)  # fo is followed by scratch in the reference's own w
        assert np.array_equal(w[:n_cmp].view(np.uint64), w_ref[:n_cmp].view(np.uint64))
        assert n > 0


@pytest.mark.parametrize("lq,terms,p,b", [(1000, 8, 4, 8), (1024, 8, 3, 16), (64, 8, 4, 32),
                                          (1024, 1, 4, 16), (1024, 8, 4, 1), (1024, 80, 4, 16)])
def test_invalid_parameters_are_rejected(fm, lq, terms, p, b):
    os.environ["FMMFFT_QUIET"] = "1"
    assert fm.getwlen2(lq, terms, p, b) == -1
    assert fm.last_error()[0] == 1
    with pytest.raises(fm.FmmFftError) as ei:
        fm.Plan(lq * p, p, terms, b, "f32")
    assert ei.value.status in (1, 4)


def test_mft_rejects_inverse_direction(fm):
    os.environ["FMMFFT_QUIET"] = "1"
    qr = np.zeros(1024, np.complex128)
    with pytest.raises(fm.FmmFftError) as ei:
        fm.mft(256, qr, -1, 4, 0, 8, 8)
    assert ei.value.status == 5


def _rank_call(fm, results, key, *args):
    try:
        fm.mft(*args)
        results[key] = 0
    except fm.FmmFftError as e:
        results[key] = e.status


def test_rank_mode_collective_refuses_mismatch_and_times_out(fm, monkeypatch):
    """Rank mode of mft (no GPU reached): a call whose (lq, p, terms, b) differ from the
    collective in progress, or that repeats a myid, is refused at once; a rank whose partners
    never come returns FMMFFT_ERR_TIMEOUT with its block untouched; the mode cannot be switched
    while a collective is open."""
    import threading
    monkeypatch.setenv("FMMFFT_RANK_TIMEOUT_MS", "1500")
    fm.mft_rank_mode(True)
    try:
        lq, p, T, b = 256, 4, 8, 8
        blk = np.arange(lq, dtype=np.complex128)
        keep = blk.copy()
        res = {}
        t0 = threading.Thread(target=_rank_call, args=(fm, res, "r0", lq, blk, 1, p, 0, T, b))
        t0.start()
        import time
        time.sleep(0.2)
        with pytest.raises(fm.FmmFftError) as ei:
            fm.mft_rank_mode(False)
        assert ei.value.status == 7
        other = np.zeros(2 * lq, dtype=np.complex128)
        _rank_call(fm, res, "mismatch", 2 * lq, other, 1, p, 1, T, b)
        dup = np.zeros(lq, dtype=np.complex128)
        _rank_call(fm, res, "dup", lq, dup, 1, p, 0, T, b)
        t0.join()
        assert res["mismatch"] == 1 and res["dup"] == 1, res
        assert res["r0"] == 6, res
        assert np.array_equal(blk, keep)
    finally:
        fm.mft_rank_mode(False)

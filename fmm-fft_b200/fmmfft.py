"""Python mirror of the FMM-FFT C-ABI (include/fmmfft.h), over ctypes.

Reference-compatible functions keep the reference's names and argument order
(97amarnathk/fmm-fft src/fmmfft.c): getwlen2 (:1160), getvlen (:1110), mfti (:337), mft (:980).
`mft` transforms the full N = p*lq vector (the P MPI ranks of the reference are P blocks of one
GPU).  `Plan` is the native API: operators resident on the GPU, execution on device buffers.

The library is loaded from this directory (libfmmfft_b200.so, built by build_lib.py).  There is no
CPU fallback: if the library or a CUDA device is missing, calls raise FmmFftError.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmmfft_b200.so")

F64, F32, F32_TC, BF16X3 = 0, 1, 2, 3
PRECISIONS = {"f64": F64, "f32": F32, "f32_tc": F32_TC, "bf16x3": BF16X3}
STATUS = {0: "OK", 1: "ERR_INVALID", 2: "ERR_NOMEM", 3: "ERR_CUDA", 4: "ERR_NO_DEVICE",
          5: "ERR_UNSUPPORTED", 6: "ERR_TIMEOUT", 7: "ERR_BUSY"}

# Every symbol include/fmmfft.h declares.
EXPORTS = ["getwlen2", "getvlen", "mfti", "mft", "fmmfft_last_error", "fmmfft_last_error_string",
           "fmmfft_plan_create", "fmmfft_plan_destroy", "fmmfft_plan_device_bytes",
           "fmmfft_execute", "fmmfft_execute_inverse", "fmmfft_execute_host", "fmmfft_execute_host_many",
           "fmmfft_debug_fetch", "fmmfft_profile_start", "fmmfft_profile_stop",
           "fmmfft_stage_name", "fmmfft_execute_noalloc", "fmmfft_plan_check",
           "fmmfft_plan_selftest_wait", "fmmfft_plan_create_batched", "fmmfft_execute_many",
           "fmmfft_execute_many_graph", "fmmfft_plan_bytes", "fmmfft_server_counts", "fmmfft_server_reserve",
           "fmmfft_plan_enable_refinement", "fmmfft_execute_refined", "fmmfft_mft_rank_mode",
           "fmmfft_execute_blocks", "fmmfft_execute_blocks_host", "fmmfft_plan_describe",
           "fmmfft_batch_create_many", "fmmfft_execute_many_ptrs",
           "fmmfft_shard_create", "fmmfft_shard_buffers", "fmmfft_shard_phase", "fmmfft_shard_destroy",
           "fmmfft_execute_graph", "fmmfft_batch_create", "fmmfft_batch_launch",
           "fmmfft_batch_destroy", "fmmfft_server_create", "fmmfft_server_destroy",
           "fmmfft_server_submit", "fmmfft_server_query", "fmmfft_server_wait",
           "fmmfft_server_stats", "fmmfft_fft_create", "fmmfft_fft_execute",
           "fmmfft_fft_device_bytes", "fmmfft_fft_destroy"]


class FmmFftError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


_lib = None
_L, _VP, _I = ctypes.c_long, ctypes.c_void_p, ctypes.c_int


class _ShardBufs(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("x_ext", "sums", "phi_send", "phi_all", "z_send", "z_recv", "y")] + \
               [(n, ctypes.c_size_t) for n in ("x_ext_elems", "halo_elems", "phi_elems", "z_elems", "y_elems")]


def load(path=LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FmmFftError(4, f"{path} is missing: run `python fmm-fft_b200/build_lib.py`")
    lib = ctypes.CDLL(path)
    lib.getwlen2.argtypes = [_L] * 4
    lib.getwlen2.restype = _L
    lib.getvlen.argtypes = [_L] * 4
    lib.getvlen.restype = _L
    lib.mfti.argtypes = [_L, _L, _L, _L, _VP, _VP, _L, _L]
    lib.mfti.restype = None
    lib.mft.argtypes = [_L, _VP, _L, _L, _L, _L, _L, _VP, _VP, _L, _L, _VP]
    lib.mft.restype = None
    lib.fmmfft_last_error.restype = _I
    lib.fmmfft_last_error_string.restype = ctypes.c_char_p
    lib.fmmfft_plan_create.argtypes = [ctypes.POINTER(_VP), _L, _L, _L, _L, _I]
    lib.fmmfft_plan_destroy.argtypes = [_VP]
    lib.fmmfft_plan_device_bytes.argtypes = [_VP, ctypes.POINTER(ctypes.c_size_t)]
    for f in ("fmmfft_execute", "fmmfft_execute_inverse", "fmmfft_execute_host"):
        getattr(lib, f).argtypes = [_VP, _VP, _VP, _VP]
        getattr(lib, f).restype = _I
    lib.fmmfft_execute_host_many.argtypes = [_VP, _I, _VP, _VP, _VP]
    lib.fmmfft_execute_host_many.restype = _I
    lib.fmmfft_debug_fetch.argtypes = [_VP, _VP, _VP, _VP, _VP]
    lib.fmmfft_profile_start.argtypes = [_VP, _I]
    lib.fmmfft_profile_stop.argtypes = [_VP, _VP, _VP, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]
    lib.fmmfft_stage_name.argtypes = [_I]
    lib.fmmfft_stage_name.restype = ctypes.c_char_p
    lib.fmmfft_execute_noalloc.argtypes = [_L, _L, _L, _L, _VP, _VP, _VP]
    lib.fmmfft_execute_noalloc.restype = _I
    lib.fmmfft_plan_check.argtypes = [_VP]
    lib.fmmfft_plan_check.restype = _I
    lib.fmmfft_plan_selftest_wait.argtypes = [_VP, _I, _L]
    lib.fmmfft_plan_selftest_wait.restype = _I
    lib.fmmfft_plan_create_batched.argtypes = [ctypes.POINTER(_VP), _L, _L, _L, _L, _I, _I]
    lib.fmmfft_plan_create_batched.restype = _I
    lib.fmmfft_execute_many.argtypes = [_VP, _I, _VP, _VP, _VP]
    lib.fmmfft_execute_many.restype = _I
    lib.fmmfft_execute_many_graph.argtypes = [_VP, _I, _VP, _VP, _VP]
    lib.fmmfft_execute_many_ptrs.argtypes = [_VP, _I, ctypes.POINTER(_VP), ctypes.POINTER(_VP), _VP]
    lib.fmmfft_execute_many_ptrs.restype = _I
    lib.fmmfft_shard_create.argtypes = [ctypes.POINTER(_VP), _L, _L, _L, _L, _I, _I, _I]
    lib.fmmfft_shard_create.restype = _I
    lib.fmmfft_shard_buffers.argtypes = [_VP, ctypes.POINTER(_ShardBufs)]
    lib.fmmfft_shard_buffers.restype = _I
    lib.fmmfft_shard_phase.argtypes = [_VP, _I, _VP]
    lib.fmmfft_shard_phase.restype = _I
    lib.fmmfft_shard_destroy.argtypes = [_VP]
    lib.fmmfft_shard_destroy.restype = _I
    lib.fmmfft_execute_many_graph.restype = _I
    lib.fmmfft_plan_bytes.argtypes = [_L, _L, _L, _L, _I, _I, ctypes.POINTER(ctypes.c_size_t)]
    lib.fmmfft_plan_bytes.restype = _I
    lib.fmmfft_server_counts.argtypes = [_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib.fmmfft_server_counts.restype = _I
    lib.fmmfft_server_reserve.argtypes = [_VP, _L, _L, _L, _L, _I, _I]
    lib.fmmfft_server_reserve.restype = _I
    lib.fmmfft_plan_enable_refinement.argtypes = [_VP]
    lib.fmmfft_plan_enable_refinement.restype = _I
    lib.fmmfft_execute_refined.argtypes = [_VP, _VP, _VP, _VP]
    lib.fmmfft_execute_refined.restype = _I
    lib.fmmfft_batch_create_many.argtypes = [ctypes.POINTER(_VP), _VP, _VP, _VP, _VP, _I, _I]
    lib.fmmfft_batch_create_many.restype = _I
    lib.fmmfft_plan_describe.argtypes = [_VP, ctypes.c_char_p, ctypes.c_size_t]
    lib.fmmfft_plan_describe.restype = _I
    lib.fmmfft_mft_rank_mode.argtypes = [_I]
    lib.fmmfft_mft_rank_mode.restype = _I
    for f in ("fmmfft_execute_blocks", "fmmfft_execute_blocks_host"):
        getattr(lib, f).argtypes = [_VP, _VP, _VP, _VP]
        getattr(lib, f).restype = _I
    lib.fmmfft_execute_graph.argtypes = [_VP, _VP, _VP, _VP]
    lib.fmmfft_execute_graph.restype = _I
    lib.fmmfft_batch_create.argtypes = [ctypes.POINTER(_VP), _VP, _VP, _VP, _I, _I]
    lib.fmmfft_batch_create.restype = _I
    lib.fmmfft_batch_launch.argtypes = [_VP, _VP]
    lib.fmmfft_batch_launch.restype = _I
    lib.fmmfft_batch_destroy.argtypes = [_VP]
    lib.fmmfft_server_create.argtypes = [ctypes.POINTER(_VP), ctypes.c_size_t, _I]
    lib.fmmfft_server_create.restype = _I
    lib.fmmfft_server_destroy.argtypes = [_VP]
    lib.fmmfft_server_submit.argtypes = [_VP, _L, _L, _L, _L, _I, _VP, _VP,
                                         ctypes.POINTER(ctypes.c_uint64)]
    lib.fmmfft_server_submit.restype = _I
    lib.fmmfft_server_query.argtypes = [_VP, ctypes.c_uint64]
    lib.fmmfft_server_query.restype = _I
    lib.fmmfft_server_wait.argtypes = [_VP, ctypes.c_uint64, _L]
    lib.fmmfft_server_wait.restype = _I
    lib.fmmfft_server_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(_I),
                                        ctypes.POINTER(_I)]
    lib.fmmfft_server_stats.restype = _I
    lib.fmmfft_fft_create.argtypes = [ctypes.POINTER(_VP), _L, _I]
    lib.fmmfft_fft_create.restype = _I
    lib.fmmfft_fft_execute.argtypes = [_VP, _VP, _VP, _VP]
    lib.fmmfft_fft_execute.restype = _I
    lib.fmmfft_fft_device_bytes.argtypes = [_VP, ctypes.POINTER(ctypes.c_size_t)]
    lib.fmmfft_fft_device_bytes.restype = _I
    lib.fmmfft_fft_destroy.argtypes = [_VP]
    lib.fmmfft_fft_destroy.restype = _I
    _lib = lib
    return lib


def last_error():
    lib = load()
    return lib.fmmfft_last_error(), lib.fmmfft_last_error_string().decode()


def _check(rc):
    if rc != 0:
        raise FmmFftError(rc, load().fmmfft_last_error_string().decode())


# ---------------------------------------------------------------- reference-compatible
def getwlen2(lq, terms, p, b):
    return load().getwlen2(lq, terms, p, b)


def getvlen(lq, terms, p, b):
    return load().getvlen(lq, terms, p, b)


def mfti(lq, p, terms, b, w, v=None, szkeep=0, sztemp=0):
    """Fills w (float64, getwlen2 entries) with the operators, reference layout; makes the
    device plan for (lq, p, terms, b) resident.  Raises on error."""
    assert w.dtype == np.float64 and w.flags.c_contiguous
    load().mfti(lq, p, terms, b, w.ctypes.data, None if v is None else v.ctypes.data, szkeep,
                sztemp)
    st, msg = last_error()
    if st:
        raise FmmFftError(st, msg)


_rank_mode = False


def mft(lq, qr, dir, p, myid=0, terms=None, b=None, w=None, v=None, sz1=0, szwk=0, plan=None):
    """In-place forward FMM-FFT of the full vector qr (complex128, p*lq values, host); in rank
    mode, rank myid's block of lq values, collectively with the other p - 1 ranks' calls."""
    assert qr.dtype == np.complex128 and qr.flags.c_contiguous
    assert qr.size == (lq if _rank_mode else p * lq)
    load().mft(lq, qr.ctypes.data, dir, p, myid, terms, b,
               None if w is None else w.ctypes.data, None if v is None else v.ctypes.data,
               sz1, szwk, plan)
    st, msg = last_error()
    if st:
        raise FmmFftError(st, msg)


def plan_bytes(N, P, terms, b, precision="f32", max_transforms=1):
    """Device bytes a plan would hold, computed without allocating."""
    v = ctypes.c_size_t()
    _check(load().fmmfft_plan_bytes(int(N), int(P), int(terms), int(b), PRECISIONS[precision],
                                    int(max_transforms), ctypes.byref(v)))
    return v.value


def mft_rank_mode(on):
    """Switch mft between full-vector calls and collective per-rank calls (see fmmfft.h)."""
    global _rank_mode
    _check(load().fmmfft_mft_rank_mode(1 if on else 0))
    _rank_mode = bool(on)


def execute_noalloc(N, P, terms, b, d_in, d_out, stream=0):
    """complex64 forward transform between caller-owned device buffers (pointers) without any
    allocation: tables and workspace live in the library's static 32 MiB device array."""
    _check(load().fmmfft_execute_noalloc(int(N), int(P), int(terms), int(b), d_in, d_out,
                                         stream or None))


# ---------------------------------------------------------------- native plans
class Plan:
    """One resident FMM-FFT plan: N points in P blocks, `terms` Chebyshev terms, b points per
    leaf box.  precision: 'f64' (complex128), 'f32' (complex64, CUDA cores) or 'f32_tc'."""

    def __init__(self, N, P, terms, b, precision="f32", max_transforms=1):
        self.N, self.P, self.terms, self.b = int(N), int(P), int(terms), int(b)
        self.M = self.N // self.P
        self.precision = precision
        self.max_transforms = int(max_transforms)
        self._p = PRECISIONS[precision]
        h = _VP()
        _check(load().fmmfft_plan_create_batched(ctypes.byref(h), self.N, self.P, self.terms,
                                                 self.b, self._p, self.max_transforms))
        self._h = h

    def describe(self):
        """The plan's stage choices (autotuned or default) as text."""
        buf = ctypes.create_string_buffer(256)
        _check(load().fmmfft_plan_describe(self._h, buf, 256))
        return buf.value.decode()

    def execute_blocks_ptr(self, ins, outs, stream=0, host=False):
        """Block-distributed transform: P input / output block pointers (M values each)."""
        n = self.P
        assert len(ins) == n and len(outs) == n
        a = (_VP * n)(*ins)
        o = (_VP * n)(*outs)
        f = load().fmmfft_execute_blocks_host if host else load().fmmfft_execute_blocks
        _check(f(self._h, a, o, stream or None))

    def enable_refinement(self):
        """Build the FP64 companion plan of the residual-correction pass (once)."""
        _check(load().fmmfft_plan_enable_refinement(self._h))

    def execute_refined_ptr(self, d_in, d_out, stream=0):
        """complex64 input -> complex128 output, one FP64 residual-correction step."""
        _check(load().fmmfft_execute_refined(self._h, d_in, d_out, stream or None))

    def execute_many_ptr(self, count, d_in, d_out, stream=0, graph=False):
        """`count` transforms in one launch sequence; transform i at d_in / d_out + i N elements."""
        f = load().fmmfft_execute_many_graph if graph else load().fmmfft_execute_many
        _check(f(self._h, int(count), d_in, d_out, stream or None))

    def execute_many_ptrs(self, d_ins, d_outs, stream=0):
        """len(d_ins) transforms in one launch sequence, transform i from device buffer d_ins[i]
        into d_outs[i]."""
        n = len(d_ins)
        ins = (_VP * n)(*d_ins)
        outs = (_VP * n)(*d_outs)
        _check(load().fmmfft_execute_many_ptrs(self._h, n, ins, outs, stream or None))

    @property
    def complex_dtype(self):
        return np.complex128 if self._p == F64 else np.complex64

    @property
    def device_bytes(self):
        v = ctypes.c_size_t()
        _check(load().fmmfft_plan_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def execute_ptr(self, d_in, d_out, stream=0, inverse=False):
        f = load().fmmfft_execute_inverse if inverse else load().fmmfft_execute
        _check(f(self._h, d_in, d_out, stream or None))

    def execute_host(self, x):
        x = np.ascontiguousarray(x, dtype=self.complex_dtype)
        assert x.size == self.N
        y = np.empty_like(x)
        _check(load().fmmfft_execute_host(self._h, x.ctypes.data, y.ctypes.data, None))
        return y

    def execute_graph_ptr(self, d_in, d_out, stream=0):
        """Forward transform through the plan's cached CUDA graph for (d_in, d_out)."""
        _check(load().fmmfft_execute_graph(self._h, d_in, d_out, stream or None))

    def execute_host_many_ptr(self, h_ins, h_outs, stream=0):
        """Pipelined host execute over a sequence of host buffers (pointers, N complex each)."""
        n = len(h_ins)
        assert len(h_outs) == n
        ins = (ctypes.c_void_p * max(1, n))(*h_ins)
        outs = (ctypes.c_void_p * max(1, n))(*h_outs)
        _check(load().fmmfft_execute_host_many(self._h, n, ins, outs, stream or None))

    def execute_host_ptr(self, h_in, h_out, stream=0):
        """Host-memory transform (pointers, e.g. pinned buffers): H2D copy, execute, D2H copy,
        synchronise, all on `stream`."""
        _check(load().fmmfft_execute_host(self._h, h_in, h_out, stream or None))

    def __call__(self, x, out=None, inverse=False, stream=None):
        """x: torch complex tensor on the GPU with N elements (complex128 for 'f64', complex64
        otherwise).  Runs on `stream` (torch.cuda.Stream) or the current stream."""
        import torch
        assert x.is_cuda and x.numel() == self.N and x.is_contiguous()
        want = torch.complex128 if self._p == F64 else torch.complex64
        assert x.dtype == want, f"plan expects {want}"
        if out is None:
            out = torch.empty_like(x)
        s = stream if stream is not None else torch.cuda.current_stream(x.device)
        self.execute_ptr(x.data_ptr(), out.data_ptr(), s.cuda_stream, inverse)
        return out

    def debug_fetch(self):
        """Intermediates of the last execute (float64): u [P-1,2,M], z [P,M] complex,
        phi/psi flat (levels 2..n, planar)."""
        P, M, T = self.P, self.M, self.terms
        s = M // self.b
        n = s.bit_length() - 1
        lv = 2 * (P - 1) * T * ((2 << n) - 4)
        u = np.zeros((P - 1, 2, M))
        z = np.zeros((P, M, 2))
        phi = np.zeros(lv)
        psi = np.zeros(lv)
        _check(load().fmmfft_debug_fetch(self._h, u.ctypes.data, z.ctypes.data, phi.ctypes.data,
                                         psi.ctypes.data))
        return dict(u=u[:, 0] + 1j * u[:, 1], z=z[..., 0] + 1j * z[..., 1], phi=phi, psi=psi)

    def check(self):
        """Synchronise; raise FmmFftError(ERR_TIMEOUT) if a bounded device wait gave up."""
        _check(load().fmmfft_plan_check(self._h))

    def selftest_wait(self, which, limit_us=2000):
        """Run the bounded-wait self-test kernel (0: an mbarrier wait holding tensor memory)
        against this plan's status word."""
        _check(load().fmmfft_plan_selftest_wait(self._h, int(which), int(limit_us)))

    def profile_start(self, max_executes):
        _check(load().fmmfft_profile_start(self._h, int(max_executes)))

    def profile_stop(self):
        """-> (nexecutes, {stage: (total_ms, launches_per_execute)})"""
        cap = 32
        ms = (ctypes.c_double * cap)()
        ln = (_I * cap)()
        ns, ne = _I(), _I()
        _check(load().fmmfft_profile_stop(self._h, ms, ln, cap, ctypes.byref(ns), ctypes.byref(ne)))
        lib = load()
        out = {}
        for i in range(ns.value):
            out[lib.fmmfft_stage_name(i).decode()] = (ms[i], ln[i])
        return ne.value, out

    def close(self):
        if getattr(self, "_h", None):
            load().fmmfft_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Transforms plans[i]: d_in[i] -> d_out[i] (device pointers) as one CUDA graph with
    `nbranch` parallel branches; launch() runs them all."""

    def __init__(self, plans, d_in, d_out, nbranch=8, counts=None):
        n = len(plans)
        self._plans = list(plans)  # keep the plans alive
        ph = (_VP * n)(*[p._h for p in plans])
        ins = (_VP * n)(*d_in)
        outs = (_VP * n)(*d_out)
        h = _VP()
        if counts is None:
            _check(load().fmmfft_batch_create(ctypes.byref(h), ph, ins, outs, n, int(nbranch)))
        else:  # entry i: counts[i] transforms of batched plan i, contiguous
            cs = (_I * n)(*[int(c) for c in counts])
            _check(load().fmmfft_batch_create_many(ctypes.byref(h), ph, cs, ins, outs, n, int(nbranch)))
        self._h = h

    def launch(self, stream=0):
        _check(load().fmmfft_batch_launch(self._h, stream or None))

    def close(self):
        if getattr(self, "_h", None):
            load().fmmfft_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request server (fmmfft_server_*): submit() admits a transform onto one of `nstreams`
    streams under an HBM budget for resident plans; returns a ticket, or raises FmmFftError
    with status ERR_BUSY (7) when the request cannot be admitted now."""

    def __init__(self, hbm_budget_bytes, nstreams=8):
        h = _VP()
        _check(load().fmmfft_server_create(ctypes.byref(h), int(hbm_budget_bytes), int(nstreams)))
        self._h = h

    def submit(self, N, P, terms, b, precision, d_in, d_out):
        t = ctypes.c_uint64()
        rc = load().fmmfft_server_submit(self._h, int(N), int(P), int(terms), int(b),
                                         PRECISIONS[precision], d_in, d_out, ctypes.byref(t))
        if rc:
            raise FmmFftError(rc, "submit refused" if rc == 7 else "submit failed")
        return t.value

    def reserve(self, N, P, terms, b, precision, nplans):
        """Make nplans plans of a shape resident (graphs instantiated) before its requests."""
        rc = load().fmmfft_server_reserve(self._h, int(N), int(P), int(terms), int(b),
                                          PRECISIONS[precision], int(nplans))
        if rc:
            raise FmmFftError(rc, "reserve refused" if rc == 7 else "reserve failed")

    def counts(self):
        """-> (requests dispatched, batched launch sequences)"""
        r, l = ctypes.c_uint64(), ctypes.c_uint64()
        _check(load().fmmfft_server_counts(self._h, ctypes.byref(r), ctypes.byref(l)))
        return r.value, l.value

    def done(self, ticket):
        rc = load().fmmfft_server_query(self._h, ticket)
        if rc not in (0, 7):
            raise FmmFftError(rc, "query failed")
        return rc == 0

    def wait(self, ticket, timeout_ms=60000):
        _check(load().fmmfft_server_wait(self._h, ticket, int(timeout_ms)))

    def stats(self):
        used, plans, streams = ctypes.c_size_t(), _I(), _I()
        _check(load().fmmfft_server_stats(self._h, ctypes.byref(used), ctypes.byref(plans),
                                          ctypes.byref(streams)))
        return {"hbm_used": used.value, "plans": plans.value, "streams": streams.value}

    def close(self):
        if getattr(self, "_h", None):
            load().fmmfft_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PlainFFT:
    """Conventional forward FFT of length N on the GPU (fmmfft_fft_*), the counterpart of the
    reference's FFTW comparators (src/fftw_serial.c:53-58, src/fftw_mpi.c:54-58).
    precision "f64" (complex128) or "f32" / "f32_tc" (complex64)."""

    def __init__(self, N, precision="f32"):
        h = _VP()
        _check(load().fmmfft_fft_create(ctypes.byref(h), int(N), PRECISIONS[precision]))
        self._h = h
        self.N = int(N)
        self.precision = precision

    def execute_ptr(self, d_in, d_out, stream=0):
        _check(load().fmmfft_fft_execute(self._h, d_in, d_out, stream or None))

    def device_bytes(self):
        v = ctypes.c_size_t()
        _check(load().fmmfft_fft_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            load().fmmfft_fft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def level_planar(flat, P, T, n, level):
    """View of level `level` of a planar expansion array as [P-1, 2, 2^level, T]."""
    off = 2 * (P - 1) * T * ((1 << level) - 4)
    cnt = 2 * (P - 1) * T * (1 << level)
    return flat[off:off + cnt].reshape(P - 1, 2, 1 << level, T)


class Shard:
    """Shard g of G of one sharded transform (fmmfft_shard_*): see include/fmmfft.h.  buffers()
    gives the device pointers and sizes of the exchange buffers; phase(k) runs phase k."""

    def __init__(self, N, P, terms, b, precision, G, g):
        h = _VP()
        _check(load().fmmfft_shard_create(ctypes.byref(h), int(N), int(P), int(terms), int(b),
                                          PRECISIONS[precision], int(G), int(g)))
        self._h = h
        self.N, self.P, self.G, self.g, self.precision = N, P, G, g, precision

    def buffers(self):
        bb = _ShardBufs()
        _check(load().fmmfft_shard_buffers(self._h, ctypes.byref(bb)))
        return {n: getattr(bb, n) for n, _ in _ShardBufs._fields_}

    def phase(self, k, stream=0):
        _check(load().fmmfft_shard_phase(self._h, int(k), stream or None))

    def close(self):
        if getattr(self, "_h", None):
            load().fmmfft_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

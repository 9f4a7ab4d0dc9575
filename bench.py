#!/usr/bin/env python
"""Throughput of the B200 FMM-FFT on one large transform (N = 2^24 complex64, P = 64 blocks,
p = 24 Chebyshev terms, b = 32 points per leaf box: 13 tree levels, near-field width 1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision f32|f32_tc|f64] [--no-cpu-baseline]

One step = one forward transform of the whole N-point vector.  `value` = Msamples/s with the
input resident in HBM (device-timed with CUDA events, L2 flushed by a 256 MB write before every
step); `e2e` = the same transform through the C-ABI from pinned host memory (H2D, execute, D2H,
synchronise).  With --gpus N (torchrun, one rank per GPU) every rank transforms its own input:
per-GPU work is fixed (weak scaling), value = all ranks' samples / max-over-ranks time.
`--impl reference` times the reference's own CPU implementation (src/fmmfft.c compiled with the
project's MPI/FFTW shims, oracle/_ref) on this host with P thread-ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "fmm-fft_b200"))

WORKLOAD = dict(workload="single large transform", N=1 << 24, P=64, terms=24, b=32,
                element="complex64", input="iid standard normal re/im, PCG64 seed 0 (+rank)")
METRIC = "Msamples/s at rel-L2 <= 1e-6 vs FP64"
UNIT = "Msamples/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", default=None, help="f32 | f32_tc | f64 (default: fastest)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--workload", choices=["single", "uneven-batch", "serving", "precision-sweep", "sharded"],
                    default="single",
                    help="single: the headline transform (default); uneven-batch: 512 transforms "
                         "of mixed N and P as one graph; serving: Poisson arrivals through the "
                         "request server; precision-sweep: N = 2^26, P = 256, tones + noise, every "
                         "order and arithmetic, error against throughput; sharded: the headline "
                         "transform as G shards (emulated in this process), each shard's device time")
    ap.add_argument("--shards", type=int, default=8, help="sharded: G")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: arrivals per second")
    ap.add_argument("--requests", type=int, default=1200, help="serving: requests per rate")
    ap.add_argument("--no-served", action="store_true", help="skip the served-vs-plain object")
    return ap.parse_args()


def seeded(n, seed, dtype):
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    re_ = rng.standard_normal(n)
    im_ = rng.standard_normal(n)
    return (re_ + 1j * im_).astype(dtype)


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append(dict(sm=float(parts[1]), smax=float(parts[2]),
                                     power=float(parts[3]) if parts[3] not in ("", "[N/A]") else 0.0,
                                     hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
                except ValueError:
                    continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows),
                "sm_max_mhz": max(r["smax"] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(r["power"] for r in rows)}


# ------------------------------------------------------------------------ roofline helpers
def stage_bytes(N, P, T, b, esz):
    """Algorithmic HBM bytes of one execute per stage: each array a stage must read or write,
    counted once (R = esz/2 bytes per real)."""
    M = N // P
    S1 = P - 1
    s = M // b
    n = s.bit_length() - 1
    R = esz // 2
    lv = lambda l: 2 * S1 * T * (1 << l) * R  # one level of expansions
    xt_all = 2 * P * M * R
    xt_sec = 2 * S1 * M * R
    u = 2 * S1 * M * R
    # levels of fewer than 4096 rows (2 (P-1) boxes each) run in the coarse-tree launch
    coarse = lambda rows: rows < 4096
    m2m = [l for l in range(2, n)]
    m2l = [l for l in range(3, n + 1)]
    m2m_c = [l for l in m2m if coarse(2 * S1 * (1 << l))]
    m2l_c = [l for l in m2l if coarse(2 * S1 * (1 << (l - 1)))]
    tile = max(1, 2048 // P)  # points per sections tile; S2M is fused there for whole boxes
    fused = tile % b == 0 and T % 4 == 0
    return {
        "sections": N * esz + xt_all + (lv(n) if fused else 0),
        "s2m": 0 if fused else xt_sec + lv(n),
        "m2m": sum(lv(l + 1) + lv(l) for l in m2m if l not in m2m_c),
        "coarse_tree": sum(lv(l + 1) + lv(l) for l in m2m_c) + 2 * lv(2) +
                       sum(lv(l - 1) + lv(l) + lv(l) for l in m2l_c),
        "m2l_l2l": sum(lv(l - 1) + lv(l) + lv(l) for l in m2l if l not in m2l_c),
        "leaf_l2t_near": lv(n) + xt_sec + u,
        "combine_dftP": 2 * M * R + u + N * esz,
        "fft_pass1": 2 * N * esz,
        "fft_pass2": 2 * N * esz,
    }


# DRAM bytes (read + write) per launch of the stage's kernel from one ncu capture of the bench
# command (profiles/k_tc_nbr_TcLeafNb_N2p24_P64_T24_b32.txt, k_sections_f32_N2p24_P64_T24_b32.txt,
# k_tc_rowgemm16_TcM2L_N2p24_P64_T24_b32.txt).  M2L: the finest of its seven launches was captured
# (213.4 MB for 2^12 parents per section plane); the mean over the seven levels scales it by the
# levels' rows, (2^13 - 2^6) / 2^12 / 7.  Only meaningful for the headline workload.
TRAFFIC_PER_LAUNCH = {
    "leaf_l2t_near": 240.520704e6 + 98.922752e6,
    "sections": 134.243840e6 + 186.710528e6,
    "m2l_l2l": (148.727808e6 + 64.687360e6) * ((1 << 13) - (1 << 6)) / (1 << 12) / 7,
}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------ reference arm
def reference_cpu(N, P, T, b, steps, warmup, budget_s=150.0):
    """Median wall time of the shim-built reference's mft (src/fmmfft.c) on this host, P
    thread-ranks; falls back to the oracle restatement when oracle/_ref was not built."""
    import numpy as np
    ref_so = os.path.join(REPO, "oracle", "_ref", "libfmmfft_ref.so")
    x = seeded(N, 0, np.complex128)
    y = np.zeros_like(x)
    times = []
    if os.path.exists(ref_so):
        lib = ctypes.CDLL(ref_so)
        L, VP = ctypes.c_long, ctypes.c_void_p
        lib.fmmref_forward.argtypes = [L, L, L, L, VP, VP, ctypes.c_int, VP]
        kind = "reference"
        t_start = time.time()
        runs = max(1, steps)
        buf = (ctypes.c_double * (runs + warmup))()
        # one process-level call: warmup + timed runs share the plan (mfti), as the reference's
        # own 6-run loop does (fmmfft.c:1251-1273); stop early if the budget is exceeded
        done = 0
        while done < runs and time.time() - t_start < budget_s:
            k = min(runs - done, 2) + (warmup if done == 0 else 0)
            t = (ctypes.c_double * k)()
            rc = lib.fmmref_forward(N, P, T, b, x.ctypes.data, y.ctypes.data, k, t)
            if rc != 0:
                raise RuntimeError(f"reference failed rc={rc}")
            vals = list(t)[(warmup if done == 0 else 0):]
            times += vals
            done += len(vals)
        del buf
        sample = (f"{len(times)} mft runs of the full workload on {P} thread-ranks "
                  f"(shim-built src/fmmfft.c: the unmodified reference with project-written MPI "
                  f"and FFTW stand-ins, the FFT a radix-2 FP64 FFT with cached twiddles, because "
                  f"neither mpicc nor libfftw3 is installed), median; plan (mfti) excluded.  "
                  f"For scale: the reference's own recorded cluster run of N = 2^24, P = 64 "
                  f"(OpenMPI + FFTW, b = 32, 15 terms) took 0.173 s = 97.2 Msamples/s "
                  f"(plotting/raw_data/cluster_out_fmmfft_32_15.txt:1552-1556)")
    else:
        sys.path.insert(0, os.path.join(REPO, "tests"))
        import oracle_lib as ol
        kind = "port"
        for i in range(max(1, min(steps, 3))):
            t0 = time.time()
            ol.forward(x, P, T, b)
            times.append(time.time() - t0)
        sample = f"{len(times)} oracle forward runs of the full workload, OpenMP threads"
    med = statistics.median(times)
    return dict(value=N / med / 1e6, unit=UNIT, cores=os.cpu_count(), kind=kind, sample=sample,
                seconds_per_transform=med, runs=len(times))


# ------------------------------------------------------------------------ uneven batch
def uneven_jobs(n, seed, lo=12, hi=22, terms=16):
    """N log-uniform over powers of two 2^lo..2^hi, P from {8,16,32,64} subject to M >= 256."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    jobs = []
    while len(jobs) < n:
        N = 1 << int(rng.integers(lo, hi + 1))
        P = int(rng.choice([8, 16, 32, 64]))
        if N // P < 256:
            continue
        jobs.append((N, P, terms, 32))
    return jobs


def run_uneven_batch(a):
    """512 transforms of uneven N and P (p = 16) as one CUDA graph: the transforms are grouped by
    shape, each group is ONE launch sequence of a batched plan (every tree stage one contraction
    over the rows of all its transforms), and the groups run as parallel graph branches.  Against
    the plain FP32 per-transform FMM-FFT (one execute after another, one stream)."""
    import numpy as np
    import torch
    import fmmfft
    torch.cuda.set_device(0)
    jobs = uneven_jobs(512, 4)
    prec = a.precision or "f32_tc"
    groups = {}
    for i, job in enumerate(jobs):
        groups.setdefault(job, []).append(i)
    shapes = sorted(groups)
    dt = torch.complex64
    total = sum(N for (N, P, T, b) in jobs)
    t0 = time.time()
    plans = [fmmfft.Plan(*sh, prec, max_transforms=len(groups[sh])) for sh in shapes]
    xin = [torch.randn(len(groups[sh]) * sh[0], dtype=dt, device="cuda") for sh in shapes]
    yout = [torch.empty_like(x) for x in xin]
    batch = fmmfft.Batch(plans, [x.data_ptr() for x in xin], [y.data_ptr() for y in yout],
                         nbranch=16, counts=[len(groups[sh]) for sh in shapes])
    build_s = time.time() - t0
    stream = torch.cuda.current_stream()
    for _ in range(max(3, a.warmup)):
        batch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    K = a.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        batch.launch(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    # plain comparator: FP32 CUDA-core plans, the same transforms one after another, one stream
    pplans = {sh: fmmfft.Plan(*sh, "f32") for sh in shapes}
    views = []
    for gi, sh in enumerate(shapes):
        N = sh[0]
        for j in range(len(groups[sh])):
            views.append((pplans[sh], xin[gi][j * N:(j + 1) * N], yout[gi][j * N:(j + 1) * N]))
    for pl, x, y in views:
        pl.execute_ptr(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0.record(stream)
    R = max(1, K // 2)
    for _ in range(R):
        for pl, x, y in views:
            pl.execute_ptr(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1) / R
    batch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    worst = 0.0
    for gi, sh in enumerate(shapes[::5]):  # accuracy of a sample against FP64
        g = shapes.index(sh)
        N = sh[0]
        x = xin[g][:N].cpu().numpy().astype(np.complex128)
        y = yout[g][:N].cpu().numpy().astype(np.complex128)
        ref = np.fft.fft(x)
        worst = max(worst, float(np.linalg.norm(y - ref) / np.linalg.norm(ref)))
    line = {"metric": "Msamples/s, uneven batch of 512 transforms as one graph", "value": total / (ms / 1e3) / 1e6,
            "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": max(3, a.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "fp32", "f32_tc": "fp32 (split-TF32 tcgen05)", "bf16x3": "fp32 (BF16x3 tcgen05)",
                      "f64": "fp64"}[prec],
            "data": "synthetic", "impl": "ours",
            "config": {"workload": "uneven batch", "transforms": len(jobs), "N": "2^12..2^22 log-uniform",
                       "P": "{8,16,32,64}, M >= 256", "terms": 16, "b": 32, "graph_branches": 16,
                       "distinct_shapes": len(shapes), "launch_sequences_per_step": len(shapes),
                       "samples_per_step": total, "plan_and_graph_build_s": build_s,
                       "autotuned": plans[0].describe()},
            "plain_per_transform": {"value": total / (ms_plain / 1e3) / 1e6, "unit": UNIT,
                                    "ms_per_step": ms_plain,
                                    "how": "FP32 plans on CUDA cores, fmmfft_execute per transform, one stream"},
            "batched_over_plain": ms_plain / ms,
            "accuracy": {"worst_rel_l2_vs_fp64_sampled": worst}}
    batch.close()
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------ serving
SERVE_CLASSES = {"1e-4": 8, "1e-6": 20}  # accuracy class -> Chebyshev terms


def serving_requests(rate, count, seed):
    """`count` Poisson arrivals at `rate` per second; N log-uniform over powers of two
    2^10..2^24 (complex64, iid normal); two accuracy classes, rel-L2 1e-4 (p = 8) and 1e-6
    (p = 20), equally likely; P = min(64, max(2, N / 512)), b = 32."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    t, reqs = 0.0, []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        N = 1 << int(rng.integers(10, 25))
        terms = SERVE_CLASSES["1e-4" if int(rng.integers(0, 2)) == 0 else "1e-6"]
        P = max(2, min(64, N // 512))
        reqs.append((t, N, P, terms, 32))
    return reqs


def serve_compare(rates, count=1200, seed=7, served_prec="f32_tc", plain_prec="f32"):
    """Open-loop Poisson arrivals through the request server (continuous batching, mixed
    precision on the tensor cores) against the plain per-request FMM-FFT (FP32 CUDA cores, one
    request after another on one stream, no batching), at each rate.  Per rate: Msamples/s =
    samples of all requests / (last completion - first arrival), and latency percentiles
    (completion - arrival).  Inputs are device-resident (4 buffers per size)."""
    import torch
    import fmmfft
    budget = 120 << 30
    nbuf = 4
    out = {}
    allreqs = {r: serving_requests(r, count, seed) for r in rates}
    sizes = sorted({q[1] for reqs in allreqs.values() for q in reqs})
    bufs = {N: [(torch.randn(N, dtype=torch.complex64, device="cuda"),
                 torch.empty(N, dtype=torch.complex64, device="cuda")) for _ in range(nbuf)]
            for N in sizes}
    shapes = sorted({q[1:] for reqs in allreqs.values() for q in reqs})

    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(q * len(v)))] * 1e3 if v else None

    def drive(reqs, submit, poll):
        lat, pend = [], []
        counter = {}
        t0 = time.perf_counter()
        i = 0
        while i < len(reqs) or pend:
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i][0] <= now:
                arr, N, P, T, b = reqs[i]
                k = counter.get(N, 0)
                x, y = bufs[N][k % nbuf]
                h = submit(N, P, T, b, x, y)
                if h is None:  # refused (admission): retried on the next pass
                    break
                counter[N] = k + 1
                pend.append((h, arr))
                i += 1
            now = time.perf_counter() - t0
            keep = []
            for h, arr in pend:
                if poll(h):
                    lat.append(now - arr)
                else:
                    keep.append((h, arr))
            pend = keep
        span = time.perf_counter() - t0 - reqs[0][0]
        return span, lat

    # served: one server for all rates, warmed so that every lane's plans and graphs exist
    srv = fmmfft.Server(budget, nstreams=3)

    def srv_submit(N, P, T, b, x, y):
        try:
            return srv.submit(N, P, T, b, served_prec, x.data_ptr(), y.data_ptr())
        except fmmfft.FmmFftError as e:
            if e.status == 7:
                return None
            raise

    for (N, P, T, b) in shapes:  # every shape's plans resident, graphs instantiated
        srv.reserve(N, P, T, b, served_prec, 3)
        srv.wait(srv_submit(N, P, T, b, *bufs[N][0]))
    torch.cuda.synchronize()
    served = {}
    for r in rates:
        reqs = allreqs[r]
        total = sum(q[1] for q in reqs)
        span, lat = drive(reqs, srv_submit, srv.done)
        served[r] = (total / span / 1e6, pct(lat, 0.5), pct(lat, 0.99), len(reqs))
    st = srv.stats()
    srv.close()

    # plain: resident FP32 plans, each request executed and synchronised before the next
    plans = {sh: fmmfft.Plan(*sh, plain_prec) for sh in shapes}
    stream = torch.cuda.current_stream()
    for sh, pl in plans.items():
        x, y = bufs[sh[0]][0]
        pl.execute_ptr(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()

    def plain_submit(N, P, T, b, x, y):
        plans[(N, P, T, b)].execute_ptr(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        return True

    for r in rates:
        reqs = allreqs[r]
        total = sum(q[1] for q in reqs)
        span, lat = drive(reqs, plain_submit, lambda h: True)
        sv = served[r]
        out[str(int(r))] = {
            "requests": sv[3], "offered_msamples_s": total / reqs[-1][0] / 1e6,
            "served": {"value": sv[0], "unit": UNIT, "p50_ms": sv[1], "p99_ms": sv[2]},
            "plain": {"value": total / span / 1e6, "unit": UNIT, "p50_ms": pct(lat, 0.5),
                      "p99_ms": pct(lat, 0.99)},
            "ratio": sv[0] / (total / span / 1e6)}
    for pl in plans.values():
        pl.close()
    return {"rates": out, "resident_plans": st["plans"], "resident_plan_bytes": st["hbm_used"],
            "config": {"N": "2^10..2^24 log-uniform, complex64 iid normal", "P": "min(64, max(2, N/512))",
                       "b": 32, "classes": {"1e-4": "p=8", "1e-6": "p=20"},
                       "served": f"request server, continuous batching, {served_prec}",
                       "plain": f"one request at a time, {plain_prec} plans on CUDA cores, no batching",
                       "hbm_budget_bytes": budget, "requests_per_rate": count}}


def run_serving(a):
    import torch
    torch.cuda.set_device(0)
    res = serve_compare([a.rate], count=a.requests)
    r = res["rates"][str(int(a.rate))]
    line = {"metric": "Msamples/s and p99 latency, served vs plain FMM-FFT (Poisson arrivals)",
            "value": r["served"]["value"], "unit": UNIT, "n_gpus": 1, "steps": r["requests"],
            "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (split-TF32 tcgen05)", "data": "synthetic",
            "impl": "ours", "config": dict(res["config"], workload="serving", rate_per_s=a.rate),
            "latency_ms": {"p50": r["served"]["p50_ms"], "p99": r["served"]["p99_ms"]},
            "plain_per_request": r["plain"], "served_over_plain": r["ratio"],
            "resident_plans": res["resident_plans"]}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------ precision sweep
def run_precision_sweep(a):
    """N = 2^26 complex64, 32 off-bin tones + 1e-3 noise (seeded), P = 256, b = 32, terms in
    {8, 16, 24, 32}; per order and arithmetic (FP32 CUDA cores, split TF32 and BF16x3 with three
    products on the tensor cores, each with and without the FP64 residual-correction pass): device-timed
    Msamples/s, and rel-L2 / max error against the FP64 FFT (numpy) and against the FP64 FMM-FFT
    of the same order (the reference's arithmetic).  One JSON line per point."""
    import numpy as np
    import torch
    import fmmfft
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib as ol
    torch.cuda.set_device(0)
    N, P, b = 1 << 26, 256, 32
    x = ol.tone_input(N, 2026).astype(np.complex64)
    ref = np.fft.fft(x.astype(np.complex128))
    nref = np.linalg.norm(ref)
    mref = np.max(np.abs(ref))
    dx = torch.from_numpy(x).cuda()
    dx64 = dx.to(torch.complex128)
    y32 = torch.empty_like(dx)
    y64 = torch.empty_like(dx64)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    K = max(3, a.steps // 2)

    def timed(fn):
        for _ in range(3):
            fn()
        evs = []
        for i in range(K):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs) / K

    def errs(y, fmm64):
        y = y.astype(np.complex128)
        return {"rel_l2_vs_fp64_fft": float(np.linalg.norm(y - ref) / nref),
                "max_err_vs_fp64_fft": float(np.max(np.abs(y - ref)) / mref),
                "rel_l2_vs_fp64_fmm": float(np.linalg.norm(y - fmm64) / np.linalg.norm(fmm64))}

    for T in (8, 16, 24, 32):
        p64 = fmmfft.Plan(N, P, T, b, "f64")
        p64.execute_ptr(dx64.data_ptr(), y64.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        fmm64 = y64.cpu().numpy()
        ms64 = timed(lambda: p64.execute_ptr(dx64.data_ptr(), y64.data_ptr(), stream.cuda_stream))
        p64.close()
        pts = [("fp64", ms64, errs(fmm64, fmm64))]
        for prec, name in (("f32", "fp32"), ("f32_tc", "tf32x3"), ("bf16x3", "bf16x3")):
            plan = fmmfft.Plan(N, P, T, b, prec)
            ms = timed(lambda: plan.execute_ptr(dx.data_ptr(), y32.data_ptr(), stream.cuda_stream))
            plan.execute_ptr(dx.data_ptr(), y32.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            pts.append((name, ms, errs(y32.cpu().numpy(), fmm64)))
            plan.enable_refinement()
            msr = timed(lambda: plan.execute_refined_ptr(dx.data_ptr(), y64.data_ptr(), stream.cuda_stream))
            plan.execute_refined_ptr(dx.data_ptr(), y64.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            pts.append((name + "+fp64_residual", msr, errs(y64.cpu().numpy(), fmm64)))
            plan.check()
            plan.close()
        for name, ms, e in pts:
            line = {"metric": "precision sweep: Msamples/s and error vs FP64", "workload": "precision-sweep",
                    "N": N, "P": P, "terms": T, "b": b, "arithmetic": name,
                    "value": N / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_transform": ms,
                    "input": "32 off-bin unit tones + 1e-3 complex white noise, PCG64 seed 2026",
                    "l2": "256 MB write before every timed step", **e}
            print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------ sharded transform
def run_sharded(a):
    """The headline transform as G shards of fmmfft_shard_*, all on this device in turn (the
    exchanges as device copies): each shard's phases timed with CUDA events, L2 flushed before
    every phase.  On G GPUs the shards' phases run at once, so a transform's device time there is
    the slowest shard's phases plus the exchanges (whose bytes are reported, not timed here)."""
    import numpy as np
    import torch
    import fmmfft
    import sharded
    torch.cuda.set_device(0)
    N, P, T, b = WORKLOAD["N"], WORKLOAD["P"], WORKLOAD["terms"], WORKLOAD["b"]
    G, prec = a.shards, a.precision or "f32_tc"
    x = torch.from_numpy(seeded(N, 0, np.complex64)).cuda()
    shards = [fmmfft.Shard(N, P, T, b, prec, G, g) for g in range(G)]
    views = [sharded._views(s) for s in shards]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()
    tr = sharded.LocalTransport(G)
    blocks = list(x.chunk(G))

    def step(timed):
        times = np.zeros((G, 3))
        for v, blk in zip(views, blocks):
            v["x_ext"][v["halo"]:v["halo"] + blk.numel()].copy_(blk)
        tr.halos(blocks, [v["x_ext"][:v["halo"]] for v in views],
                 [v["x_ext"][v["halo"] + blk.numel():] for v, blk in zip(views, blocks)])
        evs = []
        for k in range(3):
            for g, s in enumerate(shards):
                flush.fill_(k + 1)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                s.phase(k, st.cuda_stream)
                e1.record()
                evs.append((g, k, e0, e1))
            if k == 0:
                tr.sum([v["sums"] for v in views])
                tr.gather([v["phi_send"] for v in views], [v["phi_all"] for v in views])
            elif k == 1:
                tr.alltoall([v["z_send"] for v in views], [v["z_recv"] for v in views])
        torch.cuda.synchronize()
        for g, k, e0, e1 in evs:
            times[g, k] = e0.elapsed_time(e1)
        return times

    for _ in range(max(a.warmup, 3)):
        step(False)
    per = [step(True) for _ in range(a.steps)]
    worst = sorted(t.sum(axis=1).max() for t in per)[len(per) // 2]
    y = torch.cat([v["y"] for v in views]).cpu().numpy().astype(np.complex128)
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128))
    err = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
    bb = shards[0].buffers()
    esz = 8
    line = {"metric": "device time per transform, sharded over G shards (slowest shard's phases)",
            "value": worst, "unit": "ms", "higher_is_better": False, "n_gpus": 1, "steps": a.steps,
            "warmup": max(a.warmup, 3), "dtype": "fp32 (split-TF32 tcgen05)", "data": "synthetic",
            "config": {"workload": "sharded single transform", "N": N, "P": P, "terms": T, "b": b,
                       "shards": G, "precision": prec, "how": "G shards emulated on one B200, phases in turn, "
                       "256 MB L2 flush before every phase"},
            "phase_ms_median": {f"shard{g}": [float(np.median([t[g, k] for t in per])) for k in range(3)]
                                for g in range(G)},
            "exchange_bytes_per_shard": {"x_halos_in": 2 * bb["halo_elems"] * esz, "section_sums": 2 * P * esz,
                                         "coarse_allgather_in": (G - 1) * bb["phi_elems"] * 4,
                                         "alltoall_out": (G - 1) * bb["z_elems"] // G * esz},
            "accuracy": {"rel_l2_vs_fp64": err}}
    print(json.dumps(line))
    for sh in shards:
        sh.close()
    return 0


def main():
    a = parse()
    if a.workload == "sharded":
        return run_sharded(a)
    if a.workload == "precision-sweep":
        return run_precision_sweep(a)
    if a.workload == "uneven-batch":
        return run_uneven_batch(a)
    if a.workload == "serving":
        return run_serving(a)
    import replicas
    info = replicas.rank_info()
    world, rank, local = info.world, info.rank, info.local
    N, P, T, b = WORKLOAD["N"], WORKLOAD["P"], WORKLOAD["terms"], WORKLOAD["b"]
    cfg = dict(WORKLOAD)

    if a.impl == "reference":
        if rank != 0:
            return 0
        cpu = reference_cpu(N, P, T, b, a.steps, min(a.warmup, 1))
        line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": a.gpus,
                "steps": cpu["runs"], "warmup": min(a.warmup, 1),
                "ms_per_step": cpu["seconds_per_transform"] * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": cfg, "impl": "reference",
                "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch
    import fmmfft

    torch.cuda.set_device(local)
    dist = replicas.init_group(info, "nccl", device=torch.device("cuda", local))
    prec = a.precision or "f32_tc"
    plan = fmmfft.Plan(N, P, T, b, prec)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    esz = 16 if prec == "f64" else 8
    xh = seeded(N, replicas.replica_seed(0, rank), np.complex128)
    x = torch.from_numpy(xh).to(cdt).cuda()
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    acc = {}
    if rank == 0 and not a.no_accuracy:
        plan.execute_ptr(x.data_ptr(), y.data_ptr(), sp)
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.complex128)
        ref = np.fft.fft(x.cpu().numpy().astype(np.complex128))
        acc = {"rel_l2_vs_fp64": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
               "max_abs_err_over_max_abs": float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))}
        del got, ref

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, a.warmup)):
        flush.fill_(1.0)
        plan.execute_ptr(x.data_ptr(), y.data_ptr(), sp)
    torch.cuda.synchronize()

    K = a.steps
    ev_s = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ev_e = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    plan.profile_start(K)
    replicas.barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(K):
            flush.fill_(float(i))
            ev_s[i].record(stream)
            plan.execute_ptr(x.data_ptr(), y.data_ptr(), sp)
            ev_e[i].record(stream)
        torch.cuda.synchronize()
    replicas.barrier(dist)
    torch.cuda.synchronize()
    nexec, stages = plan.profile_stop()
    per = [s.elapsed_time(e) for s, e in zip(ev_s, ev_e)]
    tot = replicas.max_over_ranks(sum(per), dist, "cuda")
    clocks = clk.summary()

    # in-run comparator: the plain FP32 CUDA-core FMM-FFT on the same input, same timing rule
    plain = {}
    if prec != "f32":
        pplan = fmmfft.Plan(N, P, T, b, "f32")
        for _ in range(3):
            pplan.execute_ptr(x.data_ptr(), y.data_ptr(), sp)
        pms = []
        for i in range(max(3, K // 2)):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pplan.execute_ptr(x.data_ptr(), y.data_ptr(), sp)
            e1.record(stream)
            pms.append((e0, e1))
        torch.cuda.synchronize()
        pm = sum(e0.elapsed_time(e1) for e0, e1 in pms) / len(pms)
        plain = {"value": N * world / (pm / 1e3) / 1e6, "unit": UNIT, "ms_per_step": pm,
                 "how": "FMMFFT_F32 plan: every contraction on CUDA cores"}
        pplan.close()

    # a conventional FFT of the same N on the same GPU: the project's plain Stockham FFT (where
    # the reference's FFTW comparator programs stand) and, as library context only, cuFFT
    def timed(fn, reps):
        for _ in range(3):
            fn()
        evs = []
        for i in range(reps):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs) / reps

    fft_cmp = {}
    pfft = fmmfft.PlainFFT(N, "f64" if prec == "f64" else "f32")
    ms_pf = timed(lambda: pfft.execute_ptr(x.data_ptr(), y.data_ptr(), sp), max(3, K // 2))
    fft_cmp["plain_stockham"] = {"value": N * world / (ms_pf / 1e3) / 1e6, "unit": UNIT,
                                 "ms_per_step": ms_pf,
                                 "how": "fmmfft_fft_execute: project-written size-N FFT, "
                                        "register Stockham passes"}
    pfft.close()
    ms_cu = timed(lambda: torch.fft.fft(x), max(3, K // 2))
    fft_cmp["cufft_library"] = {"value": N * world / (ms_cu / 1e3) / 1e6, "unit": UNIT,
                                "ms_per_step": ms_cu, "how": "torch.fft.fft (cuFFT), context only"}

    # e2e through the C-ABI from pinned host memory: E host-resident transforms through the
    # pipelined host execute (copy-in of step i+1, execute of step i and copy-out of step i-1
    # overlap), and one at a time through the single host execute for comparison
    hins = [torch.from_numpy(xh).to(cdt).pin_memory()]
    hins.append(hins[0].clone().pin_memory())
    houts = [torch.empty_like(hins[0]).pin_memory() for _ in range(3)]
    E = max(3, min(K, 32))
    plan.execute_host_many_ptr([h.data_ptr() for h in hins], [o.data_ptr() for o in houts[:2]], sp)
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    plan.execute_host_many_ptr([hins[i % 2].data_ptr() for i in range(E)],
                               [houts[i % 3].data_ptr() for i in range(E)], sp)
    s1.record(stream)
    s1.synchronize()
    e2e_tot = replicas.max_over_ranks(s0.elapsed_time(s1), dist, "cuda")
    e2e_one = []
    for i in range(E):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        plan.execute_host_ptr(hins[0].data_ptr(), houts[0].data_ptr(), sp)
        s1.record(stream)
        s1.synchronize()
        e2e_one.append(s0.elapsed_time(s1))
    e2e_one_tot = replicas.max_over_ranks(sum(e2e_one), dist, "cuda")

    if rank == 0:
        ms_step = tot / K
        value = replicas.whole_job_rate(N, K, world, tot) / 1e6
        byts = stage_bytes(N, P, T, b, esz)
        hbm, peak_kind = peaks()
        stage_tab = {}
        for name, (ms, launches) in stages.items():
            if launches == 0:
                continue
            avg_launch_ms = ms / max(1, nexec) / launches
            entry = {"ms_per_execute": ms / max(1, nexec), "launches_per_execute": launches,
                     "share": ms / max(1e-12, sum(v[0] for v in stages.values()))}
            if name in byts:
                entry["alg_bytes_per_execute"] = byts[name]
                entry["gbs"] = byts[name] / (ms / max(1, nexec) / 1e3) / 1e9
            stage_tab[name] = entry
            del avg_launch_ms
        dom = max(stage_tab, key=lambda k: stage_tab[k]["ms_per_execute"])
        d = stage_tab[dom]
        achieved = d.get("gbs")
        launches_per_exec = sum(v["launches_per_execute"] for v in stage_tab.values())
        lat = sorted(per)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": max(3, a.warmup), "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "fp32", "f32_tc": "fp32 (split-TF32 tcgen05)", "f64": "fp64"}[prec],
            "data": "synthetic",
            "config": dict(cfg, precision=prec, l2="256 MB write before every timed step; "
                           "input 128 MiB > 126 MB L2", parallelism=f"replicas x{world}"),
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                           "min": lat[0], "max": lat[-1]},
            "accuracy": acc,
            "e2e": {"value": replicas.whole_job_rate(N, E, world, e2e_tot) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": N * esz, "d2h_bytes_per_step": N * esz,
                    "ms_per_step": e2e_tot / E, "steps": E,
                    "path": "fmmfft_execute_host_many over E pinned host buffers (copy-in, execute "
                            "and copy-out of consecutive steps overlapped)",
                    "one_at_a_time": {"value": replicas.whole_job_rate(N, E, world, e2e_one_tot) / 1e6,
                                      "ms_per_step": e2e_one_tot / E,
                                      "path": "fmmfft_execute_host per step (H2D, execute, D2H, sync)"}},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": TRAFFIC_PER_LAUNCH.get(dom), "peak_kind": peak_kind,
                         "alg_bytes_per_launch": d.get("alg_bytes_per_execute", 0) / d["launches_per_execute"]},
            # the transform as a whole against one read + one write of the vector (2 N e bytes)
            "transform_roofline": {"alg_bytes": 2 * N * esz, "achieved_gbs": 2 * N * esz / (ms_step / 1e3) / 1e9,
                                   "frac": 2 * N * esz / (ms_step / 1e3) / 1e9 / hbm},
            "stages": stage_tab,
            "plain_fp32_comparator": plain,
            "plain_fft_comparator": fft_cmp,
            "gpu_launches": launches_per_exec * K,
            "clocks": clocks,
        }
        if world == 1 and not a.no_served:
            # the headline comparison: served (continuous batching, tensor cores) against the
            # plain per-request FP32 FMM-FFT, Poisson arrivals at three rates
            line["served_vs_plain"] = serve_compare([2000.0, 10000.0, 50000.0], count=a.requests)
        if world == 1 and not a.no_cpu_baseline:
            cpu = reference_cpu(N, P, T, b, 2, 0, budget_s=60.0)
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line))
    plan.close()
    replicas.finish(dist)
    return 0


if __name__ == "__main__":
    sys.exit(main())

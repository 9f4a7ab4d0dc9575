"""Regenerates the golden vectors in this directory from the reference itself.

Run in the build container (it needs the reference sources, which are not shipped):

    make -C oracle REFERENCE=<reference checkout>   # builds oracle/_ref/libfmmfft_ref.so
    FMMFFT_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Outputs
  ref_forward_<tag>.npz   seeded complex128 input (from its seed) -> output y of the UNMODIFIED
                          reference src/fmmfft.c run on P thread-ranks through the project's
                          MPI/FFTW shims (oracle/ref_driver.c).  Keys: N, P, terms, b, seed,
                          x_sha256, y.
  recorded_error_envelope.csv
                          rows (N, P, b, T, err_percent) copied from the reference's own recorded
                          runs, plotting/raw_data/cluster_output_error.csv, for N <= 2^22: the
                          max pointwise relative error (percent, 6 decimals) of rank 0's block
                          for the ramp input x[i] = i + 1 (src/fmmfft_error.c:1236-1267).
"""
import csv
import ctypes
import hashlib
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("FMMFFT_REFERENCE")  # the reference checkout: required

# (N, P, terms, b): covers t = s/P = 1, 2 and > 2 (the reference's three near-field branches,
# fmmfft.c:805-954), P = 2 (only the sc = P/2 averaging case), the sc > P/2 half-shift path,
# and the N = 2^16, P = 4, p = 16, 3-level (b = 2048) transform.
CASES = [
    (256, 4, 8, 8, 0),
    (1024, 2, 8, 16, 1),
    (4096, 8, 10, 16, 2),
    (4096, 4, 12, 32, 3),
    (8192, 16, 12, 32, 4),
    (16384, 4, 16, 512, 5),
    (16384, 32, 9, 16, 6),
    (65536, 4, 16, 2048, 7),
]


def seeded_input(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    re_ = rng.standard_normal(n)
    im_ = rng.standard_normal(n)
    return (re_ + 1j * im_).astype(np.complex128)


def tag(N, P, T, b):
    return f"N{N}_P{P}_T{T}_b{b}"


def main():
    if not REFERENCE:
        sys.exit("set FMMFFT_REFERENCE to the reference checkout (its plotting/raw_data is read)")
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libfmmfft_ref.so"))
    L, VP = ctypes.c_long, ctypes.c_void_p
    lib.fmmref_forward.argtypes = [L, L, L, L, VP, VP, ctypes.c_int, VP]
    for N, P, T, b, seed in CASES:
        x = seeded_input(N, seed)
        y = np.zeros(N, np.complex128)
        rc = lib.fmmref_forward(N, P, T, b, x.ctypes.data, y.ctypes.data, 1, None)
        if rc != 0:
            sys.exit(f"reference failed on {(N, P, T, b)}: {rc}")
        out = os.path.join(HERE, f"ref_forward_{tag(N, P, T, b)}.npz")
        np.savez(out, N=N, P=P, terms=T, b=b, seed=seed,
                 x_sha256=hashlib.sha256(x.tobytes()).hexdigest(), y=y)
        print("wrote", os.path.relpath(out, REPO))

    src = os.path.join(REFERENCE, "plotting", "raw_data", "cluster_output_error.csv")
    rows = []
    pat = re.compile(r"^(\d+), (\d+), (\d+), (\d+), [\d.]+, ([\d.]+)$")
    seen = set()
    for line in open(src):
        m = pat.match(line.strip())
        if not m:
            continue
        N, P, b, T, err = int(m[1]), int(m[2]), int(m[3]), int(m[4]), m[5]
        if N > 2 ** 22 or (N, P) in seen:
            continue
        seen.add((N, P))
        rows.append((N, P, b, T, err))
    with open(os.path.join(HERE, "recorded_error_envelope.csv"), "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["N", "P", "b", "T", "err_percent"])
        w.writerows(rows)
    print("wrote", len(rows), "recorded rows")


if __name__ == "__main__":
    main()

"""Regenerates the seeded golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

The reference (Java) cannot run in this environment, so the fixtures hold the
oracle's restatement of the reference's own test cases: the seeded inputs of
GemmReference.seededArray (SplittableRandom stream, every 11th element 0), the
GemmReference.gemm output for the GemmParityTest grid, the OptimizedBLAS3
packed-path output (fma chain) and the double-double reference with the
componentwise FP64 bound.  The tests check that the oracle still reproduces
these files bit for bit, and the GPU tests compare against them.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# GemmParityTest.java:25-35: shapes and the alpha/beta grid
SHAPES = [(4, 4, 4), (12, 12, 12), (64, 64, 64), (128, 64, 16), (16, 64, 128), (96, 96, 1), (128, 3, 128)]
GRID = [0.0, 1.0, -0.5, 2.5]


FULL_ARRAYS = {(4, 4, 4), (12, 12, 12), (96, 96, 1)}


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def parity_grid():
    """Full arrays for the small shapes, SHA-256 digests of every output."""
    out, digests = {}, {}
    seed = 20260603
    for (m, k, n) in SHAPES:
        a = O.seeded_matrix(m, k, seed + 11)
        b = O.seeded_matrix(k, n, seed + 29)
        c = O.seeded_matrix(m, n, seed + 47)
        key = f"{m}x{k}x{n}"
        full = (m, k, n) in FULL_ARRAYS
        digests[f"{key}/inputs"] = [digest(a), digest(b), digest(c), seed]
        if full:
            out[f"{key}/a"], out[f"{key}/b"], out[f"{key}/c"] = a, b, c
        for alpha in GRID:
            for beta in GRID:
                tag = f"{key}/{alpha:+.1f}/{beta:+.1f}"
                ref = O.gemm_reference(a, b, c, alpha, beta, threads=1)
                fma = O.gemm_fmachain(a, b, c, alpha, beta, threads=1)
                dd, bound = O.gemm_dd(a, b, c, alpha, beta, threads=1)
                digests[tag] = {"reference": digest(ref), "fmachain": digest(fma), "dd": digest(dd),
                                "bound": digest(bound)}
                if full:
                    out[f"{tag}/reference"], out[f"{tag}/fmachain"] = ref, fma
                    out[f"{tag}/dd"], out[f"{tag}/bound"] = dd, bound
        seed += 101
    return out, digests


def seeded_streams():
    # the first values of the seeded streams used by the reference's tests
    out = {}
    for seed in (20260603 + 11, 4101 + 1, 7001, 8001, 20260604):
        out[f"seeded/{seed}"] = O.seeded_array(64, seed)
    return out


def main():
    fx, digests = parity_grid()
    fx.update(seeded_streams())
    np.savez_compressed(os.path.join(HERE, "parity_grid.npz"), **fx)
    with open(os.path.join(HERE, "parity_grid_digests.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    print(f"wrote {len(fx)} arrays and {len(digests)} digests")


if __name__ == "__main__":
    main()

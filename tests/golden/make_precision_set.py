"""Generates tests/golden/precision_n24_m4.json: the post-selected
near-degenerate instances of the n = 24, m = 4 precision study.

Draw d is the seeded SK instance sk_instances(24, 1, 24 * 1000003 + d)
(J_ij, h_i ~ N(0,1)); it is kept when the two lowest energies, in the
reference's arithmetic (the oracle's restatement of MultiQW.cpp:296-356),
differ by less than 1e-2. Draws are screened in order until 32 are kept.
The file records the kept draws, their gaps and ground-state indices; the
study re-checks every gap on the GPU before using an instance.

    python tests/golden/make_precision_set.py [--workers 8]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N, COUNT, SEED, GAP_MAX = 24, 32, 24, 1e-2


def draw_raw(d: int) -> np.ndarray:
    rng = np.random.default_rng(SEED * 1_000_003 + d)
    return rng.standard_normal(N * (N + 1) // 2)


def gap_of(d: int):
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    E, _, info = O.energies_ref(N, draw_raw(d))
    i = int(E.argmin())
    e0 = E[i]
    E[i] = np.inf
    return d, float(E.min() - e0), int(info.e_loc), float(e0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=os.cpu_count())
    a = ap.parse_args()
    kept, d0, chunk = [], 0, 8 * a.workers
    with mp.get_context("spawn").Pool(a.workers) as pool:
        while len(kept) < COUNT:
            for d, gap, eloc, e0 in pool.map(gap_of, range(d0, d0 + chunk)):
                if gap < GAP_MAX and len(kept) < COUNT:
                    kept.append({"draw": d, "gap": gap, "e_loc": eloc, "e0": e0})
            d0 += chunk
            print(f"screened {d0}, kept {len(kept)}", flush=True)
    last = kept[-1]["draw"] + 1
    out = {"n": N, "m": 4, "gap_max": GAP_MAX, "seed_rule": "numpy default_rng(24*1000003+draw).standard_normal(n(n+1)/2)",
           "screened": last, "instances": kept}
    with open(os.path.join(HERE, "precision_n24_m4.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

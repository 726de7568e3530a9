"""Generate the golden fixtures in tests/golden/ (run in a tree that has the
reference source, so that oracle/_ref can be built).

    python tests/golden/make_golden.py

Fixtures written:
  ref_normcdfinv.json   the reference's own my_normcdfinvf (MultiQW.cpp:83-86)
                        at p = 1/2^n and 1/(e 2^n), n = 1..30, as float bits.
  ref_clenshaw_step.json
                        outputs of the reference's own Clenshaw_step
                        (MultiQW.cpp:88-173, AVX-512 build) on seeded inputs
                        for n in {4, 8, 12, 17}: SHA-256 of the float32 output
                        and its first 8 values.
  oracle_config1.json   the oracle's per-instance ground-state probability
                        (FP32 reference arithmetic and FP64) for the plain
                        method at n=10, m=2 on 200 seeded SK instances
                        (J, h ~ N(0,1), numpy default_rng(0)), plus E_loc,
                        total_t and summed degree — a regression pin of the
                        oracle and the target of the GPU parity tests.
  oracle_small.json     the same for a spread of (n, m, seed) cases,
                        including m = 1 (cumulative single stage).
Seeded inputs are regenerated from numpy.random.default_rng(seed); only
outputs are stored.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def step_inputs(n: int, seed: int):
    rng = np.random.default_rng(seed)
    N = 1 << n
    b1 = rng.standard_normal(N).astype(np.float32)
    b2 = rng.standard_normal(N).astype(np.float32)
    hp = (rng.standard_normal(N) * 5).astype(np.float32)
    psi = rng.standard_normal(N).astype(np.float32)
    return b1, b2, hp, psi


STEP_CASES = [
    # n, seed, scale, gamma, coef
    (4, 1, 37.1, 2.41, 0.3),
    (8, 2, 21.1, 0.80, -0.7),
    (12, 3, 50.0, 1.7, 0.0),
    (17, 4, 80.0, 2.2, 0.05),
]

SMALL_CASES = [
    # n, m, count, seed, samples
    (4, 1, 3, 11, 100),
    (5, 2, 3, 12, 100),
    (7, 3, 3, 13, 100),
    (8, 1, 2, 14, 100),
    (10, 4, 2, 15, 20),
    (12, 2, 2, 16, 10),
    (14, 3, 1, 17, 4),
]


def main() -> None:
    O.build()
    R = O.ref_lib()
    if R is None:
        raise SystemExit("the partial reference build (oracle/_ref) is required")
    e = np.float32(2.718281828459045)
    ninv = []
    for n in range(1, 31):
        N = np.float32(1 << n)
        for p in (np.float32(1) / N, np.float32(1) / (e * N)):
            v = np.float32(R.ref_my_normcdfinvf(float(p)))
            ninv.append({"n": n, "p_bits": int(np.float32(p).view(np.uint32)),
                         "value_bits": int(v.view(np.uint32)), "value": float(v)})
    with open(os.path.join(HERE, "ref_normcdfinv.json"), "w") as f:
        json.dump({"source": "reference MultiQW.cpp:83-86 (my_normcdfinvf), partial build",
                   "values": ninv}, f, indent=1)

    steps = []
    for n, seed, scale, gamma, coef in STEP_CASES:
        b1, b2, hp, psi = step_inputs(n, seed)
        out = b2.copy()
        O.ref_clenshaw_step(b1, out, hp, psi, n, scale, gamma, coef)
        steps.append({"n": n, "seed": seed, "scale": scale, "gamma": gamma, "coef": coef,
                      "sha256": hashlib.sha256(out.tobytes()).hexdigest(),
                      "head": [float(x) for x in out[:8]]})
    with open(os.path.join(HERE, "ref_clenshaw_step.json"), "w") as f:
        json.dump({"source": "reference MultiQW.cpp:88-173 (Clenshaw_step), partial build",
                   "inputs": "numpy default_rng(seed): b1, b2, 5*hp, psi standard normal, float32",
                   "cases": steps}, f, indent=1)

    n, m, count, seed = 10, 2, 200, 0
    raw = O.sk_instances(n, count, seed)
    r32 = O.run_problems(n, m, raw, count, 100, "f32", use_ref_step=True)
    r64 = O.run_problems(n, m, raw, count, 100, "f64")
    with open(os.path.join(HERE, "oracle_config1.json"), "w") as f:
        json.dump({"n": n, "m": m, "count": count, "seed": seed, "samples": 100,
                   "generator": "numpy default_rng(seed).standard_normal(n(n+1)/2) per instance",
                   "p_f32": r32["p"].tolist(), "p_f64": r64["p"].tolist(),
                   "e_loc": r32["e_loc"].tolist(), "total_t": r32["total_t"].tolist(),
                   "terms": r32["terms"].tolist()}, f)

    small = []
    for n, m, count, seed, samples in SMALL_CASES:
        raw = O.sk_instances(n, count, seed)
        r32 = O.run_problems(n, m, raw, count, samples, "f32", use_ref_step=n >= 4)
        r64 = O.run_problems(n, m, raw, count, samples, "f64")
        small.append({"n": n, "m": m, "count": count, "seed": seed, "samples": samples,
                      "p_f32": r32["p"].tolist(), "p_f64": r64["p"].tolist(),
                      "e_loc": r32["e_loc"].tolist(), "total_t": r32["total_t"].tolist(),
                      "terms": r32["terms"].tolist()})
    with open(os.path.join(HERE, "oracle_small.json"), "w") as f:
        json.dump({"cases": small}, f, indent=1)
    print("golden fixtures written to", HERE)
    _ = math


if __name__ == "__main__":
    main()

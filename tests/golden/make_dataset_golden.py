"""Generate the dataset fixtures in tests/golden/ from the reference's own
instance files (run in a tree that has the reference checkout, so that the
files can be read and oracle/_ref can be built).

    python tests/golden/make_dataset_golden.py              # everything
    python tests/golden/make_dataset_golden.py --bench-only # bench fixtures only

The reference ships its instances as raw float64 files in the layout the
command reads (data/AdamData/description.txt:14-17: per instance n(n-1)/2
couplings of the lower triangle, then n fields). Its README's example run is
`./MultiQW 10 2 data/AdamData/SK_10n` (README.md:35-36); the TimData files
are post-selected small-gap instances. Fixtures written (instances copied
byte for byte from the start of each file, so the drop-in command can read
them unchanged):

  adam_sk10n_first200.bin   the first 200 instances of data/AdamData/SK_10n
  tim_sk10n_first100.bin    the first 100 instances of data/TimData/SK_10n
  tim_sk12n_first100.bin    the first 100 instances of data/TimData/SK_12n
  dataset_expect.json       per file and (n, m): per-instance ground-state
                            probability of a reference-driven run — the
                            reference's own FP32 Clenshaw_step (MultiQW.cpp:
                            88-173) and its own my_normcdfinvf
                            (MultiQW.cpp:83-86) in the schedule, both from the
                            partial build in oracle/_ref — with its total_t;
                            the same with this project's inverse normal (the
                            one the CUDA path uses) in FP32 and in FP64; E_loc,
                            the summed Chebyshev degree and the gap between
                            the two lowest energies (reference arithmetic),
                            plus the SHA-256 of each fixture file.
  adam_sk20n_first16.bin    the first 16 instances of data/AdamData/SK_20n,
                            the instances of bench.py's adam_n20_m4 workload
                            (bytes and SHA-256 only, under "bench_files").
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# Byte copies for the bench's workload on the reference's own instances
# (n = 20: no oracle runs, only the bytes and their SHA-256):
# (fixture, source file within the reference checkout, n, instances)
BENCH_FIXTURES = [
    ("adam_sk20n_first16.bin", "data/AdamData/SK_20n", 20, 16),
]

# (fixture, source file within the reference checkout, n, instances, m values)
CASES = [
    ("adam_sk10n_first200.bin", "data/AdamData/SK_10n", 10, 200, [2]),
    ("tim_sk10n_first100.bin", "data/TimData/SK_10n", 10, 100, [2, 3]),
    ("tim_sk12n_first100.bin", "data/TimData/SK_12n", 12, 100, [2, 4]),
]


def two_lowest_gap(n: int, raw: np.ndarray) -> float:
    E, _, _ = O.energies_ref(n, raw)
    i = int(E.argmin())
    e0 = E[i]
    E[i] = np.inf
    return float(E.min() - e0)


def write_bench_fixtures(ref: str) -> dict:
    out = {}
    for fixture, src, n, count in BENCH_FIXTURES:
        per = O.params_per_instance(n)
        with open(os.path.join(ref, src), "rb") as f:
            data = f.read(8 * per * count)
        assert len(data) == 8 * per * count, (src, len(data))
        with open(os.path.join(HERE, fixture), "wb") as f:
            f.write(data)
        out[fixture] = {"source": src, "n": n, "instances": count,
                        "sha256": hashlib.sha256(data).hexdigest()}
    return out


def main() -> None:
    ref = O.reference_dir()
    if ref is None:
        raise SystemExit("the reference checkout is required (MQW_REFERENCE_DIR)")
    if "--bench-only" in sys.argv:  # refresh only the bench fixtures' bytes and hashes
        path = os.path.join(HERE, "dataset_expect.json")
        with open(path) as f:
            out = json.load(f)
        out["bench_files"] = write_bench_fixtures(ref)
        with open(path, "w") as f:
            json.dump(out, f, indent=0)
            f.write("\n")
        return
    O.build()
    if O.ref_lib() is None:
        raise SystemExit("the partial reference build (oracle/_ref) is required")
    out = {"generator": "tests/golden/make_dataset_golden.py", "samples": O.SAMPLES, "files": {}}
    for fixture, src, n, count, m_values in CASES:
        per = O.params_per_instance(n)
        with open(os.path.join(ref, src), "rb") as f:
            data = f.read(8 * per * count)
        assert len(data) == 8 * per * count, (src, len(data))
        with open(os.path.join(HERE, fixture), "wb") as f:
            f.write(data)
        raw = np.frombuffer(data, dtype="<f8").reshape(count, per)
        entry = {"source": src, "n": n, "instances": count,
                 "sha256": hashlib.sha256(data).hexdigest(),
                 "gaps": [two_lowest_gap(n, raw[i]) for i in range(count)], "runs": {}}
        for m in m_values:
            O.use_reference_inv_norm(True)
            rr = O.run_problems(n, m, raw, count, O.SAMPLES, "f32", use_ref_step=True)
            O.use_reference_inv_norm(False)
            r32 = O.run_problems(n, m, raw, count, O.SAMPLES, "f32", use_ref_step=True)
            r64 = O.run_problems(n, m, raw, count, O.SAMPLES, "f64")
            assert np.array_equal(rr["e_loc"], r64["e_loc"])
            entry["runs"][str(m)] = {
                "p_reference_driven": rr["p"].tolist(),
                "total_t_reference_driven": rr["total_t"].astype(float).tolist(),
                "p_ref_step_f32": r32["p"].tolist(),
                "p_oracle_f64": r64["p"].tolist(),
                "e_loc": r32["e_loc"].astype(int).tolist(),
                "total_t": r32["total_t"].astype(float).tolist(),
                "terms": r32["terms"].astype(int).tolist(),
            }
            print(f"{fixture} m={m}: max |P_refdriven - P_f64| = "
                  f"{np.abs(rr['p'] - r64['p']).max():.2e}, "
                  f"max |P_refdriven - P_own_invnorm| = {np.abs(rr['p'] - r32['p']).max():.2e}")
        out["files"][fixture] = entry
    out["bench_files"] = write_bench_fixtures(ref)
    with open(os.path.join(HERE, "dataset_expect.json"), "w") as f:
        json.dump(out, f, indent=0)
        f.write("\n")


if __name__ == "__main__":
    main()

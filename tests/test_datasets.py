"""Parity on the reference's own instance files.

The fixtures are the first instances of the reference's data/AdamData/SK_10n
(the README's example run, `./MultiQW 10 2 data/AdamData/SK_10n`,
README.md:35-36) and of the small-gap post-selected data/TimData/SK_10n and
SK_12n, copied byte for byte; the expected ground-state probabilities come
from the reference pipeline driven by the reference's own FP32
Clenshaw_step (MultiQW.cpp:88-173, partial build) and from the oracle in
FP64 (tests/golden/make_dataset_golden.py).
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import GOLDEN, load_golden

EXPECT = load_golden("dataset_expect.json")


def _raw(name):
    e = EXPECT["files"][name]
    with open(os.path.join(GOLDEN, name), "rb") as f:
        data = f.read()
    n = e["n"]
    return data, np.frombuffer(data, dtype="<f8").reshape(e["instances"], n * (n + 1) // 2)


@pytest.mark.parametrize("name", sorted(EXPECT["files"]))
def test_fixture_bytes_are_the_recorded_ones(name):
    data, raw = _raw(name)
    assert hashlib.sha256(data).hexdigest() == EXPECT["files"][name]["sha256"]
    assert raw.shape[0] == EXPECT["files"][name]["instances"]


@pytest.mark.parametrize("name", sorted(EXPECT["files"]))
def test_oracle_restatement_matches_reference_step_on_dataset(orc, name):
    """The oracle's own FP32 step (a restatement) gives the same pipeline
    results as the reference's Clenshaw_step on the reference's instances;
    its FP64 path reproduces the recorded FP64 values."""
    e = EXPECT["files"][name]
    _, raw = _raw(name)
    k = 10  # a prefix keeps the CPU suite short
    for m, run in e["runs"].items():
        r32 = orc.run_problems(e["n"], int(m), raw[:k], k, orc.SAMPLES, "f32")
        assert r32["p"].tolist() == run["p_ref_step_f32"][:k]
        assert r32["e_loc"].tolist() == run["e_loc"][:k]
        assert r32["total_t"].astype(float).tolist() == run["total_t"][:k]
        r64 = orc.run_problems(e["n"], int(m), raw[:k], k, orc.SAMPLES, "f64")
        assert np.abs(r64["p"] - np.array(run["p_oracle_f64"][:k])).max() <= 1e-15


@pytest.mark.gpu
def test_readme_example_adam_sk10n_through_the_drop_in(mqw, tmp_path):
    """`MultiQW 10 2 <file>` on the first 200 AdamData SK_10n instances: one
    float32 per instance appended to output_10_2, each within 1e-5 of the
    reference pipeline run with the reference's own step; stdout's total_t
    per instance is the reference schedule's, as printed."""
    name = "adam_sk10n_first200.bin"
    run = EXPECT["files"][name]["runs"]["2"]
    f = tmp_path / "SK_10n"
    f.write_bytes(_raw(name)[0])
    r = subprocess.run([mqw.CLI_PATH, "10", "2", str(f), "0", "200"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "output_10_2", dtype=np.float32)
    assert out.shape == (200,)
    assert np.abs(out.astype(np.float64) - np.array(run["p_ref_step_f32"])).max() <= 1e-5
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 200
    # stdout prints total_t with "%g" (MultiQW.cpp:423 streams a float with
    # six significant digits): the same text as the reference's value
    assert [x.split()[0] for x in lines] == ["%g" % t for t in run["total_t"]]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EXPECT["files"]))
def test_dataset_gpu_fp32_and_fp64_against_reference(ctx, name):
    """Every instance of every fixture and m: the GPU FP32 path within 1e-5
    of the reference pipeline (reference step) and of the FP64 oracle, the
    GPU FP64 path within 1e-12 of the FP64 oracle, E_loc identical (the
    TimData instances are post-selected for small gaps)."""
    e = EXPECT["files"][name]
    _, raw = _raw(name)
    n = e["n"]
    for m, run in e["runs"].items():
        g32 = ctx.run_problems(n, int(m), raw, precision="fp32")
        g64 = ctx.run_problems(n, int(m), raw, precision="fp64")
        ref = np.array(run["p_ref_step_f32"])
        f64 = np.array(run["p_oracle_f64"])
        assert g32["e_loc"].tolist() == run["e_loc"]
        assert g64["e_loc"].tolist() == run["e_loc"]
        assert np.abs(g32["p"] - ref).max() <= 1e-5, (name, m)
        assert np.abs(g32["p"] - f64).max() <= 1e-5, (name, m)
        assert np.abs(g64["p"] - f64).max() <= 1e-12, (name, m)
        assert np.allclose(g32["total_t"], run["total_t"], rtol=0, atol=0)

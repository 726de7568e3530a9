"""CPU tests of the product's C ABI: the library loads and exports every
entry point declared in include/mqw.h, and its host-side logic (instance
unpacking, inverse normal, stage schedule, file reading, argument checking)
agrees bit-for-bit with the oracle. No kernels are launched here."""
import ctypes
import os
import subprocess

import numpy as np
import pytest


def test_exports_every_header_symbol(mqw):
    L = mqw.lib()
    names = mqw.exported_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
    assert L.mqw_abi_version() == 3


def test_cli_binary_links(mqw):
    assert os.path.exists(mqw.CLI_PATH)
    out = subprocess.run(["ldd", mqw.CLI_PATH], capture_output=True, text=True).stdout
    assert "libmqw.so" in out and "not found" not in out


def test_cli_too_few_args_returns_minus_one(mqw):
    r = subprocess.run([mqw.CLI_PATH, "10", "2"], capture_output=True)
    assert r.returncode == 255  # `return -1` (MultiQW.cpp:244)


def test_inv_norm_matches_oracle(mqw, orc):
    for n in range(1, 31):
        for p in (1.0 / (1 << n), 1.0 / (2.718281828459045 * (1 << n)), 0.3, 0.5, 0.9):
            pf = float(np.float32(p))
            a = np.float32(mqw.inv_norm_upper(pf))
            b = np.float32(orc.inv_norm_upper(pf))
            assert a.view(np.uint32) == b.view(np.uint32), (n, p)


@pytest.mark.parametrize("n", [1, 2, 3, 10, 20, 30])
def test_load_instance_matches_oracle(mqw, orc, n):
    raw = orc.sk_instances(n, 1, n)[0]
    J1, h1 = mqw.load_instance(n, raw)
    J2, h2 = orc.load_instance(n, raw)
    assert np.array_equal(J1, J2) and np.array_equal(h1, h2)
    assert np.array_equal(J1, J1.T) and not np.diag(J1).any()


@pytest.mark.parametrize("n,m", [(4, 1), (5, 2), (10, 2), (10, 4), (13, 3), (20, 4), (24, 4), (28, 3), (12, 5), (16, 8)])
def test_schedule_bit_exact_vs_oracle(mqw, orc, n, m):
    raw = orc.sk_instances(n, 3, 1000 + n * 7 + m)
    for r in raw:
        g1, s1, t1, tot1 = mqw.schedule(n, m, r)
        g2, s2, t2, tot2 = orc.schedule(n, m, r)
        assert np.array_equal(g1, g2)
        assert np.array_equal(s1, s2)
        assert np.array_equal(t1, t2)
        assert tot1 == tot2


def test_schedule_heuristic_shape(mqw, orc):
    # gamma_i decreases with the stage index; times lie in [short_t, 2 short_t).
    raw = orc.sk_instances(12, 1, 3)[0]
    g, st, t, tot = mqw.schedule(12, 4, raw)
    assert (np.diff(g) < 0).all()
    assert ((t >= st[:, None]) & (t < 2 * st[:, None])).all()
    assert np.isclose(tot, st.sum(), rtol=1e-6)


def test_read_instances_and_short_file(mqw, orc, tmp_path):
    n = 6
    raw = orc.sk_instances(n, 5, 9)
    f = tmp_path / "SK_6n"
    raw.tofile(f)
    got = mqw.read_instances(str(f), n, 1, 3)
    assert np.array_equal(got, raw[1:4])
    with pytest.raises(mqw.MQWError) as e:
        mqw.read_instances(str(f), n, 3, 3)  # runs past the end
    assert e.value.status == 4
    with pytest.raises(mqw.MQWError) as e:
        mqw.read_instances(str(tmp_path / "missing"), n, 0, 1)
    assert e.value.status == 4


def test_invalid_arguments_return_status(mqw):
    L = mqw.lib()
    raw = np.zeros(3, np.float64)
    g = np.zeros(4, np.float32)
    t = np.zeros(400, np.float32)
    P = ctypes.POINTER
    assert L.mqw_schedule(0, 2, raw.ctypes.data_as(P(ctypes.c_double)), g.ctypes.data_as(P(ctypes.c_float)),
                          None, t.ctypes.data_as(P(ctypes.c_float)), None) == 1
    assert L.mqw_schedule(2, 0, raw.ctypes.data_as(P(ctypes.c_double)), g.ctypes.data_as(P(ctypes.c_float)),
                          None, t.ctypes.data_as(P(ctypes.c_float)), None) == 1
    assert L.mqw_load_instance(31, raw.ctypes.data_as(P(ctypes.c_double)), None, None) == 1
    assert L.mqw_create(None, 0) == 1


def test_no_gpu_context_fails_loudly(mqw):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mqw.MQWError) as e:
        mqw.Context(0)
    assert e.value.status == 7


def test_sk_generator_matches_oracle(mqw, orc):
    assert np.array_equal(mqw.sk_instances(9, 4, 2), orc.sk_instances(9, 4, 2))


def test_cheb_host_build_bit_exact_vs_oracle(mqw, orc):
    s = np.array([1e-9, 2e-7, 1e-3, 0.37, 1.0, 3.3, 12.3, 37.0, 99.9, 150.0, 420.0, 901.5, 2500.0])
    coeffs, K = mqw.cheb_coeffs_host(s)
    for i, sv in enumerate(s):
        ref = orc.cheb_coeffs(sv).astype(np.float32)
        assert K[i] == len(ref), sv
        assert np.array_equal(coeffs[i].view(np.uint32), ref.view(np.uint32)), sv


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the header's sizes and field
    offsets (compiled with the system C compiler)."""
    import ctypes
    import shutil
    import subprocess
    import multistageqw_b200 as M
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    structs = {"mqw_options": M.Options, "mqw_run_stats": M.RunStats,
               "mqw_diag_info": M.DiagInfo, "mqw_grid_shape": M.GridShape,
               "mqw_tier_peaks": M.TierPeaks}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mqw.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(out[name]) == ctypes.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(out[f"{name}.{field}"]) == getattr(cls, field).offset, (name, field)


def _ranges_like_reference(problems, threads):
    """run.sh:27-33's split, restated: contiguous ranges, the first
    problems % threads of them one longer."""
    base, extra = divmod(problems, threads)
    out = []
    for t in range(threads):
        start = t * base + min(t, extra)
        count = base + (1 if t < extra else 0)
        if count:
            out.append((start, count))
    return out


@pytest.mark.parametrize("threads,problems", [(1, 2000), (3, 10), (7, 2000), (16, 30), (5, 3)])
def test_run_driver_splits_like_the_reference(mqw, tmp_path, threads, problems):
    """The run.sh-compatible driver issues exactly the reference script's
    ranges for every (n, m) of its lists, devices dealt round-robin."""
    script = os.path.join(os.path.dirname(mqw.LIB_PATH), "..", "run.sh")
    (tmp_path / "x_6n").write_bytes(b"")
    env = dict(os.environ, MQW_DRY_RUN="1", MQW_N_VALUES="6", MQW_M_VALUES="1 2",
               MQW_PROBLEMS=str(problems), MQW_DEVICES="0 1")
    r = subprocess.run(["bash", script, str(threads), "x"], cwd=tmp_path, env=env,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    want = []
    for m in (1, 2):
        for k, (s, c) in enumerate(_ranges_like_reference(problems, threads)):
            want.append((f"MQW_DEVICE={k % 2}", "6", str(m), str(s), str(c)))
    got = []
    for ln in lines:
        f = ln.split()
        got.append((f[0], f[2], f[3], f[5], f[6]))
    # ranges with no problems are not launched (the reference starts them anyway)
    assert got == [w for w in want]

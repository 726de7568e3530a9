"""Multi-GPU runs are replicas: each rank runs its own seeded batch with no
data exchange, and the job time is the maximum over ranks. This checks that
logic with two gloo ranks on the CPU (no GPU involved)."""
import os
import socket

import numpy as np
import torch.multiprocessing as tmp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import bench
    import multistageqw_b200 as M
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    t = 10.0 + 5.0 * rank  # this rank's step time
    worst = bench.max_over_ranks(t, world, dist, "cpu")
    seed = bench.replica_seed(20, rank)
    batch = M.sk_instances(12, 2, seed)
    out[rank] = (worst, seed, float(batch.sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    mgr = tmp.Manager()
    out = mgr.dict()
    tmp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 15.0          # max over ranks
    assert out[0][1] != out[1][1]                  # distinct seeds
    assert out[0][2] != out[1][2]                  # distinct batches


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_seed(20, 0) == 20
    assert np.isfinite(bench.replica_seed(20, 7))


def test_clock_summary_flags_throttling():
    """The clocks record of the bench line: median SM clock over the samples
    under load, the maximum clock, and every throttle reason seen active."""
    import bench
    lines = "\n".join([
        "1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "1950, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
        "1845, 1965, 1001.0, 0x4, Not Active, Not Active, Not Active, Active",
        "345, 1965, 90.0, 0x0, Not Active, Not Active, Not Active, Not Active",  # idle
        "garbage line",
    ])
    c = bench.ClockSampler.summarize(lines)
    assert c["sm_mhz"] == 1950.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"] and c["samples"] == 4
    hot = bench.ClockSampler.summarize(
        "1500, 1965, 900, 0x40, Not Active, Active, Not Active, Not Active")
    assert hot["reasons"] == ["hw_thermal_slowdown"]
    assert bench.ClockSampler.summarize("") is None


def test_peaks_reads_nested_measured_file(tmp_path, monkeypatch):
    """The roofline denominator: `hbm_gbs` wherever the measured-peaks file
    keeps it, else the fallback figure."""
    import json

    import bench
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (bench.PEAKS_FALLBACK, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"b200": {"hbm_gbs": 6544.7}}))
    assert bench.peaks() == ({"hbm_gbs": 6544.7}, "measured")
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert bench.peaks()[1] == "fallback"

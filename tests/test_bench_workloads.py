"""The benchmark workloads have the shapes of the benchmark configurations
(CPU): visibility-sample counts, grids, planes and oversampling, and the
bench's defaults keep the timing contract (warm-up of at least 3 steps)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _samples(w):
    nbl = w["nant"] * (w["nant"] - 1) // 2
    return nbl * int(round(w["duration"] / w["dt"])) * w["nchan"] * w["npol"]


def test_workload_shapes():
    import bench
    w0, w1, w2 = bench.workload(0), bench.workload(1), bench.workload(2)
    assert _samples(w0) == 1_814_400 and (w0["nx"], w0["nwplanes"], w0["oversample"]) == (2048, 65, 4)
    assert _samples(w1) == 1_393_459_200
    assert (w1["nx"], w1["npol"], w1["nwstacks"], w1["nwplanes"], w1["oversample"]) == (4096, 4, 17, 33, 8)
    assert _samples(w2) == 87_091_200
    assert (w2["nbeam"], w2["pitch"], w2["dish"], w2["blockage"]) == (36, 0.9, 12.0, 1.0)
    assert (w2["nx"], w2["npol"], w2["nchan"], w2["nwplanes"], w2["oversample"]) == (2048, 2, 48, 33, 4)
    assert (w2["f0"], w2["f1"]) == (700e6, 1000e6) and (w1["f0"], w1["f1"]) == (700e6, 1000e6)


def test_batched_instances():
    import bench
    ws = bench.batch_instances(64)
    assert len(ws) == 64
    assert {w["nx"] for w in ws} <= {512, 1024, 2048, 4096}
    assert all(1 <= w["nchan"] <= 32 for w in ws)
    n = [_samples(w) for w in ws]
    assert 5e4 <= min(n) and max(n) <= 6e7


def test_defaults_keep_the_timing_contract(monkeypatch):
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1 and a.config == 1 and a.impl == "b200"


def test_kernel_names_and_traffic_rates():
    """The bench line names the kernels a variant runs and scales the grid
    kernel's captured DRAM rates (None for a kernel with no capture)."""
    import bench
    assert bench.kernel_names(193, 6) == ("k_grid_pl", "k_degrid_r")
    assert bench.kernel_names(0, 6) == ("k_grid", "k_degrid_r")
    assert bench.kernel_names(193 | 256, 6) == ("k_grid_pl", "k_degrid_t")
    assert bench.kernel_names(1, 20) == ("k_grid", "k_degrid_t")
    info = {"tile": 32, "nvalid": 1000, "nitems": 10}
    per_sample, per_cell = bench.TRAFFIC_RATES["k_grid_pl"]
    assert bench.kgrid_traffic(info, 6, 4, "k_grid_pl") == int(per_sample * 1000 + per_cell * 10 * 4 * 44 * 44)
    assert bench.kgrid_traffic(info, 6, 4, "k_grid_unknown") is None

"""Host-side logic of bench.py and the scenario sampler (no GPU): the
reference arm's MPI decomposition rule and the ranges of the sampled
batched / serving scenarios."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
from cgfdm import scenarios as S  # noqa: E402


@pytest.mark.parametrize("cores", [1, 8, 16, 64])
def test_decomposition_respects_the_pml_and_core_count(cores):
    p = {"NX": 401, "NY": 401, "NZ": 201, "nPML": 20}
    px, py, pz = bench.pick_decomposition(p, cores)
    assert px * py * pz <= cores
    # every rank holds at least max(nPML, 8) cells per axis (init_grid.cpp:109-117)
    for n, k in ((401, px), (401, py), (201, pz)):
        assert n // k >= 20


def test_decomposition_uses_all_cores_when_it_can():
    p = {"NX": 401, "NY": 401, "NZ": 201, "nPML": 20}
    px, py, pz = bench.pick_decomposition(p, 16)
    assert px * py * pz == 16


def test_sampled_scenarios_follow_the_ranges():
    for seed in range(6):
        w = S.sample_scenario(seed, nsteps=10)
        p = w["params"]
        assert 121 <= p["NX"] <= 401 and 121 <= p["NY"] <= 401 and 101 <= p["NZ"] <= 201
        assert p["useMultiSource"] == 1 and len(w["stations"]) == 25
        assert np.asarray(w["terrain"]).max() <= 2000.0 + 1e-3
    w = S.sample_scenario(1, points=2e6, nsteps=10)
    n = w["params"]["NX"] * w["params"]["NY"] * w["params"]["NZ"]
    assert 0.8e6 < n < 3e6


def test_decomposition_prefers_the_least_halo():
    # 16 ranks on the 1201 x 1201 x 401 grid: a 4 x 4 column split holds
    # fewer padded points than z slabs
    p = {"NX": 1201, "NY": 1201, "NZ": 401, "nPML": 12}
    assert bench.pick_decomposition(p, 16) == (4, 4, 1)


def test_reference_memory_estimate_counts_every_rank_halo():
    p = {"NX": 100, "NY": 60, "NZ": 40, "nPML": 10}
    one = bench.reference_bytes(p, (1, 1, 1))
    assert one == 4 * 49 * 106 * 66 * 46 + 4 * 36 * (2 * 10 * 60 * 40 + 2 * 100 * 10 * 40 +
                                                      100 * 60 * 10)
    # splitting x in two adds one 6-cell halo
    assert bench.reference_bytes(p, (2, 1, 1)) - one == 4 * 49 * 6 * 66 * 46


def test_cpu_baseline_sample_of_large_grids():
    assert bench.cpu_sample_workload("c3-1201") == "c3-401"
    assert bench.cpu_sample_workload("c3-401") == "c3-401"
    assert bench.cpu_sample_workload("c2") == "c2"


def test_traffic_figure_comes_only_from_a_capture_of_the_same_workload():
    w = S.c2_workload(10)
    t = bench.measured_traffic(w["name"], "stage_stream_kernel", "fp32", 4.0e9, 4)
    assert t is not None and 1.0 < t / 1e9 < 2.0
    # another kernel, precision or workload has no figure
    assert bench.measured_traffic(w["name"], "stage_pair_kernel", "fp32", 4.0e9, 4) is None
    assert bench.measured_traffic(w["name"], "stage_stream_kernel", "bf16", 4.0e9, 4) is None
    assert bench.measured_traffic("c3-perftest-401x401x401", "stage_stream_kernel", "fp32",
                                  4.0e9, 4) is None


def test_setup_slots_follow_host_memory():
    p = {"NX": 1201, "NY": 1201, "NZ": 401}
    cjm = 13 * 1207 * 1207 * 407 * 4
    assert bench.setup_slots(p, 8, None) == 8              # unknown: no limit
    assert bench.setup_slots(p, 8, 100 * cjm) == 8         # room for all
    assert bench.setup_slots(p, 8, 5 * cjm) == 2           # two at a time
    assert bench.setup_slots(p, 8, 1 * cjm) == 1           # one at a time, never zero


def test_setup_turns_of_one_slot_serialise(tmp_path, monkeypatch):
    import multiprocessing as mp
    import time

    monkeypatch.setattr(bench.tempfile, "gettempdir", lambda: str(tmp_path))
    monkeypatch.setenv("MASTER_PORT", "4711")
    log = tmp_path / "log"
    ctx = mp.get_context("fork")

    def hold(local):
        with bench.SetupTurn(local, 1):
            with open(log, "a") as f:
                f.write("in %d\n" % local)
            time.sleep(0.3)
            with open(log, "a") as f:
                f.write("out %d\n" % local)

    ps = [ctx.Process(target=hold, args=(r,)) for r in range(2)]
    for q in ps:
        q.start()
    for q in ps:
        q.join(30)
        assert q.exitcode == 0
    lines = log.read_text().split()
    # the two holds do not interleave: in a, out a, in b, out b
    assert lines[0::2] == ["in", "out", "in", "out"]
    assert lines[1] == lines[3] and lines[5] == lines[7] and lines[1] != lines[5]

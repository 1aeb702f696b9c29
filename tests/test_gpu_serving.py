"""The request loop (cgfdm_server_*): continuous batching.

Requests of uneven sizes and two precisions arrive while others are on the
GPU; the server admits them as memory frees up and advances them together.
Each request's seismograms and PGV map must equal a lone run of the same
simulation bit for bit (the batched kernel is the kernel a lone handle runs),
under a budget that forces queuing too.  A CPU test checks that creating a
server without a device fails cleanly."""
import threading
import time

import numpy as np
import pytest

from test_gpu_batch import SHAPES, _scaled, _synthetic

cgfdm = pytest.importorskip("cgfdm")

NT = 30


def _request(sc, precision):
    nx, ny, nz, npml = sc["dims"]
    d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, NT, precision, cgfdm.KERNEL_AUTO)
    return d, dict(point=sc["src"], rickerfc=4.0, stations=sc["sta"])


def _alone(sc, precision):
    d, kw = _request(sc, precision)
    with cgfdm.Simulation(d) as s:
        s.set_tile_rows(16)
        s.set_model(sc["cjm"], sc["rdz"])
        s.set_point_source(*kw["point"], kw["rickerfc"])
        s.set_stations(kw["stations"])
        s.run(NT)
        return s.stations(), s.pgv()


def test_server_needs_a_device_on_cpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(cgfdm.CgfdmError):
        cgfdm.Server()


def _mix():
    out = []
    for q, dims in enumerate(SHAPES + SHAPES[:3]):
        prec = cgfdm.FP16 if q % 3 == 2 else cgfdm.FP32
        sc = _synthetic(*dims, seed=50 + q)
        if prec != cgfdm.FP32:
            sc = _scaled(sc)
        out.append((sc, prec))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("budget_requests", [0, 2])
def test_server_results_equal_lone_runs(gpu_available, budget_requests):
    mix = _mix()
    budget = 0
    if budget_requests:  # room for about two of the largest requests at a time
        budget = budget_requests * max(cgfdm.device_bytes(_request(sc, p)[0]) for sc, p in mix)
    with cgfdm.Server(hbm_budget_bytes=budget, chunk=7, graph=True) as srv:
        ids = {}

        def producer():  # staggered arrivals while earlier requests run
            for q, (sc, prec) in enumerate(mix):
                d, kw = _request(sc, prec)
                ids[q] = srv.submit(d, sc["cjm"], sc["rdz"], **kw)
                time.sleep(0.01)

        t = threading.Thread(target=producer)
        t.start()
        t.join()
        # streaming: rows of the first request become visible chunk by chunk
        nsta = len(mix[0][0]["sta"])
        buf = np.zeros((nsta, NT, 9), np.float32)
        seen = srv.read_rows(ids[0], buf)
        assert 0 <= seen <= NT
        results = {q: srv.wait(ids[q]) for q in ids}
        st = srv.stats()
    assert st["completed"] == len(mix)
    if budget:
        assert st["peak_bytes"] <= budget
    assert st["first_p50_ms"] <= st["done_p50_ms"]
    for q, (sc, prec) in enumerate(mix):
        wave, pgv, lat = results[q]
        ref_w, ref_p = _alone(sc, prec)
        np.testing.assert_array_equal(wave, ref_w)
        np.testing.assert_array_equal(pgv, ref_p)
        assert lat[0] <= lat[1]


@pytest.mark.gpu
def test_server_rejects_request_above_budget(gpu_available):
    sc, prec = _mix()[0]
    d, kw = _request(sc, prec)
    with cgfdm.Server(hbm_budget_bytes=cgfdm.device_bytes(d) - 1) as srv:
        with pytest.raises(cgfdm.CgfdmError) as e:
            srv.submit(d, sc["cjm"], sc["rdz"], **kw)
        assert e.value.code == 301


@pytest.mark.gpu
def test_server_cancel_queued_and_running(gpu_available):
    """Cancelling a queued request and a running one: both end as cancelled
    (their memory released), the others still equal their lone runs."""
    mix = _mix()[:4]
    budget = max(cgfdm.device_bytes(_request(sc, p)[0]) for sc, p in mix)  # one at a time
    with cgfdm.Server(hbm_budget_bytes=budget, chunk=3, graph=True) as srv:
        ids = []
        for q, (sc, prec) in enumerate(mix):
            d, kw = _request(sc, prec)
            if q == 0:
                d.nt = 3000  # long enough to be cancelled while it runs
            ids.append(srv.submit(d, sc["cjm"], sc["rdz"], **kw))
        srv.cancel(ids[3])  # still queued behind the others
        deadline = time.time() + 60
        while srv.poll(ids[0])[1] == 0 and time.time() < deadline:
            time.sleep(0.005)
        srv.cancel(ids[0])  # running (some rows streamed back already)
        for q in (0, 3):
            with pytest.raises(cgfdm.CgfdmError) as e:
                srv.wait(ids[q])
            assert e.value.code == 305
        for q in (1, 2):
            wave, pgv, _ = srv.wait(ids[q])
            ref_w, ref_p = _alone(*mix[q])
            np.testing.assert_array_equal(wave, ref_w)
        assert srv.stats()["completed"] == 2

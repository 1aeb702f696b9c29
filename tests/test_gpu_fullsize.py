"""The fast path at the full benchmark size: the 1201 x 1201 x 401
PerformanceTest grid (nPML 12, random terrain, layered medium, 80 x 40
finite fault) in FP32, 24 steps, against the exact-order kernel, which
reproduces the reference's FP32 CPU build bit for bit (tested on the
reference-built fixtures).  The whole wavefield after the last step agrees
within relative L2 1e-5 (the fast path's bar), checked field by field, and
the fault's waves are in it (non-zero).  This is the grid and the kernel
configuration (autotuned tile form, work-item depth and free-surface
kernel) that bench.py's default line measures."""
import os
import shutil
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")
from cgfdm import scenarios as S  # noqa: E402

STEPS = 24


def _run(st, kernel):
    d = st["desc"]
    desc = cgfdm.make_desc(d.nx, d.ny, d.nz, d.npml, d.dh, d.dt, STEPS, cgfdm.FP32, kernel)
    with cgfdm.Simulation(desc) as sim:
        sim.set_model(st["cjm"], st["rdz"])
        if st["point"] is not None:
            sim.set_point_source(*st["point"], st["rickerfc"])
        if st["src_index"].size:
            sim.set_fault_source(st["src_index"], st["moment_rate"], st["src_nt"], st["src_dt"],
                                 scaled=True)
        sim.set_stations(st["stations"])
        sim.run(STEPS)
        return sim.wavefield().reshape(9, -1), sim.tuning3()


def test_fast_path_at_1201_matches_exact_kernel(gpu_available):
    w = S.c3_workload(1201, STEPS + 2)
    d = tempfile.mkdtemp(prefix="cgfdm_full_")
    try:
        S.write_run_dir(d, w["params"], stations=w["stations"],
                                      terrain=w.get("terrain"), layers=w.get("layers"),
                                      source=w.get("source"))
        st = cgfdm.setup_from_directory(d)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    ref, _ = _run(st, cgfdm.KERNEL_EXACT)
    got, tuning = _run(st, cgfdm.KERNEL_AUTO)
    print("\n1201 x 1201 x 401, %d steps, fast path (form, depth, tiled surface) = %s" % (
        STEPS, tuning))
    for f in range(9):
        a, b = got[f].astype(np.float64), ref[f].astype(np.float64)
        nb = np.linalg.norm(b)
        assert nb > 0, f
        err = float(np.linalg.norm(a - b) / nb)
        print("  field %d: rel L2 %.2e" % (f, err))
        assert err <= 1e-5, (f, err)

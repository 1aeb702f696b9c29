"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Test infrastructure.  Needs the reference sources (their root is the first
argument) and builds the reference in place with ``make -C oracle ref``.  It is never run by the tests; its outputs are
committed so that the tests run without the reference.

Fixtures
--------
stage_small.npz
    Setup products of a small curvilinear grid (Gaussian-hill terrain,
    two-layer medium): coordinates, medium, CJM, free-surface matrices, PML
    profiles -- and, for four (irk, FB) cases, one RK stage of the reference's
    hot path applied to the same seeded input state (wavefield, RK buffers and
    PML auxiliaries).
c1_halfspace.npz
    The homogeneous half-space benchmark configuration (161 x 161 x 101,
    1000 steps, double-couple point source, 25 stations), one rank.
run_point_fp16.npz
    The point-source run through the reference's scalar FP16 build (outputs
    only; the inputs are those of run_point.npz).  The FP16 build overflows
    on the finite-fault run (non-finite seismograms), so it has no fixture.
c2_hill.npz, c3_201.npz
    The Gaussian-hill configuration (401 x 401 x 201, nPML 20, 121
    stations, explosive source; 400 steps; 8 x 1 ranks, so that no rank
    boundary cuts the smoothed source) and the 201 x 201 x 401
    PerformanceTest shape (random terrain, layered medium, 80 x 40 finite
    fault; 700 steps, without the per-cell medium perturbation, which the
    reference's medium reader has no counterpart for) through the
    reference's FP32 build on 8 MPI ranks (PZ = 1), the rank files merged:
    the Vx/Vy/Vz seismograms of the stations, the PGV map and the last two
    free-surface snapshots.  A multi-rank reference run equals the
    single-rank one bit for bit (checked on run_fault.npz's inputs).
srtm_run.npz
    The SRTM90 terrain reader (terrain.cpp) on a seeded DEM tile: the
    reference's own interpolated and smoothed terrain and a 120-step run on
    it (see srtm_fixture).
run_point.npz, run_fault.npz
    Complete reference runs (main.cpp -> run.cpp -> propagate.cpp) of small
    configurations: a flat half-space with the smoothed explosive point
    source, and Gaussian-hill terrain with a layered medium and a
    finite-fault (multi-point) source.  Stored: the inputs (params, stations,
    terrain, layers, source file) and the reference outputs (station
    seismograms, PGV map, free-surface snapshots).
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "tests"))
import scenarios  # noqa: E402

REF_SRC = None  # set by main() from the reference root given on the command line
REF_DIR = os.path.join(REPO, "oracle", "_ref")
DFLAGS = ("-DXFAST -DFREE_SURFACE -DPML -DSOLVE_DISPLACEMENT -DTerrain_Smooth "
          "-DDealWithFirstLayer -DLayeredStructureTerrain -DStructureTerrain").split()


def build_dumper():
    exe = os.path.join(REF_DIR, "ref_dump")
    cmd = ["g++", "-O2", "-ffp-contract=off", "-w", *DFLAGS,
           "-I" + os.path.join(REPO, "oracle", "ref_shim"), "-I" + REF_SRC,
           os.path.join(HERE, "ref_dump.cpp"), "-o", exe,
           "-L" + REF_DIR, "-lcgfdm_ref_fp32", "-Wl,-rpath," + REF_DIR, "-lm", "-lrt"]
    subprocess.check_call(cmd)
    return exe


def stage_fixture(exe):
    sc = scenarios.stage_small()
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        scenarios.write_inputs(sc, work)
        subprocess.check_call([exe, "setup"], cwd=work, stdout=subprocess.DEVNULL)
        g = scenarios.grid_dims(sc["params"])
        num = g["num"]
        out = {
            "params_json": np.array(json.dumps(sc["params"])),
            "terrain_input": sc["terrain"],
            "layers": sc["layers"],
            "coord": np.fromfile(os.path.join(work, "setup_coord.bin"), np.float32),
            "medium": np.fromfile(os.path.join(work, "setup_medium.bin"), np.float32),
            "terrain": np.fromfile(os.path.join(work, "setup_terrain.bin"), np.float32),
            "cjm": np.fromfile(os.path.join(work, "setup_cjm.bin"), np.float32),
            "rdz": np.fromfile(os.path.join(work, "setup_rdz.bin"), np.float32),
            "pml": np.fromfile(os.path.join(work, "setup_pml.bin"), np.float32),
        }
        state = scenarios.random_state(sc["params"], seed=20240607)
        for key in ("W", "t", "m", "aux"):
            out["in_" + key] = state[key]
        state["W"].tofile(os.path.join(work, "in_W.bin"))
        state["t"].tofile(os.path.join(work, "in_t.bin"))
        state["m"].tofile(os.path.join(work, "in_m.bin"))
        state["aux"].tofile(os.path.join(work, "in_aux.bin"))
        for n, (irk, fb) in enumerate(scenarios.STAGE_CASES):
            subprocess.check_call([exe, "stage", str(irk), *map(str, fb)], cwd=work,
                                  stdout=subprocess.DEVNULL)
            for key in ("h", "W", "t", "m", "aux"):
                out["case%d_%s" % (n, key)] = np.fromfile(
                    os.path.join(work, "out_%s.bin" % key), np.float32)
        assert out["cjm"].size == 13 * num
        np.savez_compressed(os.path.join(HERE, "stage_small.npz"), **out)
    finally:
        shutil.rmtree(work)


def run_fixture(name, sc, dumper):
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp32")
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        scenarios.write_inputs(sc, work)
        subprocess.check_call([exe], cwd=work, stdout=subprocess.DEVNULL)
        res = scenarios.read_outputs(sc, os.path.join(work, sc["params"]["out"]))
        out = {"params_json": np.array(json.dumps(sc["params"])),
               "stations_json": np.array(json.dumps(sc["stations"]))}
        subprocess.check_call([dumper, "setup"], cwd=work, stdout=subprocess.DEVNULL)
        out["cjm"] = np.fromfile(os.path.join(work, "setup_cjm.bin"), np.float32)
        out["rdz"] = np.fromfile(os.path.join(work, "setup_rdz.bin"), np.float32)
        if sc["params"]["useMultiSource"]:
            hdr = np.fromfile(os.path.join(work, "setup_src_hdr.bin"), np.int32)
            out["src_nt"] = hdr[1]
            out["src_index"] = np.fromfile(os.path.join(work, "setup_src_index.bin"), np.int64)
            out["src_rate"] = np.fromfile(os.path.join(work, "setup_src_rate.bin"), np.float32)
        for k in ("terrain", "layers", "source"):
            if sc.get(k) is not None:
                out[k] = sc[k]
        for k, v in res.items():
            out["out_" + k] = v
        np.savez_compressed(os.path.join(HERE, name), **out)
    finally:
        shutil.rmtree(work)


def run_fixture_fp16(name, sc):
    """The reference's scalar FP16 build (FLOAT = _Float16, Cv/Cs/Crho
    scaling) on the same inputs as an FP32 run fixture: its outputs only."""
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp16")
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        scenarios.write_inputs(sc, work)
        subprocess.check_call([exe], cwd=work, stdout=subprocess.DEVNULL)
        res = scenarios.read_outputs(sc, os.path.join(work, sc["params"]["out"]))
        out = {"params_json": np.array(json.dumps(sc["params"])),
               "stations_json": np.array(json.dumps(sc["stations"]))}
        for k, v in res.items():
            out["out_" + k] = v
        np.savez_compressed(os.path.join(HERE, name), **out)
    finally:
        shutil.rmtree(work)


def c1_fixture():
    """The half-space benchmark configuration (scenarios.c1, 1000 steps)
    through the reference's FP32 build on 8 x 1 MPI ranks (the point source
    of the multi-source path is a single cell, so a rank split changes
    nothing): seismograms, PGV and the free-surface snapshots every 333
    steps (inputs are regenerated from scenarios.c1; the setup products are
    left out, the host setup is tested bit for bit elsewhere)."""
    sc = scenarios.c1()
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp32")
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        p = dict(sc["params"], PX=8, PY=1, PZ=1)
        scenarios.write_inputs(dict(sc, params=p), work)
        env = dict(os.environ, CGFDM_SHIM_NPROC="8", CGFDM_SHIM_TIMEOUT="7200")
        subprocess.check_call([exe], cwd=work, env=env, stdout=subprocess.DEVNULL)
        res = read_outputs_ranks(sc, os.path.join(work, p["out"]), 8, 1)
        out = {"params_json": np.array(json.dumps(sc["params"])),
               "stations_json": np.array(json.dumps(sc["stations"]))}
        for k, v in res.items():
            out["out_" + k] = v
        np.savez_compressed(os.path.join(HERE, "c1_halfspace.npz"), **out)
    finally:
        shutil.rmtree(work)


def _split(n, parts, c):
    """The reference's block decomposition (init_grid.cpp:30-73): the first
    n % parts ranks get one cell more."""
    b, r = divmod(n, parts)
    return (c * (b + 1), b + 1) if c < r else (r * (b + 1) + (c - r) * b, b)


def read_outputs_ranks(sc, outdir, px, py):
    """The rank files of a PX x PY x 1 reference run merged into the
    single-rank arrays of scenarios.read_outputs (station.cpp:382-405,
    PGV.cpp:103-111, data_io.cpp:434-495)."""
    p = sc["params"]
    nt = scenarios.S.nt_of(p)
    NX, NY = p["NX"], p["NY"]
    rows = {}
    for X in range(px):
        for Y in range(py):
            fn = os.path.join(outdir, "station_mpi_%d_%d_0.bin" % (X, Y))
            if not os.path.exists(fn):
                continue
            raw = np.fromfile(fn, np.uint8)
            n = raw.size // (12 + 36 * nt)
            xyz = raw[:12 * n].view(np.int32).reshape(n, 3)
            wave = raw[12 * n:].view(np.float32).reshape(n, nt, 9)
            for q in range(n):
                rows[tuple(int(v) for v in xyz[q])] = wave[q]
    res = {"station_wave": np.stack([rows[tuple(v)] for v in sc["stations"].values()])}
    pgv = np.zeros((NY, NX, 2), np.float32)
    snaps = {}
    for X in range(px):
        x0, nx = _split(NX, px, X)
        for Y in range(py):
            y0, ny = _split(NY, py, Y)
            tag = "%d_%d_0" % (X, Y)
            pgv[y0:y0 + ny, x0:x0 + nx] = np.fromfile(
                os.path.join(outdir, "PGV_Z_mpi_%s.bin" % tag), np.float32).reshape(ny, nx, 2)
            for it in range(0, nt, p["IT_SKIP"]):
                fz = os.path.join(outdir, "FreeSurfVz_%d_Z_mpi_%s.bin" % (it, tag))
                if not os.path.exists(fz):
                    continue
                s = snaps.setdefault(it, np.zeros((3, NY, NX), np.float32))
                for c, ch in enumerate("xyz"):
                    s[c, y0:y0 + ny, x0:x0 + nx] = np.fromfile(os.path.join(
                        outdir, "FreeSurfV%s_%d_Z_mpi_%s.bin" % (ch, it, tag)),
                        np.float32).reshape(ny, nx)
    res["pgv"] = pgv
    its = sorted(snaps)
    res["freesurf"] = np.stack([snaps[k] for k in its])
    res["freesurf_its"] = np.array(its)
    return res


def bench_fixture(name, sc, px, py, keep_snaps=2):
    """A benchmark-configuration run through the reference's FP32 build on
    px * py MPI ranks (shared-memory shim); outputs merged across ranks."""
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp32")
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        p = dict(sc["params"], PX=px, PY=py, PZ=1)
        scenarios.write_inputs(dict(sc, params=p), work)
        env = dict(os.environ, CGFDM_SHIM_NPROC=str(px * py), CGFDM_SHIM_TIMEOUT="7200")
        subprocess.check_call([exe], cwd=work, env=env, stdout=subprocess.DEVNULL)
        res = read_outputs_ranks(sc, os.path.join(work, p["out"]), px, py)
        out = {"params_json": np.array(json.dumps(sc["params"])),
               "stations_json": np.array(json.dumps(sc["stations"])),
               "out_station_v": res["station_wave"][:, :, :3].copy(),
               "out_pgv": res["pgv"],
               "out_freesurf": res["freesurf"][-keep_snaps:],
               "out_freesurf_its": res["freesurf_its"][-keep_snaps:]}
        np.savez_compressed(os.path.join(HERE, name), **out)
    finally:
        shutil.rmtree(work)


FIXTURES = ["stage_small", "run_point", "run_fault", "c1_halfspace", "run_point_fp16",
            "c2_hill", "c3_201", "srtm_run"]


def srtm_fixture():
    """The SRTM90 terrain reader: scenarios.srtm_run through the reference's
    FP32 build with its own terrain.cpp (make -C oracle ref-srtm; the map
    projection is the spherical stand-in of oracle/ref_shim/proj.h), one
    rank: the interior terrain it writes (terrain_mpi_0_0_0.bin) and the run's
    seismograms, PGV and free-surface snapshots.  The 144 MB DEM tile is
    regenerated from its seed by the tests."""
    subprocess.check_call(["make", "-C", os.path.join(REPO, "oracle"), "ref-srtm", "-j8",
                           "REF_ROOT=" + os.path.dirname(REF_SRC)], stdout=subprocess.DEVNULL)
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp32_srtm")
    sc = scenarios.srtm_run()
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        scenarios.write_srtm_inputs(sc, work)
        subprocess.check_call([exe], cwd=work, stdout=subprocess.DEVNULL)
        outdir = os.path.join(work, sc["params"]["out"])
        res = scenarios.read_outputs(sc, outdir)
        p = sc["params"]
        terrain = np.fromfile(os.path.join(outdir, "terrain_mpi_0_0_0.bin"), np.float32)
        out = {"params_json": np.array(json.dumps(p)),
               "stations_json": np.array(json.dumps(sc["stations"])),
               "out_terrain": terrain.reshape(p["NY"], p["NX"])}
        for k, v in res.items():
            out["out_" + k] = v
        np.savez_compressed(os.path.join(HERE, "srtm_run.npz"), **out)
    finally:
        shutil.rmtree(work)


def main():
    """python make_golden.py REF_ROOT [fixture ...]: REF_ROOT is the
    reference project's root (the directory holding src-new-FP32-SVE); with
    no fixture names every fixture is regenerated."""
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py REF_ROOT [%s ...]" % " | ".join(FIXTURES))
    ref_root = sys.argv[1]
    global REF_SRC
    REF_SRC = os.path.join(ref_root, "src-new-FP32-SVE")
    if not os.path.isdir(REF_SRC):
        sys.exit("reference sources not found at %s" % REF_SRC)
    want = sys.argv[2:] or FIXTURES
    subprocess.check_call(["make", "-C", os.path.join(REPO, "oracle"), "ref", "-j8",
                           "REF_ROOT=" + ref_root], stdout=subprocess.DEVNULL)
    exe = build_dumper()
    if "stage_small" in want:
        stage_fixture(exe)
    if "run_point" in want:
        run_fixture("run_point.npz", scenarios.run_point(), exe)
    if "run_fault" in want:
        run_fixture("run_fault.npz", scenarios.run_fault(), exe)
    if "c1_halfspace" in want:
        c1_fixture()
    # (the FP16 build overflows on run_fault: its seismograms are not finite)
    if "run_point_fp16" in want:
        run_fixture_fp16("run_point_fp16.npz", scenarios.run_point())
    if "c2_hill" in want:
        # 8 x 1 ranks: the smoothed point source (7^3 cells around i = 170,
        # j = 200) must not straddle a rank boundary -- the reference adds it
        # only inside the rank that holds its centre, so a split source would
        # lose the part that falls into the halo
        bench_fixture("c2_hill.npz", scenarios.c2_parity(), 8, 1)
    if "c3_201" in want:
        bench_fixture("c3_201.npz", scenarios.c3_201_parity(), 4, 2)
    if "srtm_run" in want:
        srtm_fixture()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

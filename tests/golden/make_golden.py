"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Test infrastructure.  Needs the reference sources (default /root/reference,
override with CGFDM_REF_ROOT) and the in-place reference build made by
``make -C oracle ref``.  It is never run by the tests; its outputs are
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

REF_ROOT = os.environ.get("CGFDM_REF_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src-new-FP32-SVE")
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
    through the reference's FP32 build on one rank: seismograms, PGV and the
    free-surface snapshots (inputs are regenerated from scenarios.c1; the
    setup products are left out, the host setup is tested bit for bit
    elsewhere)."""
    sc = scenarios.c1()
    exe = os.path.join(REF_DIR, "cgfdm_ref_fp32")
    work = tempfile.mkdtemp(prefix="cgfdm_golden_")
    try:
        scenarios.write_inputs(sc, work)
        subprocess.check_call([exe], cwd=work, stdout=subprocess.DEVNULL)
        res = scenarios.read_outputs(sc, os.path.join(work, sc["params"]["out"]))
        out = {"params_json": np.array(json.dumps(sc["params"])),
               "stations_json": np.array(json.dumps(sc["stations"]))}
        for k, v in res.items():
            out["out_" + k] = v
        np.savez_compressed(os.path.join(HERE, "c1_halfspace.npz"), **out)
    finally:
        shutil.rmtree(work)


def main():
    if not os.path.isdir(REF_SRC):
        sys.exit("reference sources not found at %s" % REF_SRC)
    subprocess.check_call(["make", "-C", os.path.join(REPO, "oracle"), "ref", "-j8"],
                          stdout=subprocess.DEVNULL)
    exe = build_dumper()
    stage_fixture(exe)
    run_fixture("run_point.npz", scenarios.run_point(), exe)
    run_fixture("run_fault.npz", scenarios.run_fault(), exe)
    c1_fixture()
    # (the FP16 build overflows on run_fault: its seismograms are not finite)
    run_fixture_fp16("run_point_fp16.npz", scenarios.run_point())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""The TMA-staged streaming kernel (the fast path) against the reference.

It keeps FMA contraction and forms each direction's elastic combination once
(scaled by the PML beta and d afterwards), so it agrees with the reference to
rounding rather than bit for bit.  Tolerances (relative L2 norms):
  * one RK stage: the stage increment W_out - m within 1e-5 of the
    reference's increment, per field, and the PML auxiliaries within 1e-5;
  * complete runs: station seismograms within 1e-5 of the reference's and
    the PGV map within 1e-5.
Both tile heights of the kernel (32 x 16 and 32 x 8) are checked.
"""
import numpy as np
import pytest

import scenarios
from test_gpu_parity import HALO, _desc, _run_sim, _split_aux_out

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="module")
def stage_golden(gpu_available):
    return scenarios.load_golden("stage_small.npz")


@pytest.mark.parametrize("rows", [16, 8])
@pytest.mark.parametrize("case", range(len(scenarios.STAGE_CASES)))
def test_stream_stage_matches_reference(stage_golden, case, rows):
    g = stage_golden
    p = g["params"]
    irk, fb = scenarios.STAGE_CASES[case]
    with cgfdm.Simulation(_desc(p, 1, kernel=cgfdm.KERNEL_STREAM)) as sim:
        sim.set_tile_rows(rows)
        sim.set_model(g["cjm"], g["rdz"])
        sim.set_state(irk, W=g["in_W"], t=g["in_t"], m=g["in_m"], aux=g["in_aux"])
        sim.stage(irk, fb)
        st = sim.get_state()
    base = {0: g["in_W"], 1: g["in_m"], 2: g["in_m"], 3: g["in_t"]}[irk]
    ref = g["case%d_W" % case]
    for v in range(9):
        sl = slice(v * ref.size // 9, (v + 1) * ref.size // 9)
        err = rel_l2(st["W"][sl] - base[sl], ref[sl] - base[sl])
        assert err < 1e-5, (v, err)
    ref_aux = _split_aux_out(g["case%d_aux" % case], p)
    off = 0
    for n in scenarios.slab_points(p):
        n9 = 9 * n
        assert rel_l2(st["aux"][off:off + n9], ref_aux[off:off + n9]) < 1e-5
        off += 3 * n9


@pytest.mark.parametrize("rows", [16, 8])
@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_stream_full_run_matches_reference(gpu_available, name, rows):
    g = scenarios.load_golden(name)
    res = _run_sim(g, kernel=cgfdm.KERNEL_STREAM, tile_rows=rows)
    for v in range(9):
        err = rel_l2(res["station_wave"][:, :, v], g["out_station_wave"][:, :, v])
        assert err < 1e-5, (v, err)
    assert rel_l2(res["pgv"], g["out_pgv"]) < 1e-5
    assert rel_l2(res["freesurf"], g["out_freesurf"]) < 1e-5


@pytest.mark.parametrize("rows", [16, 8, 0])
def test_stream_matches_exact_on_larger_grid(gpu_available, rows):
    """A grid with several tiles in x and y, odd sizes (partial warps and
    tiles), several z chunks and all PML slabs: the fast path against the
    exact path (which is bit-identical to the reference), after 20 steps."""
    nx, ny, nz, npml = 71, 45, 90, 6
    p = scenarios.S.params(NX=nx, NY=ny, NZ=nz, nPML=npml, DH=100.0, DT=0.008)
    rng = np.random.default_rng(5)
    num = (nx + 6) * (ny + 6) * (nz + 6)
    # a smooth random medium/metric field: perturb a flat-grid CJM
    cjm = np.zeros((13, nz + 6, ny + 6, nx + 6), np.float32)
    inner = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))
    base = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 1e6, 3.2e10, 3.2e10, 1 / 2670.0], np.float32)
    pert = 1 + 0.05 * rng.standard_normal((13, nz, ny, nx)).astype(np.float32)
    cjm[inner] = base[:, None, None, None] * pert
    for f in (1, 2, 3, 5, 6, 7):  # small off-diagonal metrics (a curvilinear grid)
        cjm[f][inner[1:]] = 0.02 * rng.standard_normal((nz, ny, nx)).astype(np.float32)
    rdz = (0.1 * rng.standard_normal(18 * (nx + 6) * (ny + 6))).astype(np.float32)
    sta = np.array([[10, 10, nz + 2], [40, 20, nz + 1], [60, 40, 50]])
    out = {}
    for kern in (cgfdm.KERNEL_EXACT, cgfdm.KERNEL_STREAM):
        with cgfdm.Simulation(_desc(p, 20, kernel=kern)) as sim:
            sim.set_tile_rows(rows)
            sim.set_model(cjm.reshape(-1), rdz)
            sim.set_point_source(nx // 2, ny // 2, nz // 2, 6.0)
            sim.set_stations(sta)
            sim.run(20)
            out[kern] = (sim.stations(), sim.wavefield(), sim.pgv())
    e, s = out[cgfdm.KERNEL_EXACT], out[cgfdm.KERNEL_STREAM]
    assert np.isfinite(s[1]).all()
    assert rel_l2(s[1], e[1]) < 1e-5
    for v in range(9):
        assert rel_l2(s[0][:, :, v], e[0][:, :, v]) < 1e-5


TINY = [(1, 1, 4, 0), (2, 3, 5, 2), (5, 5, 5, 2), (33, 1, 10, 0), (1, 40, 12, 0),
        (40, 17, 7, 3), (64, 32, 60, 31), (3, 3, 4, 3), (7, 9, 4, 2)]


@pytest.mark.parametrize("rows", [16, 8])
@pytest.mark.parametrize("shape", TINY)
def test_stream_matches_exact_on_tiny_and_ragged_grids(gpu_available, shape, rows):
    """One-point-wide grids, the minimum depth (one layer below the three
    free-surface layers), a PML as wide as the grid, partial tiles and
    warps: the streaming kernel against the exact-order kernel, 12 steps.
    (Where opposite PML slabs overlap -- nPML above half the grid -- a
    handle runs the exact-order kernel even when the streaming one is
    asked for, so those shapes check that routing.)"""
    from test_gpu_batch import _synthetic
    nx, ny, nz, npml = shape
    sc = _synthetic(nx, ny, nz, npml, seed=sum(shape))
    out = {}
    for kern in (cgfdm.KERNEL_EXACT, cgfdm.KERNEL_STREAM):
        d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, 12, cgfdm.FP32, kern)
        with cgfdm.Simulation(d) as sim:
            sim.set_tile_rows(rows)
            sim.set_model(sc["cjm"], sc["rdz"])
            sim.set_point_source(nx // 2 + 3, ny // 2 + 3, nz // 2 + 3, 6.0)
            sim.set_stations(np.array([[3, 3, nz + 2], [nx + 2, ny + 2, 3]]))
            sim.run(12)
            out[kern] = (sim.stations(), sim.wavefield())
    e, s = out[cgfdm.KERNEL_EXACT], out[cgfdm.KERNEL_STREAM]
    assert np.isfinite(s[1]).all()
    assert rel_l2(s[1], e[1]) < 1e-5
    assert rel_l2(s[0], e[0]) < 1e-5


FORM_SHAPES = [(200, 60, 40, 6), (150, 45, 30, 0), (131, 83, 37, 9)]


def _run_form(sc, prec, form, steps=12):
    nx, ny, nz, npml = sc["dims"]
    d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, steps, prec, cgfdm.KERNEL_STREAM)
    with cgfdm.Simulation(d) as sim:
        sim.set_tile_rows(form)
        sim.set_model(sc["cjm"], sc["rdz"])
        sim.set_point_source(*sc["src"], 6.0)
        sim.set_stations(sc["sta"])
        sim.run(steps)
        assert sim.kernel_stats()["tile_rows"] == form
        return sim.wavefield(), sim.stations(), sim.pgv()


def _case(shape, precision):
    from test_gpu_batch import _scaled, _synthetic
    nx, ny, nz, npml = shape
    sc = _synthetic(nx, ny, nz, npml, seed=nx + ny)
    prec = {"fp32": cgfdm.FP32, "fp16": cgfdm.FP16, "bf16": cgfdm.BF16}[precision]
    return (sc if precision == "fp32" else _scaled(sc)), prec


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
@pytest.mark.parametrize("shape", [(168, 60, 40, 6), (128, 48, 30, 0)])
def test_paired_form_is_bitwise_the_one_point_kernel(gpu_available, precision, shape):
    """The paired-point kernel (64 x 8 tiles, two points per thread) computes
    each point with the one-point kernel's operations in the same order: on
    grids where both forms give the same points to the interior launch (an
    even number of interior 32-column tiles, full tiles), the paired form
    and the 32 x 8 form give bit-identical wavefields, seismograms and PGV
    over 12 steps (every RK stage and MacCormack sign triple)."""
    sc, prec = _case(shape, precision)
    ref = _run_form(sc, prec, 8)
    got = _run_form(sc, prec, 64)
    assert np.isfinite(ref[0]).all() and np.abs(ref[0]).max() > 0
    for a, b in zip(got, ref):
        assert np.array_equal(a, b), rel_l2(a, b)


@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp32"])
@pytest.mark.parametrize("shape", FORM_SHAPES)
def test_tile_forms_agree(gpu_available, precision, shape):
    """All tile forms (32 x 16, 32 x 8, and for 16-bit storage the paired
    64 x 8 form) over 12 steps on grids with an odd number of interior
    32-column tiles, partial edge tiles and no PML.  The forms split the
    grid differently between the interior and PML launches, whose variants
    round the elastic combination differently, so they agree to rounding:
    relative L2 <= 1e-6 (FP32) or 1e-3 (16-bit storage)."""
    sc, prec = _case(shape, precision)
    forms = [16, 8] + ([64] if precision != "fp32" else [])
    out = {form: _run_form(sc, prec, form) for form in forms}
    ref = out[8]
    assert np.isfinite(ref[0]).all() and np.abs(ref[0]).max() > 0
    tol = 1e-6 if precision == "fp32" else 1e-3
    for form in forms:
        for a, b in zip(out[form], ref):
            assert np.isfinite(a).all()
            assert rel_l2(a, b) <= tol, (form, rel_l2(a, b))


def test_paired_form_is_refused_for_fp32(gpu_available):
    d = cgfdm.make_desc(40, 30, 20, 4, 100.0, 0.008, 2, cgfdm.FP32, cgfdm.KERNEL_STREAM)
    with cgfdm.Simulation(d) as sim:
        with pytest.raises(Exception):
            sim.set_tile_rows(64)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_work_item_depth_does_not_change_results(gpu_available, precision):
    """The depth of the streaming work items in z (cgfdm_set_chunk) only
    changes how the planes above the bottom PML slab are cut into items, not
    how any point is computed: 0 (automatic), 32 and 7 planes give
    bit-identical results; the autotuner's choice is reported."""
    sc, prec = _case((131, 83, 37, 9), precision)
    nx, ny, nz, npml = sc["dims"]
    out = []
    for chunk in (0, 32, 7):
        d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, 12, prec, cgfdm.KERNEL_STREAM)
        with cgfdm.Simulation(d) as sim:
            sim.set_tile_rows(8)
            sim.set_chunk(chunk)
            sim.set_model(sc["cjm"], sc["rdz"])
            sim.set_point_source(*sc["src"], 6.0)
            sim.set_stations(sc["sta"])
            sim.run(12)
            assert sim.tuning() == (8, chunk)
            out.append((sim.wavefield(), sim.stations()))
    for a, b in zip(out[1:], [out[0]] * 2):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    # the autotuner picks a form and a depth among its candidates
    d = cgfdm.make_desc(nx, ny, nz, npml, 100.0, 0.008, 2, prec, cgfdm.KERNEL_STREAM)
    with cgfdm.Simulation(d) as sim:
        sim.set_model(sc["cjm"], sc["rdz"])
        sim.run(1)
        form, chunk = sim.tuning()
        assert form in ((16, 8, 64) if precision == "fp16" else (16, 8)) and chunk in (0, 64, 32)

"""cgfdm_stage_noalloc: the stage entry point for hosts that cannot call
cudaMalloc while they run (a server that splits HBM into fixed pools at
start-up, a framework whose allocator owns all device memory).  It runs one
RK stage on device buffers the caller already owns; here it is checked
against the handle path (cgfdm_stage) on the same inputs.

Both paths run the same kernels on the same inputs, so the bar is bitwise
equality of the stage output W, the RK accumulator t and the PML auxiliaries
(output and accumulator), on each of two calls in a row, in FP32, scaled
FP16 and BF16 storage, on a grid with every PML slab and on a narrow grid
whose opposite x slabs overlap (2 nPML > nx: the exact-order kernel alone).
Device free memory must not change across the second call (wait = 1
synchronizes the stream before the call returns).  The file is named to be collected last; it also passes when
run alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import scenarios

cgfdm = pytest.importorskip("cgfdm")
from cgfdm import _lib  # noqa: E402

GRIDS = [(71, 45, 40, 6), (10, 20, 12, 6)]
NX, NY, NZ, NPML = GRIDS[0]


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _params(nx, ny, nz, npml):
    return scenarios.S.params(NX=nx, NY=ny, NZ=nz, nPML=npml, DH=100.0, DT=0.008)


# Coefficients (metrics, J, mu, lambda, buoyancy) and state magnitudes.  The
# scaled FP16 form holds velocities times Cv = 5e3, stresses times Cs = 1e-6,
# mu and lambda times Cs / Cv and the buoyancy over Crho = 1e6 (macro.h:65-73,
# CJM.cpp:56-71), so every value fits the 16-bit range.
BASE = {"plain": [1, 0, 0, 0, 1, 0, 0, 0, 1, 1e6, 3.2e10, 3.2e10, 1 / 2670.0],
        "scaled": [1, 0, 0, 0, 1, 0, 0, 0, 1, 1.0, 6.4, 6.4, 1.0 / (2670.0 * 2e-10) / 1e6]}
STATE_SCALE = {"plain": (1.0, 1.0), "scaled": (5e3, 1e-6)}


def _model(nx, ny, nz, kind, seed=7):
    rng = np.random.default_rng(seed)
    cjm = np.zeros((13, nz + 6, ny + 6, nx + 6), np.float32)
    base = np.array(BASE[kind], np.float32)
    pert = 1 + 0.05 * rng.standard_normal((13, nz, ny, nx)).astype(np.float32)
    cjm[:, 3:-3, 3:-3, 3:-3] = base[:, None, None, None] * pert
    rdz = (0.1 * rng.standard_normal(18 * (nx + 6) * (ny + 6))).astype(np.float32)
    return cjm.reshape(-1), rdz


def _state(p, seed, kind):
    """scenarios.random_state, rescaled to the storage form's units."""
    st = scenarios.random_state(p, seed)
    cv, cs = STATE_SCALE[kind]
    if kind == "plain":
        return st
    g = scenarios.grid_dims(p)
    sc = np.array([cv] * 3 + [cs] * 6, np.float32)
    for key in ("W", "t", "m"):
        st[key] = (st[key].reshape(9, -1) * sc[:, None]).reshape(-1)
    aux, off = [], 0
    for n in scenarios.slab_points(p):
        for _ in range(3):
            aux.append((st["aux"][off:off + 9 * n].reshape(n, 9) * sc).reshape(-1))
            off += 9 * n
    st["aux"] = np.concatenate(aux)
    assert g["num"] * 9 == st["W"].size
    return st


def test_rejects_grid_larger_than_scratch():
    """The size check comes before any device work, so this runs without a GPU."""
    b = _lib.StageBuffers(nx=3000, ny=2000, nz=500, npml=0, dh=100.0, dt=0.008,
                          precision=cgfdm.FP32, irk=0, fb1=1, fb2=1, fb3=1,
                          w_in=256, w_out=256, w_m=256, t=256, cjm=256, rdz=256)
    rc = _lib.lib().cgfdm_stage_noalloc(ctypes.byref(b), None, 1)
    assert rc == 1
    assert b"scratch" in _lib.lib().cgfdm_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("case", range(len(scenarios.STAGE_CASES)))
def test_noalloc_stage_matches_handle_stage(gpu_available, precision, case, grid):
    import torch

    NX, NY, NZ, NPML = grid
    prec = {"fp32": cgfdm.FP32, "fp16": cgfdm.FP16, "bf16": cgfdm.BF16}[precision]
    tdt = {"fp32": torch.float32, "fp16": torch.float16, "bf16": torch.bfloat16}[precision]
    ebytes = 4 if precision == "fp32" else 2
    kind = "scaled" if precision == "fp16" else "plain"
    p = _params(NX, NY, NZ, NPML)
    irk, fb = scenarios.STAGE_CASES[case]
    cjm, rdz = _model(NX, NY, NZ, kind)
    st = _state(p, 100 + case, kind)

    # the existing entry point: a handle and cgfdm_stage (tile height 16, the
    # form the no-allocation stage launches)
    d = cgfdm.make_desc(NX, NY, NZ, NPML, 100.0, 0.008, 1, prec, cgfdm.KERNEL_AUTO)
    with cgfdm.Simulation(d) as sim:
        sim.set_tile_rows(16)
        sim.set_model(cjm, rdz)
        sim.set_state(irk, W=st["W"], t=st["t"], m=st["m"], aux=st["aux"])
        sim.stage(irk, fb)
        ref = sim.get_state()

    # the same stage on caller-owned device buffers (allocated here, by the test)
    L = cgfdm.hbm_layout(NX, NY, NZ, ebytes)
    dev = torch.device("cuda", 0)

    def view(buf, nf):
        return buf.view(nf, L["fs"])[:, :L["nz_"] * L["plane"]].view(
            nf, L["nz_"], L["ny_"], L["px"])[:, :, :, L["xoff"]:L["xoff"] + L["nx_"]]

    def to_hbm(a, nf):
        buf = torch.zeros(nf * L["fs"], dtype=tdt, device=dev)
        src = torch.from_numpy(a.reshape(nf, L["nz_"], L["ny_"], L["nx_"])).to(dev)
        view(buf, nf)[...] = src.to(tdt)
        return buf

    def from_hbm(buf, nf):
        return view(buf, nf).float().cpu().numpy().reshape(-1)

    # per slab {Aux, t, m} in the reference's [pos][9] -> the concatenations
    # cgfdm_stage_buffers takes: every slab field-major, [9][pos]
    npts = list(scenarios.slab_points(p))
    sizes = [9 * n for n in npts]
    parts = {"a": [], "t": [], "m": []}
    off = 0
    for n in npts:
        for k, key in enumerate("atm"):
            aos = st["aux"][off + k * 9 * n: off + (k + 1) * 9 * n]
            parts[key].append(aos.reshape(n, 9).T.reshape(-1))
        off += 27 * n
    aux = {k: torch.from_numpy(np.ascontiguousarray(np.concatenate(v))).to(dev)
           for k, v in parts.items()}

    def to_aos(soa):  # device order back to the reference's, slab by slab
        out, o = [], 0
        for n in npts:
            out.append(soa[o:o + 9 * n].reshape(9, n).T.reshape(-1))
            o += 9 * n
        return np.concatenate(out)

    w_in = to_hbm(st["W"], 9)
    w_m = w_in if irk == 0 else to_hbm(st["m"], 9)  # stage 0 reads its input as m
    t0 = to_hbm(st["t"], 9)
    t = t0.clone()
    w_out = torch.zeros_like(w_in)
    cjm_d = to_hbm(cjm, 13)
    rdz_d = torch.from_numpy(rdz).to(dev)
    aux_in = aux["a"]
    aux_m = aux_in if irk == 0 else aux["m"]
    aux_t = aux["t"].clone()
    aux_out = torch.zeros_like(aux_in)
    b = _lib.StageBuffers(nx=NX, ny=NY, nz=NZ, npml=NPML, dh=100.0, dt=0.008,
                          precision=prec, irk=irk, fb1=fb[0], fb2=fb[1], fb3=fb[2],
                          w_in=w_in.data_ptr(), w_out=w_out.data_ptr(), w_m=w_m.data_ptr(),
                          t=t.data_ptr(), cjm=cjm_d.data_ptr(), rdz=rdz_d.data_ptr(),
                          aux_in=aux_in.data_ptr(), aux_out=aux_out.data_ptr(),
                          aux_m=aux_m.data_ptr(), aux_t=aux_t.data_ptr())

    # the handle reports the auxiliaries per slab as {out, t, m}
    ref_slabs = np.split(ref["aux"], np.cumsum([3 * n9 for n9 in sizes])[:-1])
    ref_out = np.concatenate([r[:n9] for r, n9 in zip(ref_slabs, sizes)])
    ref_t = np.concatenate([r[n9:2 * n9] for r, n9 in zip(ref_slabs, sizes)])

    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        t.copy_(t0)  # t and aux_t are updated in place by stages 1-2
        aux_t.copy_(aux["t"])
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        cgfdm.stage_noalloc(b, stream.cuda_stream, wait=True)
        free_after = torch.cuda.mem_get_info(dev)[0]
        if call == 1:  # (the first call of a process may load the library's module)
            assert free_after == free_before, (free_before, free_after)
        got = {"W": (from_hbm(w_out, 9), ref["W"]), "t": (from_hbm(t, 9), ref["t"]),
               "aux_out": (to_aos(aux_out.cpu().numpy()), ref_out),
               "aux_t": (to_aos(aux_t.cpu().numpy()), ref_t)}
        for key, (a, r) in got.items():
            assert np.isfinite(r).all(), key
            assert np.array_equal(a, r), (call, key, rel_l2(a, r))

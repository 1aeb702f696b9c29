"""Pins the oracle (oracle/cgfdm_oracle.c) to the reference: every value the
oracle computes must equal, bit for bit, what the reference's own FP32 scalar
build produced on the same inputs (fixtures in tests/golden/)."""
import numpy as np
import pytest

import scenarios
from oracle import oracle as O

HALO = 3


def _grid(p):
    return O.make_grid(p["NX"], p["NY"], p["NZ"], p["nPML"], p["DH"])


@pytest.fixture(scope="module")
def stage_golden():
    return scenarios.load_golden("stage_small.npz")


def test_pml_profiles_bitwise(stage_golden):
    g = _grid(stage_golden["params"])
    pml = O.PmlProfiles(g)
    np.testing.assert_array_equal(pml.block, stage_golden["pml"])


@pytest.mark.parametrize("case", range(len(scenarios.STAGE_CASES)))
def test_stage_bitwise(stage_golden, case):
    d = stage_golden
    p = d["params"]
    g = _grid(p)
    irk, fb = scenarios.STAGE_CASES[case]
    st = O.State(g)
    st.W[:] = d["in_W"]
    st.t[:] = d["in_t"]
    st.m[:] = d["in_m"]
    off = 0
    for s in range(5):
        n = st.aux.bufs[s][1].size
        for b in (1, 2, 3):
            st.aux.bufs[s][b][:] = d["in_aux"][off:off + n]
            off += n
    pml = O.PmlProfiles(g)
    O.stage(g, irk, fb, p["DT"], st, d["cjm"], d["rdz"], pml)
    np.testing.assert_array_equal(st.h, d["case%d_h" % case])
    np.testing.assert_array_equal(st.W, d["case%d_W" % case])
    np.testing.assert_array_equal(st.t, d["case%d_t" % case])
    np.testing.assert_array_equal(st.m, d["case%d_m" % case])
    got = np.concatenate([np.concatenate(st.aux.bufs[s]) for s in range(5)])
    np.testing.assert_array_equal(got, d["case%d_aux" % case])


def _station_idx(p, stations):
    # global interior index -> padded local index (station.cpp:162-172)
    return np.array([[x + HALO, y + HALO, z + HALO] for x, y, z in stations.values()], np.int32)


@pytest.mark.parametrize("name", ["run_point.npz", "run_fault.npz"])
def test_full_run_bitwise(name):
    d = scenarios.load_golden(name)
    p = d["params"]
    g = _grid(p)
    NT = scenarios.S.nt_of(p)
    kw = {}
    if p["useMultiSource"]:
        kw["fault"] = dict(srcIndex=d["src_index"], momentRate=d["src_rate"],
                           nt=int(d["src_nt"]), dt=float(np.frombuffer(
                               d["source"][8:12].tobytes(), np.float32)[0]))
    else:
        kw["point"] = (p["sourceX"] + HALO, p["sourceY"] + HALO, p["sourceZ"] + HALO)
        kw["rickerfc"] = p["rickerfc"]
    res = O.run(g, p["DT"], NT, d["cjm"], d["rdz"], stations=_station_idx(p, d["stations"]),
                snapshot_every=p["IT_SKIP"], **kw)
    np.testing.assert_array_equal(res["station_wave"], d["out_station_wave"])
    np.testing.assert_array_equal(res["pgv"], d["out_pgv"])
    np.testing.assert_array_equal(res["freesurf"], d["out_freesurf"])

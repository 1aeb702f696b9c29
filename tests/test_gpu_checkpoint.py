"""Checkpoint / resume: a handle's state saved at a step boundary and loaded
into a fresh handle with the same descriptor, sources and stations continues
the run bit for bit (seismograms, PGV map, wavefield), in FP32 and scaled
FP16; a checkpoint of another configuration is refused."""
import numpy as np
import pytest

from test_gpu_batch import NT, SHAPES, _scaled, _sim, _synthetic

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")


@pytest.mark.parametrize("precision", [cgfdm.FP32, cgfdm.FP16])
def test_resume_from_checkpoint_is_bitwise(gpu_available, precision):
    sc = _synthetic(*SHAPES[2], seed=21)
    if precision != cgfdm.FP32:
        sc = _scaled(sc)
    with _sim(sc, precision) as s:
        s.run(NT)
        ref = (s.stations(), s.pgv(), s.wavefield())
    with _sim(sc, precision) as s:
        s.run(NT // 3)
        ck = s.checkpoint()
    with _sim(sc, precision) as s:
        s.set_graph(True)
        s.restore(ck)
        s.run(NT - NT // 3)
        got = (s.stations(), s.pgv(), s.wavefield())
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)


def test_checkpoint_of_another_grid_is_refused(gpu_available):
    with _sim(_synthetic(*SHAPES[1], seed=2)) as s:
        s.run(2)
        ck = s.checkpoint()
    with _sim(_synthetic(*SHAPES[3], seed=2)) as s:
        with pytest.raises(cgfdm.CgfdmError) as e:
            s.restore(ck)
        assert e.value.code == 304

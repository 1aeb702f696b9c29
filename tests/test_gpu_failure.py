"""Failure detection on the device without faulting it: a streaming launch
is made to leave one tile-plane load unissued (cgfdm_inject_fault), so that
one CTA's bounded mbarrier wait (about a second) expires.  The kernel drains
its own copies and returns; the host gets CGFDM_ERR_TIMEOUT once, and the
context stays usable: a new handle then matches an unfaulted run bit for
bit."""
import numpy as np
import pytest

from test_gpu_batch import SHAPES, _sim, _synthetic

pytestmark = pytest.mark.gpu
cgfdm = pytest.importorskip("cgfdm")


def test_expired_wait_is_reported_and_the_handle_recovers(gpu_available):
    sc = _synthetic(*SHAPES[0], seed=9)
    ref = _sim(sc)
    ref.run(6)
    ref_w = ref.wavefield()
    ref.close()

    s = _sim(sc)
    s.run(1)
    s.synchronize()
    s.inject_fault(1)  # CGFDM_FAULT_DROP_LOAD
    s.run(1)
    with pytest.raises(cgfdm.CgfdmError) as e:
        s.synchronize()
    assert e.value.code == 303
    s.synchronize()  # reported once: the flag is clear again
    s.close()

    # the device context is intact: a new handle runs and matches the
    # unfaulted run bit for bit
    s = _sim(sc)
    s.run(1)
    s.run(5)
    np.testing.assert_array_equal(s.wavefield(), ref_w)
    s.close()

"""Failure detection on the GPU without a GPU fault: a bounded device wait is
made to run out (a predecessor's status word that nothing writes), the kernel
records JC_ERR_DEVICE_TIMEOUT and finishes, and the context stays usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sort_wait_gives_up_and_the_context_survives(jc, orc):
    status, ms = ctypes.c_uint32(0), ctypes.c_float(0.0)
    assert jc.lib().jc_selftest_sort_wait(ctypes.byref(status), ctypes.byref(ms)) == jc.JC_OK
    assert status.value == jc.JC_ERR_DEVICE_TIMEOUT
    assert 1.0 < ms.value < 20000.0  # bounded: gave up after its spin limit
    # the same process keeps working: a step bit-exact against the oracle
    g = jc.gen_scale_free(500, 3, 9)
    x = jc.seed_uniform(500, 3, 9)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g, x)
    e.step()
    f, _ = e.forces()
    ref = orc.Fa2(g, x, bh=True, theta=0.8)
    ref.step()
    assert np.array_equal(f.view(np.uint32), ref.get()["force"].view(np.uint32))
    e.close()

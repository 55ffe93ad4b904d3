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


def test_gemm_wait_gives_up_and_the_context_survives(jc):
    """The tensor-core GEMM's mbarrier waits are bounded: a wait on a phase
    that no tcgen05.commit completes gives up, records the timeout, frees the
    tensor memory, and a real GEMM right after it is still correct."""
    status, ms = ctypes.c_uint32(0), ctypes.c_float(0.0)
    assert jc.lib().jc_selftest_gemm_wait(ctypes.byref(status), ctypes.byref(ms)) == jc.JC_OK
    assert status.value == jc.JC_ERR_DEVICE_TIMEOUT
    assert 500.0 < ms.value < 5000.0  # bounded to about a second of device time
    rng = np.random.default_rng(3)
    M, N, K = 256, 128, 192
    a = jc.from_bf16_bits(jc.to_bf16_bits(rng.standard_normal((M, K)).astype(np.float32)))
    b = jc.from_bf16_bits(jc.to_bf16_bits(rng.standard_normal((N, K)).astype(np.float32)))
    c = jc.tc_gemm_bf16(jc.to_bf16_bits(a), jc.to_bf16_bits(b), M, N, K)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    assert np.max(np.abs(c - ref)) <= 1e-3 * np.max(np.abs(ref))

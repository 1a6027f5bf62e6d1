"""Failure detection of the tensor-core kernels, exercised without a fault.

Every mbarrier wait of the convolution kernels is bounded by the global timer;
when one runs out the kernel stores a code in the network's error word and
returns, and the host reports LG_ERR_DEVICE (the reference instead calls
exit(1) on any CUDA error, src/pathtracer.cu:17-20).  lg_unet_wait_selftest
runs that bounded wait on an mbarrier nothing arrives at (no copy or MMA in
flight), with a 1 ms limit: the call must come back with the status within
well under a second, and the network must keep working afterwards with
unchanged results."""
import ctypes as C
import time

import numpy as np
import pytest

import lumina
from lumina import _ffi

pytestmark = pytest.mark.gpu


def test_wait_limit_expiry_is_reported_and_the_network_recovers():
    net = lumina.UNet()
    rng = np.random.default_rng(5)
    net.set_params(rng.normal(0, 0.05, net.n_params).astype(np.float32))
    x = rng.uniform(0, 1, (1, 3, 64, 96)).astype(np.float32)
    y0 = net.forward(x)
    L = _ffi.lib()
    for limit_ns in (1_000_000, 20_000_000):
        t0 = time.perf_counter()
        rc = L.lg_unet_wait_selftest(net._h, limit_ns)
        dt = time.perf_counter() - t0
        assert rc == _ffi.LG_ERR_DEVICE, rc
        assert b"wait timeout 3" in L.lg_last_error()
        assert dt < 1.0, dt  # the wait ended at its limit
        y1 = net.forward(x)  # the next call clears the word and runs normally
        assert np.array_equal(y0, y1)
    assert L.lg_unet_wait_selftest(net._h, 10) == _ffi.LG_ERR_INVALID  # limits below 1 us are refused
    net.close()

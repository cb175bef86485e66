"""Failure detection on the GPU without a fault: the grid barrier's bounded wait.

The grid-resident schedule's kernel is the library's only device-side
spin-wait (lmb::grid_barrier).  A cooperative launch whose barrier expects
more arrivals than there are blocks can never be released; its waits must
give up by themselves (about a second), report LMB_E_TIMEOUT through the
status the host reads, and leave the context usable for the next launch.
"""
import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "cpp", "_build", "libgrid_selftest.so")
LMB_OK = 0
LMB_E_TIMEOUT = -8


def _selftest():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")], check=True)
    lib = C.CDLL(LIB)
    fn = lib.lmb_selftest_grid_barrier
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_float)]

    def run(blocks, target):
        status, ms = C.c_int32(123), C.c_float(-1.0)
        err = fn(blocks, target, C.byref(status), C.byref(ms))
        return err, status.value, ms.value
    return run


@pytest.mark.gpu
def test_grid_barrier_passes_when_every_block_arrives():
    run = _selftest()
    err, status, ms = run(64, 64)
    assert err == 0 and status == LMB_OK
    assert ms < 100.0


@pytest.mark.gpu
def test_grid_barrier_wait_gives_up_and_reports_timeout():
    """Four blocks, a barrier expecting eight arrivals: every wait gives up
    after its one-second limit, the status reads LMB_E_TIMEOUT, the launch
    and the synchronisation report no CUDA error, and the next launch on the
    same context passes its barrier."""
    run = _selftest()
    err, status, ms = run(4, 8)
    assert err == 0
    assert status == LMB_E_TIMEOUT
    assert 900.0 <= ms < 10000.0
    err, status, ms = run(4, 4)
    assert err == 0 and status == LMB_OK

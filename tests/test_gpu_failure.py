"""Failure detection without a GPU fault: the engines' grid barrier gives up
after a bounded wait when a block never arrives (a flag nothing sets), the
kernel returns, the host reads the abort, and the context stays usable."""
import ctypes as C
import time

import pytest

import bfx

pytestmark = pytest.mark.gpu


def selftest(rounds, absent, timeout_ns):
    out = (C.c_uint32 * 4)()
    rc = bfx.load().bfx_barrier_selftest(0, C.c_uint32(rounds), C.c_uint32(absent), C.c_uint64(timeout_ns), out)
    assert rc == 0, bfx.load().bfx_last_error()
    return list(out)


def test_barrier_passes_when_every_block_arrives(gpu):
    aborted, passed, gave_up, grid = selftest(2000, 0xFFFFFFFF, 1_000_000_000)
    assert aborted == 0 and passed == 2000 and gave_up == 0 and grid >= 148


def test_missing_block_times_out_and_reports(gpu):
    t0 = time.time()
    aborted, passed, gave_up, grid = selftest(10, 3, 100_000_000)  # 100 ms limit
    assert time.time() - t0 < 10
    assert aborted == 1 and passed == 0 and gave_up == grid - 1
    # the context is still usable afterwards
    assert selftest(100, 0xFFFFFFFF, 1_000_000_000)[:3] == [0, 100, 0]


def test_selftest_rejects_unbounded_wait(gpu):
    out = (C.c_uint32 * 4)()
    assert bfx.load().bfx_barrier_selftest(0, 1, 0xFFFFFFFF, C.c_uint64(0), out) == 1
    assert bfx.load().bfx_barrier_selftest(0, 1, 0xFFFFFFFF, C.c_uint64(10_000_000_000), out) == 1

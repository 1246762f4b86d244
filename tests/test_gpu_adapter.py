"""GPU: the reference's own batch descriptions (its planner and
prepare_batch_device_description, in both run representations) run through
include/bfx_bfnew_adapter.hpp -- libbfx behind bf-new's engine classes --
and every status field, distance bit and predecessor equals the reference's
portable batched engines on the same descriptions."""
import ctypes as C

import pytest

from adapter_cases import ADAPTER_SO, fixture_case, load

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ADAPTER_SO.exists(), reason="adapter check (oracle/_ref) not built")]

ENGINES = {"jacobi": 0, "dense": 1, "frontier": 2}


def check(lib, h, engine, representation):
    out = (C.c_uint64 * 6)()
    rc = lib.adapter_check_plan(C.c_int(h), C.c_int(engine), C.c_int(representation), out)
    assert rc == 0, lib.ref_last_error()
    batches, lanes, dist_bad, status_bad, pred_checks, pred_bad = (int(x) for x in out)
    assert batches > 0 and lanes > 0
    assert (dist_bad, status_bad, pred_bad) == (0, 0, 0)
    return pred_checks


@pytest.mark.parametrize("engine", ["jacobi", "dense", "frontier"])
@pytest.mark.parametrize("representation", [0, 1], ids=["retained_masks", "device_materialized"])
def test_five_lane_fixture_through_adapter(gpu, engine, representation):
    lib = load()
    h = fixture_case(lib, "batched_mixed", 0, 8, (0, 1, 4, 1))
    assert check(lib, h, ENGINES[engine], representation) > 0


@pytest.mark.parametrize("suite", ["jacobi", "dense", "frontier"])
def test_single_query_fixture_suites_through_adapter(gpu, suite):
    lib = load()
    n = lib.ref_fixture_count(suite.encode())
    assert n >= 13
    for i in range(n):
        h = fixture_case(lib, suite, i, 1)
        check(lib, h, ENGINES[suite], 1)

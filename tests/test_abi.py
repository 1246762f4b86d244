"""CPU checks of the C-ABI boundary: libbfx.so loads, exports every entry
point declared in include/*.h, keeps the reference's record layouts, and
reports errors as status codes (no compute calls here)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import bfx

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared_functions():
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        text = h.read_text()
        names += re.findall(r"^\s*(?:int|const char \*)\s*(bfx_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "bfx_execute" in names and "bfx_layout_build" in names and len(names) >= 25


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    lib = bfx.load()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported by libbfx.so"


def test_record_layouts_match_reference_abi():
    # include/bfnew/gpu_api.hpp:225-251
    assert C.sizeof(bfx.GpuRunOptions) == 48
    assert bfx.GpuRunOptions.maximum_rounds.offset == 32
    assert bfx.GpuRunOptions.enable_per_lane_convergence.offset == 40
    assert C.sizeof(bfx.DeviceController) == 96
    assert bfx.DeviceController.rounds_completed.offset == 32
    assert bfx.DeviceController.frontier_size.offset == 64
    assert bfx.DeviceController.next_frontier_lane_mask.offset == 80
    assert bfx.DeviceController.error_bits.offset == 92
    assert C.sizeof(bfx.DeviceRunStatus) == 48
    assert bfx.DeviceRunStatus.rounds_completed.offset == 8
    assert bfx.DeviceRunStatus.reached_target_mask.offset == 16
    assert bfx.DeviceRunStatus.error_bits.offset == 40
    # include/bfnew/batch_layout.hpp:201-206
    assert C.sizeof(bfx.BatchVertexRange) == 12


def test_abi_version_and_errors_without_gpu():
    lib = bfx.load()
    assert lib.bfx_abi_version() == 1
    n = C.c_int(-1)
    assert lib.bfx_device_count(C.byref(n)) == 0 and n.value >= 0
    h = C.c_void_p()
    assert lib.bfx_layout_build(None, None, 0, C.byref(h)) == 1  # BFX_ERR_INVALID_ARGUMENT
    assert b"null" in lib.bfx_last_error()


def test_layout_builder_rejects_bad_input_like_reference():
    g, order, _ = bfx.synth_graph(4, 4, 4, 2, 0, [], seed=3)
    bad = bfx.InputGraph(g.x, g.y, g.has_location, g.resource_class, g.edge_source, g.edge_destination,
                         g.edge_weight.copy(), g.provenance_domain, g.provenance_kind, g.provenance_record)
    bad.edge_weight[3] = -1.0
    with pytest.raises(ValueError, match="nonnegative"):
        bfx.build_device_graph_layout(bad, order)
    bad.edge_weight[3] = np.inf
    with pytest.raises(ValueError, match="finite"):
        bfx.build_device_graph_layout(bad, order)
    bad.edge_weight[3] = 1.0
    bad.edge_destination[5] = g.vertex_count
    with pytest.raises(IndexError):
        bfx.build_device_graph_layout(bad, order)


def test_upload_without_device_fails_loudly():
    if bfx.device_count() > 0:
        pytest.skip("a GPU is visible")
    g, order, _ = bfx.synth_graph(4, 4, 4, 2, 0, [], seed=3)
    layout = bfx.build_device_graph_layout(g, order)
    with pytest.raises(bfx.BfxNoDevice):
        bfx.ResidentDeviceGraph.upload_once(layout)


def test_description_c_view_is_cached_until_a_field_is_replaced():
    """BatchDescription.c() hands the C ABI pointers into its own arrays; the
    view is reused across calls (the e2e step prepares the same set every
    step) and rebuilt when a field is replaced."""
    W = 8
    d = bfx.BatchDescription(W, 0x3, np.array([0, 1, 2] + [2] * (W - 2), np.uint32), np.array([5, 9], np.uint32),
                             np.array([0, 1, 2] + [2] * (W - 2), np.uint32), np.array([6, 7], np.uint32),
                             np.array([0], np.uint32), np.array([3], np.uint32),
                             np.array([[0, 16, 3]], np.uint32))
    a = d.c()
    assert d.c() is a
    assert C.addressof(a.sources.contents) == d.sources.ctypes.data
    d.sources = np.array([4, 9], np.uint32)
    b = d.c()
    assert b is not a
    assert C.addressof(b.sources.contents) == d.sources.ctypes.data
    assert b.lane_width == W and b.valid_lane_mask == 0x3 and b.range_count == 1

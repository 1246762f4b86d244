"""The adapter a bf-new build links against libbfx (include/bfx_bfnew_adapter.hpp):
it compiles against the reference's own headers with every record-layout
assertion (GpuRunOptions, DeviceController, DeviceRunStatus,
DeviceWorkStatistics, BatchVertexRange, CompactTargetSummary and the engine /
control-mode values), its flattened view of a reference-prepared
BatchDeviceDescription carries the description's own arrays, and without a
GPU it raises the std::runtime_error bf-new's device layer raises."""
import subprocess
from pathlib import Path

import pytest

from adapter_cases import ADAPTER_SO, REPO, fixture_case, load

pytestmark = pytest.mark.skipif(not ADAPTER_SO.exists(), reason="adapter check (oracle/_ref) not built")


def reference_include() -> Path:
    out = subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), "print-ref"], capture_output=True, text=True,
                         check=True).stdout.strip()
    return Path(out) / "include"


def test_adapter_header_compiles_against_the_reference_headers(tmp_path):
    inc = reference_include()
    if not inc.exists():
        pytest.skip("reference headers not present here")
    src = tmp_path / "use_adapter.cpp"
    src.write_text('#include "bfx_bfnew_adapter.hpp"\n'
                   "int main() { return sizeof(bfnew::cuda::BatchedFrontierPushEngine) > 0 ? 0 : 1; }\n")
    res = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", f"-I{inc}",
                          f"-I{REPO / 'include'}", str(src)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_flatten_views_reference_descriptions():
    lib = load()
    h = fixture_case(lib, "batched_mixed", 0, 8, (0, 1, 4, 1))
    assert lib.adapter_flatten_check(h) > 0, lib.ref_last_error()


def test_no_device_raises_runtime_error():
    import bfx
    if bfx.device_count() != 0:
        pytest.skip("a device is present")
    lib = load()
    h = fixture_case(lib, "frontier", 0, 1)
    assert lib.adapter_no_device_raises(h) == 1

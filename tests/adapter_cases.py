"""ctypes view of oracle/_ref/libbfx_adapter_check.so (test infrastructure):
bf-new's own batch descriptions through include/bfx_bfnew_adapter.hpp."""
import ctypes as C
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
ADAPTER_SO = REPO / "oracle" / "_ref" / "libbfx_adapter_check.so"


def load():
    lib = C.CDLL(str(ADAPTER_SO))
    lib.ref_last_error.restype = C.c_char_p
    return lib


def fixture_case(lib, suite: str, index: int, lane_width: int, policy=(0, 1, 64, 1)) -> int:
    h = lib.ref_case_fixture(suite.encode(), C.c_int(index))
    assert h >= 0, lib.ref_last_error()
    nb = lib.ref_plan(C.c_int(h), C.c_uint32(lane_width), *(C.c_uint32(x) for x in policy))
    assert nb > 0, lib.ref_last_error()
    return h

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers",
                            "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import ref_oracle
    if not ref_oracle.available("f64"):
        pytest.skip("reference oracle not built (needs the reference checkout)")
    return ref_oracle


@pytest.fixture(scope="session")
def core_host():
    """Test-only host build of the device core (tests/native)."""
    import ctypes as C
    lib_path = REPO / "tests" / "native" / "libcore_host.so"
    if not lib_path.exists():
        from detray_b200 import build
        build.build_core_host()
    lib = C.CDLL(str(lib_path))
    lib.core_host_last_error.restype = C.c_char_p
    return lib


@pytest.fixture(scope="session")
def core_host_stepped():
    """The same host build with DPROP_NO_CYCLE_SKIP: exact stepping cycles
    run to the path limit step by step, as in the reference."""
    import ctypes as C
    from detray_b200 import build
    lib_path = build.build_core_host(stepped=True)
    lib = C.CDLL(str(lib_path))
    lib.core_host_last_error.restype = C.c_char_p
    return lib

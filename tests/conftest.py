"""pytest configuration: the `gpu` marker and access to the package and the oracle.

The package directory name carries a hyphen, so it is loaded by path as the module
`jpeg2000_decoder_b200`.  The oracle (oracle/liboracle.so, oracle/_ref/libref_t1.so) is
test infrastructure and is only ever loaded from here as the checker.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def load_package():
    name = "jpeg2000_decoder_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "jpeg2000-decoder_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    # build the in-tree libraries once if they are missing (no-op when up to date)
    pkg = load_package()
    from jpeg2000_decoder_b200 import build  # noqa: F401
    try:
        build.build_library()
    except Exception as e:  # noqa: BLE001 - surfaced by the tests that need the library
        print("native build failed:", e)
    try:
        build.build_oracle()
    except Exception as e:  # noqa: BLE001
        print("oracle build failed:", e)
    return pkg


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def gpu_ctx(pkg):
    from jpeg2000_decoder_b200 import native
    ctx = native.GpuContext()
    yield ctx
    ctx.close()
